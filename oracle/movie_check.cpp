// TEST INFRASTRUCTURE (built by oracle/Makefile into _ref/, never shipped): the reference's whole movie engine,
// compiled from its sources, rendering a movie through its public API (RenderScopeMovie, ScopeMovie.h:480) on the CPU,
// then again with libiscu installed as the engine's process-wide blink splat + camera noise host
// (SetDefaultBlinkSplatGpu, ScopeMovie.cpp:5535: a SplatGpuHost, SplatGpu.h, over the CUDA named-kernel backend,
// include/iscu_gpubackend.hpp) on CUDA device 0.
//
// Checks, one output line each ("<check> ok|FAIL <figures>"), exit status 0 when all pass:
//   movie_install    the install made a host that passed the reference's own self-check (DefaultBlinkSplatGpu)
//   movie_<name>     the movie's frames with the host against the CPU's: every frame reported as drawn by the GPU
//                    splat ("blinks (splat, GPU)"), >= 99 % of the pixels equal and the mean |ADU difference| within
//                    1e-3 of the mean ADU (the engine's contract for its GPU host: frames within float32 rounding of
//                    the CPU's, a Poisson draw near a count boundary one count apart)
#include "ScopeMovie.h"
#include "SplatGpu.h"
#include "iscu_gpubackend.hpp"

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

namespace {

int failures = 0;

void Report(const std::string& name, bool ok, const std::string& detail)
{
   std::printf("%s %s %s\n", name.c_str(), ok ? "ok" : "FAIL", detail.c_str());
   std::fflush(stdout);
   if (!ok)
      ++failures;
}

bool Movie(const std::string& text, std::vector<uint16_t>& frames, long& gpuFrames, std::string& err)
{
   sim::ScopeSpec spec;
   if (!sim::ParseScopeSpec(text, spec, err))
      return false;
   frames.clear();
   gpuFrames = 0;
   sim::ScopeProgress progress = [&](const char* stage, double, const std::string& json) {
      if (std::string(stage) == "frames" && json.find("blinks (splat, GPU)") != std::string::npos)
         ++gpuFrames;
   };
   sim::ScopeMovieInfo info;
   return sim::RenderScopeMovie(spec, [&](long, const std::vector<uint16_t>& adu) {
      frames.insert(frames.end(), adu.begin(), adu.end());
      return true;
   }, info, err, &progress);
}

} // namespace

int main()
{
   const std::vector<std::pair<std::string, std::string>> movies = {
      {"dstorm", "frames=12 size=96 seed=42 psf-oversampling=4 psf-kernel-half-width-nm=2000 psf-z-range-um=2 "
                 "psf-halo-cut=0"},
      {"dstorm_halo", "frames=12 size=96 seed=7 psf-oversampling=4 psf-kernel-half-width-nm=2000 psf-z-range-um=2 "
                      "psf-halo-cut=3e-6"},
   };
   std::vector<std::vector<uint16_t>> cpu(movies.size());
   for (size_t i = 0; i < movies.size(); ++i)
   {
      std::string err;
      long g = 0;
      if (!Movie(movies[i].second, cpu[i], g, err) || cpu[i].empty())
      {
         Report("movie_" + movies[i].first, false, "CPU movie: " + err);
         cpu[i].clear();
      }
   }
   sim::SetDefaultBlinkSplatGpu([](std::string& info) -> std::unique_ptr<sim::SplatGpuHost> {
      auto be = iscu_sim::CudaGpuBackend::Create(0, info);
      return be ? sim::MakeSplatGpuHost(be, info) : nullptr;
   });
   const bool installed = sim::DefaultBlinkSplatGpu() != nullptr;
   Report("movie_install", installed, installed ? "host made, self-check passed" : sim::DefaultBlinkSplatGpuInfo());
   for (size_t i = 0; installed && i < movies.size(); ++i)
   {
      if (cpu[i].empty())
         continue;
      std::string err;
      std::vector<uint16_t> gpu;
      long gpuFrames = 0;
      if (!Movie(movies[i].second, gpu, gpuFrames, err) || gpu.size() != cpu[i].size())
      {
         Report("movie_" + movies[i].first, false, "GPU movie: " + err);
         continue;
      }
      size_t equal = 0;
      double diff = 0.0, total = 0.0;
      for (size_t k = 0; k < gpu.size(); ++k)
      {
         equal += gpu[k] == cpu[i][k];
         diff += std::fabs(static_cast<double>(gpu[k]) - cpu[i][k]);
         total += cpu[i][k];
      }
      const double eq = static_cast<double>(equal) / gpu.size(), rel = diff / std::max(1.0, total);
      char buf[200];
      std::snprintf(buf, sizeof(buf), "gpu_frames=%ld equal=%.6f rel_diff=%.3e pixels=%zu", gpuFrames, eq, rel,
                    gpu.size());
      Report("movie_" + movies[i].first, gpuFrames == 12 && eq >= 0.99 && rel <= 1e-3, buf);
   }
   sim::SetDefaultBlinkSplatGpu(nullptr);
   return failures == 0 ? 0 : 1;
}
