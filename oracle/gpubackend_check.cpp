// TEST INFRASTRUCTURE (built by oracle/Makefile into _ref/, never shipped): the reference's own GPU hosts,
// SplatGpuHost (SplatGpu.cpp) and WidefieldGpuHost (WidefieldGpuHost.cpp), compiled from its sources and driven
// unmodified over libiscu's named-kernel backend (include/iscu_gpubackend.hpp) on CUDA device 0.
//
// Checks, one output line each ("<check> ok|FAIL <figures>"), exit status 0 when all pass:
//   splat_selfcheck      MakeSplatGpuHost: the reference's own self-check (SplatGpu.cpp:464-556)
//   splat_movie_*        the host's RenderFrames over a 4-frame movie (events spanning frames, a background image per
//                        frame, sCMOS and EMCCD, with and without the halo cut) against the reference's CPU frame
//                        (RenderPhotonImage + ApplyNoiseChain): the fraction of equal pixels and the mean |ADU
//                        difference| relative to the mean ADU
//   widefield_selfcheck  WidefieldGpuHost::SelfCheck (WidefieldGpuHost.cpp:560-667): images within 1e-3 rms of the
//                        CPU's, frame noise >= 90 % equal
#include "SMLMNoise.h"
#include "SMLMSimulation.h"
#include "SplatGpu.h"
#include "WidefieldGpuHost.h"
#include "iscu_gpubackend.hpp"

#include <cmath>
#include <cstdio>
#include <random>
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

void SplatMovie(const std::shared_ptr<iscu_sim::CudaGpuBackend>& be, double haloThreshold)
{
   using namespace sim;
   std::string err;
   PsfGeneratorRequest req;
   req.model = PsfModelKind::GibsonLanniZernike;
   req.wavelengthNm = 670;
   req.na = 1.45;
   req.pixelSizeNm = 108;
   req.oversampling = 4;
   req.kernelHalfWidthPx = 8;
   req.nz = 9;
   req.zStepNm = 100;
   req.interpMode = PsfInterpMode::Cubic;
   PsfKernelCache full;
   if (!ComputePsfKernelCache(req, full, err) || !full.valid)
   {
      Report("splat_movie", false, "no kernel: " + err);
      return;
   }
   const PsfKernelCache kernel = haloThreshold > 0 ? WithHaloCut(full, haloThreshold) : full;
   const unsigned W = 96, H = 80, F = 4;
   const size_t n = static_cast<size_t>(W) * H;
   std::mt19937_64 rng(2024);
   std::uniform_real_distribution<double> u(0.0, 1.0);
   std::vector<BlinkEvent> evs(1500);
   for (BlinkEvent& e : evs)
   {
      e.xUm = (W * 0.108 + 1.0) * u(rng) - 0.5;
      e.yUm = (H * 0.108 + 1.0) * u(rng) - 0.5;
      e.zNm = 800 * u(rng) - 400;
      e.tStart = (F + 0.5) * u(rng) - 0.5;
      e.tEnd = e.tStart + 0.2 + 1.5 * u(rng);
      e.brightness = 0.3 + 1.4 * u(rng);
   }
   PixelOffsetMap off;
   PixelGainMap gain;
   PixelReadNoiseMap rn;
   off.Generate(W, H, 100, 2, rng);
   gain.Generate(W, H, 0.45, 0.02, rng);
   rn.Generate(W, H, 1.5, 0.2, rng);
   std::vector<float> bg(n);
   for (unsigned y = 0; y < H; ++y)
      for (unsigned x = 0; x < W; ++x)
         bg[static_cast<size_t>(y) * W + x] = static_cast<float>(8.0 + 6.0 * std::exp(-((x - 40.0) * (x - 40.0) +
                                                                                      (y - 30.0) * (y - 30.0)) / 900.0));
   for (int emccd = 0; emccd < 2; ++emccd)
   {
      CameraNoiseParams cam;
      cam.emccd = emccd != 0;
      cam.quantumEfficiency = 0.9;
      cam.darkCurrentElectrons = 0.02;
      cam.gainPhotonsPerAdu = 0.45;
      cam.readNoiseElectrons = 1.5;
      SplatGpuHost host(be);
      std::vector<std::vector<GpuSplatEmitter>> ems(F);
      std::vector<uint32_t> frames(F);
      std::vector<const std::vector<float>*> extras(F, &bg);
      std::vector<std::vector<uint16_t>> gpu(F);
      std::vector<std::vector<uint16_t>*> outs(F);
      for (unsigned f = 0; f < F; ++f)
      {
         CollectGpuEmitters(evs, f, W, H, 108.0, 1800.0, 0.2, -0.1, kernel, 0.03, nullptr, ems[f]);
         frames[f] = f;
         outs[f] = &gpu[f];
      }
      const std::string name = std::string("splat_movie_") + (emccd ? "emccd" : "scmos") +
                               (haloThreshold > 0 ? "_halo" : "");
      if (!host.SetKernels({&kernel}, err) ||
          !host.SetStatic(W, H, 0, off.offset, gain.gainPhotonsPerAdu, rn.readNoiseElectrons, cam, 0, err) ||
          !host.RenderFrames(ems, frames, extras, cam, 4242u, outs, err))
      {
         Report(name, false, err);
         continue;
      }
      size_t same = 0, emitters = 0;
      double diff = 0, mean = 0;
      for (unsigned f = 0; f < F; ++f)
      {
         std::vector<float> cpu(n, 0.0f);
         RenderPhotonImage(cpu, W, H, evs, f, 108.0, 1.3, 1800.0, 0.0, 0.2, -0.1, &kernel, 0.03);
         for (size_t i = 0; i < n; ++i)
            cpu[i] += bg[i];
         std::vector<uint16_t> cpuAdu;
         ApplyNoiseChain(cpu, cpuAdu, W, H, cam, off, gain, rn, 4242u, f, false, 0);
         for (size_t i = 0; i < n; ++i)
         {
            same += cpuAdu[i] == gpu[f][i];
            diff += std::abs(static_cast<double>(cpuAdu[i]) - gpu[f][i]);
            mean += cpuAdu[i];
         }
         emitters += ems[f].size();
      }
      const double frac = static_cast<double>(same) / (static_cast<double>(n) * F), rel = diff / mean;
      char buf[160];
      const double kept = kernel.halo ? kernel.halo->keptFraction : 1.0;
      std::snprintf(buf, sizeof buf, "equal=%.6f rel_diff=%.3e emitters=%zu kept=%.4f", frac, rel, emitters, kept);
      Report(name, frac >= 0.9 && rel <= 0.01 && emitters > 0 && (haloThreshold > 0) == (kept < 1.0), buf);
   }
}

} // namespace

int main()
{
   std::string err;
   std::shared_ptr<iscu_sim::CudaGpuBackend> be = iscu_sim::CudaGpuBackend::Create(0, err);
   if (!be)
   {
      Report("backend", false, err);
      return 1;
   }
   Report("backend", true, be->name);
   {
      std::string info;
      std::unique_ptr<sim::SplatGpuHost> h = sim::MakeSplatGpuHost(be, info);
      Report("splat_selfcheck", h != nullptr, info);
   }
   SplatMovie(be, 0.0);
   SplatMovie(be, 1e-3);
   {
      sim::WidefieldGpuHost wf(be);
      std::string e;
      const bool ok = wf.SelfCheck(e);
      Report("widefield_selfcheck", ok, e);
   }
   std::printf("launches %llu\n", static_cast<unsigned long long>(iscu_launch_count(be->context())));
   return failures == 0 ? 0 : 1;
}
