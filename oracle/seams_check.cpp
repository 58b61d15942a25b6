// TEST INFRASTRUCTURE (built by oracle/Makefile into _ref/, never shipped): the render engine's own code, compiled
// from the reference's sources, with libiscu behind two of its C++ seams (include/iscu_sim_seams.hpp) on CUDA
// device 0, against the same engine without them.
//
// Checks, one output line each ("<check> ok|FAIL <figures>"), exit status 0 when all pass:
//   psfcache_<name>   iscu_sim::ComputePsfKernelCacheGpu against sim::ComputePsfKernelCache for a request (the
//                     dSTORM kernel, a double-helix one, an astigmatic one): the cache's geometry fields equal, every
//                     plane within 1e-5 of its maximum, and RenderPhotonImage (SMLMSimulation.cpp:103) of 40 blinks
//                     over 3 frames with each cache within 1e-5 of the frame maximum
//   accel_<name>      WidefieldScene (GPU mode) with iscu_sim::WidefieldAcceleratorCuda installed
//                     (SetAccelerator) against the same scene on the CPU: FocusSeries images of every focus within
//                     1e-5 of the frame maximum -- a margin, a sub-cell FOV offset, 2 cells per pixel, dye planes
//                     beyond the kernel stack; then a second series on the same scene, the plane spectra resident
#include "PsfGeneratorBridge.h"
#include "SMLMSimulation.h"
#include "WidefieldRender.h"
#include "iscu_sim_seams.hpp"

#include <algorithm>
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

// max |a - b| / max |b|; infinite when a holds a NaN or the sizes differ.
double MaxRel(const std::vector<float>& a, const std::vector<float>& b)
{
   if (a.size() != b.size())
      return HUGE_VAL;
   double m = 0.0, d = 0.0;
   for (size_t i = 0; i < a.size(); ++i)
   {
      const double e = std::fabs(static_cast<double>(a[i]) - b[i]);
      if (!(e <= d))
         d = std::isnan(e) ? HUGE_VAL : e;
      m = std::max(m, std::fabs(static_cast<double>(b[i])));
   }
   return m > 0.0 ? d / m : d;
}

sim::PsfGeneratorRequest Request(double wl, int half, int nz, double zStep, int pupil)
{
   sim::PsfGeneratorRequest q;
   q.model = sim::PsfModelKind::GibsonLanniZernike;
   q.wavelengthNm = wl;
   q.na = 1.45;
   q.immersionIndex = 1.518;
   q.sampleIndex = 1.518;
   q.pixelSizeNm = 108.0;
   q.oversampling = 4;
   q.kernelHalfWidthPx = half;
   q.nz = nz;
   q.zStepNm = zStep;
   q.pupilSamples = pupil;
   q.interpMode = sim::PsfInterpMode::Cubic;
   return q;
}

void PsfCache(iscu_ctx* ctx, const std::string& name, const sim::PsfGeneratorRequest& req)
{
   std::string err;
   sim::PsfKernelCache cpu, gpu;
   if (!sim::ComputePsfKernelCache(req, cpu, err) || !cpu.valid)
   {
      Report("psfcache_" + name, false, "reference: " + err);
      return;
   }
   if (!iscu_sim::ComputePsfKernelCacheGpu(ctx, req, gpu, err) || !gpu.valid)
   {
      Report("psfcache_" + name, false, "gpu: " + err);
      return;
   }
   const bool geom = gpu.oversampling == cpu.oversampling && gpu.halfWidthOversampled == cpu.halfWidthOversampled &&
                     gpu.sizeOversampled == cpu.sizeOversampled && gpu.nz == cpu.nz && gpu.zStepNm == cpu.zStepNm &&
                     gpu.interpMode == cpu.interpMode && gpu.blockSumWidth == cpu.blockSumWidth &&
                     gpu.Planes().size() == cpu.Planes().size();
   double planeErr = 0.0;
   for (size_t z = 0; geom && z < cpu.Planes().size(); ++z)
      planeErr = std::max(planeErr, MaxRel(gpu.Planes()[z], cpu.Planes()[z]));
   // The same blinks through the CPU splat with each cache.
   std::mt19937_64 rng(7);
   std::uniform_real_distribution<double> u(0.0, 1.0);
   const unsigned W = 64, H = 56, F = 3;
   std::vector<sim::BlinkEvent> ev(40);
   for (auto& e : ev)
   {
      e.xUm = u(rng) * W * 0.108;
      e.yUm = u(rng) * H * 0.108;
      e.zNm = (u(rng) - 0.5) * 2.0 * req.zStepNm * (req.nz / 2);
      e.tStart = u(rng) * F;
      e.tEnd = e.tStart + 0.2 + u(rng);
      e.brightness = 0.5 + u(rng);
   }
   double frameErr = 0.0;
   for (unsigned f = 0; geom && f < F; ++f)
   {
      std::vector<float> a(static_cast<size_t>(W) * H, 0.0f), b(a.size(), 0.0f);
      sim::RenderPhotonImage(a, W, H, ev, static_cast<long>(f), 108.0, 1.3, 2000.0, 20.0, 0.0, 0.0, &gpu);
      sim::RenderPhotonImage(b, W, H, ev, static_cast<long>(f), 108.0, 1.3, 2000.0, 20.0, 0.0, 0.0, &cpu);
      frameErr = std::max(frameErr, MaxRel(a, b));
   }
   char buf[160];
   std::snprintf(buf, sizeof(buf), "geometry=%d plane_rel=%.3e frame_rel=%.3e planes=%zu size=%d", geom ? 1 : 0,
                 planeErr, frameErr, cpu.Planes().size(), cpu.sizeOversampled);
   Report("psfcache_" + name, geom && planeErr <= 1e-5 && frameErr <= 1e-5, buf);
}

struct SceneCase
{
   std::string name;
   int os, upscale, half, nzk;
   double zStep, plane;
   unsigned W, H, nzd;
   double originX, originY, margin;
};

void Accel(iscu_sim::WidefieldAcceleratorCuda& accel, const SceneCase& c)
{
   using namespace sim;
   std::string err;
   PsfGeneratorRequest req = Request(520.0, c.half, c.nzk, c.zStep, 0);
   req.na = 1.4;
   req.pixelSizeNm = 100.0;
   req.oversampling = c.os;
   PsfKernelCache cache;
   if (!ComputePsfKernelCache(req, cache, err))
   {
      Report("accel_" + c.name, false, "kernel: " + err);
      return;
   }
   KernelWidefieldPsf psf(cache, c.upscale);
   WidefieldSceneSpec spec;
   spec.originXUm = c.originX;
   spec.originYUm = c.originY;
   spec.width = c.W;
   spec.height = c.H;
   spec.pixelUm = 0.1;
   spec.grid.upscale = c.upscale;
   spec.grid.zPlaneNm = c.plane;
   spec.marginUm = c.margin;
   spec.kernelCapUm = 100.0;
   spec.unitDose = 1.0;
   spec.eta = 1.0;
   spec.bleachingMask = 0;
   spec.persistentMask = 1;
   spec.focusWorldUm = 0.5 * c.plane / 1000.0;
   const FlatIllumination pattern(1e6, 1e6);
   const WidefieldGridSpec g = WidefieldScene::GridSpecFor(pattern, spec);
   WidefieldDyeGrid grid;
   grid.spec = g;
   grid.k0 = 0;
   grid.nz = c.nzd;
   grid.persistent.assign(static_cast<size_t>(c.nzd) * g.nx * g.ny, 0.0f);
   std::mt19937_64 rng(11);
   std::uniform_real_distribution<double> u(0.0, 1.0);
   double total = 0.0;
   for (float& v : grid.persistent)
      if (u(rng) < 0.05)
      {
         v = static_cast<float>(1 + static_cast<int>(u(rng) * 4));
         total += v;
      }
   grid.nPersistent = static_cast<long>(total);
   std::vector<double> foci;
   for (unsigned f = 0; f < c.nzd; ++f)
      foci.push_back((f + 0.5) * c.plane / 1000.0);
   WidefieldScene cpu, gpu;
   cpu.SetGpuMode(true);
   gpu.SetGpuMode(true);
   gpu.SetAccelerator(&accel);
   std::vector<WidefieldImages> want, got, again;
   if (!cpu.UpdateFromGrid(grid, pattern, spec, psf, err) || !gpu.UpdateFromGrid(grid, pattern, spec, psf, err) ||
       !cpu.FocusSeries(foci, want, err) || !gpu.FocusSeries(foci, got, err) || !gpu.FocusSeries(foci, again, err))
   {
      Report("accel_" + c.name, false, "scene: " + err);
      return;
   }
   const bool used = gpu.UsingAccelerator() && gpu.GpuError().empty();
   const size_t cells = static_cast<size_t>(c.W) * c.upscale * c.H * c.upscale;
   double e1 = 0.0, e2 = 0.0, wantMax = 0.0, gotMax = 0.0;
   bool sizes = true;
   for (size_t f = 0; f < foci.size(); ++f)
   {
      sizes = sizes && want[f].persistent.size() == cells && got[f].persistent.size() == cells &&
              again[f].persistent.size() == cells;
      e1 = std::max(e1, MaxRel(got[f].persistent, want[f].persistent));
      e2 = std::max(e2, MaxRel(again[f].persistent, want[f].persistent));
      for (float v : want[f].persistent)
         wantMax = std::max(wantMax, std::fabs(static_cast<double>(v)));
      for (float v : got[f].persistent)
         gotMax = std::max(gotMax, std::fabs(static_cast<double>(v)));
   }
   char buf[260];
   std::snprintf(buf, sizeof(buf), "accelerated=%d sizes=%d rel=%.3e resident_rel=%.3e want_max=%.4g got_max=%.4g "
                 "foci=%zu fft=%ux%u cells=%ux%u",
                 used ? 1 : 0, sizes ? 1 : 0, e1, e2, wantMax, gotMax, foci.size(), cpu.FftSizeX(), cpu.FftSizeY(),
                 g.nx, g.ny);
   Report("accel_" + c.name, used && sizes && wantMax > 0.0 && e1 <= 1e-5 && e2 <= 1e-5, buf);
}

} // namespace

int main()
{
   iscu_ctx* ctx = nullptr;
   if (iscu_create(0, &ctx) != ISCU_OK)
   {
      Report("context", false, iscu_last_error());
      return 1;
   }
   PsfCache(ctx, "dstorm", Request(670.0, 16, 49, 25.0, 64));
   sim::PsfGeneratorRequest dh = Request(670.0, 12, 21, 50.0, 64);
   dh.maskType = sim::PsfMaskType::DoubleHelix;
   PsfCache(ctx, "double_helix", dh);
   sim::PsfGeneratorRequest astig = Request(580.0, 10, 15, 40.0, 0);
   astig.zernikeCoefficients = "0,0,0,0.245,0,0,0,0,0,0,0,0,0,0,0";
   PsfCache(ctx, "astigmatic", astig);
   {
      iscu_sim::WidefieldAcceleratorCuda accel(ctx);
      std::string err;
      if (!accel.Ok(err))
         Report("accel", false, err);
      else
      {
         Accel(accel, {"aligned", 1, 1, 8, 9, 200.0, 200.0, 40, 32, 5, 0.05, 0.05, 0.3});
         Accel(accel, {"subcell_upscale2", 4, 2, 6, 7, 200.0, 200.0, 24, 20, 6, 0.063, 0.021, 0.4});
         Accel(accel, {"clamped_planes", 2, 2, 10, 5, 200.0, 200.0, 30, 28, 7, 0.05, 0.05, 0.0});
         Accel(accel, {"blended_planes", 1, 1, 9, 11, 150.0, 100.0, 36, 30, 6, 0.071, 0.05, 0.2});
      }
   }
   iscu_destroy(ctx);
   return failures == 0 ? 0 : 1;
}
