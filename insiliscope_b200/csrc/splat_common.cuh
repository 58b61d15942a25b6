// Device pieces of the blink splat shared by the render kernels (render.cu) and the reference-record kernel
// (splat_noise.cu). Included only by units compiled with --fmad=false.
#pragma once

#include "iscu_internal.h"

#include <cstdint>

namespace iscu {

struct Kernels
{
   KernelView k[ISCU_MAX_KERNELS];
};

// The background of pixel i for a frame (RenderPhotonImage's background lambda, SMLMSimulation.cpp:124-137).
__device__ __forceinline__ float Background(const StaticView& st, uint32_t i, double bgScale)
{
   double bg = st.background ? static_cast<double>(st.background[i]) : st.flatBg;
   if (st.illum)
      bg *= static_cast<double>(st.illum[i]);
   return static_cast<float>(bg * bgScale);
}

// JS Math.round (ties toward +infinity): PsfGeneratorBridge.cpp:1245-1248.
__device__ __forceinline__ double RoundHalfUp(double v) { return floor(v + 0.5); }

__device__ __forceinline__ void CatmullRom(double f, double* w)
{
   const double f2 = f * f, f3 = f2 * f;
   w[0] = -0.5 * f3 + f2 - 0.5 * f;
   w[1] = 1.5 * f3 - 2.5 * f2 + 1.0;
   w[2] = -1.5 * f3 + 2.0 * f2 + 0.5 * f;
   w[3] = 0.5 * f3 - 0.5 * f2;
}

// One emitter's splat parameters, as SplatSetup (PsfGeneratorBridge.cpp:1382-1422) derives them.
struct StagedEmitter
{
   double photons;
   double wx[4], wy[4];
   int x0, y0, bx, by;
   int nTaps, slot, plane, pad;
};

// SplatSetup in float64 from the centre pixel (x0, y0) = (round(x), round(y)) already known.
__device__ __forceinline__ void SetupWeights(const KernelView& kv, double xPx, double yPx, StagedEmitter& s)
{
   const int os = kv.os;
   const double kc = kv.kc;
   const double tx = kc + (s.x0 - xPx - 0.5) * os + 0.5;
   const double ty = kc + (s.y0 - yPx - 0.5) * os + 0.5;
   for (int k = 0; k < 4; ++k)
   {
      s.wx[k] = k == 0 ? 1.0 : 0.0;
      s.wy[k] = k == 0 ? 1.0 : 0.0;
   }
   if (kv.interp == ISCU_INTERP_NEAREST)
   {
      s.bx = static_cast<int>(floor(tx + 0.5));
      s.by = static_cast<int>(floor(ty + 0.5));
      s.nTaps = 1;
      return;
   }
   const int bx = static_cast<int>(floor(tx)), by = static_cast<int>(floor(ty));
   const double fx = tx - bx, fy = ty - by;
   if (kv.interp == ISCU_INTERP_CUBIC)
   {
      s.bx = bx - 1;
      s.by = by - 1;
      s.nTaps = 4;
      CatmullRom(fx, s.wx);
      CatmullRom(fy, s.wy);
      return;
   }
   s.bx = bx;
   s.by = by;
   s.nTaps = 2;
   s.wx[0] = 1.0 - fx;
   s.wx[1] = fx;
   s.wy[0] = 1.0 - fy;
   s.wy[1] = fy;
}

} // namespace iscu
