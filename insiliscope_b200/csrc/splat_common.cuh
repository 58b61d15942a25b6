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

// One emitter's splat parameters, as SplatSetup (PsfGeneratorBridge.cpp:1382-1422) derives them, with what the
// render's inner loop reads staged beside them.
struct StagedEmitter
{
   double photons;
   double wx[4], wy[4];
   const double* row[4];    // phase layout (fast): tap row j's words for the centre pixel
   int xb[4];               // phase layout (fast): tap column i's word offsets
   int x0, y0, camRad, nb;  // centre pixel, splat square radius, phase-layout row pitch
   const int16_t* spanLo;   // halo cut of the emitter's plane, indexed by dy + camRad; null: the whole square
   const int16_t* spanHi;
   int bx, by, plane;
   uint8_t nTaps, slot, fast, pad;   // fast: a 4 x 4 splat whose taps all lie in the phase layout
};

// Positions the splat accepts: finite and within +-1e9 pixels (beyond, the centre pixel leaves the int range).
__host__ __device__ __forceinline__ bool PositionOk(double xPx, double yPx)
{
   return fabs(xPx) < 1e9 && fabs(yPx) < 1e9;
}

// What the splat kernels read of the context's kernel slots.
inline Kernels KernelsOfCtx(iscu_ctx* ctx)
{
   Kernels K;
   for (int s = 0; s < ISCU_MAX_KERNELS; ++s)
      K.k[s] = ctx->kernels[s].valid ? ctx->kernels[s].View() : KernelView();
   return K;
}

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
