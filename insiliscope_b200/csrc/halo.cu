// The halo cut of a kernel stack, computed on the device from its resident block sums.
//
// What is computed is the reference's PsfHaloSpans (PsfGeneratorBridge.h:228-237, built by WithHaloCut,
// PsfGeneratorBridge.cpp:1137-1243): per plane z and camera-pixel row dy of a splat, the first and last camera column
// dx whose pixel can receive at least `threshold` of the emitter's photons, and per plane the largest dx^2 + dy^2
// kept. A splat pixel (dy, dx) reads block sums in rows [halfOv - 2 + dy os, halfOv + os + 1 + dy os] and the same
// span of columns for dx (every sub-pixel offset and interpolation: SplatSetup keeps the tap origin within
// [kc - os - 1, kc]), clipped to the bw x bw array; the pixel is kept when the largest of those sums, widened to
// double, reaches threshold / overshoot (1.5625 for Catmull-Rom weights, whose absolute sum per axis reaches 1.25).
//
// Layout of the work: one warp per (plane, dy) row; lane l tests the pixels dx = -camRad + l + 32 j, each taking the
// max over its (os + 4)^2 window of sums straight from L2 (a C0 stack is 3.4 MB); a ballot per 32 pixels gives the
// row's first and last kept column; lane 0 writes them and folds the row's reach into the plane's radius2 with an
// atomic max. Max and compare are exact, so the spans equal the reference's bit for bit.

#include "iscu_internal.h"

#include <climits>

namespace iscu {
namespace {

__global__ void HaloSpansKernel(const float* __restrict__ sums, int nz, int bw, int os, int halfOv, int camRad,
                                double thr, int16_t* __restrict__ lo, int16_t* __restrict__ hi,
                                int32_t* __restrict__ radius2)
{
   const int n = 2 * camRad + 1;
   const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
   if (row >= nz * n)
      return;   // whole warps leave together: a row is a warp
   const int lane = threadIdx.x & 31;
   const int z = row / n, dy = row % n - camRad;
   const float* B = sums + static_cast<size_t>(z) * bw * bw;
   const int r0 = max(0, halfOv - 2 + dy * os), r1 = min(bw - 1, halfOv + os + 1 + dy * os);
   int first = INT_MAX, last = INT_MIN;
   for (int base = -camRad; base <= camRad; base += 32)
   {
      const int dx = base + lane;
      bool keep = false;
      if (dx <= camRad)
      {
         const int c0 = max(0, halfOv - 2 + dx * os), c1 = min(bw - 1, halfOv + os + 1 + dx * os);
         float m = 0.0f;
         for (int r = r0; r <= r1; ++r)
         {
            const float* Br = B + static_cast<size_t>(r) * bw;
            for (int c = c0; c <= c1; ++c)
               m = fmaxf(m, __ldg(Br + c));
         }
         keep = static_cast<double>(m) >= thr;
      }
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      if (mask)
      {
         first = min(first, base + __ffs(mask) - 1);
         last = max(last, base + 31 - __clz(mask));
      }
   }
   if (lane == 0)
   {
      // an empty row: lo = camRad + 1 > hi = -camRad - 1, as PsfHaloSpans marks it
      const int l = first == INT_MAX ? camRad + 1 : first;
      const int h = last == INT_MIN ? -camRad - 1 : last;
      lo[row] = static_cast<int16_t>(l);
      hi[row] = static_cast<int16_t>(h);
      if (l <= h)
         atomicMax(radius2 + z, dy * dy + max(l * l, h * h));
   }
}

} // namespace

int BuildHalo(iscu_ctx* ctx, KernelSlot& k, double threshold)
{
   k.halo = false;
   k.haloThreshold = 0.0;
   const int camRad = k.halfOv / k.os;
   // No cut (the whole square) for threshold <= 0 or a half width outside [1, 16000] camera pixels, as WithHaloCut.
   if (!(threshold > 0.0) || camRad < 1 || camRad > 16000)
      return ISCU_OK;
   const int n = 2 * camRad + 1;
   const size_t rows = static_cast<size_t>(n) * k.nz;
   ISCU_CK(k.spanLo.Reserve(rows * sizeof(int16_t)));
   ISCU_CK(k.spanHi.Reserve(rows * sizeof(int16_t)));
   ISCU_CK(k.radius2.Reserve(static_cast<size_t>(k.nz) * sizeof(int32_t)));
   ISCU_CK(cudaMemsetAsync(k.radius2.p, 0xff, static_cast<size_t>(k.nz) * sizeof(int32_t), ctx->stream));   // -1
   const double overshoot = k.interp == ISCU_INTERP_CUBIC ? 1.5625 : 1.0;
   constexpr int kWarps = 8;
   const unsigned blocks = static_cast<unsigned>((rows + kWarps - 1) / kWarps);
   HaloSpansKernel<<<blocks, kWarps * 32, 0, ctx->stream>>>(k.sums.as<float>(), k.nz, k.bw, k.os, k.halfOv, camRad,
                                                           threshold / overshoot, k.spanLo.as<int16_t>(),
                                                           k.spanHi.as<int16_t>(), k.radius2.as<int32_t>());
   ISCU_CK_LAUNCH(ctx, "HaloSpansKernel");
   // the per-plane reach stays on the host too: the binned renderer sizes its kernels from it
   k.radius2Host.assign(static_cast<size_t>(k.nz), -1);
   ISCU_CK(cudaMemcpyAsync(k.radius2Host.data(), k.radius2.p, k.radius2Host.size() * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   k.halo = true;
   k.haloThreshold = threshold;
   return ISCU_OK;
}

int GetHaloSpans(iscu_ctx* ctx, const KernelSlot& k, int16_t* lo, int16_t* hi, int32_t* radius2)
{
   const size_t rows = static_cast<size_t>(2 * (k.halfOv / k.os) + 1) * k.nz;
   ISCU_CK(cudaMemcpyAsync(lo, k.spanLo.p, rows * sizeof(int16_t), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(hi, k.spanHi.p, rows * sizeof(int16_t), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(radius2, k.radius2.p, static_cast<size_t>(k.nz) * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

} // namespace iscu
