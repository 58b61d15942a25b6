// The splat's Fft placement on sm_100a (PlanSplat with PsfInterpMode::Fft, adapter/inSiliScope/Simulation/
// PsfGeneratorBridge.cpp:1441-1456, and FftShiftKernelTile, :1293-1370), which the reference runs on the CPU only: per
// emitter, the kernel plane shifted by the emitter's sub-cell offset and that plane's block sums, which the splat then
// reads at one tap.
//
// The reference shifts each row of the n x n plane, zero-padded to N (the power of two >= 2n), by FFT, a phase
// exp(2 pi i kk s / N) over the wrapped frequencies kk = -N/2 .. N/2 - 1, inverse FFT over N, and keeps the first n
// (complex) values; then the same along the columns; the real part is the shifted plane. That line operation is a
// convolution: y[i] = sum_j x[j] h(i - j + s) with h(t) = (1/N) sum_kk exp(2 pi i kk t / N), whose geometric sum is
//   h(t) = sin(pi t) / (N tan(pi t / N)) - i sin(pi t) / N        (t not an integer;  h(d) = [d == 0] for integers),
// so each emitter is 2 n^3 complex multiply-adds in float64 with no transform: a CTA per emitter holds the plane and
// the shifted plane in shared memory, evaluates h for the 2n - 1 offsets of each axis once, and produces eight output
// columns per pass (each a row pass for those columns, then their column pass), so the complex intermediate is never
// stored whole. The shifted plane's block sums follow as BuildBlockSums (PsfGeneratorBridge.cpp:1021-1047) forms
// them: float64 row sums over each os x os block, then their sum, rounded to float.
//
// Frames in the Fft placement (RenderPhotonImage with a kernel whose interpolation is Fft, SMLMSimulation.cpp:103-160,
// SplatRows / SplatKernel.inl with one tap): a CTA per 16 x 16 pixels of a frame starts each pixel at its background,
// stages the frame's emitters whose square reaches the tile (in list order, 256 at a time) and adds, per pixel in
// that order, float(photons x the emitter's shifted sums at (by + dy os + os - 1, bx + dx os + os - 1)) where the
// pixel lies in the square and the halo cut's span; then the photon frame and/or the noise chain. Compiled with
// --fmad=false for the noise chain's exactness (the shift's explicit fma calls are unaffected).

#include "iscu_internal.h"
#include "noise_chain.cuh"
#include "splat_common.cuh"

#include <climits>

namespace iscu {
namespace {

constexpr int kThreads = 192;   // one thread per row / output index
constexpr int kCols = 8;        // output columns per pass (independent float64 chains per thread)
constexpr int kMaxN = 157;     // 2 n^2 floats + (12 n - 2) complex doubles within 227 KB of shared memory

size_t PlaceSmem(int n)
{
   return 2 * static_cast<size_t>(n) * n * sizeof(float) + 2 * (2 * static_cast<size_t>(n) - 1) * sizeof(double2) +
          static_cast<size_t>(kCols) * n * sizeof(double2);
}

// h(d + s) for the 2n - 1 offsets d = -(n - 1) .. n - 1, into h[d + n - 1].
__device__ void ShiftKernel(double s, int n, int N, double2* h)
{
   for (int i = threadIdx.x; i < 2 * n - 1; i += blockDim.x)
   {
      const int d = i - (n - 1);
      if (s == 0.0)
      {
         h[i] = make_double2(d == 0 ? 1.0 : 0.0, 0.0);
         continue;
      }
      const double t = d + s, sp = sinpi(t), u = t / N;
      h[i] = make_double2(sp * cospi(u) / (N * sinpi(u)), -sp / N);
   }
}

__global__ void __launch_bounds__(kThreads) FftPlaceKernel(const iscu_emitter* __restrict__ em,
                                                          const float* __restrict__ planes, int n, int nz, int os,
                                                          float* __restrict__ sums, int32_t* __restrict__ origins)
{
   extern __shared__ __align__(16) unsigned char smem[];
   double2* hx = reinterpret_cast<double2*>(smem);
   double2* hy = hx + (2 * n - 1);
   double2* M = hy + (2 * n - 1);                                   // kCols columns of the row pass, n each
   float* K = reinterpret_cast<float*>(M + kCols * n);              // the plane
   float* T = K + n * n;                                            // the shifted plane
   const int bw = n + os - 1;
   const iscu_emitter m = em[blockIdx.x];
   float* out = sums + static_cast<size_t>(blockIdx.x) * bw * bw;
   const int z = m.plane & 0xFFFF;
   const bool ok = m.photons > 0.0 && z < nz && fabs(m.x_px) < 1e9 && fabs(m.y_px) < 1e9;
   if (!ok)   // PlanSplat refuses: nothing to draw
   {
      for (int i = threadIdx.x; i < bw * bw; i += blockDim.x)
         out[i] = 0.f;
      if (threadIdx.x == 0)
      {
         origins[4 * blockIdx.x] = INT32_MIN;
         origins[4 * blockIdx.x + 1] = origins[4 * blockIdx.x + 2] = origins[4 * blockIdx.x + 3] = 0;
      }
      return;
   }
   // SplatSetup's nearest placement, then the sub-cell remainder as the shift (PsfGeneratorBridge.cpp:1446-1450)
   const double kc = (n - 1) / 2.0;
   const int x0 = static_cast<int>(floor(m.x_px + 0.5)), y0 = static_cast<int>(floor(m.y_px + 0.5));
   const double tx = kc + (x0 - m.x_px - 0.5) * os + 0.5, ty = kc + (y0 - m.y_px - 0.5) * os + 0.5;
   const double rx = floor(tx + 0.5), ry = floor(ty + 0.5);
   int N = 1;
   while (N < 2 * n)
      N <<= 1;
   const float* P = planes + static_cast<size_t>(z) * n * n;
   for (int i = threadIdx.x; i < n * n; i += blockDim.x)
      K[i] = P[i];
   ShiftKernel(tx - rx, n, N, hx);
   ShiftKernel(ty - ry, n, N, hy);
   __syncthreads();
   const int r = threadIdx.x;
   for (int c0 = 0; c0 < n; c0 += kCols)
   {
      // row pass for columns c0 .. c0 + 7: M[c][y] = sum_j K[y][j] h_x(c0 + c - j)
      if (r < n)
      {
         double re[kCols] = {}, im[kCols] = {};
         const float* row = K + r * n;
         for (int j = 0; j < n; ++j)
         {
            const double k = row[j];
#pragma unroll
            for (int c = 0; c < kCols; ++c)
            {
               const int x = c0 + c;
               const double2 h = hx[min(x, n - 1) - j + n - 1];
               re[c] = fma(k, h.x, re[c]);
               im[c] = fma(k, h.y, im[c]);
            }
         }
#pragma unroll
         for (int c = 0; c < kCols; ++c)
            M[c * n + r] = make_double2(re[c], im[c]);
      }
      __syncthreads();
      // column pass: T[i][x] = Re sum_y h_y(i - y) M[x][y]
      if (r < n)
      {
         double acc[kCols] = {};
         for (int y = 0; y < n; ++y)
         {
            const double2 h = hy[r - y + n - 1];
#pragma unroll
            for (int c = 0; c < kCols; ++c)
            {
               const double2 v = M[c * n + y];
               acc[c] = fma(h.x, v.x, acc[c]);
               acc[c] = fma(-h.y, v.y, acc[c]);
            }
         }
#pragma unroll
         for (int c = 0; c < kCols; ++c)
            if (c0 + c < n)
               T[r * n + c0 + c] = static_cast<float>(acc[c]);
      }
      __syncthreads();
   }
   // block sums of the shifted plane
   const int off = os - 1;
   for (int i = threadIdx.x; i < bw * bw; i += blockDim.x)
   {
      const int ai = i / bw, bi = i - ai * bw;
      const int a = ai - off, ya = max(0, a), yb = min(n - 1, a + off);
      const int b = bi - off, xa = max(0, b), xb = min(n - 1, b + off);
      double acc = 0.0;
      for (int y = ya; y <= yb; ++y)
      {
         double hsum = 0.0;
         for (int x = xa; x <= xb; ++x)
            hsum += static_cast<double>(T[y * n + x]);
         acc += hsum;
      }
      out[i] = static_cast<float>(acc);
   }
   if (threadIdx.x == 0)
   {
      origins[4 * blockIdx.x] = x0;
      origins[4 * blockIdx.x + 1] = y0;
      origins[4 * blockIdx.x + 2] = static_cast<int32_t>(rx);
      origins[4 * blockIdx.x + 3] = static_cast<int32_t>(ry);
   }
}

constexpr int kTile = 16;   // render: 16 x 16 pixels, one thread each

struct FftStaged
{
   double photons;
   const float* sums;   // the emitter's shifted block sums
   const int16_t* spanLo;
   const int16_t* spanHi;
   int x0, y0, bx, by;
};

// grid (ceil(W / 16), ceil(H / 16), frames). Frame k's emitters are ems[em_start, + em_count) cut at nEm; emitter e's
// placement is sums[e * bw * bw ..] and origins[4e ..] (x0 = INT32_MIN: not drawn).
__global__ void __launch_bounds__(kTile * kTile) RenderFftKernel(const iscu_emitter* __restrict__ ems, uint32_t nEm,
                                                                const iscu_frame* __restrict__ frames,
                                                                const float* __restrict__ sums,
                                                                const int32_t* __restrict__ origins, KernelView kv,
                                                                StaticView st, CameraView cam, int noise,
                                                                uint32_t seed, float* __restrict__ photonsOut,
                                                                uint16_t* __restrict__ aduOut)
{
   __shared__ FftStaged sEm[kTile * kTile];
   __shared__ int sWarp[kTile * kTile / 32];
   const int W = static_cast<int>(st.width), H = static_cast<int>(st.height);
   const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
   const int X = tx0 + (threadIdx.x & (kTile - 1)), Y = ty0 + (threadIdx.x >> 4);
   const int tx1 = min(tx0 + kTile, W) - 1, ty1 = min(ty0 + kTile, H) - 1;
   const bool inside = X < W && Y < H;
   const uint32_t i = static_cast<uint32_t>(Y) * st.width + static_cast<uint32_t>(X);
   const iscu_frame fr = frames[blockIdx.z];
   const int os = kv.os, off = os - 1, bw = kv.bw, cr = kv.camRad, sq = 2 * cr + 1;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   float acc = inside ? Background(st, i, fr.bg_scale) : 0.0f;
   const uint32_t count = fr.em_start < nEm ? min(fr.em_count, nEm - fr.em_start) : 0u;
   for (uint32_t e0 = 0; e0 < count; e0 += kTile * kTile)
   {
      FftStaged s;
      bool keep = false;
      const uint32_t e = fr.em_start + e0 + threadIdx.x;
      if (e0 + threadIdx.x < count)
      {
         const int x0 = origins[4 * e];
         if (x0 != INT32_MIN)
         {
            s.x0 = x0;
            s.y0 = origins[4 * e + 1];
            keep = s.x0 + cr >= tx0 && s.x0 - cr <= tx1 && s.y0 + cr >= ty0 && s.y0 - cr <= ty1;
            s.bx = origins[4 * e + 2];
            s.by = origins[4 * e + 3];
            s.photons = ems[e].photons;
            s.sums = sums + static_cast<size_t>(e) * bw * bw;
            const int plane = ems[e].plane & 0xFFFF;
            s.spanLo = kv.spanLo ? kv.spanLo + plane * sq : nullptr;
            s.spanHi = kv.spanHi ? kv.spanHi + plane * sq : nullptr;
         }
      }
      const unsigned ballot = __ballot_sync(0xFFFFFFFFu, keep);
      if (lane == 0)
         sWarp[warp] = __popc(ballot);
      __syncthreads();
      int base = 0, total = 0;
#pragma unroll
      for (int w = 0; w < kTile * kTile / 32; ++w)
      {
         base += w < warp ? sWarp[w] : 0;
         total += sWarp[w];
      }
      if (keep)
         sEm[base + __popc(ballot & ((1u << lane) - 1u))] = s;
      __syncthreads();
      if (inside)
         for (int k = 0; k < total; ++k)
         {
            const FftStaged& t = sEm[k];
            const int dx = X - t.x0, dy = Y - t.y0;
            if (dx < -cr || dx > cr || dy < -cr || dy > cr)
               continue;
            if (t.spanLo && (dx < t.spanLo[dy + cr] || dx > t.spanHi[dy + cr]))
               continue;
            const int r0 = t.by + dy * os + off, c0 = t.bx + dx * os + off;
            // one tap (weights 1): the sums value, or nothing outside the array (the reference's skipped tap)
            const double sum = r0 >= 0 && r0 < bw && c0 >= 0 && c0 < bw
                                  ? 1.0 * (1.0 * static_cast<double>(__ldg(t.sums + r0 * bw + c0)))
                                  : 0.0;
            acc += static_cast<float>(t.photons * sum);
         }
      __syncthreads();
   }
   if (!inside)
      return;
   const size_t o = static_cast<size_t>(blockIdx.z) * st.width * st.height + i;
   if (photonsOut)
      photonsOut[o] = acc;
   if (noise)
   {
      CounterRng u(seed, fr.frame);
      aduOut[o] = NoisePixel(acc, i, cam, st, u);
   }
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_fft_place_dev(iscu_ctx* ctx, int32_t slot, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                       float* sums_dev, int32_t* origins_dev)
{
   if (!ctx || (n_emitters && (!emitters_dev || !sums_dev || !origins_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (slot < 0 || slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (0..3)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const KernelSlot& k = ctx->kernels[slot];
   if (!k.valid)
      return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
   if (k.size > kMaxN)
      return Fail(ISCU_ERR_LIMIT, "the Fft placement takes planes of up to 157 x 157 samples");
   if (!n_emitters)
      return ISCU_OK;
   if (n_emitters > 0x7FFFFFFFu)
      return Fail(ISCU_ERR_LIMIT, "too many emitters per call");
   const size_t smem = PlaceSmem(k.size);
   ISCU_CK(cudaFuncSetAttribute(FftPlaceKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
   FftPlaceKernel<<<n_emitters, kThreads, smem, ctx->stream>>>(emitters_dev, k.planes.as<float>(), k.size, k.nz,
                                                               std::max(1, k.os), sums_dev, origins_dev);
   ISCU_CK_LAUNCH(ctx, "FftPlaceKernel");
   return ISCU_OK;
}

int iscu_render_fft_frames_dev(iscu_ctx* ctx, int32_t slot, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                               const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                               float* photons_dev, uint16_t* adu_dev)
{
   if (!ctx || (n_emitters && !emitters_dev) || (n_frames && !frames_dev) || (cam && !adu_dev) ||
       (!cam && !photons_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (slot < 0 || slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (0..3)");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   const KernelSlot& k = ctx->kernels[slot];
   if (!k.valid)
      return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
   if (!n_frames)
      return ISCU_OK;
   const size_t bw = static_cast<size_t>(k.bw), per = bw * bw * sizeof(float);
   if (static_cast<size_t>(n_emitters) * per > (size_t(16) << 30))
      return Fail(ISCU_ERR_LIMIT, "the batch's shifted block sums pass 16 GB: split the frames");
   ISCU_CK(ctx->dFftPlace.Reserve(std::max<size_t>(1, n_emitters) * (per + 16)));
   float* sums = ctx->dFftPlace.as<float>();
   int32_t* origins = reinterpret_cast<int32_t*>(ctx->dFftPlace.as<char>() + static_cast<size_t>(n_emitters) * per);
   int rc = iscu_fft_place_dev(ctx, slot, emitters_dev, n_emitters, sums, origins);
   if (rc != ISCU_OK)
      return rc;
   StaticView st = ctx->Static();
   const CameraView cv = cam ? MakeCameraView(*cam) : CameraView();
   const dim3 grid((st.width + kTile - 1) / kTile, (st.height + kTile - 1) / kTile, n_frames);
   RenderFftKernel<<<grid, kTile * kTile, 0, ctx->stream>>>(emitters_dev, n_emitters, frames_dev, sums, origins,
                                                            k.View(), st, cv, cam ? 1 : 0, seed, photons_dev,
                                                            adu_dev);
   ISCU_CK_LAUNCH(ctx, "RenderFftKernel");
   return ISCU_OK;
}

} // extern "C"
