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
// whose imaginary part is -(-1)^d sin(pi s) / N at t = d + s: the same magnitude at every offset. So the imaginary
// halves of both line passes collapse into one number, Z = sum of (-1)^(y + x) K[y][x] over the plane, and the shifted
// plane is two real convolutions and a rank-one term,
//   T[i][x] = sum_y Re h_y(i - y) sum_j K[y][j] Re h_x(x - j)  -  (-1)^(i + x) S_x S_y Z,   S = sin(pi s) / N,
// 2 n^3 float64 multiply-adds per emitter and no transform: a CTA per emitter holds the plane and the shifted plane in
// shared memory, evaluates Re h for the offsets of each axis once, and produces 16 output columns per pass (their
// row pass, then their column pass, each thread keeping 16 outputs along the line and a 23-value window of h in
// registers), so the intermediate is never stored whole. The shifted plane's block sums follow as BuildBlockSums
// (PsfGeneratorBridge.cpp:1021-1047) forms them: float64 row sums over each os x os block, then their sum, rounded to
// float.
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

constexpr int kThreads = 192;   // a thread per row (row pass) / per column and 16-row block (column pass)
constexpr int kCols = 16;       // output columns per pass (independent float64 chains per thread of the row pass)
constexpr int kRB = 16;         // output rows per thread of the column pass
constexpr int kMaxN = 157;      // the planes and the tables below within 227 KB of shared memory

// Re h(d + s) for the offsets d = -(n - 1) .. n + 14, at index d + n - 1 (the 15 past n - 1 are zero: the padding
// columns and rows of a pass), stored skewed -- index i in slot i + i / 8 -- so that lanes 8 indices apart read other
// banks.
__host__ __device__ constexpr int HSlot(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int HEntries(int n) { return 2 * n + (kCols > kRB ? kCols : kRB) - 2; }
__host__ __device__ constexpr int HSlots(int n) { return HSlot(HEntries(n) - 1) + 1; }
// row strides of the plane and of the row pass's columns: odd, so that lanes a row apart read other banks
__host__ __device__ constexpr int OddStride(int n) { return n | 1; }

// The shifted plane is kept as a ring of its last RingWidth(os) columns (a power of two >= kCols + os - 1: a pass's
// columns and the os - 1 before them, which its block sums read), row stride RingWidth + 1.
__host__ __device__ constexpr int RingWidth(int os)
{
   int w = 1;
   while (w < kCols + os - 1)
      w <<= 1;
   return w;
}

size_t PlaceSmem(int n, int os)
{
   const size_t ns = OddStride(n);
   return 2 * static_cast<size_t>(HSlots(n)) * sizeof(double) + static_cast<size_t>(kCols) * ns * sizeof(double) +
          (ns * n + static_cast<size_t>(n) * (RingWidth(os) + 1)) * sizeof(float);
}

__device__ void ShiftKernel(double s, int n, int N, double* h)
{
   for (int i = threadIdx.x; i < HEntries(n); i += blockDim.x)
   {
      const int d = i - (n - 1);
      double v;
      if (d > n - 1)
         v = 0.0;
      else if (s == 0.0)
         v = d == 0 ? 1.0 : 0.0;
      else
      {
         const double t = d + s, u = t / N;
         v = sinpi(t) * cospi(u) / (N * sinpi(u));
      }
      h[HSlot(i)] = v;
   }
}

__global__ void __launch_bounds__(kThreads, 2) FftPlaceKernel(const iscu_emitter* __restrict__ em,
                                                          const float* __restrict__ planes, int n, int nz, int os,
                                                          float* __restrict__ sums, int32_t* __restrict__ origins)
{
   extern __shared__ __align__(16) unsigned char smem[];
   __shared__ double warpZ[kThreads / 32];
   const int ns = OddStride(n);
   double* hx = reinterpret_cast<double*>(smem);
   double* hy = hx + HSlots(n);
   double* M = hy + HSlots(n);                                      // kCols columns of the row pass, stride ns
   float* K = reinterpret_cast<float*>(M + kCols * ns);             // the plane, row stride ns
   float* T = K + ns * n;                                           // the shifted plane's last columns (a ring)
   const int ringMask = RingWidth(os) - 1, rs = RingWidth(os) + 1;
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
   // the plane, and Z = sum over it of (-1)^(y + x) K[y][x]
   const float* P = planes + static_cast<size_t>(z) * n * n;
   double zs = 0.0;
   for (int i0 = threadIdx.x; i0 < n * n; i0 += 8 * kThreads)
   {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
         v[u] = i0 + u * kThreads < n * n ? __ldg(P + i0 + u * kThreads) : 0.f;
#pragma unroll
      for (int u = 0; u < 8; ++u)
      {
         const int i = i0 + u * kThreads;
         if (i < n * n)
         {
            const int y = i / n, x = i - y * n;
            K[y * ns + x] = v[u];
            zs += (x + y) & 1 ? -static_cast<double>(v[u]) : static_cast<double>(v[u]);
         }
      }
   }
   for (int o = 16; o; o >>= 1)
      zs += __shfl_down_sync(0xFFFFFFFFu, zs, o);
   if ((threadIdx.x & 31) == 0)
      warpZ[threadIdx.x >> 5] = zs;
   ShiftKernel(tx - rx, n, N, hx);
   ShiftKernel(ty - ry, n, N, hy);
   __syncthreads();
   double Z = 0.0;
   for (int w = 0; w < kThreads / 32; ++w)
      Z += warpZ[w];
   // Im h(d + s) = -(-1)^d sin(pi s) / N, so the imaginary halves of both passes collapse: the shifted plane is
   // T[i][x] = sum_y Re h_y(i - y) sum_j K[y][j] Re h_x(x - j)  -  (-1)^(i + x) S_x S_y Z,  S = sin(pi s) / N.
   const double corr = (sinpi(tx - rx) / N) * (sinpi(ty - ry) / N) * Z;
   const int nb8 = n & ~7;   // the steps of both passes taken eight at a time
   for (int c0 = 0; c0 < n; c0 += kCols)
   {
      // row pass for columns c0 .. c0 + 15 (a thread per row r): M[c][r] = sum_j K[r][j] Re h_x(c0 + c - j), j in
      // order. Over steps j .. j + 7 the h indices c0 + c - j' + n - 1 span 23 values: loaded once (all lanes the same).
      const int r = threadIdx.x;
      if (r < n)
      {
         double re[kCols] = {};
         const float* row = K + r * ns;
         const int base = c0 + n - 1;
         int j = 0;
         for (; j < nb8; j += 8)
         {
            double hw[kCols + 7];   // hw[t] = h index base - j - 7 + t
#pragma unroll
            for (int t = 0; t < kCols + 7; ++t)
               hw[t] = hx[HSlot(base - j - 7 + t)];
            float kv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
               kv[u] = row[j + u];
#pragma unroll
            for (int u = 0; u < 8; ++u)
            {
               const double k = kv[u];
#pragma unroll
               for (int c = 0; c < kCols; ++c)
                  re[c] = fma(k, hw[7 - u + c], re[c]);
            }
         }
         for (; j < n; ++j)
         {
            const double k = row[j];
#pragma unroll
            for (int c = 0; c < kCols; ++c)
               re[c] = fma(k, hx[HSlot(base - j + c)], re[c]);
         }
#pragma unroll
         for (int c = 0; c < kCols; ++c)
            M[c * ns + r] = re[c];
      }
      __syncthreads();
      // column pass (a thread per column c and rows i0 .. i0 + 15): T[i][c0 + c] = sum_y Re h_y(i - y) M[c][y] (y in
      // order) minus the rank-one term; over steps y .. y + 7 the h indices i - y' + n - 1 span 23 values.
      const int c = threadIdx.x & (kCols - 1), i0 = (threadIdx.x / kCols) * kRB;
      if (i0 < n)
      {
         double acc[kRB] = {};
         const double* col = M + c * ns;
         const int base = i0 + n - 1;
         int y = 0;
         for (; y < nb8; y += 8)
         {
            double hw[kRB + 7];   // hw[t] = h index base - y - 7 + t
#pragma unroll
            for (int t = 0; t < kRB + 7; ++t)
               hw[t] = hy[HSlot(base - y - 7 + t)];
#pragma unroll
            for (int u = 0; u < 8; ++u)
            {
               const double v = col[y + u];
#pragma unroll
               for (int k = 0; k < kRB; ++k)
                  acc[k] = fma(hw[7 - u + k], v, acc[k]);
            }
         }
         for (; y < n; ++y)
         {
            const double v = col[y];
#pragma unroll
            for (int k = 0; k < kRB; ++k)
               acc[k] = fma(hy[HSlot(base - y + k)], v, acc[k]);
         }
         const int x = c0 + c;
#pragma unroll
         for (int k = 0; k < kRB; ++k)
            if (i0 + k < n && x < n)
               T[(i0 + k) * rs + (x & ringMask)] = static_cast<float>(acc[k] + ((i0 + k + x) & 1 ? corr : -corr));
      }
      __syncthreads();
      // the block sums whose last column is this pass's (all the rest on the last pass), as BuildBlockSums: float64
      // row sums over the block's columns, then their sum over its rows
      const int off = os - 1;
      const int nbi = c0 + kCols >= n ? bw - c0 : kCols;
      for (int i = threadIdx.x; i < bw * nbi; i += blockDim.x)
      {
         const int ai = i / nbi, bi = c0 + (i - ai * nbi);
         const int a = ai - off, ya = max(0, a), yb = min(n - 1, a + off);
         const int b = bi - off, xa = max(0, b), xb = min(n - 1, b + off);
         double acc = 0.0;
         for (int y = ya; y <= yb; ++y)
         {
            double hsum = 0.0;
            for (int x = xa; x <= xb; ++x)
               hsum += static_cast<double>(T[y * rs + (x & ringMask)]);
            acc += hsum;
         }
         out[ai * bw + bi] = static_cast<float>(acc);
      }
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
   const size_t smem = PlaceSmem(k.size, std::max(1, k.os));
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
