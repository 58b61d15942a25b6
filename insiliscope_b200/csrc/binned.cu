// The binned blink regime on sm_100a (sim::BinnedBlinkRenderer, adapter/inSiliScope/Simulation/BinnedBlinks.h:35-60,
// BinnedBlinks.cpp:150-248): the approximate SMLM render of dense frames.
//
// A frame's emitters (the splat's: photons, position, z plane) are deposited at the nearest cell of a grid of u cells
// per camera pixel, one density per PSF plane, and each plane is convolved with that plane's kernel resampled to the
// cell pitch; the planes' images are summed, clamped at 0 per cell and summed u x u into camera pixels.
// The reference convolves by float FFTs over a grid padded by the kernel radius R (no wrap-around into the frame):
// that is the linear convolution, which this file computes directly -- every cell sums float(photons) x kernel over
// the emitters within R cells, in float64 -- so the result is the FFT's up to its float rounding.
//
// Setup (BinnedBlinkRenderer::Setup, BinnedBlinks.cpp:150-214): u = KernelWidefieldPsf::ValidUpscale (the largest
// divisor of the kernel's oversampling up to the request, WidefieldRender.cpp:262-269); the plane kernels are
// KernelWidefieldPsf::Kernel (WidefieldRender.cpp:300-322), float64 r x r block sums (r = os / u) of the oversampled
// planes; R = KernelWidefieldPsf::Radius (:288-298) capped by the halo cut; or, without a kernel, the normalized
// Gaussian of sigma_px u (BinnedBlinks.cpp:190-212), made on the host with the same std::exp calls.
//
// Render (BinnedBlinks.cpp:216-246), one CTA per 16 x 16 pixels of one frame, one thread per pixel holding its u x u
// cells: the frame's emitters are examined 256 at a time, those whose cell lies in the padded grid and within R of
// the tile staged in shared memory in event order, and every thread adds each staged emitter to its cells.

#include "iscu_internal.h"

#include <algorithm>
#include <cmath>
#include <vector>

struct iscu_binned
{
   iscu_ctx* ctx = nullptr;
   uint32_t W = 0, H = 0;
   int u = 1, R = 1, nz = 1;
   iscu::DevBuf kernels;   // nz x (2R + 1)^2 floats
};

namespace iscu {
namespace {

constexpr int kThreads = 256;   // 16 x 16 pixels per CTA
constexpr int kSide = 16;

// KernelWidefieldPsf::Kernel: cell (dx, dy) of plane p = the sum, in float64 and row order, of the oversampled plane
// over [s0 + dy r, +r) x [s0 + dx r, +r) clipped to the plane, rounded to float.
__global__ void CellKernelsKernel(const float* __restrict__ planes, int n, int nz, int r, int s0, int R,
                                  float* __restrict__ out)
{
   const int D = 2 * R + 1, i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= nz * D * D)
      return;
   const int p = i / (D * D), c = i - p * D * D, dy = c / D - R, dx = c % D - R;
   const float* P = planes + static_cast<size_t>(p) * n * n;
   const int ya = s0 + dy * r, yb = min(n, ya + r), xa = s0 + dx * r, xb = min(n, xa + r);
   double acc = 0.0;
   for (int y = max(0, ya); y < yb; ++y)
      for (int x = max(0, xa); x < xb; ++x)
         acc += P[static_cast<size_t>(y) * n + x];
   out[i] = static_cast<float>(acc);
}

} // namespace

int LaunchCellKernels(iscu_ctx* ctx, const float* planes, int n, int nz, int r, int s0, int R, float* out)
{
   const int D = 2 * R + 1, total = nz * D * D;
   CellKernelsKernel<<<(total + 255) / 256, 256, 0, ctx->stream>>>(planes, n, nz, r, s0, R, out);
   ISCU_CK_LAUNCH(ctx, "CellKernelsKernel");
   return ISCU_OK;
}

namespace {

struct Staged
{
   int cx, cy;   // the emitter's cell (unpadded grid)
   float photons;
   int plane;
};

// grid (ceil(W / 16), ceil(H / 16), frames). Frame k's emitters are emitters[em_start, em_start + em_count) cut at
// nEm. img / alone: frames x H x W, +=.
template <int U>
__global__ void __launch_bounds__(kThreads) BinnedRenderKernel(const iscu_emitter* __restrict__ em, uint32_t nEm,
                                                              const iscu_frame* __restrict__ frames,
                                                              const float* __restrict__ K, int nz, int R, uint32_t W,
                                                              uint32_t H, float* __restrict__ img,
                                                              float* __restrict__ alone)
{
   __shared__ Staged st[kThreads];
   __shared__ int warpKept[kThreads / 32];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int px = blockIdx.x * kSide + (threadIdx.x & (kSide - 1)), py = blockIdx.y * kSide + (threadIdx.x >> 4);
   const int gw = static_cast<int>(W) * U, gh = static_cast<int>(H) * U, D = 2 * R + 1;
   // the tile's cells, and the cells whose emitters reach them
   const int tx0 = blockIdx.x * kSide * U, ty0 = blockIdx.y * kSide * U;
   const int reachX0 = max(-R, tx0 - R), reachX1 = min(gw + R - 1, tx0 + kSide * U - 1 + R);
   const int reachY0 = max(-R, ty0 - R), reachY1 = min(gh + R - 1, ty0 + kSide * U - 1 + R);
   const iscu_frame fr = frames[blockIdx.z];
   const uint32_t start = min(fr.em_start, nEm), end = min(start + fr.em_count, nEm);
   const int cx = px * U, cy = py * U;   // this pixel's first cell
   double acc[U][U];
#pragma unroll
   for (int j = 0; j < U; ++j)
#pragma unroll
      for (int i = 0; i < U; ++i)
         acc[j][i] = 0.0;
   for (uint32_t base = start; base < end; base += kThreads)
   {
      Staged s{0, 0, 0.f, 0};
      bool keep = false;
      const uint32_t e = base + threadIdx.x;
      if (e < end)
      {
         const iscu_emitter m = em[e];
         if (m.photons > 0.0 && fabs(m.x_px) < 1e9 && fabs(m.y_px) < 1e9)
         {
            // pixel x spans [x - 0.5, x + 0.5): cell floor((x + 0.5) u)
            s.cx = static_cast<int>(floor((m.x_px + 0.5) * U));
            s.cy = static_cast<int>(floor((m.y_px + 0.5) * U));
            keep = s.cx >= reachX0 && s.cx <= reachX1 && s.cy >= reachY0 && s.cy <= reachY1;
            s.photons = static_cast<float>(m.photons);
            s.plane = min(nz - 1, max(0, m.plane & 0xFFFF));
         }
      }
      // staged in event order: the warps' kept counts, then each lane's rank in its warp
      const unsigned ballot = __ballot_sync(0xFFFFFFFFu, keep);
      if (lane == 0)
         warpKept[warp] = __popc(ballot);
      __syncthreads();
      int offset = 0, total = 0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w)
      {
         offset += w < warp ? warpKept[w] : 0;
         total += warpKept[w];
      }
      if (keep)
         st[offset + __popc(ballot & ((1u << lane) - 1u))] = s;
      __syncthreads();
      for (int k = 0; k < total; ++k)
      {
         const Staged t = st[k];
         const int dx0 = cx - t.cx, dy0 = cy - t.cy;
         if (dx0 > R || dx0 + U - 1 < -R || dy0 > R || dy0 + U - 1 < -R)
            continue;
         const float* Kp = K + t.plane * D * D;
         const double ph = t.photons;
         if (dx0 >= -R && dx0 + U - 1 <= R && dy0 >= -R && dy0 + U - 1 <= R)
         {
            // every cell of the pixel in reach (the common case): no per-cell test
            const float* Kc = Kp + (dy0 + R) * D + (dx0 + R);
#pragma unroll
            for (int j = 0; j < U; ++j)
#pragma unroll
               for (int i = 0; i < U; ++i)
                  acc[j][i] += ph * static_cast<double>(__ldg(Kc + j * D + i));
            continue;
         }
#pragma unroll
         for (int j = 0; j < U; ++j)
         {
            const int dy = dy0 + j;
            if (dy < -R || dy > R)
               continue;
#pragma unroll
            for (int i = 0; i < U; ++i)
            {
               const int dx = dx0 + i;
               if (dx >= -R && dx <= R)
                  acc[j][i] += ph * static_cast<double>(__ldg(Kp + (dy + R) * D + (dx + R)));
            }
         }
      }
      __syncthreads();   // the staging area is rewritten next round
   }
   if (px >= static_cast<int>(W) || py >= static_cast<int>(H))
      return;
   // a cell is the float image's value, clamped at 0; the pixel sums its cells in float64, rows first
   double sum = 0.0;
#pragma unroll
   for (int j = 0; j < U; ++j)
#pragma unroll
      for (int i = 0; i < U; ++i)
      {
         const float v = static_cast<float>(acc[j][i]);
         sum += v > 0.f ? v : 0.f;
      }
   const size_t o = (static_cast<size_t>(blockIdx.z) * H + py) * W + px;
   img[o] += static_cast<float>(sum);
   if (alone)
      alone[o] += static_cast<float>(sum);
}

// KernelWidefieldPsf::ValidUpscale (WidefieldRender.cpp:262-269).
int ValidUpscale(int oversampling, int requested)
{
   const int os = std::max(1, oversampling);
   for (int u = std::max(1, std::min(requested, os)); u > 1; --u)
      if (os % u == 0)
         return u;
   return 1;
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_binned_create(iscu_ctx* ctx, int32_t slot, double sigma_px, uint32_t width, uint32_t height, int32_t upscale,
                       iscu_binned** out)
{
   if (!ctx || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   if (width == 0 || height == 0)
      return Fail(ISCU_ERR_ARG, "binned render: width and height >= 1");
   if (slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (-1..3)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   std::unique_ptr<iscu_binned> b(new iscu_binned());
   b->ctx = ctx;
   b->W = width;
   b->H = height;
   if (slot >= 0)
   {
      const KernelSlot& k = ctx->kernels[slot];
      if (!k.valid)
         return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
      const int os = std::max(1, k.os), n = k.size;
      b->u = ValidUpscale(os, upscale);
      // KernelWidefieldPsf: blocks of r oversampled samples per cell, the cell at offset 0 from s0 (a dye at a cell
      // centre, as SplatSetup places it: tx = kc - r/2 + 0.5 rounded half up)
      const int r = std::max(1, os / b->u);
      const double kc = (n - 1) / 2.0;
      const int s0 = static_cast<int>(std::floor(kc - r / 2.0 + 1.0));
      const int dMin = static_cast<int>(std::ceil((-s0 - r + 1) / static_cast<double>(r)));
      const int dMax = static_cast<int>(std::floor((n - 1 - s0) / static_cast<double>(r)));
      b->R = std::max(1, std::max(-dMin, dMax));
      // the halo cut bounds what the splat draws; the cell kernel stops there too
      if (k.halo && !k.radius2Host.empty())
      {
         const int32_t r2 = *std::max_element(k.radius2Host.begin(), k.radius2Host.end());
         if (r2 >= 0)
            b->R = std::min(b->R, static_cast<int>(std::ceil((std::sqrt(static_cast<double>(r2)) + 1.0) * b->u)));
      }
      b->R = std::max(1, b->R);
      b->nz = std::max(1, k.nz);
      const int D = 2 * b->R + 1;
      ISCU_CK(b->kernels.Reserve(static_cast<size_t>(b->nz) * D * D * sizeof(float)));
      const int total = b->nz * D * D;
      CellKernelsKernel<<<(total + 255) / 256, 256, 0, ctx->stream>>>(k.planes.as<float>(), n, b->nz, r, s0, b->R,
                                                                        b->kernels.as<float>());
      ISCU_CK_LAUNCH(ctx, "CellKernelsKernel");
   }
   else
   {
      if (!(sigma_px > 0.0))
         return Fail(ISCU_ERR_ARG, "binned render: no kernel slot and no Gaussian sigma");
      b->u = std::max(1, std::min(upscale, 8));
      b->R = std::max(1, static_cast<int>(std::ceil(3.0 * sigma_px * b->u)));
      b->nz = 1;
      const int R = b->R, D = 2 * R + 1;
      const double sc = sigma_px * b->u, twoS2 = 2.0 * sc * sc;
      std::vector<double> g(static_cast<size_t>(D) * D);
      double sum = 0.0;
      for (int y = -R; y <= R; ++y)
         for (int x = -R; x <= R; ++x)
         {
            const double v = std::exp(-(static_cast<double>(x) * x + static_cast<double>(y) * y) / twoS2);
            g[static_cast<size_t>(y + R) * D + (x + R)] = v;
            sum += v;
         }
      std::vector<float> gf(g.size());
      for (size_t i = 0; i < g.size(); ++i)
         gf[i] = static_cast<float>(g[i] / sum);
      ISCU_CK(b->kernels.Reserve(gf.size() * sizeof(float)));
      ISCU_CK(cudaMemcpyAsync(b->kernels.p, gf.data(), gf.size() * sizeof(float), cudaMemcpyHostToDevice,
                              ctx->stream));
   }
   if (b->u > 8)
      return Fail(ISCU_ERR_LIMIT, "binned render: at most 8 cells per pixel");
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   *out = b.release();
   return ISCU_OK;
}

int iscu_binned_info(iscu_binned* b, int32_t* upscale, int32_t* radius_cells, int32_t* planes)
{
   if (!b)
      return Fail(ISCU_ERR_ARG, "null renderer");
   if (upscale)
      *upscale = b->u;
   if (radius_cells)
      *radius_cells = b->R;
   if (planes)
      *planes = b->nz;
   return ISCU_OK;
}

int iscu_binned_kernels(iscu_binned* b, float* out)
{
   if (!b || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
   ClearError();
   const size_t D = 2 * static_cast<size_t>(b->R) + 1;
   ISCU_CK(cudaMemcpyAsync(out, b->kernels.p, b->nz * D * D * sizeof(float), cudaMemcpyDeviceToHost,
                           b->ctx->stream));
   ISCU_CK(cudaStreamSynchronize(b->ctx->stream));
   return ISCU_OK;
}

void iscu_binned_destroy(iscu_binned* b)
{
   if (!b)
      return;
   cudaStreamSynchronize(b->ctx->stream);
   delete b;
}

int iscu_binned_render_dev(iscu_binned* b, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                           const iscu_frame* frames_dev, uint32_t n_frames, float* img_dev, float* alone_dev)
{
   if (!b || (n_frames && (!frames_dev || !img_dev)) || (n_emitters && !emitters_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   iscu_ctx* ctx = b->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (!n_frames)
      return ISCU_OK;
   const dim3 grid((b->W + kSide - 1) / kSide, (b->H + kSide - 1) / kSide, n_frames);
   const float* K = b->kernels.as<float>();
#define ISCU_BINNED_LAUNCH(UU)                                                                                          \
   BinnedRenderKernel<UU><<<grid, kThreads, 0, ctx->stream>>>(emitters_dev, n_emitters, frames_dev, K, b->nz, b->R,  \
                                                              b->W, b->H, img_dev, alone_dev)
   switch (b->u)
   {
   case 1: ISCU_BINNED_LAUNCH(1); break;
   case 2: ISCU_BINNED_LAUNCH(2); break;
   case 3: ISCU_BINNED_LAUNCH(3); break;
   case 4: ISCU_BINNED_LAUNCH(4); break;
   case 5: ISCU_BINNED_LAUNCH(5); break;
   case 6: ISCU_BINNED_LAUNCH(6); break;
   case 7: ISCU_BINNED_LAUNCH(7); break;
   default: ISCU_BINNED_LAUNCH(8); break;
   }
#undef ISCU_BINNED_LAUNCH
   ISCU_CK_LAUNCH(ctx, "BinnedRenderKernel");
   return ISCU_OK;
}

} // extern "C"
