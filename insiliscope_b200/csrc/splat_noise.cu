// sm_100a kernels beside the render (render.cu): the reference's 64-byte GPU records (the D3D11/WebGPU shader's
// semantics), the noise chain on given photon images, the bare counter RNG, and the block sums the splat reads.
//
// Compiled with --fmad=false: every float64/float32 multiply and add rounds on its own, as the reference's
// -ffp-contract=off build does.

#include "counter_rng.cuh"
#include "iscu_internal.h"
#include "noise_chain.cuh"
#include "splat_common.cuh"

#include <cstdint>

namespace iscu {

namespace {

constexpr int kTileX = 16, kTileY = 16, kThreads = kTileX * kTileY, kChunk = kThreads;

// ------------------------------------------------------------------- the reference's 64-byte record (D3D11 path)
struct StagedRecord
{
   double photons;
   double wx[4], wy[4];
   int x0, y0, bx, by;
   int nTaps, slot, plane, cutR2;
};

// GpuSimD3D11.cpp:169-248 / SplatGpu.wgsl: one thread per pixel gathers the frame's records in list order (the
// record's float weights, the halo radius test, the halo spans), taps summed in float64 here; the frame's other light
// (background, extra image) first, as SplatGpuHost splats the blinks onto it; then the noise chain.
__global__ void __launch_bounds__(kThreads) RenderGpuRecordsKernel(const iscu_gpu_splat_emitter* __restrict__ ems,
                                                                     const iscu_frame* __restrict__ frames,
                                                                     Kernels K, StaticView st,
                                                                     const float* __restrict__ extras,
                                                                     CameraView cam, uint32_t seed,
                                                                     uint16_t* __restrict__ aduOut)
{
   __shared__ StagedRecord sEm[kChunk];
   __shared__ int sWarp[kThreads / 32];
   const iscu_frame fr = frames[blockIdx.z];
   const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
   const int tx0 = blockIdx.x * kTileX, ty0 = blockIdx.y * kTileY;
   const int X = tx0 + (t % kTileX), Y = ty0 + (t / kTileX);
   const int W = static_cast<int>(st.width), H = static_cast<int>(st.height);
   const int tx1 = min(tx0 + kTileX, W) - 1, ty1 = min(ty0 + kTileY, H) - 1;
   const bool inside = X < W && Y < H;
   const uint32_t i = static_cast<uint32_t>(Y) * st.width + static_cast<uint32_t>(X);
   const size_t o = static_cast<size_t>(blockIdx.z) * st.width * st.height + i;
   float acc = inside ? Background(st, i, fr.bg_scale) : 0.0f;
   if (inside && extras)
      acc += extras[o];
   for (uint32_t e0 = 0; e0 < fr.em_count; e0 += kChunk)
   {
      const uint32_t cnt = min(static_cast<uint32_t>(kChunk), fr.em_count - e0);
      bool keep = false;
      StagedRecord s;
      if (static_cast<uint32_t>(t) < cnt)
      {
         const iscu_gpu_splat_emitter em = ems[fr.em_start + e0 + t];
         const int slot = static_cast<int>(static_cast<uint32_t>(em.plane) >> 16), plane = em.plane & 0xffff;
         if (slot < ISCU_MAX_KERNELS && K.k[slot].sums && plane < K.k[slot].nz)
         {
            const int r = K.k[slot].camRad;
            s.photons = static_cast<double>(em.photons);
            for (int k = 0; k < 4; ++k)
            {
               s.wx[k] = static_cast<double>(em.wx[k]);
               s.wy[k] = static_cast<double>(em.wy[k]);
            }
            s.x0 = em.x0;
            s.y0 = em.y0;
            s.bx = em.bx;
            s.by = em.by;
            s.nTaps = em.n_taps < 1 ? 1 : (em.n_taps > 4 ? 4 : em.n_taps);
            s.slot = slot;
            s.plane = plane;
            s.cutR2 = em.cut_radius2;
            keep = s.x0 + r >= tx0 && s.x0 - r <= tx1 && s.y0 + r >= ty0 && s.y0 - r <= ty1;
         }
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, keep);
      if (lane == 0)
         sWarp[warp] = __popc(ballot);
      __syncthreads();
      int base = 0, total = 0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w)
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
            const StagedRecord& e = sEm[k];
            const KernelView& kv = K.k[e.slot];
            const int dx = X - e.x0, dy = Y - e.y0;
            if (dx < -kv.camRad || dx > kv.camRad || dy < -kv.camRad || dy > kv.camRad)
               continue;
            if (dx * dx + dy * dy > e.cutR2)
               continue;
            if (kv.spanLo)
            {
               const int row = e.plane * (2 * kv.camRad + 1) + dy + kv.camRad;
               if (dx < kv.spanLo[row] || dx > kv.spanHi[row])
                  continue;
            }
            const int os = kv.os, off = os - 1, bw = kv.bw;
            const int r0 = e.by + dy * os + off, c0 = e.bx + dx * os + off;
            const float* B = kv.sums + static_cast<size_t>(e.plane) * bw * bw;
            double sum = 0.0;
            for (int j = max(0, -r0); j < min(e.nTaps, bw - r0); ++j)
            {
               double row = 0.0;
               for (int ii = max(0, -c0); ii < min(e.nTaps, bw - c0); ++ii)
                  row += e.wx[ii] * static_cast<double>(B[static_cast<size_t>(r0 + j) * bw + c0 + ii]);
               sum += e.wy[j] * row;
            }
            acc += static_cast<float>(e.photons * sum);
         }
      __syncthreads();
   }
   if (!inside)
      return;
   CounterRng u(seed, fr.frame);
   aduOut[o] = NoisePixel(acc, i, cam, st, u);
}

// ---------------------------------------------------------------------------------------------- noise only
__global__ void NoiseFramesKernel(const float* __restrict__ photons, const uint32_t* __restrict__ frames,
                                  StaticView st, CameraView cam, uint32_t seed, uint16_t* __restrict__ adu)
{
   const size_t n = static_cast<size_t>(st.width) * st.height;
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n)
      return;
   const size_t o = static_cast<size_t>(blockIdx.y) * n + i;
   CounterRng u(seed, frames[blockIdx.y]);
   adu[o] = NoisePixel(photons[o], i, cam, st, u);
}

// ---------------------------------------------------------------------------------------------- bare RNG
__global__ void Pcg4dKernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t n)
{
   const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
   if (i >= n)
      return;
   uint32_t a = in[4 * i], b = in[4 * i + 1], c = in[4 * i + 2], d = in[4 * i + 3];
   Pcg4d(a, b, c, d);
   out[4 * i] = a;
   out[4 * i + 1] = b;
   out[4 * i + 2] = c;
   out[4 * i + 3] = d;
}

__global__ void CounterUniformsKernel(uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix,
                                      uint32_t perPixel, double* __restrict__ out)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= npix)
      return;
   CounterRng u(seed, frame);
   u.Pixel(pixel0 + i);
   for (uint32_t j = 0; j < perPixel; ++j)
      out[static_cast<size_t>(i) * perPixel + j] = u.Uniform();
}

// ---------------------------------------------------------------------------------------------- block sums
// BuildBlockSums (PsfGeneratorBridge.cpp:1021-1047): out[ai][bi] = sum_y (sum_x kernel[y][x]) over the os x os block
// that starts at (ai - (os-1), bi - (os-1)), clipped to the kernel; float64 sums in the reference's order (the
// horizontal sums per row first, then the vertical sum of those), one thread per output.
__global__ void BlockSumsKernel(const float* __restrict__ planes, int n, int os, float* __restrict__ sums)
{
   const int off = os - 1, bw = n + off;
   const int bi = blockIdx.x * blockDim.x + threadIdx.x;
   const int ai = blockIdx.y;
   const int z = blockIdx.z;
   if (bi >= bw)
      return;
   const float* k = planes + static_cast<size_t>(z) * n * n;
   const int a = ai - off, y0 = max(0, a), y1 = min(n - 1, a + off);
   const int b = bi - off, x0 = max(0, b), x1 = min(n - 1, b + off);
   double acc = 0.0;
   for (int y = y0; y <= y1; ++y)
   {
      double h = 0.0;
      for (int x = x0; x <= x1; ++x)
         h += static_cast<double>(k[static_cast<size_t>(y) * n + x]);
      acc += h;
   }
   sums[(static_cast<size_t>(z) * bw + ai) * bw + bi] = static_cast<float>(acc);
}

} // namespace

// ------------------------------------------------------------------------------------------------ launchers
int LaunchRenderGpuRecords(iscu_ctx* ctx, const iscu_gpu_splat_emitter* ems, const iscu_frame* frames,
                           uint32_t nFrames, const float* extras, const CameraView* cam, uint32_t seed, uint16_t* adu)
{
   if (nFrames == 0)
      return ISCU_OK;
   const StaticView st = ctx->Static();
   const dim3 grid((st.width + kTileX - 1) / kTileX, (st.height + kTileY - 1) / kTileY, nFrames);
   RenderGpuRecordsKernel<<<grid, kThreads, 0, ctx->stream>>>(ems, frames, KernelsOfCtx(ctx), st, extras, *cam, seed,
                                                              adu);
   ISCU_CK_LAUNCH(ctx, "RenderGpuRecordsKernel");
   return ISCU_OK;
}

int LaunchNoiseFrames(iscu_ctx* ctx, const float* photons, uint32_t nFrames, const uint32_t* frames,
                      const CameraView& cam, uint32_t seed, uint16_t* adu)
{
   const StaticView st = ctx->Static();
   const size_t n = static_cast<size_t>(st.width) * st.height;
   if (nFrames == 0 || n == 0)
      return ISCU_OK;
   const dim3 grid(static_cast<unsigned>((n + 255) / 256), nFrames);
   NoiseFramesKernel<<<grid, 256, 0, ctx->stream>>>(photons, frames, st, cam, seed, adu);
   ISCU_CK_LAUNCH(ctx, "NoiseFramesKernel");
   return ISCU_OK;
}

int LaunchPcg4d(iscu_ctx* ctx, const uint32_t* in, uint32_t* out, size_t n)
{
   if (n == 0)
      return ISCU_OK;
   Pcg4dKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(in, out, n);
   ISCU_CK_LAUNCH(ctx, "Pcg4dKernel");
   return ISCU_OK;
}

int LaunchCounterUniforms(iscu_ctx* ctx, uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix,
                          uint32_t perPixel, double* out)
{
   if (npix == 0 || perPixel == 0)
      return ISCU_OK;
   CounterUniformsKernel<<<(npix + 255) / 256, 256, 0, ctx->stream>>>(seed, frame, pixel0, npix, perPixel, out);
   ISCU_CK_LAUNCH(ctx, "CounterUniformsKernel");
   return ISCU_OK;
}

int LaunchBlockSums(iscu_ctx* ctx, const float* planes, int n, int os, int nz, float* sums)
{
   const int bw = n + os - 1;
   const dim3 grid((bw + 127) / 128, bw, nz);
   BlockSumsKernel<<<grid, 128, 0, ctx->stream>>>(planes, n, os, sums);
   ISCU_CK_LAUNCH(ctx, "BlockSumsKernel");
   return ISCU_OK;
}

} // namespace iscu
