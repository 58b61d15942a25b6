// The per-frame hot path on sm_100a: blink splat fused with the camera noise chain (RenderPhotonImage +
// ApplyNoiseChain, adapter/inSiliScope/Simulation/SMLMSimulation.cpp:103-160, SMLMNoise.cpp:142-216).
//
// Compiled with --fmad=false: every float64 multiply and add rounds on its own, as the reference's
// -ffp-contract=off build does, so the noise-free image and the ADU are bit for bit the CPU's.
//
// A CTA owns one TX x TY pixel tile of one frame. It streams the frame's emitter list through shared memory 256
// records at a time; a record whose (2 camRad + 1)^2 square misses the tile is dropped on its centre pixel alone,
// the others get their SplatSetup (PsfGeneratorBridge.cpp:1382-1422) and are kept, in list order, by a warp-ballot
// compaction. Each thread then adds every kept emitter to its own pixel, in list order:
// float(photons * sum_j wy[j] * (sum_i wx[i] * B[r0 + j][c0 + i])) in float64 (SplatKernel.inl:51-171), the block
// sums read as float64 copies of the float sums (the same values; no per-tap conversion), taps outside the array
// skipped, the halo cut's columns only. The noise chain follows in registers.
//
// Frames with very different emitter counts (10 to 8,000 in one movie) are balanced by the persistent form: a grid
// of resident CTAs takes (frame, tile) items from an atomic counter, heaviest frames first (a rank of the frames by
// emitter count made on the device). Tile shape and form are chosen by a small autotuner (iscu_render_autotune); a
// batch's device work can be captured once into a CUDA graph and replayed (iscu_render_graph_*).

#include "counter_rng.cuh"
#include "iscu_internal.h"
#include "noise_chain.cuh"
#include "splat_common.cuh"

#include <algorithm>
#include <cstdint>

struct iscu_render_graph
{
   iscu_ctx* ctx = nullptr;
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   int kernels = 0;
   iscu::DevBuf order;   // the persistent form's frame order + work counter, owned by the graph
};

namespace iscu {

namespace {

constexpr int kThreads = 256, kChunk = 256;

// One staged emitter's contribution to pixel (X, Y), added to acc.
__device__ __forceinline__ void SplatOne(const StagedEmitter& e, const KernelView& kv, int X, int Y, float& acc)
{
   const int camRad = kv.camRad;
   const int dx = X - e.x0, dy = Y - e.y0;
   if (dx < -camRad || dx > camRad || dy < -camRad || dy > camRad)
      return;
   if (kv.spanLo)
   {
      const int row = e.plane * (2 * camRad + 1) + dy + camRad;
      if (dx < kv.spanLo[row] || dx > kv.spanHi[row])
         return;
   }
   const int os = kv.os, off = os - 1, bw = kv.bw, nt = e.nTaps;
   const int r0 = e.by + dy * os + off, c0 = e.bx + dx * os + off;
   const double* B = kv.sums64 + static_cast<size_t>(e.plane) * bw * bw;
   double sum;
   if (nt == 4 && r0 >= 0 && r0 + 4 <= bw && c0 >= 0 && c0 + 4 <= bw)
   {
      // all 16 taps inside: the reference's row = 0; row += wx[i] B; sum += wy[j] row, unrolled (starting from the
      // first product instead of 0 changes at most the sign of a zero sum, which the float add cannot see)
      const double* b = B + static_cast<size_t>(r0) * bw + c0;
      double row[4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
      {
         const double* br = b + j * bw;
         double r = e.wx[0] * __ldg(br);
         r += e.wx[1] * __ldg(br + 1);
         r += e.wx[2] * __ldg(br + 2);
         r += e.wx[3] * __ldg(br + 3);
         row[j] = r;
      }
      sum = e.wy[0] * row[0];
      sum += e.wy[1] * row[1];
      sum += e.wy[2] * row[2];
      sum += e.wy[3] * row[3];
   }
   else
   {
      const int jLo = max(0, -r0), jHi = min(nt, bw - r0);
      const int iLo = max(0, -c0), iHi = min(nt, bw - c0);
      sum = 0.0;
      for (int j = jLo; j < jHi; ++j)
      {
         const double* brow = B + static_cast<size_t>(r0 + j) * bw + c0;
         double row = 0.0;
         for (int i = iLo; i < iHi; ++i)
            row += e.wx[i] * __ldg(brow + i);
         sum += e.wy[j] * row;
      }
   }
   acc += static_cast<float>(e.photons * sum);
}

// Stages one chunk of a frame's emitters: the ones whose square reaches the tile, in list order, with their setup.
// Every thread of the CTA calls it (it synchronizes). Returns how many were kept.
__device__ __forceinline__ int StageChunk(const iscu_emitter* __restrict__ ems, uint32_t start, uint32_t count,
                                          const Kernels& K, int tx0, int ty0, int tx1, int ty1, StagedEmitter* sEm,
                                          int* sWarp)
{
   const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
   bool keep = false;
   StagedEmitter s;
   double xPx = 0.0, yPx = 0.0;
   if (static_cast<uint32_t>(t) < count)
   {
      const iscu_emitter em = ems[start + t];
      const int slot = static_cast<int>(static_cast<uint32_t>(em.plane) >> 16), plane = em.plane & 0xffff;
      if (slot < ISCU_MAX_KERNELS && em.photons > 0.0 && K.k[slot].sums64 && plane < K.k[slot].nz)
      {
         s.x0 = static_cast<int>(RoundHalfUp(em.x_px));
         s.y0 = static_cast<int>(RoundHalfUp(em.y_px));
         const int r = K.k[slot].camRad;
         keep = s.x0 + r >= tx0 && s.x0 - r <= tx1 && s.y0 + r >= ty0 && s.y0 - r <= ty1;
         s.photons = em.photons;
         s.slot = slot;
         s.plane = plane;
         xPx = em.x_px;
         yPx = em.y_px;
      }
   }
   if (keep)
      SetupWeights(K.k[s.slot], xPx, yPx, s);
   const unsigned ballot = __ballot_sync(0xffffffffu, keep);
   if (lane == 0)
      sWarp[warp] = __popc(ballot);
   __syncthreads();
   int base = 0, total = 0;
#pragma unroll
   for (int w = 0; w < kThreads / 32; ++w)
   {
      const int c = sWarp[w];
      base += w < warp ? c : 0;
      total += c;
   }
   if (keep)
      sEm[base + __popc(ballot & ((1u << lane) - 1u))] = s;
   __syncthreads();
   return total;
}

struct RenderArgs
{
   const iscu_emitter* ems;
   const iscu_frame* frames;
   uint32_t nFrames;
   const uint32_t* order;   // persistent form: frames, heaviest first
   uint32_t* counter;       // persistent form: the next work item
   Kernels K;
   StaticView st;
   CameraView cam;
   uint32_t seed;
   float* photonsOut;
   uint16_t* aduOut;
};

template <int TX, int TY, bool kNoise, bool kPersistent>
__global__ void __launch_bounds__(kThreads) RenderTilesKernel(RenderArgs a)
{
   static_assert(TX * TY == kThreads, "one thread per pixel of the tile");
   __shared__ StagedEmitter sEm[kChunk];
   __shared__ int sWarp[kThreads / 32];
   __shared__ uint32_t sItem;
   const int W = static_cast<int>(a.st.width), H = static_cast<int>(a.st.height);
   const uint32_t tilesX = (W + TX - 1) / TX, tilesY = (H + TY - 1) / TY, tilesPerFrame = tilesX * tilesY;
   const uint32_t total = a.nFrames * tilesPerFrame;
   for (;;)
   {
      uint32_t f, tile;
      if (kPersistent)
      {
         if (threadIdx.x == 0)
            sItem = atomicAdd(a.counter, 1u);
         __syncthreads();
         const uint32_t item = sItem;
         __syncthreads();
         if (item >= total)
            return;
         f = a.order[item / tilesPerFrame];
         tile = item % tilesPerFrame;
      }
      else
      {
         f = blockIdx.z;
         tile = blockIdx.y * tilesX + blockIdx.x;
      }
      const iscu_frame fr = a.frames[f];
      const int tx0 = static_cast<int>(tile % tilesX) * TX, ty0 = static_cast<int>(tile / tilesX) * TY;
      const int X = tx0 + static_cast<int>(threadIdx.x % TX), Y = ty0 + static_cast<int>(threadIdx.x / TX);
      const int tx1 = min(tx0 + TX, W) - 1, ty1 = min(ty0 + TY, H) - 1;
      const bool inside = X < W && Y < H;
      const uint32_t i = static_cast<uint32_t>(Y) * a.st.width + static_cast<uint32_t>(X);
      float acc = inside ? Background(a.st, i, fr.bg_scale) : 0.0f;
      for (uint32_t e0 = 0; e0 < fr.em_count; e0 += kChunk)
      {
         const uint32_t cnt = min(static_cast<uint32_t>(kChunk), fr.em_count - e0);
         const int kept = StageChunk(a.ems, fr.em_start + e0, cnt, a.K, tx0, ty0, tx1, ty1, sEm, sWarp);
         if (inside)
            for (int k = 0; k < kept; ++k)
               SplatOne(sEm[k], a.K.k[sEm[k].slot], X, Y, acc);
         __syncthreads();
      }
      if (inside)
      {
         const size_t o = static_cast<size_t>(f) * a.st.width * a.st.height + i;
         if (a.photonsOut)
            a.photonsOut[o] = acc;
         if (kNoise)
         {
            CounterRng u(a.seed, fr.frame);
            a.aduOut[o] = NoisePixel(acc, i, a.cam, a.st, u);
         }
      }
      if (!kPersistent)
         return;
   }
}

// order[rank] = frame: frames by emitter count, heaviest first (ties by index).
__global__ void FrameOrderKernel(const iscu_frame* __restrict__ frames, uint32_t n, uint32_t* __restrict__ order)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n)
      return;
   const uint32_t c = frames[i].em_count;
   uint32_t rank = 0;
   for (uint32_t j = 0; j < n; ++j)
   {
      const uint32_t cj = frames[j].em_count;
      rank += (cj > c || (cj == c && j < i)) ? 1u : 0u;
   }
   order[rank] = i;
}

__global__ void IdentityOrderKernel(uint32_t n, uint32_t* __restrict__ order)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n)
      order[i] = i;
}

__global__ void SumsToDoubleKernel(const float* __restrict__ in, size_t n, double* __restrict__ out)
{
   const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
   if (i < n)
      out[i] = static_cast<double>(in[i]);
}

// The six configurations: tile 16 x 16, 32 x 8, 8 x 32; grid or persistent.
using RenderFn = void (*)(RenderArgs);
template <bool kNoise>
RenderFn Variant(int config)
{
   switch (config)
   {
   case 0: return RenderTilesKernel<16, 16, kNoise, false>;
   case 1: return RenderTilesKernel<32, 8, kNoise, false>;
   case 2: return RenderTilesKernel<8, 32, kNoise, false>;
   case 3: return RenderTilesKernel<16, 16, kNoise, true>;
   case 4: return RenderTilesKernel<32, 8, kNoise, true>;
   default: return RenderTilesKernel<8, 32, kNoise, true>;
   }
}
constexpr int kTileW[3] = {16, 32, 8}, kTileH[3] = {16, 8, 32};

Kernels KernelsOf(iscu_ctx* ctx)
{
   Kernels K;
   for (int s = 0; s < ISCU_MAX_KERNELS; ++s)
      K.k[s] = ctx->kernels[s].valid ? ctx->kernels[s].View() : KernelView();
   return K;
}

size_t OrderBytes(uint32_t nFrames) { return (static_cast<size_t>(nFrames + 3) & ~size_t(3)) * 4 + 16; }

// orderBuf: OrderBytes(nFrames) bytes of device scratch (the persistent forms' frame order and work counter).
int LaunchConfig(iscu_ctx* ctx, int config, const iscu_emitter* ems, const iscu_frame* frames, uint32_t nFrames,
                 const CameraView* cam, uint32_t seed, float* photons, uint16_t* adu, uint32_t* orderBuf)
{
   RenderArgs a;
   a.ems = ems;
   a.frames = frames;
   a.nFrames = nFrames;
   a.K = KernelsOf(ctx);
   a.st = ctx->Static();
   a.cam = cam ? *cam : CameraView();
   a.seed = seed;
   a.photonsOut = photons;
   a.aduOut = cam ? adu : nullptr;
   const bool persistent = config >= 3;
   const int tw = kTileW[config % 3], th = kTileH[config % 3];
   RenderFn fn = cam ? Variant<true>(config) : Variant<false>(config);
   if (persistent)
   {
      a.order = orderBuf;
      a.counter = orderBuf + ((nFrames + 3) & ~3u);
      ISCU_CK(cudaMemsetAsync(a.counter, 0, sizeof(uint32_t), ctx->stream));
      if (nFrames <= 8192)
         FrameOrderKernel<<<(nFrames + 127) / 128, 128, 0, ctx->stream>>>(frames, nFrames, orderBuf);
      else
         IdentityOrderKernel<<<(nFrames + 255) / 256, 256, 0, ctx->stream>>>(nFrames, orderBuf);
      ISCU_CK_LAUNCH(ctx, "FrameOrderKernel");
      int perSm = 0;
      ISCU_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, kThreads, 0));
      const uint32_t tiles = ((a.st.width + tw - 1) / tw) * ((a.st.height + th - 1) / th);
      const uint32_t grid = std::min<uint32_t>(static_cast<uint32_t>(std::max(1, perSm) * ctx->smCount),
                                               tiles * nFrames);
      fn<<<grid, kThreads, 0, ctx->stream>>>(a);
   }
   else
   {
      a.order = nullptr;
      a.counter = nullptr;
      const dim3 grid((a.st.width + tw - 1) / tw, (a.st.height + th - 1) / th, nFrames);
      fn<<<grid, kThreads, 0, ctx->stream>>>(a);
   }
   ISCU_CK_LAUNCH(ctx, "RenderTilesKernel");
   return ISCU_OK;
}

} // namespace

int LaunchSumsToDouble(iscu_ctx* ctx, const float* in, size_t n, double* out)
{
   SumsToDoubleKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(in, n, out);
   ISCU_CK_LAUNCH(ctx, "SumsToDoubleKernel");
   return ISCU_OK;
}

int LaunchRenderFrames(iscu_ctx* ctx, const iscu_emitter* ems, const iscu_frame* frames, uint32_t nFrames,
                       const CameraView* cam, uint32_t seed, float* photons, uint16_t* adu)
{
   if (nFrames == 0)
      return ISCU_OK;
   if (ctx->renderConfig >= 3)
      ISCU_CK(ctx->dOrder.Reserve(OrderBytes(nFrames)));
   return LaunchConfig(ctx, ctx->renderConfig, ems, frames, nFrames, cam, seed, photons, adu,
                       ctx->dOrder.as<uint32_t>());
}

} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_render_set_config(iscu_ctx* ctx, int32_t config)
{
   if (!ctx || config < 0 || config > 5)
      return Fail(ISCU_ERR_ARG, "render config 0..5 (tile 16x16, 32x8, 8x32; +3: persistent)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ctx->renderConfig = config;
   return ISCU_OK;
}

int iscu_render_get_config(iscu_ctx* ctx, int32_t* config, int32_t* tile_w, int32_t* tile_h, int32_t* persistent)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null context");
   const int c = ctx->renderConfig;
   if (config)
      *config = c;
   if (tile_w)
      *tile_w = kTileW[c % 3];
   if (tile_h)
      *tile_h = kTileH[c % 3];
   if (persistent)
      *persistent = c >= 3;
   return ISCU_OK;
}

int iscu_render_autotune(iscu_ctx* ctx, const iscu_emitter* emitters_dev, const iscu_frame* frames_dev,
                         uint32_t n_frames, const iscu_camera* cam, uint32_t seed, uint16_t* adu_dev, float* ms6)
{
   if (!ctx || !frames_dev || !cam || !adu_dev || n_frames == 0)
      return Fail(ISCU_ERR_ARG, "null argument or no frames");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   const CameraView cv = MakeCameraView(*cam);
   ISCU_CK(ctx->dOrder.Reserve(OrderBytes(n_frames)));
   uint32_t* order = ctx->dOrder.as<uint32_t>();
   cudaEvent_t e0, e1;
   ISCU_CK(cudaEventCreate(&e0));
   ISCU_CK(cudaEventCreate(&e1));
   float best = 1e30f;
   int bestConfig = 0;
   for (int c = 0; c < 6; ++c)
   {
      int rc = LaunchConfig(ctx, c, emitters_dev, frames_dev, n_frames, &cv, seed, nullptr, adu_dev, order);   // warm
      ISCU_CK(cudaEventRecord(e0, ctx->stream));
      for (int r = 0; r < 2 && rc == ISCU_OK; ++r)
         rc = LaunchConfig(ctx, c, emitters_dev, frames_dev, n_frames, &cv, seed, nullptr, adu_dev, order);
      ISCU_CK(cudaEventRecord(e1, ctx->stream));
      if (rc != ISCU_OK)
      {
         cudaEventDestroy(e0);
         cudaEventDestroy(e1);
         return rc;
      }
      ISCU_CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      ISCU_CK(cudaEventElapsedTime(&ms, e0, e1));
      ms *= 0.5f;
      if (ms6)
         ms6[c] = ms;
      if (ms < best)
      {
         best = ms;
         bestConfig = c;
      }
   }
   cudaEventDestroy(e0);
   cudaEventDestroy(e1);
   ctx->renderConfig = bestConfig;
   return ISCU_OK;
}

int iscu_render_graph_create(iscu_ctx* ctx, const iscu_emitter* emitters_dev, const iscu_frame* frames_dev,
                             uint32_t n_frames, const iscu_camera* cam, uint32_t seed, float* photons_dev,
                             uint16_t* adu_dev, iscu_render_graph** out)
{
   if (!ctx || !out || !frames_dev || n_frames == 0 || (cam && !adu_dev))
      return Fail(ISCU_ERR_ARG, "null argument or no frames");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   *out = nullptr;
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   CameraView cv;
   if (cam)
      cv = MakeCameraView(*cam);
   std::unique_ptr<iscu_render_graph> g(new iscu_render_graph());
   g->ctx = ctx;
   ISCU_CK(g->order.Reserve(OrderBytes(n_frames)));   // scratch the capture bakes in, alive as long as the graph
   const uint64_t before = ctx->launches.load();
   ISCU_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
   const int rc = LaunchConfig(ctx, ctx->renderConfig, emitters_dev, frames_dev, n_frames, cam ? &cv : nullptr, seed,
                               photons_dev, adu_dev, g->order.as<uint32_t>());
   cudaGraph_t graph = nullptr;
   const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
   if (rc != ISCU_OK)
   {
      if (graph)
         cudaGraphDestroy(graph);
      return rc;
   }
   ISCU_CK(ec);
   g->graph = graph;
   g->kernels = static_cast<int>(ctx->launches.load() - before);
   ctx->launches.fetch_sub(static_cast<uint64_t>(g->kernels));   // counted when the graph runs
   ISCU_CK(cudaGraphInstantiate(&g->exec, graph, 0));
   *out = g.release();
   return ISCU_OK;
}

int iscu_render_graph_launch(iscu_render_graph* g)
{
   if (!g)
      return Fail(ISCU_ERR_ARG, "null graph");
   std::lock_guard<std::recursive_mutex> lock(g->ctx->mu);
   ClearError();
   ISCU_CK(cudaGraphLaunch(g->exec, g->ctx->stream));
   g->ctx->launches.fetch_add(static_cast<uint64_t>(g->kernels));
   return ISCU_OK;
}

void iscu_render_graph_destroy(iscu_render_graph* g)
{
   if (!g)
      return;
   cudaStreamSynchronize(g->ctx->stream);
   if (g->exec)
      cudaGraphExecDestroy(g->exec);
   if (g->graph)
      cudaGraphDestroy(g->graph);
   delete g;
}

} // extern "C"
