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
   iscu::DevBuf order;            // the persistent form's frame order + work counter, owned by the graph
   iscu::ContribScratch contrib;  // the two-pass forms' scratch, owned by the graph
};

namespace iscu {

namespace {

constexpr int kThreads = 256, kChunk = 256;

// Whether pixel (X, Y) lies in the emitter's splat square and halo cut; its offset (dx, dy) from the centre pixel.
__device__ __forceinline__ bool Covers(const StagedEmitter& e, int X, int Y, int& dx, int& dy)
{
   dx = X - e.x0;
   dy = Y - e.y0;
   const int cr = e.camRad;
   if (dx < -cr || dx > cr || dy < -cr || dy > cr)
      return false;
   if (e.spanLo && (dx < e.spanLo[dy + cr] || dx > e.spanHi[dy + cr]))
      return false;
   return true;
}

// The 16 taps of a fast emitter for the pixel p words from its centre pixel in the phase layout: the reference's
// row = 0; row += wx[i] B; sum += wy[j] row, unrolled. Taps outside the bw x bw array read the layout's zero margin
// where the reference skips them, and the sums start from the first product instead of 0: both change at most the
// sign of a zero partial sum, which the final float add cannot see (a pixel that starts at a background other than
// -0 is never -0).
__device__ __forceinline__ double PhaseTaps(const StagedEmitter& e, int p)
{
   int q[4];
#pragma unroll
   for (int i = 0; i < 4; ++i)
      q[i] = p + e.xb[i];
   double row[4];
#pragma unroll
   for (int j = 0; j < 4; ++j)
   {
      const double* pr = e.row[j];
      double r = e.wx[0] * __ldg(pr + q[0]);
      r += e.wx[1] * __ldg(pr + q[1]);
      r += e.wx[2] * __ldg(pr + q[2]);
      r += e.wx[3] * __ldg(pr + q[3]);
      row[j] = r;
   }
   double sum = e.wy[0] * row[0];
   sum += e.wy[1] * row[1];
   sum += e.wy[2] * row[2];
   sum += e.wy[3] * row[3];
   return sum;
}

// Any splat (1, 2 or 4 taps) from the row-major float64 block sums, taps outside the array skipped, in the
// reference's order (SplatKernel.inl:51-171).
__device__ __forceinline__ double GeneralTaps(const StagedEmitter& e, const KernelView& kv, int dx, int dy)
{
   const int os = kv.os, off = os - 1, bw = kv.bw, nt = e.nTaps;
   const int r0 = e.by + dy * os + off, c0 = e.bx + dx * os + off;
   const double* B = kv.sums64 + static_cast<size_t>(e.plane) * bw * bw;
   const int jLo = max(0, -r0), jHi = min(nt, bw - r0);
   const int iLo = max(0, -c0), iHi = min(nt, bw - c0);
   double sum = 0.0;
   for (int j = jLo; j < jHi; ++j)
   {
      const double* brow = B + static_cast<size_t>(r0 + j) * bw + c0;
      double row = 0.0;
      for (int i = iLo; i < iHi; ++i)
         row += e.wx[i] * __ldg(brow + i);
      sum += e.wy[j] * row;
   }
   return sum;
}

// One staged emitter's contribution to pixel (X, Y), added to acc.
__device__ __forceinline__ void SplatSingle(const StagedEmitter& e, const Kernels& K, bool inside, int X, int Y,
                                            float& acc)
{
   int dx, dy;
   if (!inside || !Covers(e, X, Y, dx, dy))
      return;
   const double sum = e.fast ? PhaseTaps(e, dy * e.nb + dx) : GeneralTaps(e, K.k[e.slot], dx, dy);
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
      if (slot < ISCU_MAX_KERNELS && em.photons > 0.0 && K.k[slot].sums64 && plane < K.k[slot].nz &&
          PositionOk(em.x_px, em.y_px))
      {
         s.x0 = static_cast<int>(RoundHalfUp(em.x_px));
         s.y0 = static_cast<int>(RoundHalfUp(em.y_px));
         const int r = K.k[slot].camRad;
         keep = s.x0 + r >= tx0 && s.x0 - r <= tx1 && s.y0 + r >= ty0 && s.y0 - r <= ty1;
         s.photons = em.photons;
         s.slot = static_cast<uint8_t>(slot);
         s.plane = plane;
         xPx = em.x_px;
         yPx = em.y_px;
      }
   }
   if (keep)
   {
      const KernelView& kv = K.k[s.slot];
      SetupWeights(kv, xPx, yPx, s);
      s.camRad = kv.camRad;
      s.nb = kv.nb;
      const int sq = 2 * kv.camRad + 1;
      s.spanLo = kv.spanLo ? kv.spanLo + s.plane * sq : nullptr;
      s.spanHi = kv.spanHi ? kv.spanHi + s.plane * sq : nullptr;
      // The phase layout serves the splat when every tap of every pixel of its square lies inside it (rows
      // R + dy os + j, columns C + dx os + i in padded coordinates, |dx|, |dy| <= camRad, i, j < 4).
      const int os = kv.os, ext = kv.nb * os, span = kv.camRad * os;
      const int R = s.by + os - 1 + kv.padLo, Cc = s.bx + os - 1 + kv.padLo;
      s.fast = kv.phase && s.nTaps == 4 && R - span >= 0 && R + span + 3 < ext && Cc - span >= 0 &&
               Cc + span + 3 < ext;
      if (s.fast)
      {
         const int nb2 = kv.nb * kv.nb;
         const double* base = kv.phase + static_cast<size_t>(s.plane) * os * os * nb2;
#pragma unroll
         for (int k = 0; k < 4; ++k)
         {
            s.row[k] = base + ((R + k) % os) * os * nb2 + ((R + k) / os) * kv.nb;
            s.xb[k] = ((Cc + k) % os) * nb2 + (Cc + k) / os;
         }
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
      const int c = sWarp[w];
      base += w < warp ? c : 0;
      total += c;
   }
   if (keep)
      sEm[base + __popc(ballot & ((1u << lane) - 1u))] = s;
   __syncthreads();
   return total;
}

// The warp's own list: the staged emitters whose square reaches the warp's pixel rectangle [wx0, wx1] x [wy0, wy1],
// in staged order. Returns its length.
__device__ __forceinline__ int WarpList(const StagedEmitter* sEm, int kept, int wx0, int wx1, int wy0, int wy1,
                                        uint16_t* list)
{
   const int lane = threadIdx.x & 31;
   int n = 0;
   for (int b = 0; b < kept; b += 32)
   {
      const int k = b + lane;
      bool hit = false;
      if (k < kept)
      {
         const StagedEmitter& e = sEm[k];
         const int cr = e.camRad;
         hit = e.x0 + cr >= wx0 && e.x0 - cr <= wx1 && e.y0 + cr >= wy0 && e.y0 - cr <= wy1;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (hit)
         list[n + __popc(bal & ((1u << lane) - 1u))] = static_cast<uint16_t>(k);
      n += __popc(bal);
   }
   __syncwarp();
   return n;
}

struct RenderArgs
{
   const iscu_emitter* ems;
   uint32_t nEm;            // emitter runs are cut at nEm
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

// kPair: two emitters per step (their taps in flight together; 2 CTAs per SM by registers), else one (3 CTAs).
template <int TX, int TY, bool kNoise, bool kPersistent, bool kPair>
__global__ void __launch_bounds__(kThreads, kPair ? 2 : 3) RenderTilesKernel(RenderArgs a)
{
   static_assert(TX * TY == kThreads, "one thread per pixel of the tile");
   static_assert(TX % 32 == 0 || 32 % TX == 0, "a warp covers a rectangle of the tile");
   __shared__ StagedEmitter sEm[kChunk];
   __shared__ uint16_t sList[kThreads / 32][kChunk];
   __shared__ int sWarp[kThreads / 32];
   __shared__ uint32_t sItem;
   const int W = static_cast<int>(a.st.width), H = static_cast<int>(a.st.height);
   const uint32_t tilesX = (W + TX - 1) / TX, tilesY = (H + TY - 1) / TY, tilesPerFrame = tilesX * tilesY;
   const uint32_t total = a.nFrames * tilesPerFrame;
   const int warp = threadIdx.x >> 5;
   uint16_t* list = sList[warp];
   // the warp's pixel rectangle within the tile
   const int wcx = TX >= 32 ? (32 * warp) % TX : 0, wcw = TX >= 32 ? 32 : TX;
   const int wry = (32 * warp) / TX, wrh = TX >= 32 ? 1 : 32 / TX;
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
      const int wx0 = tx0 + wcx, wy0 = ty0 + wry;
      float acc = inside ? Background(a.st, i, fr.bg_scale) : 0.0f;
      const uint32_t emCount = fr.em_start < a.nEm ? min(fr.em_count, a.nEm - fr.em_start) : 0u;
      for (uint32_t e0 = 0; e0 < emCount; e0 += kChunk)
      {
         const uint32_t cnt = min(static_cast<uint32_t>(kChunk), emCount - e0);
         const int kept = StageChunk(a.ems, fr.em_start + e0, cnt, a.K, tx0, ty0, tx1, ty1, sEm, sWarp);
         const int n = WarpList(sEm, kept, wx0, wx0 + wcw - 1, wy0, wy0 + wrh - 1, list);
         // Two emitters per step, their taps independent (more loads in flight), their adds in list order.
         int m = 0;
         for (; kPair && m + 1 < n; m += 2)
         {
            const StagedEmitter& ea = sEm[list[m]];
            const StagedEmitter& eb = sEm[list[m + 1]];
            if (ea.fast && eb.fast)
            {
               int dxa, dya, dxb, dyb;
               const bool ina = inside && Covers(ea, X, Y, dxa, dya);
               const bool inb = inside && Covers(eb, X, Y, dxb, dyb);
               // a pixel outside a square reads the centre pixel's taps (in the layout) and adds nothing
               const double sa = PhaseTaps(ea, ina ? dya * ea.nb + dxa : 0);
               const double sb = PhaseTaps(eb, inb ? dyb * eb.nb + dxb : 0);
               if (ina)
                  acc += static_cast<float>(ea.photons * sa);
               if (inb)
                  acc += static_cast<float>(eb.photons * sb);
            }
            else
            {
               SplatSingle(ea, a.K, inside, X, Y, acc);
               SplatSingle(eb, a.K, inside, X, Y, acc);
            }
         }
         for (; m < n; ++m)
            SplatSingle(sEm[list[m]], a.K, inside, X, Y, acc);
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

// phase[z][qy][qx][ky][kx] = sums[z][ky os + qy - padLo][kx os + qx - padLo], 0 outside the array.
__global__ void PhaseSplitKernel(const float* __restrict__ sums, int bw, int os, int padLo, int nb,
                                 double* __restrict__ out)
{
   const int kx = blockIdx.x * blockDim.x + threadIdx.x;
   const int ky = blockIdx.y;
   const int z = blockIdx.z / (os * os), q = blockIdx.z % (os * os), qy = q / os, qx = q % os;
   if (kx >= nb)
      return;
   const int r = ky * os + qy - padLo, c = kx * os + qx - padLo;
   const double v = (r >= 0 && r < bw && c >= 0 && c < bw)
                       ? static_cast<double>(sums[(static_cast<size_t>(z) * bw + r) * bw + c])
                       : 0.0;
   out[((static_cast<size_t>(blockIdx.z) * nb) + ky) * nb + kx] = v;
}

__global__ void SumsToDoubleKernel(const float* __restrict__ in, size_t n, double* __restrict__ out)
{
   const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
   if (i < n)
      out[i] = static_cast<double>(in[i]);
}

// The forms: config % 3 the tile (16 x 16, 32 x 8, 8 x 32), (config / 3) % 2 grid or persistent, config / 6 one or
// two emitters per step.
using RenderFn = void (*)(RenderArgs);
template <bool kNoise, bool kPersistent, bool kPair>
RenderFn TileVariant(int tile)
{
   switch (tile)
   {
   case 0: return RenderTilesKernel<16, 16, kNoise, kPersistent, kPair>;
   case 1: return RenderTilesKernel<32, 8, kNoise, kPersistent, kPair>;
   default: return RenderTilesKernel<8, 32, kNoise, kPersistent, kPair>;
   }
}
template <bool kNoise>
RenderFn Variant(int config)
{
   const int tile = config % 3;
   switch (config / 3)
   {
   case 0: return TileVariant<kNoise, false, false>(tile);
   case 1: return TileVariant<kNoise, true, false>(tile);
   case 2: return TileVariant<kNoise, false, true>(tile);
   default: return TileVariant<kNoise, true, true>(tile);
   }
}
constexpr int kTileW[3] = {16, 32, 8}, kTileH[3] = {16, 8, 32};

// The forms 0..11 (one pass) and 12..17 (two passes, render_contrib.cu). orderBuf: OrderBytes(nFrames) bytes of
// device scratch (the persistent forms' frame order and work counter). A two-pass form whose contributions would
// pass the context's limit renders in the one-pass form of the same tile and scheduling (the same bits).
int LaunchConfig(iscu_ctx* ctx, int config, const iscu_emitter* ems, uint32_t nEm, const iscu_frame* frames,
                 uint32_t nFrames, const CameraView* cam, uint32_t seed, float* photons, uint16_t* adu,
                 uint32_t* orderBuf, ContribScratch& sc)
{
   if (config >= 12)
   {
      const int rc = LaunchContribRender(ctx, config - 12, ems, nEm, frames, nFrames, cam, seed, photons, adu,
                                         orderBuf, sc);
      if (rc != ISCU_ERR_LIMIT)
         return rc;
      ClearError();
      config -= 12;
   }
   cudaEvent_t* marks = RenderMarks(ctx);
   if (marks)
      for (int m = 0; m < 3; ++m)
         ISCU_CK(cudaEventRecord(marks[m], ctx->stream));
   RenderArgs a;
   a.ems = ems;
   a.nEm = nEm;
   a.frames = frames;
   a.nFrames = nFrames;
   a.K = KernelsOfCtx(ctx);
   a.st = ctx->Static();
   a.cam = cam ? *cam : CameraView();
   a.seed = seed;
   a.photonsOut = photons;
   a.aduOut = cam ? adu : nullptr;
   const bool persistent = (config / 3) % 2 == 1;
   const int tw = kTileW[config % 3], th = kTileH[config % 3];
   RenderFn fn = cam ? Variant<true>(config) : Variant<false>(config);
   if (persistent)
   {
      const int rc = LaunchFrameOrder(ctx, frames, nFrames, orderBuf);
      if (rc != ISCU_OK)
         return rc;
      a.order = orderBuf;
      a.counter = orderBuf + ((nFrames + 3) & ~3u);
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
   if (marks)
      ISCU_CK(cudaEventRecord(marks[3], ctx->stream));
   return ISCU_OK;
}

} // namespace

size_t OrderBytes(uint32_t nFrames) { return (static_cast<size_t>(nFrames + 3) & ~size_t(3)) * 4 + 16; }

int LaunchFrameOrder(iscu_ctx* ctx, const iscu_frame* frames, uint32_t nFrames, uint32_t* orderBuf)
{
   ISCU_CK(cudaMemsetAsync(orderBuf + ((nFrames + 3) & ~3u), 0, sizeof(uint32_t), ctx->stream));
   if (nFrames <= 8192)
      FrameOrderKernel<<<(nFrames + 127) / 128, 128, 0, ctx->stream>>>(frames, nFrames, orderBuf);
   else
      IdentityOrderKernel<<<(nFrames + 255) / 256, 256, 0, ctx->stream>>>(nFrames, orderBuf);
   ISCU_CK_LAUNCH(ctx, "FrameOrderKernel");
   return ISCU_OK;
}

int LaunchSumsToDouble(iscu_ctx* ctx, const float* in, size_t n, double* out)
{
   SumsToDoubleKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(in, n, out);
   ISCU_CK_LAUNCH(ctx, "SumsToDoubleKernel");
   return ISCU_OK;
}

int LaunchPhaseSplit(iscu_ctx* ctx, const float* sums, int nz, int bw, int os, int padLo, int nb, double* out)
{
   const dim3 grid((nb + 127) / 128, nb, nz * os * os);
   PhaseSplitKernel<<<grid, 128, 0, ctx->stream>>>(sums, bw, os, padLo, nb, out);
   ISCU_CK_LAUNCH(ctx, "PhaseSplitKernel");
   return ISCU_OK;
}

cudaEvent_t* RenderMarks(iscu_ctx* ctx)
{
   if (!ctx->renderTiming)
      return nullptr;
   cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
   if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
      return nullptr;
   const size_t need = 4 * (ctx->renderCalls + 1);
   while (ctx->renderMarks.size() < need)
   {
      cudaEvent_t e = nullptr;
      if (cudaEventCreate(&e) != cudaSuccess)
         return nullptr;
      ctx->renderMarks.push_back(e);
   }
   return ctx->renderMarks.data() + 4 * ctx->renderCalls++;
}

int LaunchRenderFrames(iscu_ctx* ctx, const iscu_emitter* ems, uint32_t nEmitters, const iscu_frame* frames,
                       uint32_t nFrames, const CameraView* cam, uint32_t seed, float* photons, uint16_t* adu)
{
   if (nFrames == 0)
      return ISCU_OK;
   ISCU_CK(ctx->dOrder.Reserve(OrderBytes(nFrames)));
   return LaunchConfig(ctx, ctx->renderConfig, ems, nEmitters, frames, nFrames, cam, seed, photons, adu,
                       ctx->dOrder.as<uint32_t>(), ctx->contrib);
}

} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_render_set_config(iscu_ctx* ctx, int32_t config)
{
   if (!ctx || config < 0 || config >= ISCU_RENDER_CONFIGS)
      return Fail(ISCU_ERR_ARG, "render config 0..17 (tile 16x16, 32x8, 8x32; +3: persistent; +6: two emitters "
                                "per step; 12..17: two passes)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ctx->renderConfig = config;
   return ISCU_OK;
}

int iscu_render_set_contrib_limit(iscu_ctx* ctx, uint64_t bytes)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null context");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ctx->contribLimit = static_cast<size_t>(bytes);
   return ISCU_OK;
}

int iscu_render_set_timing(iscu_ctx* ctx, int32_t on)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null context");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   ctx->renderTiming = on != 0;
   ctx->renderCalls = 0;
   return ISCU_OK;
}

int iscu_render_pass_times(iscu_ctx* ctx, float* ms3, uint32_t* calls)
{
   if (!ctx || !ms3)
      return Fail(ISCU_ERR_ARG, "null argument");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (!ctx->renderTiming)
      return Fail(ISCU_ERR_STATE, "render timing is off (iscu_render_set_timing)");
   ms3[0] = ms3[1] = ms3[2] = 0.0f;
   if (calls)
      *calls = static_cast<uint32_t>(ctx->renderCalls);
   if (ctx->renderCalls == 0)
      return ISCU_OK;
   ISCU_CK(cudaEventSynchronize(ctx->renderMarks[4 * ctx->renderCalls - 1]));
   for (size_t c = 0; c < ctx->renderCalls; ++c)
      for (int k = 0; k < 3; ++k)
      {
         float t = 0.0f;
         ISCU_CK(cudaEventElapsedTime(&t, ctx->renderMarks[4 * c + k], ctx->renderMarks[4 * c + k + 1]));
         ms3[k] += t;
      }
   for (int k = 0; k < 3; ++k)
      ms3[k] /= static_cast<float>(ctx->renderCalls);
   return ISCU_OK;
}

int iscu_render_get_config(iscu_ctx* ctx, int32_t* config, int32_t* tile_w, int32_t* tile_h, int32_t* persistent,
                           int32_t* paired)
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
      *persistent = (c / 3) % 2;
   if (paired)
      *paired = c < 12 ? c / 6 : 2;
   return ISCU_OK;
}

int iscu_render_autotune(iscu_ctx* ctx, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                         const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                         uint16_t* adu_dev, float* ms)
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
   struct Events
   {
      cudaEvent_t e[2] = {nullptr, nullptr};
      ~Events()
      {
         for (cudaEvent_t x : e)
            if (x)
               cudaEventDestroy(x);
      }
   } ev;
   ISCU_CK(cudaEventCreate(&ev.e[0]));
   ISCU_CK(cudaEventCreate(&ev.e[1]));
   float best = 1e30f;
   int bestConfig = 0;
   for (int c = 0; c < ISCU_RENDER_CONFIGS; ++c)
   {
      int rc = LaunchConfig(ctx, c, emitters_dev, n_emitters, frames_dev, n_frames, &cv, seed, nullptr, adu_dev,
                            order, ctx->contrib);   // warm
      ISCU_CK(cudaEventRecord(ev.e[0], ctx->stream));
      for (int r = 0; r < 2 && rc == ISCU_OK; ++r)
         rc = LaunchConfig(ctx, c, emitters_dev, n_emitters, frames_dev, n_frames, &cv, seed, nullptr, adu_dev,
                           order, ctx->contrib);
      ISCU_CK(cudaEventRecord(ev.e[1], ctx->stream));
      if (rc != ISCU_OK)
         return rc;
      ISCU_CK(cudaEventSynchronize(ev.e[1]));
      float t = 0.f;
      ISCU_CK(cudaEventElapsedTime(&t, ev.e[0], ev.e[1]));
      t *= 0.5f;
      if (ms)
         ms[c] = t;
      if (t < best)
      {
         best = t;
         bestConfig = c;
      }
   }
   ctx->renderConfig = bestConfig;
   return ISCU_OK;
}

int iscu_render_graph_create(iscu_ctx* ctx, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                             const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                             float* photons_dev, uint16_t* adu_dev, iscu_render_graph** out)
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
   // the scratch the capture bakes in, alive as long as the graph, allocated before the capture
   ISCU_CK(g->order.Reserve(OrderBytes(n_frames)));
   int config = ctx->renderConfig;
   if (config >= 12)
   {
      const int rr = ReserveContrib(ctx, n_emitters, g->contrib);
      if (rr == ISCU_ERR_LIMIT)
      {
         ClearError();
         config -= 12;   // the one-pass form of the same tile and scheduling
      }
      else if (rr != ISCU_OK)
         return rr;
   }
   const uint64_t before = ctx->launches.load();
   ISCU_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
   const int rc = LaunchConfig(ctx, config, emitters_dev, n_emitters, frames_dev, n_frames, cam ? &cv : nullptr,
                               seed, photons_dev, adu_dev, g->order.as<uint32_t>(), g->contrib);
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
