// The two-pass render on sm_100a: the same frames, bit for bit, as the one-pass tile render (render.cu), with the
// float64 tap arithmetic regrouped so that the FP64 pipe, not the tap loads, bounds it.
//
// A splat's value at pixel (dx, dy) of its square is float(photons * sum_j wy[j] (sum_i wx[i] B[r0 + j][c0 + i]))
// (SplatKernel.inl:51-171) with r0 = by + dy os + os - 1, c0 = bx + dx os + os - 1: the block sums it reads depend
// only on the kernel slot, the z plane and the tap origin (bx, by), which takes at most os + 1 values per axis. So:
//
//  1. setup (one thread per emitter): SplatSetup (PsfGeneratorBridge.cpp:1382-1422), and the emitter's group
//     (slot, plane, bx, by) counted;
//  2. the groups' offsets (one CTA scan) and 3. each emitter listed under its group;
//  4. contributions: a CTA takes a group's block of square pixels and up to 64 of its emitters; each thread loads its
//     pixel's taps into registers once and computes every emitter's float contribution, in the reference's operation
//     order, into HBM (emitter-major, one float per pixel of the square);
//  5. gather (one CTA per frame tile, or a persistent grid heaviest frame first): every pixel adds, in the frame's
//     emitter order, the contributions of the emitters whose square (and halo cut) covers it -- the same float
//     additions in the same order as RenderPhotonImage (SMLMSimulation.cpp:103-160) -- then the noise chain
//     (ApplyNoiseChain, SMLMNoise.cpp:142-216) in registers.
//
// Compiled with --fmad=false: every float64 multiply and add rounds on its own, as the reference's -ffp-contract=off
// build does.

#include "counter_rng.cuh"
#include "iscu_internal.h"
#include "noise_chain.cuh"
#include "splat_common.cuh"

#include <algorithm>
#include <cstdint>

namespace iscu {

namespace {

constexpr int kE = 64;          // emitters per contribution work item
// Contribution CTAs: at most 384 computing threads and a staging warp, two per SM (72 registers: the 16 float64 taps
// in registers without spills). A 33 x 33 square is three pixel blocks, so a group's per-item work (its taps from L2,
// its geometry, the barrier) is paid three times rather than five as with 224-thread CTAs four to an SM, while the
// other CTA keeps the FP64 pipe busy through one CTA's barrier.
constexpr int kMaxCT = 384;
constexpr int kContribPerSm = 2;
constexpr int kGT = 256;        // gather CTA size (one thread per pixel of the tile)
constexpr int kGChunk = 256;    // gather staging chunk

// One emitter's setup, as the contribution pass reads it.
struct SplatRec
{
   double photons;
   double wx[4], wy[4];
   int bx, by;
   int key, plane;
};

// The group keys: slot s owns keys [base[s], base[s + 1]); key base[s] + (plane n1 + (by - lo)) n1 + (bx - lo) is the
// group (s, plane, bx, by); the slot's last key collects tap origins outside [lo, lo + n1) (none arise from finite
// positions: SplatSetup keeps by, bx within [kc - os - 1, kc + 1]).
struct KeyMap
{
   int base[ISCU_MAX_KERNELS + 1];
   int lo[ISCU_MAX_KERNELS];
   int n1[ISCU_MAX_KERNELS];
   int pbs[ISCU_MAX_KERNELS];    // pixel blocks of a group's square (ceil(side^2 / contribution CTA size))
   int side[ISCU_MAX_KERNELS];   // splat square side, 2 camRad + 1
};

__device__ __forceinline__ int SlotOfKey(const KeyMap& km, int key)
{
   int s = 0;
#pragma unroll
   for (int t = 1; t < ISCU_MAX_KERNELS; ++t)
      if (key >= km.base[t])
         s = t;
   return s;
}

__device__ __forceinline__ int TapsOf(const KernelView& kv)
{
   return kv.interp == ISCU_INTERP_CUBIC ? 4 : (kv.interp == ISCU_INTERP_LINEAR ? 2 : 1);
}

// ------------------------------------------------------------------------------------------------ 1. setup
struct SetupArgs
{
   const iscu_emitter* ems;
   uint32_t n;
   Kernels K;
   KeyMap km;
   SplatRec* rec;
   int4* grec;        // per emitter (x0, y0, slot, plane); slot -1: not splatted
   uint32_t* count;   // per key
};

__global__ void ContribSetupKernel(SetupArgs a)
{
   const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
   bool valid = false;
   int key = 0;
   if (g < a.n)
   {
      const iscu_emitter em = a.ems[g];
      const int slot = static_cast<int>(static_cast<uint32_t>(em.plane) >> 16), plane = em.plane & 0xffff;
      int4 gr = make_int4(0, 0, -1, 0);
      if (slot < ISCU_MAX_KERNELS && em.photons > 0.0 && a.K.k[slot].sums64 && plane < a.K.k[slot].nz &&
          PositionOk(em.x_px, em.y_px))
      {
         const KernelView& kv = a.K.k[slot];
         StagedEmitter s;
         s.x0 = static_cast<int>(RoundHalfUp(em.x_px));
         s.y0 = static_cast<int>(RoundHalfUp(em.y_px));
         SetupWeights(kv, em.x_px, em.y_px, s);
         SplatRec r;
         r.photons = em.photons;
#pragma unroll
         for (int k = 0; k < 4; ++k)
         {
            r.wx[k] = s.wx[k];
            r.wy[k] = s.wy[k];
         }
         r.bx = s.bx;
         r.by = s.by;
         r.plane = plane;
         const int n1 = a.km.n1[slot], cy = s.by - a.km.lo[slot], cx = s.bx - a.km.lo[slot];
         key = (cy >= 0 && cy < n1 && cx >= 0 && cx < n1) ? a.km.base[slot] + (plane * n1 + cy) * n1 + cx
                                                          : a.km.base[slot + 1] - 1;
         r.key = key;
         a.rec[g] = r;
         gr = make_int4(s.x0, s.y0, slot, plane);
         valid = true;
      }
      a.grec[g] = gr;
   }
   const unsigned vm = __ballot_sync(0xffffffffu, valid);
   if (valid)
   {
      const unsigned peers = __match_any_sync(vm, key);
      if ((threadIdx.x & 31) == __ffs(peers) - 1)
         atomicAdd(&a.count[key], static_cast<uint32_t>(__popc(peers)));
   }
}

// ------------------------------------------------------------------------------------------------ 2. offsets
// One CTA of 1024 threads, kScanPer consecutive keys a thread per pass of 4,096 keys (one round trip for the counts):
// start[k] = exclusive sum of count, itemStart[k] = exclusive sum of the keys' work items (ceil(count / kE) emitter
// chunks x the slot's pixel blocks), itemKey[i] = k for each of key k's items; itemStart[nKeys] and ctr[0] = the
// total; ctr[1] = 0.
constexpr int kScanPer = 4;
__global__ void __launch_bounds__(1024) ContribScanKernel(KeyMap km, const uint32_t* __restrict__ count,
                                                          uint32_t* __restrict__ start, uint32_t* __restrict__ cursor,
                                                          uint32_t* __restrict__ itemStart,
                                                          uint32_t* __restrict__ itemKey, uint32_t* __restrict__ ctr)
{
   const int nKeys = km.base[ISCU_MAX_KERNELS];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   __shared__ uint32_t sw[2][32];
   __shared__ uint32_t carry[2];
   if (threadIdx.x == 0)
      carry[0] = carry[1] = 0;
   __syncthreads();
   for (int k0 = 0; k0 < nKeys; k0 += 1024 * kScanPer)
   {
      const int kb = k0 + static_cast<int>(threadIdx.x) * kScanPer;
      uint32_t c[kScanPer], it[kScanPer], tc = 0, ti = 0;
#pragma unroll
      for (int j = 0; j < kScanPer; ++j)
         c[j] = kb + j < nKeys ? count[kb + j] : 0u;
#pragma unroll
      for (int j = 0; j < kScanPer; ++j)
      {
         it[j] = c[j] ? ((c[j] + kE - 1) / kE) * static_cast<uint32_t>(km.pbs[SlotOfKey(km, kb + j)]) : 0u;
         tc += c[j];
         ti += it[j];
      }
      uint32_t xc = tc, xi = ti;   // inclusive warp scans of the threads' totals
#pragma unroll
      for (int d = 1; d < 32; d <<= 1)
      {
         const uint32_t u = __shfl_up_sync(0xffffffffu, xc, d), v = __shfl_up_sync(0xffffffffu, xi, d);
         if (lane >= d)
         {
            xc += u;
            xi += v;
         }
      }
      if (lane == 31)
      {
         sw[0][warp] = xc;
         sw[1][warp] = xi;
      }
      __syncthreads();
      if (warp == 0)
      {
         uint32_t u = sw[0][lane], v = sw[1][lane];
#pragma unroll
         for (int d = 1; d < 32; d <<= 1)
         {
            const uint32_t pu = __shfl_up_sync(0xffffffffu, u, d), pv = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d)
            {
               u += pu;
               v += pv;
            }
         }
         sw[0][lane] = u;
         sw[1][lane] = v;
      }
      __syncthreads();
      uint32_t ec = carry[0] + (warp ? sw[0][warp - 1] : 0u) + xc - tc;
      uint32_t ei = carry[1] + (warp ? sw[1][warp - 1] : 0u) + xi - ti;
#pragma unroll
      for (int j = 0; j < kScanPer; ++j)
      {
         const int k = kb + j;
         if (k < nKeys)
         {
            start[k] = ec;
            cursor[k] = ec;
            itemStart[k] = ei;
            for (uint32_t q = 0; q < it[j]; ++q)
               itemKey[ei + q] = static_cast<uint32_t>(k);
         }
         ec += c[j];
         ei += it[j];
      }
      __syncthreads();
      if (threadIdx.x == 1023)
      {
         carry[0] = ec;
         carry[1] = ei;
      }
      __syncthreads();
   }
   if (threadIdx.x == 0)
   {
      itemStart[nKeys] = carry[1];
      ctr[0] = carry[1];
      ctr[1] = 0;
   }
}

// ------------------------------------------------------------------------------------------------ 3. lists
// An emitter as the contribution pass stages it; the lists hold these records in group order.
struct CStage
{
   double photons;
   double wx[4], wy[4];
   uint32_t g;
   int bx, by, plane;
};

__global__ void ContribScatterKernel(uint32_t n, const SplatRec* __restrict__ rec, const int4* __restrict__ grec,
                                     uint32_t* __restrict__ cursor, CStage* __restrict__ stage)
{
   const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
   const bool valid = g < n && grec[g].z >= 0;
   const int key = valid ? rec[g].key : 0;
   const unsigned vm = __ballot_sync(0xffffffffu, valid);
   if (!valid)
      return;
   const int lane = threadIdx.x & 31;
   const unsigned peers = __match_any_sync(vm, key);
   const int leader = __ffs(peers) - 1;
   uint32_t base = 0;
   if (lane == leader)
      base = atomicAdd(&cursor[key], static_cast<uint32_t>(__popc(peers)));
   base = __shfl_sync(peers, base, leader);
   const SplatRec& r = rec[g];
   CStage s;
   s.photons = r.photons;
#pragma unroll
   for (int k = 0; k < 4; ++k)
   {
      s.wx[k] = r.wx[k];
      s.wy[k] = r.wy[k];
   }
   s.g = g;
   s.bx = r.bx;
   s.by = r.by;
   s.plane = r.plane;
   stage[base + __popc(peers & ((1u << lane) - 1u))] = s;
}

// ------------------------------------------------------------------------------------------------ 4. contributions
struct ContribArgs
{
   KeyMap km;
   Kernels K;
   const uint32_t* count;
   const uint32_t* start;
   const uint32_t* itemStart;
   const uint32_t* itemKey;
   const CStage* stage;  // the emitters in group order
   uint32_t* ctr;        // [0] work items, [1] the next item
   float* contrib;       // emitter g's square at contrib[g S ..]
   uint32_t S;
};

// The reference's row = 0; row += wx[i] B; sum += wy[j] row over NT x NT taps held in registers, started from the
// first product (the same values; at most the sign of a zero partial sum differs, which the pixel's float add cannot
// see). Taps outside the bw x bw array are the layout's zero margin where the reference skips them.
template <int NT>
__device__ __forceinline__ double RegisterTaps(const double (&t)[4][4], const CStage& e)
{
   double row[NT];
#pragma unroll
   for (int j = 0; j < NT; ++j)
   {
      double r = e.wx[0] * t[j][0];
#pragma unroll
      for (int i = 1; i < NT; ++i)
         r += e.wx[i] * t[j][i];
      row[j] = r;
   }
   double sum = e.wy[0] * row[0];
#pragma unroll
   for (int j = 1; j < NT; ++j)
      sum += e.wy[j] * row[j];
   return sum;
}

// Any tap origin, from the row-major float64 sums with the reference's bounds (the misc group).
__device__ __forceinline__ double BoundedTaps(const KernelView& kv, const CStage& e, int nt, int dx, int dy)
{
   const int os = kv.os, off = os - 1, bw = kv.bw;
   const long long r0 = static_cast<long long>(e.by) + static_cast<long long>(dy) * os + off;
   const long long c0 = static_cast<long long>(e.bx) + static_cast<long long>(dx) * os + off;
   const double* B = kv.sums64 + static_cast<size_t>(e.plane) * bw * bw;
   double sum = 0.0;
   for (int j = 0; j < nt; ++j)
   {
      const long long r = r0 + j;
      if (r < 0 || r >= bw)
         continue;
      double row = 0.0;
      for (int i = 0; i < nt; ++i)
      {
         const long long c = c0 + i;
         if (c >= 0 && c < bw)
            row += e.wx[i] * __ldg(B + static_cast<size_t>(r) * bw + static_cast<size_t>(c));
      }
      sum += e.wy[j] * row;
   }
   return sum;
}

__device__ __forceinline__ bool HaloKeeps(const KernelView& kv, int plane, int dx, int dy)
{
   if (!kv.spanLo)
      return true;
   const int cr = kv.camRad, row = plane * (2 * cr + 1) + dy + cr;
   return dx >= kv.spanLo[row] && dx <= kv.spanHi[row];
}

template <int NT>
__device__ __forceinline__ void GroupContrib(const ContribArgs& a, const KernelView& kv, const CStage* sE, int cnt,
                                             int plane, int bx, int by, int p, int dx, int dy, bool active)
{
   const int os = kv.os, ext = kv.nb * os, span = kv.camRad * os;
   const int R = by + os - 1 + kv.padLo, C = bx + os - 1 + kv.padLo;
   const bool fits = kv.phase && R - span >= 0 && R + span + NT - 1 < ext && C - span >= 0 &&
                     C + span + NT - 1 < ext;
   if (!fits)
   {
      for (int k = 0; k < cnt; ++k)
         if (active)
            a.contrib[static_cast<size_t>(sE[k].g) * a.S + p] =
               static_cast<float>(sE[k].photons * BoundedTaps(kv, sE[k], NT, dx, dy));
      return;
   }
   double t[4][4];
   const int nb = kv.nb, nb2 = nb * nb;
   const double* base = kv.phase + static_cast<size_t>(plane) * os * os * nb2 + (active ? dy * nb + dx : 0);
#pragma unroll
   for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int i = 0; i < NT; ++i)
         t[j][i] = __ldg(base + ((R + j) % os * os + (C + i) % os) * nb2 + ((R + j) / os) * nb + (C + i) / os);
   float* out = a.contrib + p;
   // two emitters per step: independent FP64 chains in flight
   int k = 0;
   for (; k + 1 < cnt; k += 2)
   {
      const CStage& e0 = sE[k];
      const CStage& e1 = sE[k + 1];
      const double s0 = RegisterTaps<NT>(t, e0);
      const double s1 = RegisterTaps<NT>(t, e1);
      if (active)
      {
         out[static_cast<size_t>(e0.g) * a.S] = static_cast<float>(e0.photons * s0);
         out[static_cast<size_t>(e1.g) * a.S] = static_cast<float>(e1.photons * s1);
      }
   }
   if (k < cnt && active)
      out[static_cast<size_t>(sE[k].g) * a.S] = static_cast<float>(sE[k].photons * RegisterTaps<NT>(t, sE[k]));
}

// The work item's key, first stage record, record count and pixel block (key -1: no items left).
__device__ __forceinline__ void FetchItem(const ContribArgs& a, int* info)
{
   const uint32_t item = atomicAdd(&a.ctr[1], 1u);
   int key = -1, first = 0, cnt = 0, pbi = 0;
   if (item < a.ctr[0])
   {
      key = static_cast<int>(a.itemKey[item]);
      const int pbs = a.km.pbs[SlotOfKey(a.km, key)];
      const uint32_t local = item - a.itemStart[key];
      pbi = static_cast<int>(local % pbs);
      const uint32_t chunk = local / pbs;
      first = static_cast<int>(a.start[key] + chunk * kE);
      cnt = static_cast<int>(min(static_cast<uint32_t>(kE), a.count[key] - chunk * kE));
   }
   info[0] = key;
   info[1] = first;
   info[2] = cnt;
   info[3] = pbi;
}

// blockDim.x = computing threads + one staging warp: while the others compute item i, the last warp fetches item
// i + 1 and stages its emitters into the other buffer.
__global__ void __launch_bounds__(kMaxCT + 32, kContribPerSm) ContribKernel(ContribArgs a)
{
   __shared__ CStage sE[2][kE];
   __shared__ int sInfo[2][4];
   const int nc = static_cast<int>(blockDim.x) - 32;   // computing threads
   const bool stager = static_cast<int>(threadIdx.x) >= nc;
   const int sl = static_cast<int>(threadIdx.x) - nc;  // lane of the staging warp
   if (stager)
   {
      if (sl == 0)
         FetchItem(a, sInfo[0]);
      __syncwarp();
      for (int t = sl; t < sInfo[0][2]; t += 32)
         sE[0][t] = a.stage[sInfo[0][1] + t];
   }
   __syncthreads();
   for (int cur = 0;; cur ^= 1)
   {
      const int key = sInfo[cur][0], cnt = sInfo[cur][2], pbi = sInfo[cur][3];
      if (key < 0)
         return;
      if (stager)
      {
         if (sl == 0)
            FetchItem(a, sInfo[cur ^ 1]);
         __syncwarp();
         if (sInfo[cur ^ 1][0] >= 0)
            for (int t = sl; t < sInfo[cur ^ 1][2]; t += 32)
               sE[cur ^ 1][t] = a.stage[sInfo[cur ^ 1][1] + t];
      }
      else
      {
         const int slot = SlotOfKey(a.km, key);
         const KernelView& kv = a.K.k[slot];
         const int side = a.km.side[slot], cr = kv.camRad;
         const int p = pbi * nc + static_cast<int>(threadIdx.x);
         const bool inSquare = p < side * side;
         const int dx = inSquare ? p % side - cr : 0, dy = inSquare ? p / side - cr : 0;
         const int nt = TapsOf(kv);
         const int local = key - a.km.base[slot];
         const CStage* E = sE[cur];
         if (key == a.km.base[slot + 1] - 1)
         {
            // the misc group: every emitter with its own plane and tap origin
            for (int k = 0; k < cnt; ++k)
               if (inSquare && HaloKeeps(kv, E[k].plane, dx, dy))
                  a.contrib[static_cast<size_t>(E[k].g) * a.S + p] =
                     static_cast<float>(E[k].photons * BoundedTaps(kv, E[k], nt, dx, dy));
         }
         else
         {
            const int n1 = a.km.n1[slot], plane = local / (n1 * n1), cls = local % (n1 * n1);
            const int by = a.km.lo[slot] + cls / n1, bx = a.km.lo[slot] + cls % n1;
            const bool active = inSquare && HaloKeeps(kv, plane, dx, dy);
            if (nt == 4)
               GroupContrib<4>(a, kv, E, cnt, plane, bx, by, p, dx, dy, active);
            else if (nt == 2)
               GroupContrib<2>(a, kv, E, cnt, plane, bx, by, p, dx, dy, active);
            else
               GroupContrib<1>(a, kv, E, cnt, plane, bx, by, p, dx, dy, active);
         }
      }
      __syncthreads();
   }
}

// ------------------------------------------------------------------------------------------------ 5. gather
struct GStage
{
   const float* centre;   // the emitter's contributions at its square's centre pixel: contrib + g S + cr side + cr
   int x0, y0;            // (the first 16 bytes: what every pixel's test and address read)
   int cr, side;
   const int16_t* lo;     // halo cut of the emitter's plane, by dy + cr; null: the whole square
   const int16_t* hi;
};

struct GatherArgs
{
   const iscu_frame* frames;
   uint32_t nFrames;
   uint32_t nEm;
   const uint32_t* order;    // persistent form: frames, heaviest first
   uint32_t* counter;        // persistent form: the next work item
   const int4* grec;
   const float* contrib;
   uint32_t S;
   Kernels K;
   StaticView st;
   CameraView cam;
   uint32_t seed;
   float* photonsOut;
   uint16_t* aduOut;
};

// Stages one chunk of a frame's emitters whose square reaches the tile, in list order. Every thread calls it.
__device__ __forceinline__ int GatherStage(const GatherArgs& a, uint32_t start, uint32_t count, int tx0, int ty0,
                                           int tx1, int ty1, GStage* sG, int* sWarp, bool& anyHalo)
{
   const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
   bool keep = false;
   GStage s;
   if (static_cast<uint32_t>(t) < count)
   {
      const uint32_t g = start + t;
      const int4 gr = a.grec[g];
      if (gr.z >= 0)
      {
         const KernelView& kv = a.K.k[gr.z];
         const int cr = kv.camRad;
         keep = gr.x + cr >= tx0 && gr.x - cr <= tx1 && gr.y + cr >= ty0 && gr.y - cr <= ty1;
         s.x0 = gr.x;
         s.y0 = gr.y;
         s.cr = cr;
         s.side = 2 * cr + 1;
         s.centre = a.contrib + static_cast<size_t>(g) * a.S + static_cast<size_t>(cr) * s.side + cr;
         s.lo = kv.spanLo ? kv.spanLo + gr.w * s.side : nullptr;
         s.hi = kv.spanHi ? kv.spanHi + gr.w * s.side : nullptr;
      }
   }
   const unsigned ballot = __ballot_sync(0xffffffffu, keep);
   if (lane == 0)
      sWarp[warp] = __popc(ballot);
   anyHalo = __syncthreads_or(keep && s.lo != nullptr) != 0;
   int base = 0, total = 0;
#pragma unroll
   for (int w = 0; w < kGT / 32; ++w)
   {
      const int c = sWarp[w];
      base += w < warp ? c : 0;
      total += c;
   }
   if (keep)
      sG[base + __popc(ballot & ((1u << lane) - 1u))] = s;
   __syncthreads();
   return total;
}

__device__ __forceinline__ int GatherWarpList(const GStage* sG, int kept, int wx0, int wx1, int wy0, int wy1,
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
         const GStage& e = sG[k];
         hit = e.x0 + e.cr >= wx0 && e.x0 - e.cr <= wx1 && e.y0 + e.cr >= wy0 && e.y0 - e.cr <= wy1;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (hit)
         list[n + __popc(bal & ((1u << lane) - 1u))] = static_cast<uint16_t>(k);
      n += __popc(bal);
   }
   __syncwarp();
   return n;
}

// Whether the emitter's square and halo cut cover pixel (X, Y); the contribution's address if so.
template <bool kHalo>
__device__ __forceinline__ bool GatherCovers(const GStage& e, int X, int Y, const float*& src)
{
   const int dx = X - e.x0, dy = Y - e.y0, cr = e.cr;
   const unsigned w = static_cast<unsigned>(2 * cr);   // |dx|, |dy| <= cr as one unsigned compare each
   if (static_cast<unsigned>(dx + cr) > w || static_cast<unsigned>(dy + cr) > w)
      return false;
   if (kHalo && e.lo && (dx < e.lo[dy + cr] || dx > e.hi[dy + cr]))
      return false;
   src = e.centre + dy * e.side + dx;
   return true;
}

// A pixel's adds of the warp list's contributions, in list order, four loads in flight.
template <bool kHalo>
__device__ __forceinline__ float GatherAdds(const GStage* sG, const uint16_t* list, int n, int X, int Y, float acc)
{
   int m = 0;
   for (; m + 4 <= n; m += 4)
   {
      float v[4];
      bool in[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
         const float* src = nullptr;
         in[u] = GatherCovers<kHalo>(sG[list[m + u]], X, Y, src);
         v[u] = in[u] ? __ldg(src) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
         if (in[u])
            acc += v[u];
   }
   for (; m < n; ++m)
   {
      const float* src = nullptr;
      if (GatherCovers<kHalo>(sG[list[m]], X, Y, src))
         acc += __ldg(src);
   }
   return acc;
}

// Six CTAs per SM (40 registers; the noise chain spills a little): the gather's loads and the Knuth loops are latency-
// bound, and the extra warps hide more than the spills cost (C0 tiles 0.228 -> 0.211 ms, C3 4.60 -> 4.12 ms).
template <int TX, int TY, bool kNoise, bool kPersistent>
__global__ void __launch_bounds__(kGT, 6) GatherTilesKernel(GatherArgs a)
{
   static_assert(TX * TY == kGT, "one thread per pixel of the tile");
   static_assert(TX % 32 == 0 || 32 % TX == 0, "a warp covers a rectangle of the tile");
   __shared__ GStage sG[kGChunk];
   __shared__ uint16_t sList[kGT / 32][kGChunk];
   __shared__ int sWarp[kGT / 32];
   __shared__ uint32_t sItem;
   const int W = static_cast<int>(a.st.width), H = static_cast<int>(a.st.height);
   const uint32_t tilesX = (W + TX - 1) / TX, tilesY = (H + TY - 1) / TY, tilesPerFrame = tilesX * tilesY;
   const uint32_t total = a.nFrames * tilesPerFrame;
   const int warp = threadIdx.x >> 5;
   uint16_t* list = sList[warp];
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
      const uint32_t emCount = fr.em_start < a.nEm ? min(fr.em_count, a.nEm - fr.em_start) : 0u;
      const int tx0 = static_cast<int>(tile % tilesX) * TX, ty0 = static_cast<int>(tile / tilesX) * TY;
      const int X = tx0 + static_cast<int>(threadIdx.x % TX), Y = ty0 + static_cast<int>(threadIdx.x / TX);
      const int tx1 = min(tx0 + TX, W) - 1, ty1 = min(ty0 + TY, H) - 1;
      const bool inside = X < W && Y < H;
      const uint32_t i = static_cast<uint32_t>(Y) * a.st.width + static_cast<uint32_t>(X);
      const int wx0 = tx0 + wcx, wy0 = ty0 + wry;
      float acc = inside ? Background(a.st, i, fr.bg_scale) : 0.0f;
      for (uint32_t e0 = 0; e0 < emCount; e0 += kGChunk)
      {
         const uint32_t cnt = min(static_cast<uint32_t>(kGChunk), emCount - e0);
         bool anyHalo = false;
         const int kept = GatherStage(a, fr.em_start + e0, cnt, tx0, ty0, tx1, ty1, sG, sWarp, anyHalo);
         const int n = GatherWarpList(sG, kept, wx0, wx0 + wcw - 1, wy0, wy0 + wrh - 1, list);
         // the chunk's adds in list order; the halo test only where a staged emitter has a cut (the same for the CTA)
         if (inside)
            acc = anyHalo ? GatherAdds<true>(sG, list, n, X, Y, acc) : GatherAdds<false>(sG, list, n, X, Y, acc);
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

using GatherFn = void (*)(GatherArgs);
template <bool kNoise, bool kPersistent>
GatherFn GatherTile(int tile)
{
   switch (tile)
   {
   case 0: return GatherTilesKernel<16, 16, kNoise, kPersistent>;
   case 1: return GatherTilesKernel<32, 8, kNoise, kPersistent>;
   default: return GatherTilesKernel<8, 32, kNoise, kPersistent>;
   }
}
constexpr int kTileW[3] = {16, 32, 8}, kTileH[3] = {16, 8, 32};

} // namespace

namespace {

struct ContribGeometry
{
   KeyMap km = {};
   int nKeys = 0, ct = 32;
   size_t S = 1;
};

ContribGeometry GeometryOf(const iscu_ctx* ctx)
{
   ContribGeometry G;
   int maxS2 = 1;
   for (int s = 0; s < ISCU_MAX_KERNELS; ++s)
   {
      G.km.base[s] = G.nKeys;
      const KernelSlot& k = ctx->kernels[s];
      if (!k.valid)
         continue;
      const int cr = k.halfOv / k.os, side = 2 * cr + 1;
      G.km.side[s] = side;
      G.km.n1[s] = k.os + 4;
      G.km.lo[s] = k.halfOv - k.os - 2;
      G.nKeys += k.nz * G.km.n1[s] * G.km.n1[s] + 1;
      maxS2 = std::max(maxS2, side * side);
   }
   G.km.base[ISCU_MAX_KERNELS] = G.nKeys;
   const int blocks = (maxS2 + kMaxCT - 1) / kMaxCT;
   G.ct = std::min(kMaxCT, ((maxS2 + blocks - 1) / blocks + 31) / 32 * 32);
   for (int s = 0; s < ISCU_MAX_KERNELS; ++s)
      G.km.pbs[s] = std::max(1, (G.km.side[s] * G.km.side[s] + G.ct - 1) / G.ct);
   G.S = static_cast<size_t>(maxS2);
   return G;
}

// An upper bound of the work items: every key's emitter chunks (one partial chunk per key at most) times the largest
// number of pixel blocks.
size_t MaxItems(const ContribGeometry& G, uint32_t nEm)
{
   int maxPbs = 1;
   for (int s = 0; s < ISCU_MAX_KERNELS; ++s)
      maxPbs = std::max(maxPbs, G.km.pbs[s]);
   return (static_cast<size_t>(nEm) / kE + static_cast<size_t>(G.nKeys) + 1) * static_cast<size_t>(maxPbs);
}

} // namespace

int ReserveContrib(iscu_ctx* ctx, uint32_t nEm, ContribScratch& sc)
{
   const ContribGeometry G = GeometryOf(ctx);
   if (ctx->contribLimit == 0)
   {
      size_t freeB = 0, totalB = 0;
      ISCU_CK(cudaMemGetInfo(&freeB, &totalB));
      ctx->contribLimit = totalB / 4;
   }
   const size_t contribBytes = static_cast<size_t>(nEm) * G.S * sizeof(float);
   if (contribBytes > ctx->contribLimit)
      return Fail(ISCU_ERR_LIMIT, "two-pass render: contributions of " + std::to_string(nEm) + " emitters need " +
                                     std::to_string(contribBytes >> 20) + " MiB, over the limit");
   const size_t n = std::max<uint32_t>(nEm, 1u);
   ISCU_CK(sc.rec.Reserve(n * sizeof(SplatRec)));
   ISCU_CK(sc.grec.Reserve(n * sizeof(int4)));
   ISCU_CK(sc.list.Reserve(n * sizeof(CStage)));
   ISCU_CK(sc.contrib.Reserve(std::max<size_t>(contribBytes, 16)));
   ISCU_CK(sc.keys.Reserve((4 * static_cast<size_t>(G.nKeys) + 1 + MaxItems(G, nEm)) * sizeof(uint32_t)));
   ISCU_CK(sc.ctr.Reserve(4 * sizeof(uint32_t)));
   return ISCU_OK;
}

int LaunchContribRender(iscu_ctx* ctx, int tileConfig, const iscu_emitter* ems, uint32_t nEm,
                        const iscu_frame* frames, uint32_t nFrames, const CameraView* cam, uint32_t seed,
                        float* photons, uint16_t* adu, uint32_t* orderBuf, ContribScratch& sc)
{
   if (nFrames == 0)
      return ISCU_OK;
   const int rcReserve = ReserveContrib(ctx, nEm, sc);
   if (rcReserve != ISCU_OK)
      return rcReserve;
   const ContribGeometry G = GeometryOf(ctx);
   const KeyMap& km = G.km;
   const int nKeys = G.nKeys, ct = G.ct;
   const size_t S = G.S;
   cudaEvent_t* marks = RenderMarks(ctx);
   if (marks)
      ISCU_CK(cudaEventRecord(marks[0], ctx->stream));
   uint32_t* count = sc.keys.as<uint32_t>();
   uint32_t* start = count + nKeys;
   uint32_t* cursor = start + nKeys;
   uint32_t* itemStart = cursor + nKeys;
   uint32_t* itemKey = itemStart + nKeys + 1;
   const Kernels K = KernelsOfCtx(ctx);
   if (nEm > 0)
   {
      if (nKeys > 0)
         ISCU_CK(cudaMemsetAsync(count, 0, static_cast<size_t>(nKeys) * sizeof(uint32_t), ctx->stream));
      SetupArgs sa{ems, nEm, K, km, sc.rec.as<SplatRec>(), sc.grec.as<int4>(), count};
      ContribSetupKernel<<<(nEm + 255) / 256, 256, 0, ctx->stream>>>(sa);
      ISCU_CK_LAUNCH(ctx, "ContribSetupKernel");
      if (nKeys > 0)
      {
         ContribScanKernel<<<1, 1024, 0, ctx->stream>>>(km, count, start, cursor, itemStart, itemKey,
                                                        sc.ctr.as<uint32_t>());
         ISCU_CK_LAUNCH(ctx, "ContribScanKernel");
         ContribScatterKernel<<<(nEm + 255) / 256, 256, 0, ctx->stream>>>(nEm, sc.rec.as<SplatRec>(),
                                                                           sc.grec.as<int4>(), cursor,
                                                                           sc.list.as<CStage>());
         ISCU_CK_LAUNCH(ctx, "ContribScatterKernel");
         if (marks)
            ISCU_CK(cudaEventRecord(marks[1], ctx->stream));
         ContribArgs ca{km, K, count, start, itemStart, itemKey, sc.list.as<CStage>(), sc.ctr.as<uint32_t>(),
                        sc.contrib.as<float>(), static_cast<uint32_t>(S)};
         int perSm = 0;
         ISCU_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, ContribKernel, ct + 32, 0));
         ContribKernel<<<std::max(1, perSm) * ctx->smCount, ct + 32, 0, ctx->stream>>>(ca);
         ISCU_CK_LAUNCH(ctx, "ContribKernel");
      }
   }
   if (marks)
   {
      if (nEm == 0 || nKeys == 0)
         ISCU_CK(cudaEventRecord(marks[1], ctx->stream));
      ISCU_CK(cudaEventRecord(marks[2], ctx->stream));
   }
   GatherArgs ga;
   ga.frames = frames;
   ga.nFrames = nFrames;
   ga.nEm = nEm;
   ga.grec = sc.grec.as<int4>();
   ga.contrib = sc.contrib.as<float>();
   ga.S = static_cast<uint32_t>(S);
   ga.K = K;
   ga.st = ctx->Static();
   ga.cam = cam ? *cam : CameraView();
   ga.seed = seed;
   ga.photonsOut = photons;
   ga.aduOut = cam ? adu : nullptr;
   const int tile = tileConfig % 3;
   const bool persistent = tileConfig / 3 == 1;
   const int tw = kTileW[tile], th = kTileH[tile];
   GatherFn fn = cam ? (persistent ? GatherTile<true, true>(tile) : GatherTile<true, false>(tile))
                     : (persistent ? GatherTile<false, true>(tile) : GatherTile<false, false>(tile));
   if (persistent)
   {
      int rc = LaunchFrameOrder(ctx, frames, nFrames, orderBuf);
      if (rc != ISCU_OK)
         return rc;
      ga.order = orderBuf;
      ga.counter = orderBuf + ((nFrames + 3) & ~3u);
      int perSm = 0;
      ISCU_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fn, kGT, 0));
      const uint32_t tiles = ((ga.st.width + tw - 1) / tw) * ((ga.st.height + th - 1) / th);
      const uint32_t grid = std::min<uint32_t>(static_cast<uint32_t>(std::max(1, perSm) * ctx->smCount),
                                               tiles * nFrames);
      fn<<<grid, kGT, 0, ctx->stream>>>(ga);
   }
   else
   {
      ga.order = nullptr;
      ga.counter = nullptr;
      const dim3 grid((ga.st.width + tw - 1) / tw, (ga.st.height + th - 1) / th, nFrames);
      fn<<<grid, kGT, 0, ctx->stream>>>(ga);
   }
   ISCU_CK_LAUNCH(ctx, "GatherTilesKernel");
   if (marks)
      ISCU_CK(cudaEventRecord(marks[3], ctx->stream));
   return ISCU_OK;
}

} // namespace iscu
