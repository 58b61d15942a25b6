// Split-precision chirp-Z on the 5th-generation tensor cores (tcgen05): the PSF library's two complex products as
// TF32 x 3 real GEMMs with float32 accumulation in tensor memory.
//
// Both passes of the reference's separable chirp-Z (ChirpZ.h:28-142; ZernikePsf.cpp:264-334) are products with the
// same DFT matrix A[p][q] = exp(i (kMin + q dk)(x0 + p dx)):
//   row pass     T   = A U        (T[p][m]  = sum_n A[p][n] U[n][m])
//   column pass  E^T = A T^T      (E[y][x]  = sum_m T[y][m] A[x][m])
// In real arithmetic each is one GEMM with the stacked operand  Ahat = [[Ar, -Ai], [Ai, Ar]]  (rows: the real and
// the imaginary part of each output index p; columns: the real and the imaginary part of each input index q), so a
// CTA keeps one A operand for both passes: M = 2P <= 128 rows, K = 2M <= 256, N = M (row pass) or P (column pass).
// Rows and columns are interleaved in groups of 16 -- row r = 32 g + 16 h + i is output p = 16 g + i, part h; column
// k = 32 j + 16 h' + c is input q = 16 j + c, part h' -- so one 32-wide K block holds 16 input indices' real and
// imaginary parts, and one warp's 32 TMEM lanes hold 16 outputs' real and imaginary parts.
//
// TF32 x 3: every operand x is split into hi = tf32(x) and lo = x - hi (read by the tensor cores as TF32); a product
// is hi*hi + hi*lo + lo*hi (the dropped lo*lo and the roundings are ~2^-21 relative), accumulated in float32 in TMEM.
// The pupil phasors come from float64 phases (the per-set phase tables) and are split in registers; the row-pass
// result is read from TMEM, split and written as the column pass's B operand; |E|^2 and the plane's sum-1
// normalization finish in registers.
//
// The kernel (CztTf32x3Kernel, below) is persistent and warp-specialized: producer warps build the pupil operand, a
// copy thread streams the DFT operand with bulk copies, two threads issue the MMAs (row passes, column passes) and
// four warps drain TMEM; the roles meet only at mbarriers with bounded waits.

#include "iscu_internal.h"
#include "psf_common.cuh"
#include "tcgen05.cuh"

#include <algorithm>
#include <vector>

namespace iscu {

namespace {

using namespace tc;

constexpr int kThreads = 512;
constexpr int kRows = 128;             // UMMA M (2P rows, padded)
constexpr int kBlockBytes = 128 * 128; // one operand K block: 128 rows x 32 TF32 (128 B per row)

// ------------------------------------------------------------------------------------------ PTX helpers

// TF32 rounding (to nearest, ties away from zero: cvt.rna.tf32.f32) on the integer pipe: adding half a TF32 unit in
// the last place to the magnitude bits and clearing the 13 bits TF32 drops rounds the magnitude half away from zero,
// the carry moving into the exponent where it must (finite inputs).
__device__ __forceinline__ float ToTf32(float x)
{
   return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// hi = tf32(x), lo = x - hi (exact in float32; the tensor cores read its TF32 part, truncated: |x - hi - lo_tf32| <
// 2^-21 |x|)
__device__ __forceinline__ void Split(float x, float& hi, float& lo)
{
   hi = ToTf32(x);
   lo = x - hi;
}

// Instruction descriptor, kind::tf32: D float32, A and B TF32, both K-major, M x N.
__host__ __device__ constexpr uint32_t InstrDesc(int M, int N)
{
   return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
          (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void Mma(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc, uint32_t accum)
{
   asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dTmem),
                "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accum));
}

// Byte offset of element (row, col) (col: TF32 index 0..31 within the K block) in a swizzled K block.
__device__ __forceinline__ uint32_t SwOff(int row, int col)
{
   return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((((col >> 2) ^ (row & 7)) & 7) << 4) +
                                ((col & 3) << 2));
}

// ------------------------------------------------------------------------------------------ the stacked operand
// Ahat for one set, already split, in K-block order and in the shared-memory image the MMA reads (128-byte-swizzled
// K-major atoms): [kb][hi, lo][16 KB image of 128 rows x 32 TF32], so one 32 KB bulk copy stages a K block.
// P <= 64 outputs, M <= 128 inputs (M % 16 == 0); rows beyond 2P and columns beyond 2M are zero.
__global__ void AhatKernel(const float2* __restrict__ A, int M, int P, float* __restrict__ Ahat)
{
   const int s = blockIdx.y;
   const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (kb, row, col)
   const int nKb = 8;
   if (e >= nKb * kRows * 32)
      return;
   const int kb = e / (kRows * 32), row = (e / 32) % kRows, col = e % 32;
   const int g = row >> 5, h = (row >> 4) & 1, i = row & 15;
   const int p = 16 * g + i;
   const int hp = col >> 4, q = 16 * kb + (col & 15);
   float v = 0.f;
   if (p < P && q < M)
   {
      const float2 a = A[(static_cast<size_t>(s) * P + p) * M + q];
      // [[Ar, -Ai], [Ai, Ar]]: output part h, input part hp
      v = h == 0 ? (hp == 0 ? a.x : -a.y) : (hp == 0 ? a.y : a.x);
   }
   float hi, lo;
   Split(v, hi, lo);
   unsigned char* base = reinterpret_cast<unsigned char*>(Ahat) +
                         (static_cast<size_t>(s) * nKb + kb) * 2 * kBlockBytes;
   *reinterpret_cast<float*>(base + SwOff(row, col)) = hi;
   *reinterpret_cast<float*>(base + kBlockBytes + SwOff(row, col)) = lo;
}

// The pupil's phase table for the split-precision kernel: per set and sample (base, opd3F) with
// base = k0 opd1 + (zernike + mask) and the defocus term's obliquity opd3F (ZernikePsf.cpp:240-248), so a PSF's
// phase is base + (k0 ni dti) opd3F: one float64 multiply-add before the reduction mod 2 pi. opd3F < 0 outside the
// aperture.
__global__ void PhaseTableKernel(const SetParams* __restrict__ sets, const double3* __restrict__ tables, int MM,
                                 double2* __restrict__ out)
{
   const int s = blockIdx.y;
   const int m = blockIdx.x * blockDim.x + threadIdx.x;
   if (m >= MM)
      return;
   const double3 t = tables[static_cast<size_t>(s) * MM + m];
   out[static_cast<size_t>(s) * MM + m] = t.y < 0.0 ? make_double2(0.0, -1.0)
                                                    : make_double2(sets[s].k0 * t.x + t.z, t.y);
}

// ------------------------------------------------------------------------------------------ the fused kernel
struct TcParams
{
   const SetParams* sets;
   const double2* phase;     // [set][M * M] (base, opd3F)
   const float* ahat;
   const PsfItem* items;
   float* out;
   int* error;
   int nPsf, M, P, normalize;
};

constexpr int kAStages = 3;                        // Ahat K blocks in flight, in MMA order (both passes)
constexpr int kRowStages = 3;                      // row-pass B blocks (pupil phasors)
constexpr int kColStages = 2;                      // column-pass B blocks (T, split)
constexpr int kStageBytes = 2 * kBlockBytes;       // an A or row-pass B block: hi and lo images of 128 rows
constexpr int kColStageBytes = kBlockBytes;        // a column-pass B block: hi and lo images of 64 rows
// Warp roles. Warps share an SM sub-partition (scheduler) when equal mod 4: the MMA warp's (0) holds no producer.
constexpr int kDrainWarps = 4;                     // warps 0-3, one per TMEM lane quadrant
constexpr int kMmaWarp = 4;                        // lane 0 issues the row-pass MMAs
constexpr int kLoadWarp = 8;                       // lane 0 issues the Ahat copies
constexpr int kColMmaWarp = 12;                    // lane 0 issues the column-pass MMAs
constexpr int kProducerWarps = 9;                  // warps 5-7, 9-11, 13-15 make the pupil phasors
constexpr int kProducerThreads = 32 * kProducerWarps;
constexpr int kItemsPerBlock = 512;                // (pupil column, 4 pupil rows) items of one row-pass block
constexpr int kItemRounds = (kItemsPerBlock + kProducerThreads - 1) / kProducerThreads;

// A producer warp's index 0..8 (warps 5-7, 9-11, 13-15).
__device__ __forceinline__ int ProducerIndex(int warp) { return warp - 5 - (warp >= 9) - (warp >= 13); }
constexpr int kTmemRow = 0;                        // T of PSF j: columns [128 (j % 2), +128)
constexpr int kTmemCol = 256;                      // E of PSF j: columns [256 + 64 (j % 2), +64)
constexpr int kSetCache = 96;                      // PSFs whose set and defocus factor are staged in shared memory

struct Shared
{
   uint64_t aFull[kAStages], aEmpty[kAStages];
   uint64_t rowFull[kRowStages], rowEmpty[kRowStages];
   uint64_t colFull[kColStages], colEmpty[kColStages];
   uint64_t rowDone[2], colDone[2], tFree[2], eFree[2], red[2];
   uint64_t final[2];
   double sum[2][kDrainWarps];
   double aDef[kSetCache];   // k0 ni (ti - ti0) of the CTA's j-th PSF, j < kSetCache
   int set[kSetCache];       // its set
   uint32_t tmemSlot;
   int err;
};
constexpr size_t kSmemBytes = static_cast<size_t>(kAStages + kRowStages) * kStageBytes +
                              static_cast<size_t>(kColStages) * kColStageBytes + sizeof(Shared) + 1024;

// Per CTA, persistent over a contiguous run of PSFs (neighbours in the item list usually share their request set),
// warp-specialized; the roles meet only at mbarriers:
//   producers (warps 5-7, 9-11, 13-15): per row-pass K block the pupil phasors of 16 pupil rows (float64 phase,
//     reduced by quarter turns, float32 sine and cosine, TF32 hi/lo split) into a row-B stage -> rowFull;
//   the copy thread (warp 8, lane 0): the Ahat K blocks by bulk copy into the A ring, in the MMA order, each once the
//     MMAs that used the stage kAStages slots earlier are done (aEmpty);
//   the MMA threads (warp 4 the row passes R(j), warp 12 the column passes C(j), each lane 0): the Ahat order is R(0),
//     then per PSF j >= 1 R(j) and C(j - 1) K block by K block, then C(n - 1), so the column pass of one PSF runs
//     beside the row pass of the next; when PSFs j and j - 1 share their set, one Ahat copy serves both blocks (its
//     stage frees when both threads' MMAs are done). Per K block 12 MMAs (hi*hi, hi*lo, lo*hi over 4 K steps);
//     commits free the stages and mark a pass done (rowDone / colDone);
//   drain warps (0-3, one TMEM lane quadrant each): T of PSF j from TMEM, split, into col-B stages -> colFull (then
//     tFree: T's columns may take PSF j + 2); then E of PSF j: |E|^2, the plane sum, the normalized plane (eFree).
// T and E are double-buffered in TMEM (512 columns). Every wait is bounded (kWaitNs) and also ends when another role
// has failed (Shared::err); a failed CTA stops issuing, waits for its copies and MMAs in flight, frees TMEM and
// reports through prm.error.
__global__ void __launch_bounds__(kThreads, 1) CztTf32x3Kernel(TcParams prm)
{
   extern __shared__ __align__(1024) unsigned char smemRaw[];
   unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
   unsigned char* sA = smem;                                            // [kAStages] x 32 KB
   unsigned char* sRowB = sA + kAStages * kStageBytes;                  // [kRowStages] x 32 KB
   unsigned char* sColB = sRowB + kRowStages * kStageBytes;             // [kColStages] x 16 KB
   Shared* sh = reinterpret_cast<Shared*>(sColB + kColStages * kColStageBytes);
   volatile int* err = &sh->err;

   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   const int M = prm.M, P = prm.P, nKb = M / 16;
   // this CTA's PSFs: psf0 .. psf0 + nLocal - 1
   const int perCta = prm.nPsf / static_cast<int>(gridDim.x), extra = prm.nPsf % static_cast<int>(gridDim.x);
   const int cta = static_cast<int>(blockIdx.x);
   const int psf0 = cta * perCta + min(cta, extra), nLocal = perCta + (cta < extra ? 1 : 0);
   auto psfOf = [&](int j) { return psf0 + j; };

   if (warp == 0)
   {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(&sh->tmemSlot)),
                   "r"(512));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   if (tid == 0)
   {
      for (int s = 0; s < kAStages; ++s)
      {
         MbarInit(&sh->aFull[s], 1);
         MbarInit(&sh->aEmpty[s], 2);   // the row-pass and the column-pass MMA threads
      }
      for (int s = 0; s < kRowStages; ++s)
      {
         MbarInit(&sh->rowFull[s], kProducerWarps);
         MbarInit(&sh->rowEmpty[s], 1);
      }
      for (int s = 0; s < kColStages; ++s)
      {
         MbarInit(&sh->colFull[s], kDrainWarps);
         MbarInit(&sh->colEmpty[s], 1);
      }
      for (int s = 0; s < 2; ++s)
      {
         MbarInit(&sh->rowDone[s], 1);
         MbarInit(&sh->colDone[s], 1);
         MbarInit(&sh->tFree[s], kDrainWarps);
         MbarInit(&sh->eFree[s], kDrainWarps);
         MbarInit(&sh->red[s], kDrainWarps);
      }
      MbarInit(&sh->final[0], 1);
      MbarInit(&sh->final[1], 1);
      sh->err = 0;
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   for (int j = tid; j < nLocal && j < kSetCache; j += kThreads)
   {
      const PsfItem it = prm.items[psfOf(j)];
      sh->set[j] = it.set;
      sh->aDef[j] = prm.sets[it.set].k0 * prm.sets[it.set].ni * it.dtiM;
   }
   TcFenceBefore();
   __syncthreads();
   TcFenceAfter();
   const uint32_t tmem = sh->tmemSlot;
   bool ok = true;
   auto setOf = [&](int j) { return j < kSetCache ? sh->set[j] : prm.items[psfOf(j)].set; };

   if (warp > kMmaWarp && warp != kLoadWarp && warp != kColMmaWarp)
   {
      // ---------------------------------------------------------------- producers: row-pass B blocks
      // A thread's work per row-pass block: items ptid + r kProducerThreads (pupil column m, pupil rows n .. n + 3).
      // The table entries of the next block are in flight while a block computes.
      const int ptid = 32 * ProducerIndex(warp) + lane;
      auto load = [&](const double2* tab, int kb, double2 (*dst)[4]) {
#pragma unroll
         for (int r = 0; r < kItemRounds; ++r)
         {
            const int item = ptid + r * kProducerThreads, m = item & 127, n = 16 * kb + 4 * (item >> 7);
            const bool in = item < kItemsPerBlock && m < M;
#pragma unroll
            for (int c = 0; c < 4; ++c)
               dst[r][c] = in ? tab[static_cast<size_t>(n + c) * M + m] : make_double2(0.0, -1.0);
         }
      };
      // the defocus factor of PSF j (staged in shared memory for j < kSetCache)
      auto aDefOf = [&](int j) {
         if (j < kSetCache)
            return sh->aDef[j];
         const PsfItem it = prm.items[psfOf(j)];
         return prm.sets[it.set].k0 * prm.sets[it.set].ni * it.dtiM;
      };
      double2 nxt[kItemRounds][4];
      load(prm.phase + static_cast<size_t>(setOf(0)) * M * M, 0, nxt);
      uint32_t rowCount = 0;
      for (int j = 0; j < nLocal && ok; ++j)
      {
         const double aDef = aDefOf(j);
         const double2* tab = prm.phase + static_cast<size_t>(setOf(j)) * M * M;
         const double2* tabNext = j + 1 < nLocal ? prm.phase + static_cast<size_t>(setOf(j + 1)) * M * M : tab;
         for (int kb = 0; kb < nKb; ++kb, ++rowCount)
         {
            double2 cur[kItemRounds][4];
#pragma unroll
            for (int r = 0; r < kItemRounds; ++r)
#pragma unroll
               for (int c = 0; c < 4; ++c)
                  cur[r][c] = nxt[r][c];
            if (kb + 1 < nKb)
               load(tab, kb + 1, nxt);
            else if (j + 1 < nLocal)
               load(tabNext, 0, nxt);
            const int rs = static_cast<int>(rowCount % kRowStages);
            ok = __all_sync(0xffffffffu, MbarWait(&sh->rowEmpty[rs], ((rowCount / kRowStages) & 1u) ^ 1u, err));
            if (!ok)
               break;
            unsigned char* b = sRowB + rs * kStageBytes;
#pragma unroll
            for (int r = 0; r < kItemRounds; ++r)
            {
               const int item = ptid + r * kProducerThreads;
               if (item < kItemsPerBlock)
               {
                  const int m = item & 127, nl = 4 * (item >> 7);
                  float rh[4], rl[4], ih[4], il[4];
#pragma unroll
                  for (int c = 0; c < 4; ++c)
                  {
                     const float2 u = TablePhasor(cur[r][c], aDef);
                     Split(u.x, rh[c], rl[c]);
                     Split(u.y, ih[c], il[c]);
                  }
                  // B[m][nl + c]: the real part of pupil row 16 kb + nl + c; B[m][16 + nl + c]: the imaginary part
                  *reinterpret_cast<float4*>(b + SwOff(m, nl)) = make_float4(rh[0], rh[1], rh[2], rh[3]);
                  *reinterpret_cast<float4*>(b + SwOff(m, 16 + nl)) = make_float4(ih[0], ih[1], ih[2], ih[3]);
                  *reinterpret_cast<float4*>(b + kBlockBytes + SwOff(m, nl)) = make_float4(rl[0], rl[1], rl[2], rl[3]);
                  *reinterpret_cast<float4*>(b + kBlockBytes + SwOff(m, 16 + nl)) =
                     make_float4(il[0], il[1], il[2], il[3]);
               }
            }
            FenceProxyAsync();
            __syncwarp();
            if (lane == 0)
               MbarArrive(&sh->rowFull[rs]);
         }
      }
   }
   else if (warp == kLoadWarp)
   {
      // ---------------------------------------------------------------- the Ahat copies, in MMA order
      if (lane == 0 && nLocal > 0)
      {
         int slot = 0;
         int last[kAStages] = {-1, -1, -1};   // the latest slot copied into each stage
         for (int seg = 0; seg <= nLocal && ok; ++seg)
         {
            const int jR = seg < nLocal ? seg : -1, jC = seg - 1;
            const bool shared = jR >= 0 && jC >= 0 && setOf(jR) == setOf(jC);
            for (int kb = 0; kb < nKb && ok; ++kb)
               for (int part = 0; part < 2 && ok; ++part)
               {
                  const int jj = part == 0 ? jR : jC;
                  if (jj < 0 || (part == 1 && shared))
                     continue;
                  const int st = slot % kAStages;
                  if (slot >= kAStages)   // the MMAs of the slot kAStages earlier are done with the stage
                     ok = MbarWait(&sh->aEmpty[st], static_cast<uint32_t>(slot / kAStages - 1) & 1u, err);
                  if (!ok)
                     break;
                  MbarExpectTx(&sh->aFull[st], kStageBytes);
                  BulkLoad(sA + st * kStageBytes,
                           prm.ahat + (static_cast<size_t>(setOf(jj)) * 8 + kb) * (kStageBytes / 4), kStageBytes,
                           &sh->aFull[st]);
                  last[st] = slot++;
               }
         }
         if (!ok)
         {
            *err = 1;
            for (int st = 0; st < kAStages; ++st)   // the copies in flight land before the CTA frees its memory
               if (last[st] >= 0)
                  MbarWait(&sh->aFull[st], static_cast<uint32_t>(last[st] / kAStages) & 1u, nullptr);
         }
      }
   }
   else if (warp == kMmaWarp || warp == kColMmaWarp)
   {
      // ---------------------------------------------------------------- the MMA threads
      // Warp 4 issues the row passes, warp 12 the column passes: their accumulators are apart in TMEM, so each
      // thread's waits and bookkeeping overlap the other's MMAs (one thread's queue of MMAs is short).
      const int mine = warp == kMmaWarp ? 0 : 1;
      if (lane == 0 && nLocal > 0)
      {
         const bool row = mine == 0;
         const uint32_t idesc = row ? InstrDesc(kRows, M) : InstrDesc(kRows, 64);
         uint32_t count = 0;   // this thread's K blocks so far (its B ring's position)
         int slot = 0;
         for (int seg = 0; seg <= nLocal && ok; ++seg)
         {
            const int jR = seg < nLocal ? seg : -1, jC = seg - 1;
            const bool shared = jR >= 0 && jC >= 0 && setOf(jR) == setOf(jC);
            for (int kb = 0; kb < nKb && ok; ++kb)
               for (int part = 0; part < 2 && ok; ++part)
               {
                  const int jj = part == 0 ? jR : jC;
                  if (jj < 0)
                     continue;
                  const int st = slot % kAStages;
                  const uint32_t aParity = static_cast<uint32_t>(slot / kAStages) & 1u;
                  if (!shared || part == 1)   // the next block takes the next Ahat slot
                     ++slot;
                  if (part != mine)
                     continue;
                  // K block kb of PSF jj's pass on Ahat stage st
                  const uint32_t use = static_cast<uint32_t>(jj >> 1) & 1u;
                  if (kb == 0)   // the accumulator's TMEM columns are free (PSF jj - 2 is past them)
                     ok = MbarWait(row ? &sh->tFree[jj & 1] : &sh->eFree[jj & 1], use ^ 1u, err, false);
                  uint64_t* full;
                  uint64_t* empty;
                  uint32_t parity, bH, bL, d;
                  if (row)
                  {
                     const int rs = static_cast<int>(count % kRowStages);
                     full = &sh->rowFull[rs];
                     empty = &sh->rowEmpty[rs];
                     parity = (count / kRowStages) & 1u;
                     bH = SmemAddr(sRowB + rs * kStageBytes);
                     bL = bH + kBlockBytes;
                     d = tmem + kTmemRow + 128u * static_cast<uint32_t>(jj & 1);
                  }
                  else
                  {
                     const int cs = static_cast<int>(count % kColStages);
                     full = &sh->colFull[cs];
                     empty = &sh->colEmpty[cs];
                     parity = (count / kColStages) & 1u;
                     bH = SmemAddr(sColB + cs * kColStageBytes);
                     bL = bH + kColStageBytes / 2;
                     d = tmem + kTmemCol + 64u * static_cast<uint32_t>(jj & 1);
                  }
                  ok = ok && MbarWait(&sh->aFull[st], aParity, err, false);
                  ok = ok && MbarWait(full, parity, err, false);
                  if (!ok)
                     break;
                  TcFenceAfter();
                  const uint32_t aH = SmemAddr(sA + st * kStageBytes), aL = aH + kBlockBytes;
#pragma unroll
                  for (int kk = 0; kk < 4; ++kk)
                  {
                     const uint32_t off = kk * 32;   // 8 TF32 = 32 bytes along K
                     Mma(d, SmemDesc(aH + off), SmemDesc(bH + off), idesc, (kb == 0 && kk == 0) ? 0u : 1u);
                     Mma(d, SmemDesc(aH + off), SmemDesc(bL + off), idesc, 1u);
                     Mma(d, SmemDesc(aL + off), SmemDesc(bH + off), idesc, 1u);
                  }
                  Commit(empty);
                  Commit(&sh->aEmpty[st]);
                  if (!shared)   // the slot's only user arrives for both
                     Commit(&sh->aEmpty[st]);
                  if (kb == nKb - 1)
                     Commit(row ? &sh->rowDone[jj & 1] : &sh->colDone[jj & 1]);
                  ++count;
               }
         }
         if (!ok)
         {
            *err = 1;
            Commit(&sh->final[mine]);   // this thread's MMAs in flight finish before the CTA frees its TMEM
            MbarWait(&sh->final[mine], 0u, nullptr);
         }
      }
   }
   else if (warp < kDrainWarps)
   {
      // ---------------------------------------------------------------- drain warps
      // TMEM lane r = 32 w + 16 h + i of T holds row y = 16 w + i, part h (columns: the pupil column m); of E, output
      // x = 16 w + i, part h (columns: y).
      const int h = (lane >> 4) & 1, y = 16 * warp + (lane & 15), x = y;
      const uint32_t quad = static_cast<uint32_t>(32 * warp) << 16;
      uint32_t colCount = 0;
      for (int j = 0; j < nLocal && ok; ++j)
      {
         const uint32_t use = static_cast<uint32_t>(j >> 1) & 1u;
         ok = __all_sync(0xffffffffu, MbarWait(&sh->rowDone[j & 1], use, err));
         if (!ok)
            break;
         TcFenceAfter();
         for (int kb = 0; kb < nKb; ++kb, ++colCount)
         {
            const int cs = static_cast<int>(colCount % kColStages);
            ok = __all_sync(0xffffffffu, MbarWait(&sh->colEmpty[cs], ((colCount / kColStages) & 1u) ^ 1u, err));
            if (!ok)
               break;
            float v[16];
            TmemLoad16(tmem + quad + kTmemRow + 128u * static_cast<uint32_t>(j & 1) + 16u * kb, v);
            float hi[16], lo[16];
#pragma unroll
            for (int c = 0; c < 16; ++c)
               Split(y < P ? v[c] : 0.f, hi[c], lo[c]);
            // B[y][16 h + c] = part h of T[y][16 kb + c]
            unsigned char* b = sColB + cs * kColStageBytes;
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
               *reinterpret_cast<float4*>(b + SwOff(y, 16 * h + 4 * q)) =
                  make_float4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
               *reinterpret_cast<float4*>(b + kColStageBytes / 2 + SwOff(y, 16 * h + 4 * q)) =
                  make_float4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
            }
            FenceProxyAsync();
            __syncwarp();
            if (lane == 0)
               MbarArrive(&sh->colFull[cs]);
         }
         if (!ok)
            break;
         TcFenceBefore();
         __syncwarp();
         if (lane == 0)
            MbarArrive(&sh->tFree[j & 1]);
         // ------------------------------------------------ |E|^2, the plane sum, the normalized plane
         ok = __all_sync(0xffffffffu, MbarWait(&sh->colDone[j & 1], use, err));
         if (!ok)
            break;
         TcFenceAfter();
         float I[64];
         float part[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};   // eight float partial sums of 8 values each
#pragma unroll
         for (int c0 = 0; c0 < 64; c0 += 32)
         {
            float vv[32];
            TmemLoad32(tmem + quad + kTmemCol + 64u * static_cast<uint32_t>(j & 1) + c0, vv);
#pragma unroll
            for (int c = 0; c < 32; ++c)
            {
               const float o = __shfl_xor_sync(0xffffffffu, vv[c], 16);
               const float e = vv[c] * vv[c] + o * o;
               I[c0 + c] = e;
               if (c0 + c < P)
                  part[(c0 + c) >> 3] += e;
            }
         }
         double local = 0.0;
         if (lane < 16 && x < P)
#pragma unroll
            for (int k = 0; k < 8; ++k)
               local += static_cast<double>(part[k]);
         TcFenceBefore();
         __syncwarp();
         if (lane == 0)
            MbarArrive(&sh->eFree[j & 1]);
         double total = 0.0;
         if (prm.normalize)
         {
            for (int o = 16; o > 0; o >>= 1)
               local += __shfl_xor_sync(0xffffffffu, local, o);
            if (lane == 0)
            {
               sh->sum[j & 1][warp] = local;
               MbarArrive(&sh->red[j & 1]);
            }
            ok = __all_sync(0xffffffffu, MbarWait(&sh->red[j & 1], use, err));
            if (!ok)
               break;
            const volatile double* s = sh->sum[j & 1];
            total = s[0] + s[1] + s[2] + s[3];
         }
         // lanes 0-15 store rows y < 32 of column x, lanes 16-31 rows y >= 32; the plane times 1 / sum (the float
         // product is within an ulp or two of the float64 quotient)
         if (x < P)
         {
            float* plane = prm.out + static_cast<size_t>(psfOf(j)) * P * P;
            const float scale = (prm.normalize && total > 0.0) ? static_cast<float>(1.0 / total) : 1.0f;
            const int y0 = 32 * h;
#pragma unroll
            for (int c = 0; c < 32; ++c)
            {
               const int yy = y0 + c;
               const float e = h ? I[32 + c] : I[c];
               if (yy < P)
                  plane[static_cast<size_t>(yy) * P + x] = e * scale;
            }
         }
      }
   }
   if (!ok)
      *err = 1;
   TcFenceBefore();
   __syncthreads();
   TcFenceAfter();
   if (tid == 0 && *err)
      atomicExch(prm.error, 1);
   if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

} // namespace

bool Tf32x3Supports(int M, int P) { return M <= 128 && M % 16 == 0 && P <= 64 && P >= 1; }

size_t AhatBytes(int nSets) { return static_cast<size_t>(nSets) * 8 * kStageBytes; }

static_assert(kSmemBytes <= 227 * 1024, "the chirp-Z kernel's shared memory");

size_t SplitImageBytes(int method, int nSets)
{
   return method == ISCU_CZT_F16X3 ? AhatF16Bytes(nSets) : AhatBytes(nSets);
}

int BuildAhat(iscu_ctx* ctx, const float2* A, const SetParams* sets, const double3* tables, int nSets, int M, int P,
              int method, DevBuf& ahat)
{
   const bool f16 = method == ISCU_CZT_F16X3;
   if (f16 ? !F16x3Supports(M, P) : !Tf32x3Supports(M, P))
      return Fail(ISCU_ERR_ARG, std::string(f16 ? "f16x3" : "tf32x3") +
                                   " chirp-Z: needs pupil samples M <= 128 (a multiple of 16) and planes of at most "
                                   "64 x 64 (else use the fp32 method)");
   // the K-block images, then the phase tables (FP16 form: (tx, tx, ty, ty) float4 per pair of pupil rows, in
   // revolutions, the size of a float2 per sample; TF32 form: double2 in radians)
   const size_t images = SplitImageBytes(method, nSets);
   ISCU_CK(ahat.Reserve(images + static_cast<size_t>(nSets) * M * M * (f16 ? sizeof(float2) : sizeof(double2))));
   if (f16)
      return BuildAhatF16(ctx, A, sets, tables, nSets, M, P, ahat.as<unsigned char>());
   AhatKernel<<<dim3((8 * kRows * 32 + 255) / 256, nSets), 256, 0, ctx->stream>>>(A, M, P, ahat.as<float>());
   ISCU_CK_LAUNCH(ctx, "AhatKernel");
   PhaseTableKernel<<<dim3((M * M + 255) / 256, nSets), 256, 0, ctx->stream>>>(
      sets, tables, M * M, reinterpret_cast<double2*>(ahat.as<char>() + images));
   ISCU_CK_LAUNCH(ctx, "PhaseTableKernel");
   return ISCU_OK;
}

int LaunchCztTf32x3Core(iscu_ctx* ctx, const SetParams* sets, const float* ahat, int nSets, const PsfItem* items,
                        uint32_t nPsf, int M, int P, int normalize, float* out, int* dErr)
{
   const size_t smem = kSmemBytes;
   ISCU_CK(cudaFuncSetAttribute(CztTf32x3Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
   TcParams prm;
   prm.sets = sets;
   prm.phase = reinterpret_cast<const double2*>(reinterpret_cast<const char*>(ahat) + AhatBytes(nSets));
   prm.ahat = ahat;
   prm.items = items;
   prm.out = out;
   prm.error = dErr;
   prm.nPsf = static_cast<int>(nPsf);
   prm.M = M;
   prm.P = P;
   prm.normalize = normalize;
   const int grid = static_cast<int>(std::min<uint32_t>(nPsf, static_cast<uint32_t>(ctx->smCount)));
   CztTf32x3Kernel<<<grid, kThreads, smem, ctx->stream>>>(prm);
   ISCU_CK_LAUNCH(ctx, "CztTf32x3Kernel");
   return ISCU_OK;
}

int LaunchCztSplit(iscu_ctx* ctx, int method, const SetParams* sets, const double3* tables, const float2* A,
                   uint32_t nSets, const PsfItem* items, uint32_t nPsf, int M, int P, int normalize, float* out)
{
   DevBuf dAhat, dErr;
   int rc = BuildAhat(ctx, A, sets, tables, static_cast<int>(nSets), M, P, method, dAhat);
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(dErr.Reserve(sizeof(int)));
   ISCU_CK(cudaMemsetAsync(dErr.p, 0, sizeof(int), ctx->stream));
   rc = method == ISCU_CZT_F16X3
           ? LaunchCztF16x3Core(ctx, sets, dAhat.as<unsigned char>(), static_cast<int>(nSets), items, nPsf, M, P,
                                normalize, out, dErr.as<int>())
           : LaunchCztTf32x3Core(ctx, sets, dAhat.as<float>(), static_cast<int>(nSets), items, nPsf, M, P, normalize,
                                 out, dErr.as<int>());
   if (rc != ISCU_OK)
      return rc;
   int err = 0;
   ISCU_CK(cudaMemcpyAsync(&err, dErr.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   if (err)
      return Fail(ISCU_ERR_TIMEOUT, "split-precision chirp-Z: a tensor-core completion wait ran out");
   return ISCU_OK;
}

} // namespace iscu
