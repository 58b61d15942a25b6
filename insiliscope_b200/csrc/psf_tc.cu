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
// TF32 x 3: every operand x is split into hi = tf32(x) and lo = tf32(x - hi); a product is hi*hi + hi*lo + lo*hi
// (the dropped lo*lo and the roundings are ~2^-21 relative), accumulated in float32 in TMEM. The pupil phasors come
// from float64 phases (psf_common.cuh) and are split in registers; the row-pass result is read from TMEM, split and
// written as the column pass's B operand; |E|^2 and the plane's sum-1 normalization finish in registers.
//
// Per CTA (persistent over PSFs, 256 threads): operands staged in shared memory in the canonical 128-byte-swizzled
// K-major layout (8-row x 128-byte atoms, 1024-byte aligned), two stages for the A/B K blocks of the row pass; one
// thread issues tcgen05.mma (M = 128, K = 8 per instruction) and tcgen05.commit to an mbarrier per stage; warps 0-3
// read TMEM back with tcgen05.ld. Every mbarrier wait is bounded: on timeout the CTA records an error, stops issuing,
// frees its TMEM and returns.

#include "iscu_internal.h"
#include "psf_common.cuh"

#include <algorithm>
#include <vector>

namespace iscu {

namespace {

constexpr int kThreads = 512;
constexpr int kRows = 128;             // UMMA M (2P rows, padded)
constexpr int kBlockBytes = 128 * 128; // one operand K block: 128 rows x 32 TF32 (128 B per row)

// ------------------------------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t SmemAddr(const void* p)
{
   return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float ToTf32(float x)
{
   uint32_t r;
   asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
   return __uint_as_float(r);
}

// hi = tf32(x), lo = tf32(x - hi)
__device__ __forceinline__ void Split(float x, float& hi, float& lo)
{
   hi = ToTf32(x);
   lo = ToTf32(x - hi);
}

__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count));
}

__device__ __forceinline__ void FenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void TcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void TcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: canonical K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t SmemDesc(uint32_t addr)
{
   uint64_t d = 0;
   d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);          // start address
   d |= static_cast<uint64_t>(1u) << 16;                       // leading byte offset (unused for this layout)
   d |= static_cast<uint64_t>(1024u >> 4) << 32;               // stride byte offset: 8-row group pitch
   d |= static_cast<uint64_t>(1u) << 46;                       // descriptor version (sm_100)
   d |= static_cast<uint64_t>(2u) << 61;                       // layout: 128-byte swizzle
   return d;
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

__device__ __forceinline__ void Commit(uint64_t* bar)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(bar))
                : "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes into v[0..31] (thread = lane).
__device__ __forceinline__ void TmemLoad32(uint32_t taddr, float* v)
{
   uint32_t r[32];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int i = 0; i < 32; ++i)
      v[i] = __uint_as_float(r[i]);
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

// The pupil phasor of one sample from the phase table: float64 phase, reduced mod 2 pi, then the float32 sine and
// cosine of the reduced phase by the special-function unit (absolute error ~4e-7 over [-pi, pi]).
__device__ __forceinline__ float2 TablePhasor(double2 t, double a)
{
   if (t.y < 0.0)
      return make_float2(0.f, 0.f);
   const double ph = ReduceTwoPi(fma(a, t.y, t.x));
   float sn, cs;
   __sincosf(static_cast<float>(ph), &sn, &cs);
   return make_float2(cs, sn);
}

// ------------------------------------------------------------------------------------------ async copies
__device__ __forceinline__ void MbarExpectTx(uint64_t* bar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
                : "memory");
}

// A bulk copy global -> this CTA's shared memory (no multicast), completing `bytes` on the mbarrier.
__device__ __forceinline__ void BulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   SmemAddr(dst)),
                "l"(src), "r"(bytes), "r"(SmemAddr(bar))
                : "memory");
}

// 4 consecutive TMEM columns of this warp's 32 lanes into v[0..3].
__device__ __forceinline__ void TmemLoad4(uint32_t taddr, float* v)
{
   uint32_t r[4];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int i = 0; i < 4; ++i)
      v[i] = __uint_as_float(r[i]);
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
constexpr int kDrainWarps = 4;                     // warps 0-3, one per TMEM lane quadrant
constexpr int kMmaWarp = 4;                        // lane 0 issues the MMAs and the Ahat copies
constexpr int kFirstProducer = 5;                  // warps 5-15 make the pupil phasors
constexpr int kProducerThreads = kThreads - 32 * kFirstProducer;
constexpr int kItemsPerBlock = 1024;               // (pupil column, pair of pupil rows) items of one row-pass block
constexpr int kItemRounds = (kItemsPerBlock + kProducerThreads - 1) / kProducerThreads;
constexpr int kTmemRow = 0;                        // T of PSF j: columns [128 (j % 2), +128)
constexpr int kTmemCol = 256;                      // E of PSF j: columns [256 + 64 (j % 2), +64)
constexpr uint64_t kWaitNs = 4000000000ull;        // a wait gives up after 4 s

struct Shared
{
   uint64_t aFull[kAStages], aEmpty[kAStages];
   uint64_t rowFull[kRowStages], rowEmpty[kRowStages];
   uint64_t colFull[kColStages], colEmpty[kColStages];
   uint64_t rowDone[2], colDone[2], tFree[2], eFree[2], red[2];
   uint64_t final;
   double sum[2][kDrainWarps];
   uint32_t tmemSlot;
   int err;
};
constexpr size_t kSmemBytes = static_cast<size_t>(kAStages + kRowStages) * kStageBytes +
                              static_cast<size_t>(kColStages) * kColStageBytes + sizeof(Shared) + 1024;

__device__ __forceinline__ uint64_t GlobalNs()
{
   uint64_t t;
   asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
   return t;
}

// Waits for the phase of the given parity to complete. false after kWaitNs, or (err non-null) once *err is set.
__device__ __forceinline__ bool MbarWait(uint64_t* bar, uint32_t parity, const volatile int* err)
{
   const uint32_t a = SmemAddr(bar);
   uint64_t t0 = 0;
   for (unsigned it = 0;; ++it)
   {
      uint32_t done;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done)
                   : "r"(a), "r"(parity)
                   : "memory");
      if (done)
         return true;
      if ((it & 15) == 15)
      {
         if (err && *err)
            return false;
         const uint64_t now = GlobalNs();
         if (t0 == 0)
            t0 = now;
         else if (now - t0 > kWaitNs)
            return false;
      }
   }
}

__device__ __forceinline__ void MbarArrive(uint64_t* bar)
{
   asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar)) : "memory");
}

// 16 consecutive TMEM columns of this warp's 32 lanes into v[0..15].
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, float* v)
{
   uint32_t r[16];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int i = 0; i < 16; ++i)
      v[i] = __uint_as_float(r[i]);
}

// The CTA's j-th PSF.
__device__ __forceinline__ int PsfOf(int j) { return static_cast<int>(blockIdx.x) + j * static_cast<int>(gridDim.x); }

// The MMA order of a CTA's K blocks: R(0), R(1), C(0), R(2), C(1), ..., R(n - 1), C(n - 2), C(n - 1), each pass nKb
// blocks (R: row pass, C: column pass), so the column pass of one PSF runs on the tensor cores while the producers
// make the next PSFs' pupils. Block t -> its PSF j, its pass and K block kb.
__device__ __forceinline__ void JobOf(int t, int nKb, int nLocal, int& j, bool& row, int& kb)
{
   const int seg = t / nKb;
   kb = t % nKb;
   if (seg == 0)
   {
      j = 0;
      row = true;
      return;
   }
   const int u = seg - 1;
   if ((u & 1) == 0 && u / 2 + 1 < nLocal)
   {
      j = u / 2 + 1;
      row = true;
   }
   else
   {
      j = (u & 1) ? (u - 1) / 2 : nLocal - 1;
      row = false;
   }
}

// Per CTA, persistent over its PSFs (blockIdx.x + j gridDim.x), warp-specialized; the roles meet only at mbarriers:
//   producers (warps 5-15): per row-pass K block the pupil phasors of 16 pupil rows (float64 phase, reduced mod 2 pi,
//     SFU sine and cosine, TF32 hi/lo split) into a row-B stage -> rowFull;
//   the MMA thread (warp 4, lane 0): the Ahat K blocks by bulk copy into the A ring (two blocks ahead), and per K
//     block 12 MMAs (hi*hi, hi*lo, lo*hi over 4 K steps) in the MMA order of JobOf; commits free the stages and mark
//     a pass done (rowDone / colDone);
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
   const int nLocal = prm.nPsf > static_cast<int>(blockIdx.x)
                         ? (prm.nPsf - static_cast<int>(blockIdx.x) + static_cast<int>(gridDim.x) - 1) /
                              static_cast<int>(gridDim.x)
                         : 0;

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
         MbarInit(&sh->aEmpty[s], 1);
      }
      for (int s = 0; s < kRowStages; ++s)
      {
         MbarInit(&sh->rowFull[s], kThreads / 32 - kFirstProducer);
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
      MbarInit(&sh->final, 1);
      sh->err = 0;
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   TcFenceBefore();
   __syncthreads();
   TcFenceAfter();
   const uint32_t tmem = sh->tmemSlot;
   bool ok = true;

   if (warp >= kFirstProducer)
   {
      // ---------------------------------------------------------------- producers: row-pass B blocks
      const int ptid = tid - 32 * kFirstProducer;
      uint32_t rowCount = 0;
      for (int j = 0; j < nLocal && ok; ++j)
      {
         const PsfItem it = prm.items[PsfOf(j)];
         const double aDef = prm.sets[it.set].k0 * prm.sets[it.set].ni * it.dtiM;
         const double2* tab = prm.phase + static_cast<size_t>(it.set) * M * M;
         for (int kb = 0; kb < nKb; ++kb, ++rowCount)
         {
            const int rs = static_cast<int>(rowCount % kRowStages);
            ok = __all_sync(0xffffffffu, MbarWait(&sh->rowEmpty[rs], ((rowCount / kRowStages) & 1u) ^ 1u, err));
            if (!ok)
               break;
            double2 t[kItemRounds][2];
#pragma unroll
            for (int r = 0; r < kItemRounds; ++r)
            {
               const int item = ptid + r * kProducerThreads, m = item & 127, n = 16 * kb + 2 * (item >> 7);
               const bool in = item < kItemsPerBlock && m < M;
               t[r][0] = in ? tab[static_cast<size_t>(n) * M + m] : make_double2(0.0, -1.0);
               t[r][1] = in ? tab[static_cast<size_t>(n + 1) * M + m] : make_double2(0.0, -1.0);
            }
            unsigned char* b = sRowB + rs * kStageBytes;
#pragma unroll
            for (int r = 0; r < kItemRounds; ++r)
            {
               const int item = ptid + r * kProducerThreads;
               if (item < kItemsPerBlock)
               {
                  const int m = item & 127, nl = 2 * (item >> 7);
                  const float2 u0 = TablePhasor(t[r][0], aDef), u1 = TablePhasor(t[r][1], aDef);
                  float rh0, rl0, ih0, il0, rh1, rl1, ih1, il1;
                  Split(u0.x, rh0, rl0);
                  Split(u0.y, ih0, il0);
                  Split(u1.x, rh1, rl1);
                  Split(u1.y, ih1, il1);
                  // B[m][nl], B[m][nl + 1]: the real parts of pupil rows n, n + 1; B[m][16 + nl ..]: the imaginary
                  *reinterpret_cast<float2*>(b + SwOff(m, nl)) = make_float2(rh0, rh1);
                  *reinterpret_cast<float2*>(b + SwOff(m, 16 + nl)) = make_float2(ih0, ih1);
                  *reinterpret_cast<float2*>(b + kBlockBytes + SwOff(m, nl)) = make_float2(rl0, rl1);
                  *reinterpret_cast<float2*>(b + kBlockBytes + SwOff(m, 16 + nl)) = make_float2(il0, il1);
               }
            }
            FenceProxyAsync();
            __syncwarp();
            if (lane == 0)
               MbarArrive(&sh->rowFull[rs]);
         }
      }
   }
   else if (warp == kMmaWarp)
   {
      // ---------------------------------------------------------------- the MMA thread
      if (lane == 0 && nLocal > 0)
      {
         const int nJobs = 2 * nLocal * nKb;
         const uint32_t idesc1 = InstrDesc(kRows, M), idesc2 = InstrDesc(kRows, 64);
         int loaded = 0;   // A blocks whose copy was started
         // block t's Ahat K block into stage t % kAStages, once the MMAs of block t - kAStages are done
         auto loadA = [&](int t) -> bool {
            const int st = t % kAStages;
            if (t >= kAStages && !MbarWait(&sh->aEmpty[st], static_cast<uint32_t>(t / kAStages - 1) & 1u, err))
               return false;
            int j, kb;
            bool row;
            JobOf(t, nKb, nLocal, j, row, kb);
            const float* src = prm.ahat + (static_cast<size_t>(prm.items[PsfOf(j)].set) * 8 + kb) * (kStageBytes / 4);
            MbarExpectTx(&sh->aFull[st], kStageBytes);
            BulkLoad(sA + st * kStageBytes, src, kStageBytes, &sh->aFull[st]);
            loaded = t + 1;
            return true;
         };
         int consumed = 0;
         uint32_t rowCount = 0, colCount = 0;
         for (int t = 0; t < kAStages - 1 && t < nJobs && ok; ++t)
            ok = loadA(t);
         for (int t = 0; t < nJobs && ok; ++t)
         {
            int j, kb;
            bool row;
            JobOf(t, nKb, nLocal, j, row, kb);
            const uint32_t use = static_cast<uint32_t>(j >> 1) & 1u;
            if (kb == 0)   // the accumulator's TMEM columns are free (PSF j - 2 is past them)
               ok = MbarWait(row ? &sh->tFree[j & 1] : &sh->eFree[j & 1], use ^ 1u, err);
            uint64_t* full;
            uint64_t* empty;
            uint32_t parity, bH, bL, d, idesc;
            if (row)
            {
               const int rs = static_cast<int>(rowCount % kRowStages);
               full = &sh->rowFull[rs];
               empty = &sh->rowEmpty[rs];
               parity = (rowCount / kRowStages) & 1u;
               bH = SmemAddr(sRowB + rs * kStageBytes);
               bL = bH + kBlockBytes;
               d = tmem + kTmemRow + 128u * static_cast<uint32_t>(j & 1);
               idesc = idesc1;
            }
            else
            {
               const int cs = static_cast<int>(colCount % kColStages);
               full = &sh->colFull[cs];
               empty = &sh->colEmpty[cs];
               parity = (colCount / kColStages) & 1u;
               bH = SmemAddr(sColB + cs * kColStageBytes);
               bL = bH + kColStageBytes / 2;
               d = tmem + kTmemCol + 64u * static_cast<uint32_t>(j & 1);
               idesc = idesc2;
            }
            ok = ok && MbarWait(full, parity, err);
            ok = ok && MbarWait(&sh->aFull[t % kAStages], static_cast<uint32_t>(t / kAStages) & 1u, err);
            if (!ok)
               break;
            consumed = t + 1;
            TcFenceAfter();
            const uint32_t aH = SmemAddr(sA + (t % kAStages) * kStageBytes), aL = aH + kBlockBytes;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
            {
               const uint32_t off = kk * 32;   // 8 TF32 = 32 bytes along K
               Mma(d, SmemDesc(aH + off), SmemDesc(bH + off), idesc, (kb == 0 && kk == 0) ? 0u : 1u);
               Mma(d, SmemDesc(aH + off), SmemDesc(bL + off), idesc, 1u);
               Mma(d, SmemDesc(aL + off), SmemDesc(bH + off), idesc, 1u);
            }
            Commit(empty);
            Commit(&sh->aEmpty[t % kAStages]);
            if (kb == nKb - 1)
               Commit(row ? &sh->rowDone[j & 1] : &sh->colDone[j & 1]);
            if (row)
               ++rowCount;
            else
               ++colCount;
            if (t + kAStages - 1 < nJobs)
               ok = loadA(t + kAStages - 1);   // waits for the MMAs of block t - 1
         }
         if (!ok)
         {
            *err = 1;
            // let the copies and MMAs in flight land before the CTA frees its memory
            for (int t = consumed; t < loaded; ++t)
               MbarWait(&sh->aFull[t % kAStages], static_cast<uint32_t>(t / kAStages) & 1u, nullptr);
            Commit(&sh->final);
            MbarWait(&sh->final, 0u, nullptr);
         }
      }
   }
   else
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
         double local = 0.0;
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
               if (lane < 16 && x < P && c0 + c < P)
                  local += static_cast<double>(e);
            }
         }
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
         // lanes 0-15 store rows y < 32 of column x, lanes 16-31 rows y >= 32
         if (x < P)
         {
            float* plane = prm.out + static_cast<size_t>(PsfOf(j)) * P * P;
            const int y0 = 32 * h;
#pragma unroll
            for (int c = 0; c < 32; ++c)
            {
               const int yy = y0 + c;
               const float e = h ? I[32 + c] : I[c];
               if (yy < P)
                  plane[static_cast<size_t>(yy) * P + x] =
                     (prm.normalize && total > 0.0) ? static_cast<float>(static_cast<double>(e) / total) : e;
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

int BuildAhat(iscu_ctx* ctx, const float2* A, const SetParams* sets, const double3* tables, int nSets, int M, int P,
              DevBuf& ahat)
{
   if (!Tf32x3Supports(M, P))
      return Fail(ISCU_ERR_ARG, "tf32x3 chirp-Z: needs pupil samples M <= 128 (a multiple of 16) and planes of at "
                                "most 64 x 64 (else use the fp32 method)");
   // the K-block images, then the phase tables
   ISCU_CK(ahat.Reserve(AhatBytes(nSets) + static_cast<size_t>(nSets) * M * M * sizeof(double2)));
   AhatKernel<<<dim3((8 * kRows * 32 + 255) / 256, nSets), 256, 0, ctx->stream>>>(A, M, P, ahat.as<float>());
   ISCU_CK_LAUNCH(ctx, "AhatKernel");
   PhaseTableKernel<<<dim3((M * M + 255) / 256, nSets), 256, 0, ctx->stream>>>(
      sets, tables, M * M, reinterpret_cast<double2*>(ahat.as<char>() + AhatBytes(nSets)));
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

int LaunchCztTf32x3(iscu_ctx* ctx, const SetParams* sets, const double3* tables, const float2* A, uint32_t nSets,
                    const PsfItem* items, uint32_t nPsf, int M, int P, int normalize, float* out)
{
   DevBuf dAhat, dErr;
   int rc = BuildAhat(ctx, A, sets, tables, static_cast<int>(nSets), M, P, dAhat);
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(dErr.Reserve(sizeof(int)));
   ISCU_CK(cudaMemsetAsync(dErr.p, 0, sizeof(int), ctx->stream));
   rc = LaunchCztTf32x3Core(ctx, sets, dAhat.as<float>(), static_cast<int>(nSets), items, nPsf, M, P, normalize, out,
                            dErr.as<int>());
   if (rc != ISCU_OK)
      return rc;
   int err = 0;
   ISCU_CK(cudaMemcpyAsync(&err, dErr.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   if (err)
      return Fail(ISCU_ERR_TIMEOUT, "tf32x3 chirp-Z: a tensor-core completion wait ran out");
   return ISCU_OK;
}

} // namespace iscu
