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
constexpr int kTmemCols = 256;         // row pass: columns [0, 128); column pass: [128, 192)
constexpr unsigned kSpinLimit = 1u << 26;

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

// Waits for the phase with the given parity to complete; false after kSpinLimit polls.
__device__ __forceinline__ bool MbarWait(uint64_t* bar, uint32_t parity)
{
   const uint32_t a = SmemAddr(bar);
   for (unsigned it = 0; it < kSpinLimit; ++it)
   {
      uint32_t done;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done)
                   : "r"(a), "r"(parity)
                   : "memory");
      if (done)
         return true;
      if (it > 64)
         __nanosleep(64);
   }
   return false;
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

constexpr int kStages = 2;
constexpr int kStageBytes = 2 * kBlockBytes;   // a K block's hi and lo images (A: 128 rows; B: up to 128 rows)
constexpr int kPerThread = 16 * 128 / kThreads; // pupil samples of a row-pass B block per thread

// Per CTA, persistent over PSFs. Per K block kb of each pass, stage s = kb % 2:
//   wait until the MMAs that last read stage s are done (tcgen05.commit -> mma[s]);
//   thread 0 starts the bulk copy of Ahat's K block into sA[s] (-> full[s]);
//   the threads write the B block into sB[s]: row pass, the pupil phasors of rows [16 kb, 16 kb + 16) (their table
//   entries loaded one K block ahead); column pass, T's columns [16 kb, 16 kb + 16) read from TMEM and split;
//   then thread 0 waits for full[s] and issues the 12 MMAs (hi*hi, hi*lo, lo*hi over 4 K steps) and the commit.
__global__ void __launch_bounds__(kThreads, 1) CztTf32x3Kernel(TcParams prm)
{
   extern __shared__ __align__(1024) unsigned char smemRaw[];
   unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
   unsigned char* sA = smem;                                   // [kStages] x 32 KB
   unsigned char* sB = smem + kStages * kStageBytes;           // [kStages] x 32 KB
   unsigned char* tail = smem + 2 * kStages * kStageBytes;
   double* sRed = reinterpret_cast<double*>(tail);             // 4 doubles
   uint64_t* full = reinterpret_cast<uint64_t*>(tail + 64);    // kStages
   uint64_t* mmaBar = reinterpret_cast<uint64_t*>(tail + 96);  // kStages
   uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(tail + 128);
   int* sErr = reinterpret_cast<int*>(tail + 132);

   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   const int M = prm.M, P = prm.P, nKb = M / 16;

   if (warp == 0)
   {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(tmemSlot)),
                   "r"(kTmemCols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   if (tid == 0)
   {
      for (int s = 0; s < kStages; ++s)
      {
         MbarInit(&full[s], 1);
         MbarInit(&mmaBar[s], 1);
      }
      *sErr = 0;
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   TcFenceBefore();
   __syncthreads();
   TcFenceAfter();
   const uint32_t tmem = *tmemSlot;
   uint32_t fullPhase[kStages] = {0u, 0u}, mmaPhase[kStages] = {0u, 0u};
   int pending[kStages] = {0, 0};
   bool ok = true;
   const uint32_t idesc1 = InstrDesc(kRows, M), idesc2 = InstrDesc(kRows, 64);

   // every thread waits for stage s's last MMAs; the outcome (and a failed copy wait of thread 0, whose flag is
   // read after the barrier) is made uniform
   auto drain = [&](int s) {
      if (pending[s])
      {
         ok = __syncthreads_and(MbarWait(&mmaBar[s], mmaPhase[s]) && ok) != 0;
         if (*sErr)
            ok = false;
         mmaPhase[s] ^= 1u;
         pending[s] = 0;
      }
   };
   // thread 0: wait for the stage's A copy, then the MMAs and the commit (a commit with no MMA completes at once,
   // so the other threads' waits end after a failure too)
   auto issue = [&](int s, uint32_t dTmem, uint32_t bH, uint32_t bL, uint32_t idesc, bool first) {
      if (tid != 0)
         return;
      const bool copied = MbarWait(&full[s], fullPhase[s]);
      fullPhase[s] ^= 1u;
      if (!copied)
         *sErr = 1;
      TcFenceAfter();
      if (copied && *sErr == 0)
      {
         const uint32_t aH = SmemAddr(sA + s * kStageBytes), aL = aH + kBlockBytes;
#pragma unroll
         for (int kk = 0; kk < 4; ++kk)
         {
            const uint32_t off = kk * 32;   // 8 TF32 = 32 bytes along K
            Mma(dTmem, SmemDesc(aH + off), SmemDesc(bH + off), idesc, (first && kk == 0) ? 0u : 1u);
            Mma(dTmem, SmemDesc(aH + off), SmemDesc(bL + off), idesc, 1u);
            Mma(dTmem, SmemDesc(aL + off), SmemDesc(bH + off), idesc, 1u);
         }
      }
      Commit(&mmaBar[s]);
   };
   auto loadA = [&](int s, const float* ahat, int kb) {
      if (tid == 0)
      {
         MbarExpectTx(&full[s], kStageBytes);
         BulkLoad(sA + s * kStageBytes, ahat + static_cast<size_t>(kb) * (kStageBytes / 4), kStageBytes, &full[s]);
      }
   };

   for (int psf = blockIdx.x; psf < prm.nPsf && ok; psf += gridDim.x)
   {
      const PsfItem it = prm.items[psf];
      const SetParams& sp = prm.sets[it.set];
      const double2* tab = prm.phase + static_cast<size_t>(it.set) * M * M;
      const double aDef = sp.k0 * sp.ni * it.dtiM;
      const float* ahat = prm.ahat + static_cast<size_t>(it.set) * 8 * (kStageBytes / 4);

      // ---------------------------------------------------------------- row pass: T = A U
      double2 pre[kPerThread];
#pragma unroll
      for (int q = 0; q < kPerThread; ++q)
      {
         const int e = tid + q * kThreads, m = e & 127, nl = e >> 7;
         pre[q] = m < M ? tab[static_cast<size_t>(nl) * M + m] : make_double2(0.0, -1.0);
      }
      for (int kb = 0; kb < nKb; ++kb)
      {
         const int s = kb % kStages;
         drain(s);
         if (!ok)
            break;
         loadA(s, ahat, kb);
         double2 cur[kPerThread];
#pragma unroll
         for (int q = 0; q < kPerThread; ++q)
            cur[q] = pre[q];
         if (kb + 1 < nKb)
#pragma unroll
            for (int q = 0; q < kPerThread; ++q)
            {
               const int e = tid + q * kThreads, m = e & 127, n = 16 * (kb + 1) + (e >> 7);
               pre[q] = m < M ? tab[static_cast<size_t>(n) * M + m] : make_double2(0.0, -1.0);
            }
         unsigned char* b = sB + s * kStageBytes;
#pragma unroll
         for (int q = 0; q < kPerThread; ++q)
         {
            const int e = tid + q * kThreads, m = e & 127, nl = e >> 7;
            const float2 u = TablePhasor(cur[q], aDef);
            float rh, rl, ih, il;
            Split(u.x, rh, rl);
            Split(u.y, ih, il);
            *reinterpret_cast<float*>(b + SwOff(m, nl)) = rh;
            *reinterpret_cast<float*>(b + SwOff(m, 16 + nl)) = ih;
            *reinterpret_cast<float*>(b + kBlockBytes + SwOff(m, nl)) = rl;
            *reinterpret_cast<float*>(b + kBlockBytes + SwOff(m, 16 + nl)) = il;
         }
         FenceProxyAsync();
         __syncthreads();
         const uint32_t bH = SmemAddr(b);
         issue(s, tmem, bH, bH + kBlockBytes, idesc1, kb == 0);
         pending[s] = 1;
      }
      for (int s = 0; s < kStages; ++s)
         drain(s);
      if (!ok)
         break;
      TcFenceAfter();

      // ---------------------------------------------------------------- column pass: E^T = A T^T
      // TMEM lane r = 32 g + 16 h + i holds T row y = 16 g + i, part h; column m. B2 block kb: row y, column
      // 16 h + (m - 16 kb). Warps w, w + 4, w + 8, w + 12 share lanes 32 (w % 4) ..; warp w reads the 4 columns
      // 16 kb + 4 (w / 4) ..
      const int lg = warp & 3, ch = warp >> 2;
      const int r = 32 * lg + lane, h = (r >> 4) & 1, y = 16 * lg + (r & 15);
      for (int kb = 0; kb < nKb; ++kb)
      {
         const int s = kb % kStages;
         drain(s);
         if (!ok)
            break;
         loadA(s, ahat, kb);
         float v[4];
         TmemLoad4(tmem + (static_cast<uint32_t>(32 * lg) << 16) + 16 * kb + 4 * ch, v);
         unsigned char* b = sB + s * kStageBytes;
#pragma unroll
         for (int j = 0; j < 4; ++j)
         {
            const int col = 16 * h + 4 * ch + j;
            float hi, lo;
            Split(y < P ? v[j] : 0.f, hi, lo);
            *reinterpret_cast<float*>(b + SwOff(y, col)) = hi;
            *reinterpret_cast<float*>(b + kBlockBytes / 2 + SwOff(y, col)) = lo;
         }
         TcFenceBefore();
         FenceProxyAsync();
         __syncthreads();
         const uint32_t bH = SmemAddr(b);
         issue(s, tmem + 128, bH, bH + kBlockBytes / 2, idesc2, kb == 0);
         pending[s] = 1;
      }
      for (int s = 0; s < kStages; ++s)
         drain(s);
      if (!ok)
         break;
      TcFenceAfter();
      // ------------------------------------------------ |E|^2, the plane sum, the normalized plane
      // TMEM lane r = 32 g + 16 h + i holds x = 16 g + i, part h; columns 128 + y.
      float I[64];
      double local = 0.0;
      const int x = 16 * warp + (lane & 15);
      if (warp < 4)
      {
         for (int c0 = 0; c0 < 64; c0 += 32)
         {
            float vv[32];
            TmemLoad32(tmem + (static_cast<uint32_t>(32 * warp) << 16) + 128 + c0, vv);
#pragma unroll
            for (int j = 0; j < 32; ++j)
            {
               const float o = __shfl_xor_sync(0xffffffffu, vv[j], 16);
               const float e = vv[j] * vv[j] + o * o;
               I[c0 + j] = e;
               if (lane < 16 && x < P && c0 + j < P)
                  local += static_cast<double>(e);
            }
         }
      }
      TcFenceBefore();
      double total = 0.0;
      if (prm.normalize)
      {
         for (int o = 16; o > 0; o >>= 1)
            local += __shfl_xor_sync(0xffffffffu, local, o);
         __syncthreads();
         if (lane == 0 && warp < 4)
            sRed[warp] = local;
         __syncthreads();
         total = sRed[0] + sRed[1] + sRed[2] + sRed[3];
      }
      if (warp < 4 && lane < 16 && x < P)
      {
         float* plane = prm.out + static_cast<size_t>(psf) * P * P;
         for (int yy = 0; yy < P; ++yy)
            plane[static_cast<size_t>(yy) * P + x] =
               (prm.normalize && total > 0.0) ? static_cast<float>(static_cast<double>(I[yy]) / total) : I[yy];
      }
      __syncthreads();
   }
   if (!ok && tid == 0)
      atomicExch(prm.error, 1);
   TcFenceBefore();
   __syncthreads();
   TcFenceAfter();
   if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

} // namespace

bool Tf32x3Supports(int M, int P) { return M <= 128 && M % 16 == 0 && P <= 64 && P >= 1; }

size_t AhatBytes(int nSets) { return static_cast<size_t>(nSets) * 8 * kStageBytes; }

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
   const size_t smem = 2 * kStages * kStageBytes + 256 + 1024;
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
