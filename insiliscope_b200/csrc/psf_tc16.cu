// Split-precision chirp-Z on the 5th-generation tensor cores with FP16 operands: the PSF library's two complex
// products as FP16 x 3 real GEMMs (tcgen05 kind::f16, float32 accumulation in tensor memory), the DFT operand resident
// in tensor memory.
//
// The products and the stacked operand are the TF32 x 3 kernel's (psf_tc.cu): row pass T = A U, column pass
// E^T = A T^T, Ahat = [[Ar, -Ai], [Ai, Ar]], rows interleaved in groups of 16 (row r = 32 g + 16 h + i is output
// p = 16 g + i, part h) so one warp's 32 TMEM lanes hold 16 outputs' real and imaginary parts. A K block is one row of
// a 128-byte swizzle atom, 64 FP16: 32 input indices as [16 real, 16 imaginary, 16 real, 16 imaginary] (column c is
// input q = 32 kb + 16 (c >> 5) + (c & 15), part (c >> 4) & 1). A K step (16 FP16, one MMA) is one of those groups;
// the steps whose inputs lie at or past M are skipped.
//
// FP16 x 3: every operand x is split into hi = fp16(x) and lo = fp16(x - hi), both rounded to nearest (x - hi is
// exact in float32); a product is hi*hi + hi*lo + lo*hi. With 11-bit significands |x - hi - lo| <= 2^-22 |x| and
// the dropped lo*lo is <= 2^-22 |a b|, half the TF32 split's error (its lo is truncated to TF32 by the tensor
// cores). FP16's narrow range is kept by exact power-of-two scales: the DFT operand and the pupil phasors (|x| <= 1)
// enter times 2^12, so a part falls below FP16's normal range only where it is under 2^-26 of the unit; the row-pass
// result T (|T| <= M <= 128, accumulated as 2^24 T) is scaled by 2^-16 to 2^8 T (<= 32,768) before its split; E is
// 2^20 E in TMEM (|2^20 E| <= 2^34), so |2^20 E|^2 <= 2^68 stays finite in float32 and the sum-1 normalization
// cancels the 2^40 (an unnormalized plane is multiplied by 2^-40, exactly).
//
// The pupil phasors come from a per-set float32 table in revolutions: (tx, ty) = ((base mod 2 pi) / 2 pi, opd3F /
// 2 pi), reduced in float64 when the table is built, so a PSF's phase is x = a ty + tx revolutions (a = k0 ni dti, one
// float32 multiply-add; |x| < 4 at these defocus ranges, so its rounding is < 2.4e-7 revolutions, 1.5e-6 rad), reduced
// exactly as x - rint(x) and turned into sine and cosine by the special-function unit. Those per-sample phase errors
// are independent, so their effect on a plane, a sum over ~10^4 samples, stays orders of magnitude below float32
// resolution of its peak; the float64 form of the TF32 kernel costs twice the table bytes and a float64 chain.
//
// Against the TF32 form: a K step does twice the inputs, so the MMAs take half the time; and the DFT operand (both
// parts, 2M inputs: 128 KB at M = 128) is loaded once per run of PSFs that share a request set, into tensor memory
// (256 of the 512 columns), instead of streamed through shared memory per K block. An MMA then reads only its B
// operand from shared memory (4 KB per row-pass step, 2 KB per column-pass step, where an A operand in shared memory
// doubled that and made the N = 64 column pass shared-memory bound), the two passes run out of lockstep, and shared
// memory holds four row-pass and four column-pass stages. A set change waits until both passes of the previous set
// are done with the operand (the drain warps, which load it, have by then taken the previous PSF's E). The other
// 256 columns hold T of the current PSF (128) and E of two PSFs (2 x 64).
//
// Instruction count is what the warps spend their time on, so the library's shape (a 128-sample pupil to 64 x 64) is
// compiled in as its own instantiation, the phase table is laid out by pairs of pupil rows, and the producers' phase,
// reduction and split residual and the drain's scaling, |E|^2, sums and normalization use the sm_100 two-lane float
// instructions (fma/add/sub/mul.rn.f32x2; each lane rounds as the one-lane instruction would).

#include "iscu_internal.h"
#include "psf_common.cuh"
#include "tcgen05.cuh"

#include <cuda_fp16.h>

#include <algorithm>

namespace iscu {

namespace {

using namespace tc;

constexpr int kThreads = 640;
constexpr int kRows = 128;                        // UMMA M (2P rows, padded)
constexpr int kImgBytes = 128 * 128;              // one B operand image: 128 rows x 64 FP16 (128 B per row)
constexpr int kKbBytes = 2 * kImgBytes;           // a row-pass B block: its hi and lo images
constexpr int kACols = 128;                       // TMEM columns of one part of the DFT operand (256 FP16 per row)
constexpr int kAImageBytes = 2 * kRows * kACols * 4;   // the DFT operand of one set, both parts: 128 KB
constexpr int kRowStages = 4;                     // row-pass B blocks (pupil phasors)
constexpr int kColStages = 4;                     // column-pass B blocks (T, split): a whole PSF's at M = 128
constexpr int kColImgBytes = 64 * 128;            // a column-pass B image: 64 rows x 64 FP16
constexpr int kColStageBytes = 2 * kColImgBytes;
constexpr float kScaleOp = 4096.0f;               // 2^12: the DFT operand and the pupil phasors
constexpr float kScaleT = 1.0f / 65536.0f;        // 2^-16: 2^24 T -> 2^8 T
constexpr float kScaleI = 0x1p-40f;               // 2^-40: |2^20 E|^2 -> |E|^2 (unnormalized planes)

// Warp roles. Warps share an SM sub-partition (scheduler) when equal mod 4, and warp w reaches TMEM lanes
// [32 (w % 4), +32) only.
constexpr int kDrainWarps = 8;                    // warps 0-7: two per TMEM lane quadrant, each half the columns
constexpr int kRowMmaWarp = 8;                    // lane 0: the row-pass MMAs
constexpr int kColMmaWarp = 12;                   // lane 0: the column-pass MMAs
constexpr int kProducerWarps = 10;                // warps 9-11 and 13-19 make the pupil phasors
constexpr int kProducerThreads = 32 * kProducerWarps;
constexpr int kItemsPerBlock = 512;               // (pupil column, 8 pupil rows) items of one row-pass K block
constexpr int kTmemAHi = 0;                       // the DFT operand's hi part: columns [0, 128)
constexpr int kTmemALo = 128;                     // its lo part: columns [128, 256)
constexpr int kTmemRow = 256;                     // T of the current PSF: columns [256, 384)
constexpr int kTmemCol = 384;                     // E of PSF j: columns [384 + 64 (j % 2), +64)
constexpr int kSetCache = 96;                     // PSFs whose set and defocus factor are staged in shared memory

static_assert(kItemsPerBlock <= 2 * kProducerThreads, "a producer thread makes at most two items per K block");

// A producer warp's index 0..9 (warps 9-11, 13-19).
__device__ __forceinline__ int ProducerIndex(int warp) { return warp - 9 - (warp > kColMmaWarp ? 1 : 0); }

// Instruction descriptor, kind::f16: D float32, A and B FP16, both K-major, M x N.
__host__ __device__ constexpr uint32_t InstrDescF16(int M, int N)
{
   return (1u << 4) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// D (TMEM) += A (TMEM, 8 columns: 16 FP16 per row) x B (shared memory descriptor); accum 0 overwrites D.
__device__ __forceinline__ void MmaF16Ts(uint32_t dTmem, uint32_t aTmem, uint64_t bDesc, uint32_t idesc,
                                         uint32_t accum)
{
   asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(dTmem),
                "r"(aTmem), "l"(bDesc), "r"(idesc), "r"(accum));
}

// Byte offset of FP16 element (row, col) (col 0..63 within the K block) in a 128-byte-swizzled image.
__host__ __device__ __forceinline__ uint32_t SwOff16(int row, int col)
{
   return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((((col >> 3) ^ (row & 7)) & 7) << 4) +
                                ((col & 7) << 1));
}

// (a, b) -> hi = fp16x2(a, b) and lo = fp16x2(a - hi.a, b - hi.b), rounded to nearest; a in the low half.
__device__ __forceinline__ void SplitH2(float a, float b, uint32_t& hi, uint32_t& lo)
{
   const __half2 h = __floats2half2_rn(a, b);
   const float2 f = __half22float2(h);
   const __half2 l = __floats2half2_rn(a - f.x, b - f.y);
   hi = *reinterpret_cast<const uint32_t*>(&h);
   lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void StoreShared16(unsigned char* p, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
   *reinterpret_cast<uint4*>(p) = make_uint4(a, b, c, d);
}

// ------------------------------------------------------------------------------------------ the stacked operand
// Ahat for one set, times 2^12 and split, in the order the drain warps move it into tensor memory: [part hi, lo]
// [column group g = 0..31][row r][4 columns], so that a warp's 32 rows of a column group are 512 consecutive bytes.
// Column c of row r holds K elements 2c and 2c + 1 (the even one in the low half); K element k = 64 kb + c' is input
// q = 32 kb + 16 (c' >> 5) + (c' & 15), part (c' >> 4) & 1, the order of the B operands' K blocks. Rows beyond 2P and
// inputs at or past M are zero.
__global__ void AhatTmemKernel(const float2* __restrict__ A, int M, int P, uint32_t* __restrict__ out)
{
   const int s = blockIdx.y;
   const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (row, column)
   if (e >= kRows * kACols)
      return;
   const int row = e / kACols, col = e % kACols;
   const int p = 16 * (row >> 5) + (row & 15), h = (row >> 4) & 1;
   float v[2];
#pragma unroll
   for (int t = 0; t < 2; ++t)
   {
      const int k = 2 * col + t, kb = k >> 6, c = k & 63;
      const int hp = (c >> 4) & 1, q = 32 * kb + 16 * (c >> 5) + (c & 15);
      v[t] = 0.f;
      if (p < P && q < M)
      {
         const float2 a = A[(static_cast<size_t>(s) * P + p) * M + q];
         // [[Ar, -Ai], [Ai, Ar]]: output part h, input part hp
         v[t] = (h == 0 ? (hp == 0 ? a.x : -a.y) : (hp == 0 ? a.y : a.x)) * kScaleOp;
      }
   }
   uint32_t hi, lo;
   SplitH2(v[0], v[1], hi, lo);
   uint32_t* base = out + static_cast<size_t>(s) * (kAImageBytes / 4);
   const size_t idx = (static_cast<size_t>(col >> 2) * kRows + row) * 4 + (col & 3);
   base[idx] = hi;
   base[kRows * kACols + idx] = lo;
}

// The phase table in revolutions: per set and sample (tx, ty) = ((k0 opd1 + zernike + mask) mod 2 pi, opd3F) / 2 pi
// (ZernikePsf.cpp:240-248), the reduction in float64; (0, -1) outside the aperture (opd3F < 0). Laid out by pairs of
// pupil rows, [set][n / 2][m] float4 = (tx of rows n, n + 1; ty of rows n, n + 1), so that one 16-byte load gives
// a producer two samples' (tx, ty) already paired for the two-lane float instructions (M is even).
__global__ void RevTableKernel(const SetParams* __restrict__ sets, const double3* __restrict__ tables, int M,
                               float* __restrict__ out)
{
   const int s = blockIdx.y;
   const int i = blockIdx.x * blockDim.x + threadIdx.x, MM = M * M;
   if (i >= MM)
      return;
   const int n = i / M, m = i - n * M;
   const double3 t = tables[static_cast<size_t>(s) * MM + i];
   const double kInvTwoPi = 0.15915494309189533577;
   const double b = ReduceTwoPi(sets[s].k0 * t.x + t.z) * kInvTwoPi;
   // set s holds M / 2 row pairs of M float4 (2 MM floats, the float2 table's size)
   float* o = out + ((static_cast<size_t>(s) * (M / 2) + static_cast<size_t>(n >> 1)) * M + m) * 4 + (n & 1);
   o[0] = t.y < 0.0 ? 0.f : static_cast<float>(b);
   o[2] = t.y < 0.0 ? -1.f : static_cast<float>(t.y * kInvTwoPi);
}

// Two float lanes in one 64-bit register for the sm_100 two-lane float instructions (each lane rounds as the
// one-lane instruction does).
__device__ __forceinline__ uint64_t Pack2(float a, float b)
{
   uint64_t r;
   asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
   return r;
}
__device__ __forceinline__ float2 Unpack2(uint64_t v)
{
   float2 r;
   asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
   return r;
}
__device__ __forceinline__ uint64_t Fma2(uint64_t a, uint64_t b, uint64_t c)
{
   uint64_t d;
   asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
   return d;
}
__device__ __forceinline__ uint64_t Add2(uint64_t a, uint64_t b)
{
   uint64_t d;
   asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
   return d;
}
__device__ __forceinline__ uint64_t Sub2(uint64_t a, uint64_t b)
{
   uint64_t d;
   asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
   return d;
}
__device__ __forceinline__ uint64_t Mul2(uint64_t a, uint64_t b)
{
   uint64_t d;
   asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
   return d;
}

// Two pupil phasors from the revolution table, times amp inside the aperture (0 outside): x = a ty + tx, r = x -
// rint(x) (rint by adding and taking away 1.5 2^23, exact for |x| < 2^22; r in [-1/2, 1/2] exactly), then the float32
// sine and cosine of 2 pi r (absolute error ~4e-7 over [-pi, pi]). The two samples t = (tx0, tx1, ty0, ty1) go through
// two-lane instructions, each lane rounding as the one-lane form would: re = (cs0 s0, cs1 s1), im = (sn0 s0, sn1 s1).
__device__ __forceinline__ void RevPhasor2(float4 t, uint64_t a2, float amp, uint64_t& re, uint64_t& im)
{
   const uint64_t kRound2 = 0x4B4000004B400000ull;      // (1.5 2^23, 1.5 2^23)
   const uint64_t kTwoPi2 = 0x40C90FDB40C90FDBull;      // (6.28318530718f, 6.28318530718f)
   const uint64_t x = Fma2(a2, Pack2(t.z, t.w), Pack2(t.x, t.y));
   const uint64_t n = Sub2(Add2(x, kRound2), kRound2);
   const float2 r = Unpack2(Mul2(kTwoPi2, Sub2(x, n)));
   float sn0, cs0, sn1, cs1;
   __sincosf(r.x, &sn0, &cs0);
   __sincosf(r.y, &sn1, &cs1);
   const uint64_t s = Pack2(t.z >= 0.f ? amp : 0.f, t.w >= 0.f ? amp : 0.f);
   re = Mul2(Pack2(cs0, cs1), s);
   im = Mul2(Pack2(sn0, sn1), s);
}

// SplitH2 of a two-lane value, the residual in one two-lane subtraction.
__device__ __forceinline__ void SplitH2P(uint64_t v, uint32_t& hi, uint32_t& lo)
{
   const float2 ab = Unpack2(v);
   const __half2 h = __floats2half2_rn(ab.x, ab.y);
   const float2 f = __half22float2(h);
   const float2 d = Unpack2(Sub2(v, Pack2(f.x, f.y)));
   const __half2 l = __floats2half2_rn(d.x, d.y);
   hi = *reinterpret_cast<const uint32_t*>(&h);
   lo = *reinterpret_cast<const uint32_t*>(&l);
}

// ------------------------------------------------------------------------------------------ the fused kernel
struct Tc16Params
{
   const SetParams* sets;
   const float4* phase;        // [set][M / 2][M] (tx, tx, ty, ty) of two pupil rows, revolutions
   const unsigned char* ahat;  // [set] DFT operand images in tensor-memory order (AhatTmemKernel)
   const PsfItem* items;
   float* out;
   int* error;
   int nPsf, M, P, normalize;
};

struct Shared16
{
   uint64_t aFull;
   uint64_t rowFull[kRowStages], rowEmpty[kRowStages];
   uint64_t colFull[kColStages], colEmpty[kColStages];
   uint64_t rowDone, tFree;
   uint64_t colDone[2], eFree[2], red[2];
   uint64_t final[2];
   double sum[2][kDrainWarps];
   float aDef[kSetCache];    // k0 ni (ti - ti0) of the CTA's j-th PSF, j < kSetCache (ty carries the 1 / 2 pi)
   int set[kSetCache];       // its set
   uint32_t tmemSlot;
   int err;
};
constexpr size_t kSmemBytes = static_cast<size_t>(kRowStages) * kKbBytes +
                              static_cast<size_t>(kColStages) * kColStageBytes + sizeof(Shared16) + 1024;
static_assert(kSmemBytes <= 227 * 1024, "the FP16 chirp-Z kernel's shared memory");

// Per CTA, persistent over a contiguous run of PSFs, warp-specialized; the roles meet only at mbarriers:
//   producers (warps 9-11, 13-19): per row-pass K block the pupil phasors of 32 pupil rows (float32 phase in
//     revolutions reduced exactly, float32 sine and cosine, times 2^12, FP16 hi/lo split) into a row-B stage ->
//     rowFull; the phase-table entries of a thread's next item are in flight while it computes the current one;
//   the row-pass thread (warp 8, lane 0): per PSF its row pass R(j), K block by K block as the producers fill the
//     stages, into T's columns once the drain warps have taken T(j - 1) (tFree), with the set's DFT operand from TMEM
//     (aFull at the first PSF of each run of one set); commits free the stages and mark the pass done (rowDone);
//   the column-pass thread (warp 12, lane 0): per PSF its column pass C(j) into E's buffer j % 2 once E(j - 2) has
//     been taken (eFree), K block by K block as the drain warps fill the col-B stages; commits colEmpty / colDone;
//   drain warps (0-7, two per TMEM lane quadrant, each half of every block's columns): T of PSF j from TMEM, times
//     2^-16, split, into col-B stages -> colFull (then tFree); then E of PSF j - 1: |E|^2, the plane sum, the
//     normalized plane (eFree). At the first PSF of each set's run, once E of the previous PSF is taken (both passes of
//     every earlier PSF complete), the set's DFT operand from global memory into TMEM (aFull).
// R(j + 1) runs beside C(j) on the tensor pipe. Every wait is bounded (kWaitNs) and also ends when another role has
// failed (Shared16::err); a failed CTA stops issuing, waits for its MMAs in flight, frees TMEM and reports through
// prm.error.
template <int kM, int kP>
__global__ void __launch_bounds__(kThreads, 1) CztF16x3Kernel(Tc16Params prm)
{
   extern __shared__ __align__(1024) unsigned char smemRaw[];
   unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
   unsigned char* sRowB = smem;                               // [kRowStages] x 32 KB
   unsigned char* sColB = sRowB + kRowStages * kKbBytes;      // [kColStages] x 16 KB
   Shared16* sh = reinterpret_cast<Shared16*>(sColB + kColStages * kColStageBytes);
   volatile int* err = &sh->err;

   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   // kM, kP > 0: the shape compiled in (the library's 128 -> 64); 0: the request's
   const int M = kM > 0 ? kM : prm.M, P = kP > 0 ? kP : prm.P, nKb = (M + 31) / 32;
   // this CTA's PSFs: psf0 .. psf0 + nLocal - 1
   const int perCta = prm.nPsf / static_cast<int>(gridDim.x), extra = prm.nPsf % static_cast<int>(gridDim.x);
   const int cta = static_cast<int>(blockIdx.x);
   const int psf0 = cta * perCta + min(cta, extra), nLocal = perCta + (cta < extra ? 1 : 0);

   if (warp == 0)
   {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(&sh->tmemSlot)),
                   "r"(512));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   if (tid == 0)
   {
      MbarInit(&sh->aFull, kDrainWarps);   // once per set run
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
      MbarInit(&sh->rowDone, 1);
      MbarInit(&sh->tFree, kDrainWarps);
      for (int s = 0; s < 2; ++s)
      {
         MbarInit(&sh->colDone[s], 1);
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
      const PsfItem it = prm.items[psf0 + j];
      sh->set[j] = it.set;
      sh->aDef[j] = static_cast<float>(prm.sets[it.set].k0 * prm.sets[it.set].ni * it.dtiM);
   }
   TcFenceBefore();
   __syncthreads();
   TcFenceAfter();
   const uint32_t tmem = sh->tmemSlot;
   bool ok = true;
   auto setOf = [&](int j) { return j < kSetCache ? sh->set[j] : prm.items[psf0 + j].set; };
   auto firstOfSet = [&](int j) { return j == 0 || setOf(j) != setOf(j - 1); };

   if (warp > kRowMmaWarp && warp != kColMmaWarp)
   {
      // ---------------------------------------------------------------- producers: row-pass B blocks
      // Item r (0, 1) of K block kb: pupil column m = item & 127 and pupil rows n0 .. n0 + 7, n0 = 32 kb + 8 (item >>
      // 7), item = slot + r kProducerThreads with slot = (ptid + rot) mod kProducerThreads.
      const int ptid = 32 * ProducerIndex(warp) + lane;
      // A block's 512 items over 320 threads: 192 threads make two, 128 one. Which do is rotated by 64 threads (two
      // warps, so a warp's count stays uniform) from one K block to the next: over any five blocks every thread
      // makes eight items, 1.6 a block, where a fixed split would give some threads two every block. rot = 64 (block
      // count mod 5), stepped with the blocks rather than divided out.
      auto slotAt = [&](int rot) { return ptid + rot >= kProducerThreads ? ptid + rot - kProducerThreads : ptid + rot; };
      auto nextRot = [](int rot) { return rot == kProducerThreads - 64 ? 0 : rot + 64; };
      auto load = [&](const float4* tab, int kb, int item, float4* dst) {
         const int m = item & 127, n0 = 32 * kb + 8 * (item >> 7);
         const bool in = m < M && n0 < M;
         const float4* t = tab + (n0 >> 1) * M + m;
#pragma unroll
         for (int c = 0; c < 4; ++c)
            dst[c] = in ? t[c * M] : make_float4(0.f, 0.f, -1.f, -1.f);
      };
      // the defocus factor of PSF j (staged in shared memory for j < kSetCache)
      auto aDefOf = [&](int j) {
         if (j < kSetCache)
            return sh->aDef[j];
         const PsfItem it = prm.items[psf0 + j];
         return static_cast<float>(prm.sets[it.set].k0 * prm.sets[it.set].ni * it.dtiM);
      };
      auto tabOf = [&](int j) { return prm.phase + static_cast<size_t>(setOf(j)) * (M / 2) * M; };
      float4 nxt[4];
      if (nLocal > 0)
         load(tabOf(0), 0, slotAt(0), nxt);
      uint32_t rowCount = 0;
      int rot = 0;   // (rowCount % 5) 64
      for (int j = 0; j < nLocal && ok; ++j)
      {
         const float aDef = aDefOf(j);
         const uint64_t aDef2 = Pack2(aDef, aDef);
         const float4* tab = tabOf(j);
         for (int kb = 0; kb < nKb; ++kb, ++rowCount, rot = nextRot(rot))
         {
            const int rs = static_cast<int>(rowCount % kRowStages);
            ok = __all_sync(0xffffffffu, MbarWait(&sh->rowEmpty[rs], ((rowCount / kRowStages) & 1u) ^ 1u, err));
            if (!ok)
               break;
            unsigned char* b = sRowB + rs * kKbBytes;
            const int slot = slotAt(rot), nR = slot + kProducerThreads < kItemsPerBlock ? 2 : 1;
#pragma unroll
            for (int r = 0; r < 2; ++r)
            {
               if (r >= nR)
                  break;
               float4 cur[4];
#pragma unroll
               for (int c = 0; c < 4; ++c)
                  cur[c] = nxt[c];
               // the next item's table entries while this one computes
               if (r + 1 < nR)
                  load(tab, kb, slot + kProducerThreads, nxt);
               else if (kb + 1 < nKb)
                  load(tab, kb + 1, slotAt(nextRot(rot)), nxt);
               else if (j + 1 < nLocal)
                  load(tabOf(j + 1), 0, slotAt(nextRot(rot)), nxt);
               const int item = slot + r * kProducerThreads, m = item & 127, l = 8 * (item >> 7);
               if (m < M && 32 * kb + l < M)   // pupil columns >= M are not read (N = M); K steps >= M are skipped
               {
                  uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
                  for (int c = 0; c < 4; ++c)
                  {
                     uint64_t re, im;   // rows n0 + 2c, n0 + 2c + 1
                     RevPhasor2(cur[c], aDef2, kScaleOp, re, im);
                     SplitH2P(re, rh[c], rl[c]);
                     SplitH2P(im, ih[c], il[c]);
                  }
                  // B[m][c0 + i]: the real part of pupil row n0 + i; B[m][c0 + 16 + i]: the imaginary part
                  const int c0 = 32 * (l >> 4) + (l & 15);
                  StoreShared16(b + SwOff16(m, c0), rh[0], rh[1], rh[2], rh[3]);
                  StoreShared16(b + SwOff16(m, c0 + 16), ih[0], ih[1], ih[2], ih[3]);
                  StoreShared16(b + kImgBytes + SwOff16(m, c0), rl[0], rl[1], rl[2], rl[3]);
                  StoreShared16(b + kImgBytes + SwOff16(m, c0 + 16), il[0], il[1], il[2], il[3]);
               }
            }
            FenceProxyAsync();
            __syncwarp();
            if (lane == 0)
               MbarArrive(&sh->rowFull[rs]);
         }
      }
   }
   else if (warp == kRowMmaWarp)
   {
      // ---------------------------------------------------------------- the row passes
      if (lane == 0 && nLocal > 0)
      {
         const uint32_t idesc = InstrDescF16(kRows, M);
         uint32_t count = 0, runs = 0;
         for (int j = 0; j < nLocal && ok; ++j)
         {
            if (firstOfSet(j))
            {
               ok = MbarWait(&sh->aFull, runs & 1u, err, false);   // this set's operand is in TMEM
               ++runs;
               if (!ok)
                  break;
            }
            if (j > 0)   // T(j - 1) has left TMEM
               ok = MbarWait(&sh->tFree, static_cast<uint32_t>(j - 1) & 1u, err, false);
            const uint32_t d = tmem + kTmemRow;
            for (int kb = 0; kb < nKb && ok; ++kb, ++count)
            {
               const int rs = static_cast<int>(count % kRowStages);
               ok = MbarWait(&sh->rowFull[rs], (count / kRowStages) & 1u, err, false);
               if (!ok)
                  break;
               TcFenceAfter();
               const uint32_t bH = SmemAddr(sRowB + rs * kKbBytes), bL = bH + kImgBytes;
#pragma unroll
               for (int kk = 0; kk < 4; ++kk)
               {
                  if (32 * kb + 16 * (kk >> 1) >= M)
                     continue;
                  const uint32_t off = kk * 32;   // 16 FP16 = 32 bytes along K
                  const uint32_t aH = tmem + kTmemAHi + 8u * (4 * kb + kk), aL = aH + (kTmemALo - kTmemAHi);
                  MmaF16Ts(d, aH, SmemDesc(bH + off), idesc, (kb == 0 && kk == 0) ? 0u : 1u);
                  MmaF16Ts(d, aH, SmemDesc(bL + off), idesc, 1u);
                  MmaF16Ts(d, aL, SmemDesc(bH + off), idesc, 1u);
               }
               Commit(&sh->rowEmpty[rs]);
            }
            if (!ok)
               break;
            Commit(&sh->rowDone);
         }
         if (!ok)
         {
            *err = 1;
            Commit(&sh->final[0]);   // this thread's MMAs in flight finish before the CTA frees its TMEM
            MbarWait(&sh->final[0], 0u, nullptr);
         }
      }
   }
   else if (warp == kColMmaWarp)
   {
      // ---------------------------------------------------------------- the column passes
      if (lane == 0 && nLocal > 0)
      {
         const uint32_t idesc = InstrDescF16(kRows, 64);
         uint32_t count = 0, runs = 0;
         for (int j = 0; j < nLocal && ok; ++j)
         {
            if (firstOfSet(j))
            {
               ok = MbarWait(&sh->aFull, runs & 1u, err, false);   // this set's operand has landed
               ++runs;
               if (!ok)
                  break;
            }
            const uint32_t use = static_cast<uint32_t>(j >> 1) & 1u;
            ok = MbarWait(&sh->eFree[j & 1], use ^ 1u, err, false);   // E(j - 2) has left the buffer
            const uint32_t d = tmem + kTmemCol + 64u * static_cast<uint32_t>(j & 1);
            for (int kb = 0; kb < nKb && ok; ++kb, ++count)
            {
               const int cs = static_cast<int>(count % kColStages);
               ok = MbarWait(&sh->colFull[cs], (count / kColStages) & 1u, err, false);
               if (!ok)
                  break;
               TcFenceAfter();
               const uint32_t bH = SmemAddr(sColB + cs * kColStageBytes), bL = bH + kColImgBytes;
#pragma unroll
               for (int kk = 0; kk < 4; ++kk)
               {
                  if (32 * kb + 16 * (kk >> 1) >= M)
                     continue;
                  const uint32_t off = kk * 32;
                  const uint32_t aH = tmem + kTmemAHi + 8u * (4 * kb + kk), aL = aH + (kTmemALo - kTmemAHi);
                  MmaF16Ts(d, aH, SmemDesc(bH + off), idesc, (kb == 0 && kk == 0) ? 0u : 1u);
                  MmaF16Ts(d, aH, SmemDesc(bL + off), idesc, 1u);
                  MmaF16Ts(d, aL, SmemDesc(bH + off), idesc, 1u);
               }
               Commit(&sh->colEmpty[cs]);
            }
            if (!ok)
               break;
            Commit(&sh->colDone[j & 1]);
         }
         if (!ok)
         {
            *err = 1;
            Commit(&sh->final[1]);
            MbarWait(&sh->final[1], 0u, nullptr);
         }
      }
   }
   else if (warp < kDrainWarps)
   {
      // ---------------------------------------------------------------- drain warps
      // Warp w drains TMEM lane quadrant q = w % 4, columns half w / 4 of each block. TMEM lane r = 32 q + 16 h + i of
      // T holds row y = 16 q + i, part h (columns: the pupil column m); of E, output x = 16 q + i, part h (columns:
      // y).
      const int q = warp & 3, half = warp >> 2;
      const int h = (lane >> 4) & 1, y = 16 * q + (lane & 15), x = y;
      const uint32_t quad = static_cast<uint32_t>(32 * q) << 16;
      // The DFT operand of a set into this quadrant's 32 TMEM lanes (rows 32 q + lane): both parts, this warp's half
      // of the columns, 32 columns per store.
      auto loadOperand = [&](int set) {
         const uint4* src = reinterpret_cast<const uint4*>(prm.ahat + static_cast<size_t>(set) * kAImageBytes);
         const int r = 32 * q + lane;
#pragma unroll 1
         for (int part = 0; part < 2; ++part)
#pragma unroll 1
            for (int c0 = half * (kACols / 2); c0 < (half + 1) * (kACols / 2); c0 += 32)
            {
               uint32_t v[32];
#pragma unroll
               for (int g = 0; g < 8; ++g)
               {
                  const uint4 w4 = src[static_cast<size_t>(part * (kACols / 4) + c0 / 4 + g) * kRows + r];
                  v[4 * g] = w4.x;
                  v[4 * g + 1] = w4.y;
                  v[4 * g + 2] = w4.z;
                  v[4 * g + 3] = w4.w;
               }
               TmemStore32(tmem + quad + (part ? kTmemALo : kTmemAHi) + c0, v);
            }
         TmemWaitStore();
      };
      // T(j): wait for its row pass, then K block by K block from TMEM into the col-B stages (this warp: pupil
      // columns 32 kb + 16 half .. + 15); tFree when all is taken. The drain's waits spin without sleeping: its warps
      // are on the critical path of both passes.
      const float tScale = y < P ? kScaleT : 0.f;
      const uint64_t tScale2 = Pack2(tScale, tScale);
      uint32_t colCount = 0;
      auto drainT = [&](int j) -> bool {
         if (!__all_sync(0xffffffffu, MbarWait(&sh->rowDone, static_cast<uint32_t>(j) & 1u, err, false)))
            return false;
         TcFenceAfter();
         for (int kb = 0; kb < nKb; ++kb, ++colCount)
         {
            const int cs = static_cast<int>(colCount % kColStages);
            if (!__all_sync(0xffffffffu,
                            MbarWait(&sh->colEmpty[cs], ((colCount / kColStages) & 1u) ^ 1u, err, false)))
               return false;
            float v[16];
            TmemLoad16(tmem + quad + kTmemRow + 32u * kb + 16u * half, v);
            uint32_t hi[8], lo[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)   // rows y >= P of T are exact zeros (so are those of the DFT operand)
               SplitH2P(Mul2(Pack2(v[2 * c], v[2 * c + 1]), tScale2), hi[c], lo[c]);
            // B[y][32 half + 16 h + i] = part h of T[y][32 kb + 16 half + i]
            unsigned char* b = sColB + cs * kColStageBytes;
#pragma unroll
            for (int g = 0; g < 2; ++g)
            {
               const int col = 32 * half + 16 * h + 8 * g;
               StoreShared16(b + SwOff16(y, col), hi[4 * g], hi[4 * g + 1], hi[4 * g + 2], hi[4 * g + 3]);
               StoreShared16(b + kColImgBytes + SwOff16(y, col), lo[4 * g], lo[4 * g + 1], lo[4 * g + 2],
                             lo[4 * g + 3]);
            }
            FenceProxyAsync();
            __syncwarp();
            if (lane == 0)
               MbarArrive(&sh->colFull[cs]);
         }
         TcFenceBefore();
         __syncwarp();
         if (lane == 0)
            MbarArrive(&sh->tFree);
         return true;
      };
      // E(j) (this warp: y = 32 half .. + 31): wait for its column pass, |E|^2, the plane sum, the normalized plane;
      // eFree once E is in registers.
      auto drainE = [&](int j) -> bool {
         const uint32_t use = static_cast<uint32_t>(j >> 1) & 1u;
         if (!__all_sync(0xffffffffu, MbarWait(&sh->colDone[j & 1], use, err, false)))
            return false;
         TcFenceAfter();
         uint64_t I2[16];   // |E|^2 of columns (2c, 2c + 1)
         uint64_t part2[4] = {0ull, 0ull, 0ull, 0ull};   // four two-lane float partial sums of 8 values each
         {
            float vv[32];
            TmemLoad32(tmem + quad + kTmemCol + 64u * static_cast<uint32_t>(j & 1) + 32u * half, vv);
#pragma unroll
            for (int c = 0; c < 16; ++c)   // |2^20 E|^2 = 2^40 |E|^2; the 2^-40 goes into the final scale
            {
               const uint64_t me = Pack2(vv[2 * c], vv[2 * c + 1]);
               const uint64_t o = Pack2(__shfl_xor_sync(0xffffffffu, vv[2 * c], 16),
                                        __shfl_xor_sync(0xffffffffu, vv[2 * c + 1], 16));
               const uint64_t e = Fma2(me, me, Mul2(o, o));
               I2[c] = e;
               const int col = 32 * half + 2 * c;   // planes' rows y < P are summed
               if (col + 1 < P)
                  part2[c >> 2] = Add2(part2[c >> 2], e);
               else if (col < P)
                  part2[c >> 2] = Add2(part2[c >> 2], Pack2(Unpack2(e).x, 0.f));
            }
         }
         double local = 0.0;
         if (lane < 16 && x < P)
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
               const float2 p = Unpack2(part2[k]);
               local += static_cast<double>(p.x + p.y);
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
            if (!__all_sync(0xffffffffu, MbarWait(&sh->red[j & 1], use, err, false)))
               return false;
            const volatile double* sm = sh->sum[j & 1];
#pragma unroll
            for (int w = 0; w < kDrainWarps; ++w)
               total += sm[w];
         }
         // lanes 0-15 store rows y = 32 half .. + 15 of column x, lanes 16-31 rows 32 half + 16 .. + 31; the plane
         // times 1 / sum (the float product is within an ulp or two of the float64 quotient)
         float* plane = prm.out + static_cast<size_t>(psf0 + j) * P * P;
         const float scale = (prm.normalize && total > 0.0) ? static_cast<float>(1.0 / total) : kScaleI;
         const int y0 = 32 * half + 16 * h;
         const uint64_t scale2 = Pack2(scale, scale);
         if (x < P)
         {
#pragma unroll
            for (int c = 0; c < 8; ++c)
            {
               const float2 e = Unpack2(Mul2(h ? I2[8 + c] : I2[c], scale2));
               const int yy = y0 + 2 * c;
               if (yy < P)
                  plane[static_cast<size_t>(yy) * P + x] = e.x;
               if (yy + 1 < P)
                  plane[static_cast<size_t>(yy + 1) * P + x] = e.y;
            }
         }
         return true;
      };
      // T(j), then E(j - 1): the column pass of PSF j follows the T drain K block by K block and the row pass of PSF
      // j + 1 starts once T(j) is taken, while these warps take E(j - 1), whose column pass has had all of R(j) to
      // finish (E(j) right after T(j) would wait for C(j)). At a set change E(j - 1) is taken first: then both passes of
      // every earlier PSF are complete and no MMA reads the operand being replaced.
      int eNext = 0;   // the next PSF whose E is taken
      for (int j = 0; j < nLocal && ok; ++j)
      {
         if (firstOfSet(j))
         {
            while (ok && eNext < j)
               ok = drainE(eNext++);
            if (!ok)
               break;
            loadOperand(setOf(j));
            TcFenceBefore();
            __syncwarp();
            if (lane == 0)
               MbarArrive(&sh->aFull);
         }
         ok = drainT(j);
         if (ok && eNext < j)
            ok = drainE(eNext++);
      }
      while (ok && eNext < nLocal)
         ok = drainE(eNext++);
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

bool F16x3Supports(int M, int P) { return M <= 128 && M % 16 == 0 && P <= 64 && P >= 1; }

size_t AhatF16Bytes(int nSets) { return static_cast<size_t>(nSets) * kAImageBytes; }

int BuildAhatF16(iscu_ctx* ctx, const float2* A, const SetParams* sets, const double3* tables, int nSets, int M,
                 int P, unsigned char* out)
{
   AhatTmemKernel<<<dim3((kRows * kACols + 255) / 256, nSets), 256, 0, ctx->stream>>>(A, M, P,
                                                                                  reinterpret_cast<uint32_t*>(out));
   ISCU_CK_LAUNCH(ctx, "AhatTmemKernel");
   RevTableKernel<<<dim3((M * M + 255) / 256, nSets), 256, 0, ctx->stream>>>(
      sets, tables, M, reinterpret_cast<float*>(out + AhatF16Bytes(nSets)));
   ISCU_CK_LAUNCH(ctx, "RevTableKernel");
   return ISCU_OK;
}

int LaunchCztF16x3Core(iscu_ctx* ctx, const SetParams* sets, const unsigned char* ahat, int nSets,
                       const PsfItem* items, uint32_t nPsf, int M, int P, int normalize, float* out, int* dErr)
{
   if (!F16x3Supports(M, P))
      return Fail(ISCU_ERR_ARG, "f16x3 chirp-Z: needs pupil samples M <= 128 (a multiple of 16) and planes of at "
                                "most 64 x 64");
   if (nPsf == 0)
      return ISCU_OK;
   const size_t smem = kSmemBytes;
   const bool fixed = M == 128 && P == 64;
   auto kernel = fixed ? CztF16x3Kernel<128, 64> : CztF16x3Kernel<0, 0>;
   ISCU_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
   Tc16Params prm;
   prm.sets = sets;
   prm.phase = reinterpret_cast<const float4*>(ahat + AhatF16Bytes(nSets));
   prm.ahat = ahat;
   prm.items = items;
   prm.out = out;
   prm.error = dErr;
   prm.nPsf = static_cast<int>(nPsf);
   prm.M = M;
   prm.P = P;
   prm.normalize = normalize;
   const int grid = static_cast<int>(std::min<uint32_t>(nPsf, static_cast<uint32_t>(ctx->smCount)));
   kernel<<<grid, kThreads, smem, ctx->stream>>>(prm);
   ISCU_CK_LAUNCH(ctx, "CztF16x3Kernel");
   return ISCU_OK;
}

} // namespace iscu
