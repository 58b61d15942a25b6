// Widefield mean-field image formation on sm_100a: the dye volume convolved with a 3D PSF by FFT, then background and
// the camera noise chain per focal plane.
//
// The reference renders a focus series one focus at a time: every dye plane's 2D spectrum is paired with the PSF
// plane at its defocus and summed (WidefieldScene, adapter/inSiliScope/Simulation/WidefieldRender.h:360-620,
// ChannelImageStep WidefieldRender.cpp:1724) -- for dye planes and foci on one z grid that sum over planes is a
// linear convolution along z. Here the whole series is one 3D linear convolution on a zero-padded power-of-two grid
// (GX x GY x GZ >= the linear-convolution lengths), cropped to the volume ("same"), so image plane f is
// sum_k dye plane k (x) PSF plane f - k + kz/2. Then max(0, .) + background per pixel (WidefieldImages::Render,
// WidefieldRender.cpp:547) and ApplyNoiseChain per plane (SMLMNoise.cpp:142-216) in the same kernel.
//
// Passes (each a batch of 1D transforms; the padded halves are never loaded, stored or transformed beyond the first
// butterfly stage that reads their zeros):
//   XForward   rows of nx reals -> GX-point real FFT through a GX/2-point complex FFT of packed pairs -> GX/2+1 bins,
//              stored k-major, y contiguous: A[z][k][y]
//   YForward   A rows (ny values, zero-padded to GY) -> GY-point FFT -> B[z][k][ky]
//   ZConvolve  B columns along z (nz values, padded to GZ) -> GZ-point FFT, times the PSF spectrum, inverse FFT,
//              keep the nz cropped planes -> B in place
//   YInverse   B rows -> inverse GY-point FFT, keep the ny cropped rows -> A
//   XInverse   A -> GX/2-point inverse complex FFT of the re-packed half spectrum -> GX reals, keep nx cropped
//              columns, scale 1/(GX GY GZ), max(0, .) + background, noise chain -> uint16 frames (and the image)
// Forward transforms are decimation in frequency (natural order in, bit-reversed out) and inverse transforms
// decimation in time (bit-reversed in, natural out), so no pass ever permutes: the spectra B and the PSF spectrum
// are stored with ky and kz in bit-reversed order.
//
// Each N-point transform is split into groups of up to five radix-2 stages (N = R_0 R_1 ... , R_g <= 32). A thread
// holds the R_g points of one group in registers -- points j + q m, m < R_g, q the group's smallest span -- does
// the R_g-point DFT there (constant roots of unity only) and then one table twiddle per point: DIF group g of
// block size M = q R_g is, per j < q, an R_g-point DFT of the stride-q points followed by W_M^(j rev(m)) on output
// slot m. The inverse groups are the conjugate transposes (conjugate twiddle first, then the R_g-point inverse DFT
// with bit-reversed input), run in reverse group order. The first group loads straight from global memory and the
// last one of an inverse stores straight back, so a 1024-point transform is one shared-memory exchange. Layouts:
// rows (Y) pad one point per R_last points, so both the stride-q reads of the first group and the contiguous reads
// of the last one hit 16 distinct 8-byte bank pairs per half warp; columns (Z, X: lines fastest) pad X's line
// stride to an odd count for the passes that walk along a line.
//
// Compiled with --fmad=false for the noise chain's exactness; the FFT arithmetic uses explicit __fmaf_rn.

#include "iscu_internal.h"
#include "noise_chain.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace iscu {

// One transform length's group plan: groups of r[g] radix-2 stages from the largest span down; tw[g] is the offset of
// group g's twiddle table (q R entries, slot-major) in the plan's table buffer, -1 where q = 1.
struct LinePlan
{
   int logN = 0, groups = 0;
   int r[4] = {0, 0, 0, 0};
   int tw[4] = {-1, -1, -1, -1};
};

__host__ __device__ inline int LogQ(const LinePlan& P, int g)
{
   int s = 0;
   for (int i = 0; i <= g; ++i)
      s += P.r[i];
   return P.logN - s;
}

// Group sizes for an N = 2^logN point transform: one group up to 32 points; else groups of 2^3..2^5. Rows: the
// last (span-1) group at least 16 points, so that every group but the last has a smallest span q >= 16 (the padded
// row layout is conflict-free for those). Columns (lanes walk the lines, any q is conflict-free): the larger group
// first, for more loads in flight per thread where group 0 reads global memory.
__host__ __device__ constexpr LinePlan MakeLinePlan(int logN, bool cols)
{
   LinePlan P;
   P.logN = logN;
   if (logN <= 5)
   {
      P.groups = 1;
      P.r[0] = logN;
   }
   else if (logN <= 10)
   {
      P.groups = 2;
      if (cols)
         P.r[0] = (logN + 1) / 2 < 5 ? (logN + 1) / 2 : 5;
      else
         P.r[0] = logN - (logN >= 9 ? logN - 5 : 4);
      P.r[1] = logN - P.r[0];
   }
   else
   {
      P.groups = 3;
      P.r[1] = 4;
      P.r[2] = 4;
      P.r[0] = logN - 8;
   }
   return P;
}

// Assigns the tables of the groups with q > 1 at `offset` (float2 entries) onwards; returns the entries used.
// The z pass's plan: groups of at most 16 points, the smaller group first (it reads the zero-padded half).
__host__ __device__ constexpr LinePlan MakeZPlan(int logN)
{
   LinePlan P;
   P.logN = logN;
   P.groups = (logN + 3) / 4;
   for (int g = 1; g < P.groups; ++g)
      P.r[g] = 4;
   P.r[0] = logN - 4 * (P.groups - 1);
   return P;
}

} // namespace iscu

struct iscu_wf_plan
{
   iscu_ctx* ctx = nullptr;
   uint32_t nx = 0, ny = 0, nz = 0, kx = 0, ky = 0, kz = 0;
   uint32_t GX = 0, GY = 0, GZ = 0, H = 0, NK = 0, G = 0;
   int logH = 0, logGY = 0, logGZ = 0;
   iscu::LinePlan px, py, pz;
   iscu::DevBuf A, B, Kh, tw, twg, image, adu;
   // The camera (iscu_wf_plan_from_kernel): frames are the FOV cells [fovX0, fovX0 + up fovW) x [fovY0, fovY0 + up
   // fovH) of the grid, up x up cells per pixel; without one (camera false) a frame is the whole nx x ny grid.
   bool camera = false;
   uint32_t fovX0 = 0, fovY0 = 0, fovW = 0, fovH = 0, up = 1;
   iscu::DevBuf cells;   // camera plans: the clamped cell images before binning
   uint32_t FrameW() const { return camera ? fovW : nx; }
   uint32_t FrameH() const { return camera ? fovH : ny; }
   size_t FrameElems() const { return static_cast<size_t>(FrameW()) * FrameH() * nz; }
   // Pipelined renders (iscu_wf_render_async): per I/O slot the volume, the frames and the three stage events.
   struct Io
   {
      bool busy = false;
      iscu::DevBuf density, image, adu;
      cudaEvent_t uploaded = nullptr, rendered = nullptr, downloaded = nullptr;
   } io[ISCU_EVENT_IO_SLOTS];
   // Pass timing (iscu_wf_set_timing): events before XForward and after each of the ISCU_WF_PASSES passes.
   bool timing = false;
   cudaEvent_t ev[ISCU_WF_PASSES + 1] = {};
   void Mark(int i) const
   {
      if (timing)
         cudaEventRecord(ev[i], ctx->stream);
   }
};

// Frames of a drifting widefield sample from its channels' spectra (iscu_wf_shifted_frames_dev): the grid's plans and
// twiddle tables, and the spectra of the frames between the two passes.
struct iscu_wf_shift
{
   iscu_ctx* ctx = nullptr;
   uint32_t nx = 0, ny = 0, H = 0, W = 0, G = 0;
   iscu::LinePlan px, py;
   iscu::DevBuf tw, twg, T;
};

namespace iscu {

namespace {

// Resident CTAs per SM the FFT passes are compiled for (registers per thread <= 64K / (256 x this)).
#ifndef ISCU_WF_MIN_CTAS
#define ISCU_WF_MIN_CTAS 2
#endif
// Stage buffers of the z pass: 2 = persistent CTAs copying the next column block in while transforming one; 1 = a
// CTA per column block.
#ifndef ISCU_WF_Z_STAGES
#define ISCU_WF_Z_STAGES 1
#endif
// Columns per z block with one stage buffer (a power of two).
#ifndef ISCU_WF_Z_COLUMNS
#define ISCU_WF_Z_COLUMNS 32
#endif
constexpr int kThreads = 256;
constexpr int kMinCtas = ISCU_WF_MIN_CTAS;
constexpr size_t kSmemBudget = 100 * 1024;   // lines per CTA are sized to this
constexpr size_t kSmemMax = 227 * 1024;
constexpr size_t kSmemPair = 112 * 1024;   // dynamic shared memory of a CTA that leaves room for a second on its SM

__device__ __forceinline__ float2 Cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 Csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 Cmul(float2 a, float2 b)
{
   return make_float2(__fmaf_rn(a.x, b.x, -(a.y * b.y)), __fmaf_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 Conj(float2 a) { return make_float2(a.x, -a.y); }

// 8-byte asynchronous global -> shared copies (no registers held while in flight); a thread waits for its own.
__device__ __forceinline__ void CopyAsync8(float2* dst, const float2* src)
{
   asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                "l"(src)
                : "memory");
}
__device__ __forceinline__ void CopyAsync16(float2* dst, const float2* src)
{
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                "l"(src)
                : "memory");
}
__device__ __forceinline__ void CopyAsyncWait() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void CopyAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits for all of this thread's copy groups but the most recently committed one.
__device__ __forceinline__ void CopyAsyncWaitPrior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ int Rev(int n, int logN) { return static_cast<int>(__brev(static_cast<unsigned>(n)) >> (32 - logN)); }

__host__ __device__ constexpr int Log2i(int v) { return v <= 1 ? 0 : 1 + Log2i(v >> 1); }

// cos(2 pi e / 32) for e = 0..8 (the first octant of the 32nd roots of unity).
__device__ __forceinline__ float Cos32Octant(int e)
{
   switch (e)
   {
   case 0: return 1.0f;
   case 1: return 0.98078528040323044913f;
   case 2: return 0.92387953251128675613f;
   case 3: return 0.83146961230254523708f;
   case 4: return 0.70710678118654752440f;
   case 5: return 0.55557023301960222474f;
   case 6: return 0.38268343236508977173f;
   case 7: return 0.19509032201612826785f;
   default: return 0.0f;
   }
}

__device__ __forceinline__ float Cos32(int e)
{
   e &= 31;
   if (e <= 8)
      return Cos32Octant(e);
   if (e <= 16)
      return -Cos32Octant(16 - e);
   if (e <= 24)
      return -Cos32Octant(e - 16);
   return Cos32Octant(32 - e);
}

// x W_32^e, W_32 = exp(-2 pi i / 32), conjugated for inverse transforms. Every call site has e fixed once its loops
// are unrolled, so the branches fold away.
template <bool kInv>
__device__ __forceinline__ float2 RootMul(float2 x, int e)
{
   e &= 31;
   if (e == 0)
      return x;
   if (e == 16)
      return make_float2(-x.x, -x.y);
   if (e == 8 || e == 24)
      return ((e == 8) != kInv) ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);   // times -i : times +i
   const float c = Cos32(e), s = Cos32(e - 8);                                       // sin(2 pi e / 32)
   return Cmul(x, make_float2(c, kInv ? s : -s));
}

// R-point DFT in registers, decimation in frequency: natural order in, bit-reversed order out. kHalf: the upper
// half of the input is zero (and not read).
template <int R, bool kInv, bool kHalf>
__device__ __forceinline__ void DifReg(float2 (&v)[R])
{
#pragma unroll
   for (int s = R / 2; s >= 1; s >>= 1)
   {
#pragma unroll
      for (int i = 0; i < R / 2; ++i)
      {
         const int lo = (i / s) * 2 * s + i % s, hi = lo + s, e = (i % s) * (32 / (2 * s));
         if (kHalf && s == R / 2)
         {
            v[hi] = RootMul<kInv>(v[lo], e);
         }
         else
         {
            const float2 a = v[lo], b = v[hi];
            v[lo] = Cadd(a, b);
            v[hi] = RootMul<kInv>(Csub(a, b), e);
         }
      }
   }
}

// R-point DFT in registers, decimation in time: bit-reversed order in, natural order out.
template <int R, bool kInv>
__device__ __forceinline__ void DitReg(float2 (&v)[R])
{
#pragma unroll
   for (int s = 1; s < R; s <<= 1)
   {
#pragma unroll
      for (int i = 0; i < R / 2; ++i)
      {
         const int lo = (i / s) * 2 * s + i % s, hi = lo + s;
         const float2 a = v[lo], b = RootMul<kInv>(v[hi], (i % s) * (32 / (2 * s)));
         v[lo] = Cadd(a, b);
         v[hi] = Csub(a, b);
      }
   }
}

// Output slot m (m >= 1) of a group times its table twiddle W_M^(j rev(m)) (conjugated for inverse transforms);
// table entry m q + j, so the lanes of a warp walking j read consecutive entries.
template <int R, bool kInv>
__device__ __forceinline__ void Twiddle(float2 (&v)[R], const float2* __restrict__ tw, int q, int j)
{
#pragma unroll
   for (int m = 1; m < R; ++m)
   {
      float2 w = __ldg(tw + m * q + j);
      if (kInv)
         w.y = -w.y;
      v[m] = Cmul(v[m], w);
   }
}

// Shared-memory layouts. Rows: point i of line b at b * np + i + (i >> rl), np = N + N / 2^rl. Columns: point i of
// line b at i * ls + b.
struct RowAddr
{
   float2* s;
   int np, rl;
   __device__ __forceinline__ float2& operator()(int b, int i) const { return s[b * np + i + (i >> rl)]; }
};

struct ColAddr
{
   float2* s;
   int ls;
   __device__ __forceinline__ float2& operator()(int b, int i) const { return s[i * ls + b]; }
};

// One group on lines held in shared memory, in place: the DIF group (then its twiddles) or, for kInv, the inverse
// group (conjugate twiddles, then the DIT DFT). Rows: lanes walk the tasks of a line; columns: lanes walk the lines
// (BL of them, a power of two; lines >= nb are skipped).
template <int R, bool kInv, bool kCols, class Addr>
__device__ __forceinline__ void SmemGroup(const Addr& S, int nb, int BL, int logBL, int logN, int logQ, const float2* __restrict__ tw)
{
   constexpr int r = Log2i(R);
   const int logT = logN - r, q = 1 << logQ;
   const int total = kCols ? (BL << logT) : (nb << logT);
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      int b, u;
      if (kCols)
      {
         b = t & (BL - 1);
         u = t >> logBL;
         if (b >= nb)
            continue;
      }
      else
      {
         b = t >> logT;
         u = t & ((1 << logT) - 1);
      }
      const int j = u & (q - 1), base = ((u >> logQ) << (logQ + r)) | j;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
         v[m] = S(b, base + m * q);
      if (!kInv)
      {
         DifReg<R, false, false>(v);
         if (tw)
            Twiddle<R, false>(v, tw, q, j);
      }
      else
      {
         if (tw)
            Twiddle<R, true>(v, tw, q, j);
         DitReg<R, true>(v);
      }
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, base + m * q) = v[m];
   }
}

#define ISCU_RADIX_SWITCH(r, ...)                                                                                       \
   switch (r)                                                                                                          \
   {                                                                                                                   \
   case 1: { constexpr int R = 2; __VA_ARGS__; } break;                                                                \
   case 2: { constexpr int R = 4; __VA_ARGS__; } break;                                                                \
   case 3: { constexpr int R = 8; __VA_ARGS__; } break;                                                                \
   case 4: { constexpr int R = 16; __VA_ARGS__; } break;                                                               \
   default: { constexpr int R = 32; __VA_ARGS__; } break;                                                              \
   }

// The z pass runs groups of at most 16 points (its plans keep r <= 4), so its kernels carry no 32-point code.
#define ISCU_RADIX_SWITCH16(r, ...)                                                                                     \
   switch (r)                                                                                                          \
   {                                                                                                                   \
   case 1: { constexpr int R = 2; __VA_ARGS__; } break;                                                                \
   case 2: { constexpr int R = 4; __VA_ARGS__; } break;                                                                \
   case 3: { constexpr int R = 8; __VA_ARGS__; } break;                                                                \
   default: { constexpr int R = 16; __VA_ARGS__; } break;                                                              \
   }

__device__ __forceinline__ const float2* GroupTw(const LinePlan& P, const float2* twg, int g)
{
   return P.tw[g] >= 0 ? twg + P.tw[g] : nullptr;
}

// The plan a pass runs: for a codelet (kLogN > 0) the compile-time plan of that length -- every span, pad and index
// shift then folds into the instructions -- with the runtime plan's table offsets; else the runtime plan.
// kKind: 0 rows (y), 1 columns (x), 2 the z pass.
template <int kLogN, int kKind>
__device__ __forceinline__ LinePlan Fixed(const LinePlan& runtime)
{
   if constexpr (kLogN == 0)
      return runtime;
   else
   {
      constexpr LinePlan C = kKind == 2 ? MakeZPlan(kLogN) : MakeLinePlan(kLogN, kKind == 1);
      LinePlan P = runtime;
      P.logN = C.logN;
      P.groups = C.groups;
#pragma unroll
      for (int g = 0; g < 4; ++g)
         P.r[g] = C.r[g];
      return P;
   }
}

// Forward groups 1 .. groups-1 of lines already in shared memory (group 0 done by the pass's loader).
template <bool kCols, class Addr>
__device__ __forceinline__ void ForwardRest(const LinePlan& P, const float2* twg, const Addr& S, int nb, int BL, int logBL)
{
   for (int g = 1; g < P.groups; ++g)
   {
      const int logQ = LogQ(P, g);
      const float2* tw = GroupTw(P, twg, g);
      ISCU_RADIX_SWITCH(P.r[g], (SmemGroup<R, false, kCols>(S, nb, BL, logBL, P.logN, logQ, tw)));
      __syncthreads();
   }
}

// Inverse groups last .. first of lines in shared memory (kMax16: plans of groups of at most 16 points).
template <bool kCols, bool kMax16 = false, class Addr>
__device__ __forceinline__ void InverseRest(const LinePlan& P, const float2* twg, const Addr& S, int nb, int BL, int logBL, int last,
                            int first)
{
   for (int g = last; g >= first; --g)
   {
      const int logQ = LogQ(P, g);
      const float2* tw = GroupTw(P, twg, g);
      if (kMax16)
         ISCU_RADIX_SWITCH16(P.r[g], (SmemGroup<R, true, kCols>(S, nb, BL, logBL, P.logN, logQ, tw)))
      else
         ISCU_RADIX_SWITCH(P.r[g], (SmemGroup<R, true, kCols>(S, nb, BL, logBL, P.logN, logQ, tw)))
      __syncthreads();
   }
}

// ------------------------------------------------------------------------------------------------ passes
struct Dims
{
   int nxv, nyv, nzv;   // valid extent of the input (volume or PSF)
   int GX, GY, GZ, H, NK, G, logH, logGY, logGZ, logG, logGX;
   LinePlan px, py, pz;   // group plans of the H-, GY- and GZ-point transforms
};

// X forward group 0: packed pairs z[n] = x[2n] + i x[2n+1] of row b straight from global memory (lanes walk j, so
// the loads coalesce), DIF group, twiddles, into the column layout.
template <int R, bool kHalf>
__device__ __forceinline__ void XFirst(const ColAddr& S, const float* __restrict__ src, int nxv, int nb, int logQ,
                       const float2* __restrict__ tw, bool pairs)
{
   const int q = 1 << logQ, total = nb << logQ;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t >> logQ, j = t & (q - 1);
      const float* row = src + static_cast<size_t>(b) * nxv;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < (kHalf ? R / 2 : R); ++m)
      {
         const int n = j + m * q;
         if (pairs)
            v[m] = 2 * n < nxv ? __ldg(reinterpret_cast<const float2*>(row) + n) : make_float2(0.f, 0.f);
         else
            v[m] = make_float2(2 * n < nxv ? __ldg(row + 2 * n) : 0.f, 2 * n + 1 < nxv ? __ldg(row + 2 * n + 1) : 0.f);
      }
      DifReg<R, false, kHalf>(v);
      if (tw)
         Twiddle<R, false>(v, tw, q, j);
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, j + m * q) = v[m];
   }
}

// Rows of `in` (nzv x nyv x nxv) -> A[z][k][y], k <= H, y < nyv. grid (ceil(nyv / BY), nzv); BY a power of two;
// smem H * (BY + 1) float2. kLogH: the codelet's log2 H (0: any H).
template <int kLogH>
__global__ void __launch_bounds__(kThreads, kMinCtas) XForwardKernel(const float* __restrict__ in, Dims d, int BY, int logBY,
                                                           const float2* __restrict__ tw, const float2* __restrict__ twg,
                                                           float2* __restrict__ A)
{
   extern __shared__ float2 s[];
   const LinePlan P = Fixed<kLogH, 1>(d.px);
   const int z = blockIdx.y, y0 = blockIdx.x * BY;
   const int nb = min(BY, d.nyv - y0), H = 1 << P.logN, logH = P.logN;
   const ColAddr S{s, BY + 1};
   const float* src = in + (static_cast<size_t>(z) * d.nyv + y0) * d.nxv;
   const bool pairs = (d.nxv & 1) == 0 && (reinterpret_cast<uintptr_t>(in) & 7) == 0;
   const int logQ0 = LogQ(P, 0);
   const float2* tw0 = GroupTw(P, twg, 0);
   if (d.nxv <= H)
      ISCU_RADIX_SWITCH(P.r[0], (XFirst<R, true>(S, src, d.nxv, nb, logQ0, tw0, pairs)))
   else
      ISCU_RADIX_SWITCH(P.r[0], (XFirst<R, false>(S, src, d.nxv, nb, logQ0, tw0, pairs)))
   __syncthreads();
   ForwardRest<true>(P, twg, S, nb, BY, logBY);
   // X[k] = ((Z[k] + conj Z[H-k]) - i W_GX^k (Z[k] - conj Z[H-k])) / 2, Z in bit-reversed order
   for (int t = threadIdx.x; t < (H + 1) * BY; t += blockDim.x)
   {
      const int k = t >> logBY, b = t & (BY - 1);
      if (b >= nb)
         continue;
      const float2 zk = S(b, Rev(k & (H - 1), logH));
      const float2 zm = Conj(S(b, Rev((H - k) & (H - 1), logH)));
      const float2 e = Cadd(zk, zm), o = Csub(zk, zm);
      const float2 w = __ldg(tw + (k << (d.logG - d.logGX)));
      const float2 wo = Cmul(w, o);   // then times -i: (x, y) -> (y, -x)
      const float2 X = make_float2(0.5f * (e.x + wo.y), 0.5f * (e.y - wo.x));
      A[(static_cast<size_t>(z) * d.NK + k) * d.nyv + y0 + b] = X;
   }
}

// Y forward group 0: rows of A (nyv values, zero beyond) straight from global memory, lanes walking j.
template <int R, bool kHalf>
__device__ __forceinline__ void YFirst(const RowAddr& S, const float2* __restrict__ rows, int nyv, int nb, int logQ,
                       const float2* __restrict__ tw)
{
   const int q = 1 << logQ, total = nb << logQ;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t >> logQ, j = t & (q - 1);
      const float2* row = rows + static_cast<size_t>(b) * nyv;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < (kHalf ? R / 2 : R); ++m)
      {
         const int n = j + m * q;
         v[m] = n < nyv ? __ldg(row + n) : make_float2(0.f, 0.f);
      }
      DifReg<R, false, kHalf>(v);
      if (tw)
         Twiddle<R, false>(v, tw, q, j);
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, j + m * q) = v[m];
   }
}

__device__ __forceinline__ RowAddr RowsOf(float2* s, const LinePlan& P)
{
   const int rl = P.r[P.groups - 1];
   return RowAddr{s, (1 << P.logN) + ((1 << P.logN) >> rl), rl};
}

// A rows (nyv values per (z, k)) -> B[z][k][p], p = bit-reversed ky. grid (ceil(NK / BK), nzv); smem BK rows.
// kLogN: the codelet's log2 GY (0: any GY).
template <int kLogN>
__global__ void __launch_bounds__(kThreads, kMinCtas) YForwardKernel(const float2* __restrict__ A, Dims d, int BK,
                                                           const float2* __restrict__ twg, float2* __restrict__ B)
{
   extern __shared__ float2 s[];
   const LinePlan P = Fixed<kLogN, 0>(d.py);
   const int z = blockIdx.y, k0 = blockIdx.x * BK, nb = min(BK, d.NK - k0), N = 1 << P.logN;
   const RowAddr S = RowsOf(s, P);
   const float2* rows = A + (static_cast<size_t>(z) * d.NK + k0) * d.nyv;
   const int logQ0 = LogQ(P, 0);
   const float2* tw0 = GroupTw(P, twg, 0);
   if (2 * d.nyv <= N)
      ISCU_RADIX_SWITCH(P.r[0], (YFirst<R, true>(S, rows, d.nyv, nb, logQ0, tw0)))
   else
      ISCU_RADIX_SWITCH(P.r[0], (YFirst<R, false>(S, rows, d.nyv, nb, logQ0, tw0)))
   __syncthreads();
   ForwardRest<false>(P, twg, S, nb, 1, 0);
   float2* out = B + (static_cast<size_t>(z) * d.NK + k0) * N;
   for (int t = threadIdx.x; t < nb * N; t += blockDim.x)
   {
      const int b = t >> P.logN, p = t & (N - 1);
      out[static_cast<size_t>(b) * N + p] = S(b, p);
   }
}

// Y inverse group 0: conjugate twiddles, DIT, natural order out; rows [oy, oy + nyv) to global memory.
template <int R>
__device__ __forceinline__ void YLast(const RowAddr& S, float2* __restrict__ rows, int nyv, int oy, int nb, int logQ,
                      const float2* __restrict__ tw)
{
   const int q = 1 << logQ, total = nb << logQ;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t >> logQ, j = t & (q - 1);
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
         v[m] = S(b, j + m * q);
      if (tw)
         Twiddle<R, true>(v, tw, q, j);
      DitReg<R, true>(v);
      float2* row = rows + static_cast<size_t>(b) * nyv;
#pragma unroll
      for (int m = 0; m < R; ++m)
      {
         const int y = j + m * q - oy;
         if (y >= 0 && y < nyv)
            row[y] = v[m];
      }
   }
}

// B rows (bit-reversed ky) -> inverse GY-point FFT -> rows [oy, oy + nyv) into A[z][k][y]. grid (ceil(NK / BK), nzv).
template <int kLogN>
__global__ void __launch_bounds__(kThreads, kMinCtas) YInverseKernel(const float2* __restrict__ B, Dims d, int BK, int oy,
                                                           const float2* __restrict__ twg, float2* __restrict__ A)
{
   extern __shared__ float2 s[];
   const LinePlan P = Fixed<kLogN, 0>(d.py);
   const int z = blockIdx.y, k0 = blockIdx.x * BK, nb = min(BK, d.NK - k0), N = 1 << P.logN;
   const RowAddr S = RowsOf(s, P);
   const float2* in = B + (static_cast<size_t>(z) * d.NK + k0) * N;
   for (int t = threadIdx.x; t < nb * N; t += blockDim.x)
      CopyAsync8(&S(t >> P.logN, t & (N - 1)), in + t);
   CopyAsyncWait();
   __syncthreads();
   InverseRest<false>(P, twg, S, nb, 1, 0, P.groups - 1, 1);
   float2* rows = A + (static_cast<size_t>(z) * d.NK + k0) * d.nyv;
   ISCU_RADIX_SWITCH(P.r[0], (YLast<R>(S, rows, d.nyv, oy, nb, LogQ(P, 0), GroupTw(P, twg, 0))));
}

// The asynchronous copies of one block of columns into a stage buffer: B's nzv planes at in[n BZ + b] and, when
// convolving, the PSF spectrum's GZ planes after them. 16-byte copies of column pairs (nb is even whenever BZ >= 2:
// GY and BZ are powers of two, GY >= 4), else 8-byte ones.
template <bool kConvolve>
__device__ __forceinline__ void ZPrefetch(const float2* __restrict__ B, const float2* __restrict__ Kh, size_t plane, size_t col,
                          int nzv, int GZ, int nb, int BZ, int logBZ, float2* in)
{
   float2* ks = in + (static_cast<size_t>(nzv) << logBZ);
   if ((nb & 1) == 0)
   {
      const int logPairs = logBZ - 1, pairs = BZ >> 1;
      for (int t = threadIdx.x; t < (nzv << logPairs); t += blockDim.x)
      {
         const int n = t >> logPairs, b = (t & (pairs - 1)) << 1;
         if (b < nb)
            CopyAsync16(in + (n << logBZ) + b, B + n * plane + col + b);
      }
      if (kConvolve)
         for (int t = threadIdx.x; t < (GZ << logPairs); t += blockDim.x)
         {
            const int n = t >> logPairs, b = (t & (pairs - 1)) << 1;
            if (b < nb)
               CopyAsync16(ks + (n << logBZ) + b, Kh + n * plane + col + b);
         }
   }
   else
   {
      for (int t = threadIdx.x; t < (nzv << logBZ); t += blockDim.x)
      {
         const int n = t >> logBZ, b = t & (BZ - 1);
         if (b < nb)
            CopyAsync8(in + t, B + n * plane + col + b);
      }
      if (kConvolve)
         for (int t = threadIdx.x; t < (GZ << logBZ); t += blockDim.x)
         {
            const int n = t >> logBZ, b = t & (BZ - 1);
            if (b < nb)
               CopyAsync8(ks + t, Kh + n * plane + col + b);
         }
   }
}

// Z forward group 0: the block's columns from its stage buffer (lanes walk the columns), DIF group, twiddles.
template <int R, bool kHalf>
__device__ __forceinline__ void ZFirst(const ColAddr& S, const float2* in, int nzv, int nb, int BL, int logBL, int logQ,
                       const float2* __restrict__ tw)
{
   const int q = 1 << logQ, total = BL << logQ;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t & (BL - 1), j = t >> logBL;
      if (b >= nb)
         continue;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < (kHalf ? R / 2 : R); ++m)
      {
         const int n = j + m * q;
         v[m] = n < nzv ? in[(n << logBL) + b] : make_float2(0.f, 0.f);
      }
      DifReg<R, false, kHalf>(v);
      if (tw)
         Twiddle<R, false>(v, tw, q, j);
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, j + m * q) = v[m];
   }
}

// The last forward group (span 1, contiguous points; skipped when group 0 was the only one), then either the
// spectrum out to Kh (kConvolve false) or times the PSF spectrum (KS: this CTA's columns of Kh, prefetched into
// shared memory) and the first inverse group, back into shared memory.
template <int R, bool kConvolve>
__device__ __forceinline__ void ZTurn(const ColAddr& S, const float2* KS, float2* __restrict__ Kh, size_t plane, size_t col, int nb,
                      int BL, int logBL, int logN, bool dif, bool dit)
{
   constexpr int r = Log2i(R);
   const int logT = logN - r, total = BL << logT;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t & (BL - 1), base = (t >> logBL) << r;
      if (b >= nb)
         continue;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
         v[m] = S(b, base + m);
      if (dif)
         DifReg<R, false, false>(v);
      if constexpr (!kConvolve)
      {
#pragma unroll
         for (int m = 0; m < R; ++m)
            Kh[(base + m) * plane + col + b] = v[m];
      }
      else
      {
#pragma unroll
         for (int m = 0; m < R; ++m)
            v[m] = Cmul(v[m], KS[(base + m) * BL + b]);
         if (dit)
            DitReg<R, true>(v);
#pragma unroll
         for (int m = 0; m < R; ++m)
            S(b, base + m) = v[m];
      }
   }
}

// Z inverse group 0: conjugate twiddles, DIT (skipped when group 0 was the only one, ZTurn did it), planes
// [oz, oz + nzv) to global memory.
template <int R>
__device__ __forceinline__ void ZLast(const ColAddr& S, float2* __restrict__ B, size_t plane, size_t col, int nzv, int oz, int nb,
                      int BL, int logBL, int logQ, const float2* __restrict__ tw, bool dit)
{
   const int q = 1 << logQ, total = BL << logQ;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t & (BL - 1), j = t >> logBL;
      if (b >= nb)
         continue;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
         v[m] = S(b, j + m * q);
      if (dit)
      {
         if (tw)
            Twiddle<R, true>(v, tw, q, j);
         DitReg<R, true>(v);
      }
#pragma unroll
      for (int m = 0; m < R; ++m)
      {
         const int zz = j + m * q - oz;
         if (zz >= 0 && zz < nzv)
            B[zz * plane + col + b] = v[m];
      }
   }
}

// Columns along z of B (nzv planes) -> GZ-point forward FFT -> either the PSF spectrum Kh[pz][k][p] (all GZ planes,
// forward only) or, times Kh, the inverse FFT cropped to planes [oz, oz + nzv) back into B. Persistent: CTA c takes
// column blocks c, c + gridDim.x, ... (block blk: k = blk / blocksPerK, columns from p0 = (blk % blocksPerK) BZ),
// and with stages = 2 the next block's B planes and PSF spectrum are copied into shared memory while this one is
// transformed (stages = 1 where two stage buffers do not fit: the copies then follow the block). BZ a power of two;
// smem (GZ + stages (nzv + GZ when convolving)) BZ float2, column layout.
template <bool kConvolve, int kLogN>
__global__ void __launch_bounds__(kThreads, kMinCtas) ZKernel(float2* __restrict__ B, Dims d, int BZ, int logBZ,
                                                              int blocksPerK, int nBlocks, int stages, int oz,
                                                              const float2* __restrict__ twg, float2* __restrict__ Kh)
{
   extern __shared__ float2 s[];
   const size_t plane = static_cast<size_t>(d.NK) * d.GY;
   const LinePlan P = Fixed<kLogN, 2>(d.pz);
   const int GZ = 1 << P.logN;
   const ColAddr S{s, BZ};
   const size_t stageElems = static_cast<size_t>(d.nzv + (kConvolve ? GZ : 0)) << logBZ;
   float2* stage0 = s + (static_cast<size_t>(GZ) << logBZ);
   const int logQ0 = LogQ(P, 0);
   const float2* tw0 = GroupTw(P, twg, 0);
   const bool half = 2 * d.nzv <= (1 << P.logN), single = P.groups == 1;
   auto colOf = [&](int blk, int& nb) {
      const int k = blk / blocksPerK, p0 = (blk - k * blocksPerK) << logBZ;
      nb = min(BZ, d.GY - p0);
      return static_cast<size_t>(k) * d.GY + p0;
   };
   int blk = blockIdx.x;
   if (blk < nBlocks)
   {
      int nb;
      const size_t col = colOf(blk, nb);
      ZPrefetch<kConvolve>(B, Kh, plane, col, d.nzv, GZ, nb, BZ, logBZ, stage0);
   }
   CopyAsyncCommit();
   for (int i = 0; blk < nBlocks; ++i, blk += gridDim.x)
   {
      const int buf = stages == 2 ? (i & 1) : 0, next = blk + gridDim.x;
      if (stages == 2 && next < nBlocks)
      {
         int nbn;
         const size_t coln = colOf(next, nbn);
         ZPrefetch<kConvolve>(B, Kh, plane, coln, d.nzv, GZ, nbn, BZ, logBZ, stage0 + (buf ^ 1) * stageElems);
      }
      CopyAsyncCommit();
      CopyAsyncWaitPrior();   // this block's copies (the group before the one just committed)
      __syncthreads();
      int nb;
      const size_t col = colOf(blk, nb);
      const float2* in = stage0 + buf * stageElems;
      const float2* KS = in + (static_cast<size_t>(d.nzv) << logBZ);
      if (half)
         ISCU_RADIX_SWITCH16(P.r[0], (ZFirst<R, true>(S, in, d.nzv, nb, BZ, logBZ, logQ0, tw0)))
      else
         ISCU_RADIX_SWITCH16(P.r[0], (ZFirst<R, false>(S, in, d.nzv, nb, BZ, logBZ, logQ0, tw0)))
      __syncthreads();
      for (int g = 1; g < P.groups - 1; ++g)
      {
         ISCU_RADIX_SWITCH16(P.r[g],
                           (SmemGroup<R, false, true>(S, nb, BZ, logBZ, P.logN, LogQ(P, g), GroupTw(P, twg, g))));
         __syncthreads();
      }
      ISCU_RADIX_SWITCH16(P.r[P.groups - 1],
                        (ZTurn<R, kConvolve>(S, KS, Kh, plane, col, nb, BZ, logBZ, P.logN, !single, true)));
      if (kConvolve)
      {
         __syncthreads();
         if (!single)
            InverseRest<true, true>(P, twg, S, nb, BZ, logBZ, P.groups - 2, 1);
         ISCU_RADIX_SWITCH16(P.r[0], (ZLast<R>(S, B, plane, col, d.nzv, oz, nb, BZ, logBZ, logQ0, tw0, !single)));
      }
      __syncthreads();   // the block's shared memory (S and its stage buffer) is free again
      if (stages == 1 && next < nBlocks)
      {
         int nbn;
         const size_t coln = colOf(next, nbn);
         ZPrefetch<kConvolve>(B, Kh, plane, coln, d.nzv, GZ, nbn, BZ, logBZ, stage0);
         CopyAsyncCommit();
      }
   }
   CopyAsyncWait();
}

// X inverse, the last DIF group's inverse (span 1, no twiddles) straight from A: Z'[k] = (X[k] + conj X[H-k]) +
// i W_GX^-k (X[k] - conj X[H-k]) at bit-reversed slots, lanes walking the rows.
template <int R>
__device__ __forceinline__ void XLoad(const ColAddr& S, const float2* __restrict__ Az, int nyv, int y0, int nb, int BL, int logBL,
                      int H, int logH, const float2* __restrict__ tw, int twShift)
{
   constexpr int r = Log2i(R);
   const int logT = logH - r, total = BL << logT;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t & (BL - 1), base = (t >> logBL) << r;
      if (b >= nb)
         continue;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
      {
         const int k = Rev(base + m, logH);
         const float2 xk = __ldg(Az + static_cast<size_t>(k) * nyv + y0 + b);
         const float2 xm = Conj(__ldg(Az + static_cast<size_t>(H - k) * nyv + y0 + b));
         const float2 w = Conj(__ldg(tw + (k << twShift)));
         const float2 e = Cadd(xk, xm), o = Cmul(Csub(xk, xm), w);
         v[m] = make_float2(e.x - o.y, e.y + o.x);   // e + i o
      }
      DitReg<R, true>(v);
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, base + m) = v[m];
   }
}

// A (half spectrum along x, per (z, y)) -> GX reals -> columns [ox, ox + nxv), scaled, max(0, .) + background ->
// the photon frames. grid (ceil(nyv / BY), nzv), BY a power of two; smem H * (BY + 1) float2.
template <int kLogH>
__global__ void __launch_bounds__(kThreads, kMinCtas) XInverseKernel(const float2* __restrict__ A, Dims d, int BY,
                                                                     int logBY, int ox, float scale, float background,
                                                                     int clamp, const float2* __restrict__ tw,
                                                                     const float2* __restrict__ twg,
                                                                     float* __restrict__ image)
{
   extern __shared__ float2 s[];
   const LinePlan P = Fixed<kLogH, 1>(d.px);
   const int z = blockIdx.y, y0 = blockIdx.x * BY, nb = min(BY, d.nyv - y0), H = 1 << P.logN;
   const ColAddr S{s, BY + 1};
   const float2* Az = A + static_cast<size_t>(z) * d.NK * d.nyv;
   ISCU_RADIX_SWITCH(P.r[P.groups - 1],
                     (XLoad<R>(S, Az, d.nyv, y0, nb, BY, logBY, H, P.logN, tw, d.logG - d.logGX)));
   __syncthreads();
   InverseRest<true>(P, twg, S, nb, BY, logBY, P.groups - 2, 0);
   float* out = image + (static_cast<size_t>(z) * d.nyv + y0) * d.nxv;
   for (int t = threadIdx.x; t < nb * d.nxv; t += blockDim.x)
   {
      const int b = t / d.nxv, x = t % d.nxv;
      const int m = x + ox;
      const float2 c = S(b, m >> 1);
      const float v = (m & 1 ? c.y : c.x) * scale;
      out[t] = (clamp && !(v > 0.f) ? 0.f : v) + background;
   }
}

// The noise chain of every pixel of the photon frames (frame frame0 + plane) -> ADU. A kernel of its own: the
// float64 chain wants many resident warps, the transforms wants registers. grid (ceil(nx ny / 256), nz).
__global__ void __launch_bounds__(256) WfNoiseKernel(const float* __restrict__ photons, uint32_t npix, StaticView st,
                                                     CameraView cam, uint32_t seed, uint32_t frame0,
                                                     uint16_t* __restrict__ adu)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= npix)
      return;
   const size_t o = static_cast<size_t>(blockIdx.y) * npix + i;
   CounterRng u(seed, frame0 + blockIdx.y);
   adu[o] = NoisePixel(photons[o], i, cam, st, u);
}

// A camera plan's photon frames (WidefieldImages::Render, WidefieldRender.cpp:547-586): pixel (X, Y) of plane z is the
// float64 sum, row by row, of its up x up cells (already clamped at 0) of the FOV window, as float, plus the
// background. grid (ceil(fovW fovH / 256), nz).
__global__ void __launch_bounds__(256) WfBinKernel(const float* __restrict__ cells, uint32_t nx, uint32_t ny,
                                                   uint32_t fovX0, uint32_t fovY0, uint32_t fovW, uint32_t fovH,
                                                   uint32_t up, float background, float* __restrict__ photons)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= fovW * fovH)
      return;
   const uint32_t X = i % fovW, Y = i / fovW;
   const float* plane = cells + static_cast<size_t>(blockIdx.y) * nx * ny;
   double acc = 0.0;
   for (uint32_t sy = 0; sy < up; ++sy)
   {
      const float* row = plane + static_cast<size_t>(fovY0 + Y * up + sy) * nx + fovX0 + X * up;
      for (uint32_t sx = 0; sx < up; ++sx)
         acc += row[sx];
   }
   photons[static_cast<size_t>(blockIdx.y) * fovW * fovH + i] = static_cast<float>(acc) + background;
}

// The kernel volume of a plan made from a kernel slot: plane j = w0[j] K[p0[j]] + w1[j] K[p1[j]] of the D x D cell
// kernels K (the second term only where w1 != 0), the blend WidefieldScene applies to kernel spectra
// (ChannelImageStep, WidefieldRender.cpp:1790-1801) made here on the cells.
__global__ void WfKernelVolumeKernel(const float* __restrict__ K, int D2, const int2* __restrict__ planes,
                                     const float2* __restrict__ weights, int kz, float* __restrict__ out)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= kz * D2)
      return;
   const int j = i / D2, c = i - j * D2;
   const int2 p = planes[j];
   const float2 w = weights[j];
   float v = w.x * K[static_cast<size_t>(p.x) * D2 + c];
   if (w.y != 0.0f)
      v = v + w.y * K[static_cast<size_t>(p.y) * D2 + c];
   out[i] = v;
}

// ---------------------------------------------------------------------------- drifting sample (RenderShiftedImages)
// The frame's spectrum S = sum_c coef[c] spec[c] (float complex, channels in order, zero coefficients skipped, as
// RenderShiftedImages adds them, WidefieldRender.cpp:2905-2935), times ApplyShiftRamp's phase (DriftShift.cpp:23-48:
// exp(2 pi i (kx sx / nx + ky' sy / ny)), ky' the signed row frequency, the Nyquist terms their cosine only; the
// product formed in float64 and rounded to float), then the inverse transform, as conj(forward(conj S)): column pass
// (along ky, every kx) here, row pass (the packed real inverse along kx, the window's rows) in ShiftRowsKernel.

struct ShiftArgs
{
   const float2* spec;   // channels x ny x W, RealFft2d's layout
   const float* coef;    // frames x channels
   const double* shift;  // frames x 2: (fracX, fracY) in cells
   int nChannels, nx, ny, W;
};

// Column pass group 0: S conjugated, straight from the channels (lanes walk kx), DIF group, twiddles.
template <int R>
__device__ __forceinline__ void ShiftFirst(const ColAddr& S, const ShiftArgs& a, int f, int kx0, int nb, int BL,
                                          int logBL, int logQ, const float2* __restrict__ tw, const double2* py)
{
   const int q = 1 << logQ, total = BL << logQ;
   const float* coef = a.coef + static_cast<size_t>(f) * a.nChannels;
   const double sx = a.shift[2 * f];
   const bool ramp = a.shift[2 * f] != 0.0 || a.shift[2 * f + 1] != 0.0;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t & (BL - 1), j = t >> logBL, kx = kx0 + b;
      if (b >= nb)
         continue;
      double2 pxv = make_double2(1.0, 0.0);
      if (ramp)
      {
         double sn, cs;
         sincospi(2.0 * kx * sx / a.nx, &sn, &cs);
         pxv = make_double2(cs, kx == a.nx / 2 ? 0.0 : sn);
      }
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
         v[m] = make_float2(0.f, 0.f);
      // channels in order, a channel's loads issued eight at a time (every point's sum keeps the channel order)
      constexpr int kBatch = R < 8 ? R : 8;
      for (int c = 0; c < a.nChannels; ++c)
      {
         const float w = coef[c];
         if (w == 0.0f)
            continue;
         const float2* sc = a.spec + (static_cast<size_t>(c) * a.ny + j) * a.W + kx;
#pragma unroll
         for (int m0 = 0; m0 < R; m0 += kBatch)
         {
            float2 sp[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
               sp[u] = __ldg(sc + static_cast<size_t>(m0 + u) * q * a.W);
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
            {
               v[m0 + u].x = v[m0 + u].x + w * sp[u].x;
               v[m0 + u].y = v[m0 + u].y + w * sp[u].y;
            }
         }
      }
#pragma unroll
      for (int m = 0; m < R; ++m)
      {
         float2 acc = v[m];
         if (ramp)
         {
            const double2 pyv = py[j + m * q];
            const double pr = pxv.x * pyv.x - pxv.y * pyv.y, pi = pxv.x * pyv.y + pxv.y * pyv.x;
            const double vr = acc.x, vi = acc.y;
            acc = make_float2(static_cast<float>(vr * pr - vi * pi), static_cast<float>(vr * pi + vi * pr));
         }
         v[m] = make_float2(acc.x, -acc.y);   // conjugated: the forward transform then gives the inverse's conjugate
      }
      DifReg<R, false, false>(v);
      if (tw)
         Twiddle<R, false>(v, tw, q, j);
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, j + m * q) = v[m];
   }
}

// grid (ceil(W / BZ), frames), BZ a power of two; smem ny * BZ float2 + ny double2 (the row ramp).
// T[f][p][kx] = forward_y(conj S)[rev p], every column kx < W.
__global__ void __launch_bounds__(kThreads, kMinCtas) ShiftColumnsKernel(ShiftArgs a, LinePlan P, int BZ, int logBZ,
                                                                        const float2* __restrict__ twg,
                                                                        float2* __restrict__ T)
{
   extern __shared__ __align__(16) unsigned char smem[];
   double2* py = reinterpret_cast<double2*>(smem);
   float2* s = reinterpret_cast<float2*>(py + a.ny);
   const ColAddr S{s, BZ};
   const int f = blockIdx.y, kx0 = blockIdx.x * BZ, nb = min(BZ, a.W - kx0);
   const double sy = a.shift[2 * f + 1];
   for (int ky = threadIdx.x; ky < a.ny; ky += blockDim.x)
   {
      const int k = ky <= a.ny / 2 ? ky : ky - a.ny;
      double sn, cs;
      sincospi(2.0 * k * sy / a.ny, &sn, &cs);
      py[ky] = make_double2(cs, ky == a.ny / 2 ? 0.0 : sn);
   }
   __syncthreads();
   ISCU_RADIX_SWITCH(P.r[0], (ShiftFirst<R>(S, a, f, kx0, nb, BZ, logBZ, LogQ(P, 0), GroupTw(P, twg, 0), py)));
   __syncthreads();
   ForwardRest<true>(P, twg, S, nb, BZ, logBZ);
   float2* out = T + static_cast<size_t>(f) * a.ny * a.W;
   for (int t = threadIdx.x; t < (a.ny << logBZ); t += blockDim.x)
   {
      const int b = t & (BZ - 1), p = t >> logBZ;
      if (b < nb)
         out[static_cast<size_t>(p) * a.W + kx0 + b] = S(b, p);
   }
}

// Row pass, the last DIF group's inverse (span 1) from the staged rows: Z'[k] = (X[k] + conj X[H-k]) +
// i W_nx^-k (X[k] - conj X[H-k]) at bit-reversed slots, X the row's half spectrum.
template <int R>
__device__ __forceinline__ void ShiftRowLoad(const ColAddr& S, const float2* rows, int W, int nb, int BL, int logBL,
                                            int H, int logH, const float2* __restrict__ tw, int twShift)
{
   constexpr int r = Log2i(R);
   const int logT = logH - r, total = BL << logT;
   for (int t = threadIdx.x; t < total; t += blockDim.x)
   {
      const int b = t & (BL - 1), base = (t >> logBL) << r;
      if (b >= nb)
         continue;
      const float2* X = rows + b * W;
      float2 v[R];
#pragma unroll
      for (int m = 0; m < R; ++m)
      {
         const int k = Rev(base + m, logH);
         const float2 xk = X[k], xm = Conj(X[H - k]);
         const float2 w = Conj(__ldg(tw + (k << twShift)));
         const float2 e = Cadd(xk, xm), o = Cmul(Csub(xk, xm), w);
         v[m] = make_float2(e.x - o.y, e.y + o.x);
      }
      DitReg<R, true>(v);
#pragma unroll
      for (int m = 0; m < R; ++m)
         S(b, base + m) = v[m];
   }
}

// grid (ceil(camRows / rowsPerCta), frames); BL lines (a power of two >= rowsPerCta up); smem BL W float2 (the rows)
// + H (BL + 1) float2 (the transform). cam[f][Y][X] += float(sum over up x up cells of max(0, cell) (float64) x
// scale), the cells at rows y0 + Y up + sy, columns x0 + X up + sx of the image (1 / (nx ny)) x inverse.
__global__ void __launch_bounds__(kThreads, kMinCtas) ShiftRowsKernel(const float2* __restrict__ T, LinePlan P, int nx,
                                                                     int ny, int W, int BL, int logBL, int rowsPerCta,
                                                                     int up, int x0, int y0, int camW, int camH,
                                                                     float scale, const float2* __restrict__ tw,
                                                                     int twShift, const float2* __restrict__ twg,
                                                                     float* __restrict__ cam)
{
   extern __shared__ __align__(16) unsigned char smem[];
   float2* rows = reinterpret_cast<float2*>(smem);
   const ColAddr S{rows + BL * W, BL + 1};
   const int f = blockIdx.y, Y0 = blockIdx.x * rowsPerCta, camRows = min(rowsPerCta, camH - Y0);
   const int nb = camRows * up, H = nx / 2;
   const int logNy = Log2i(ny);
   // the window's rows, conjugated back: the unnormalised inverse along y, half spectrum along x
   const float2* Tf = T + static_cast<size_t>(f) * ny * W;
   constexpr int kU = 8;   // loads in flight per thread
   const int nIn = nb * W;
   for (int t0 = threadIdx.x; t0 < nIn; t0 += kU * blockDim.x)
   {
      float2 v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u)
      {
         const int t = t0 + u * blockDim.x;
         if (t < nIn)
         {
            const int b = t / W, k = t - b * W;
            const int y = y0 + Y0 * up + b;
            v[u] = __ldg(Tf + static_cast<size_t>(Rev(y, logNy)) * W + k);
         }
      }
#pragma unroll
      for (int u = 0; u < kU; ++u)
      {
         const int t = t0 + u * blockDim.x;
         if (t < nIn)
            rows[t] = Conj(v[u]);
      }
   }
   __syncthreads();
   ISCU_RADIX_SWITCH(P.r[P.groups - 1], (ShiftRowLoad<R>(S, rows, W, nb, BL, logBL, H, P.logN, tw, twShift)));
   __syncthreads();
   InverseRest<true>(P, twg, S, nb, BL, logBL, P.groups - 2, 0);
   const float norm = 1.0f / (static_cast<float>(nx) * static_cast<float>(ny));
   const int nOut = camRows * camW;
   float* camF = cam + (static_cast<size_t>(f) * camH + Y0) * camW;
   for (int t0 = threadIdx.x; t0 < nOut; t0 += kU * blockDim.x)
   {
      float o[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u)
      {
         const int t = t0 + u * blockDim.x;
         if (t < nOut)
            o[u] = camF[t];
      }
#pragma unroll
      for (int u = 0; u < kU; ++u)
      {
         const int t = t0 + u * blockDim.x;
         if (t >= nOut)
            continue;
         const int Yc = t / camW, X = t - Yc * camW;
         double acc = 0.0;
         for (int sy = 0; sy < up; ++sy)
            for (int sx = 0; sx < up; ++sx)
            {
               const int b = Yc * up + sy, x = x0 + X * up + sx;
               const float2 c = S(b, x >> 1);
               const float v = (x & 1 ? c.y : c.x) * norm;
               acc += v > 0.f ? v : 0.f;
            }
         camF[t] = o[u] + static_cast<float>(acc * scale);
      }
   }
}

__global__ void TwiddleKernel(int G, float2* tw)
{
   const int j = blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= G)
      return;
   double sn, cs;
   sincospi(-2.0 * j / G, &sn, &cs);
   tw[j] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
}

// A group's table: entry m q + j = W_M^(j rev_r(m)), M = q 2^r, rounded from float64.
__global__ void GroupTwiddleKernel(int logQ, int r, float2* out)
{
   const int M = 1 << (logQ + r), i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= M)
      return;
   const int m = i >> logQ, j = i & ((1 << logQ) - 1);
   const int e = j * (r ? static_cast<int>(__brev(static_cast<unsigned>(m)) >> (32 - r)) : 0);
   double sn, cs;
   sincospi(-2.0 * e / M, &sn, &cs);
   out[i] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
}

int Log2(uint32_t v)
{
   int l = 0;
   while ((1u << l) < v)
      ++l;
   return l;
}

uint32_t Pow2AtLeast(uint32_t v)
{
   uint32_t p = 1;
   while (p < v)
      p <<= 1;
   return p;
}

int PlaceTables(LinePlan& P, int offset)
{
   int used = 0;
   for (int g = 0; g < P.groups; ++g)
   {
      const int logQ = LogQ(P, g);
      if (logQ == 0)
         continue;
      P.tw[g] = offset + used;
      used += 1 << (logQ + P.r[g]);
   }
   return used;
}

int PowTwoAtMost(int v)
{
   int p = 1;
   while (p * 2 <= v)
      p *= 2;
   return p;
}

// Lines per CTA for each pass, sized to the shared-memory budget.
int XLines(int H) { return PowTwoAtMost(std::max<int>(1, std::min<int>(16, kSmemBudget / (static_cast<size_t>(H) * sizeof(float2)) - 1))); }
size_t XSmem(int H, int BY) { return static_cast<size_t>(H) * (BY + 1) * sizeof(float2); }
size_t RowBytes(const LinePlan& P)
{
   const int N = 1 << P.logN;
   return static_cast<size_t>(N + (N >> P.r[P.groups - 1])) * sizeof(float2);
}
int YLines(const LinePlan& P)
{
   const int N = 1 << P.logN;
   return std::max<int>(1, std::min<int>(std::max(1, 8192 / N), static_cast<int>(kSmemBudget / RowBytes(P))));
}
// The z pass's column blocks: BZ columns per block (a power of two), `stages` stage buffers, the persistent grid.
struct ZLaunch
{
   int BZ = 1, logBZ = 0, stages = 1, blocksPerK = 1, nBlocks = 1, grid = 1;
   size_t smem = 0;
};

size_t ZSmem(const Dims& d, int BZ, int stages, bool convolve)
{
   return (static_cast<size_t>(d.GZ) + stages * static_cast<size_t>(d.nzv + (convolve ? d.GZ : 0))) * BZ *
          sizeof(float2);
}

template <bool kConvolve, int kLogN>
int ZPlan(const iscu_ctx* ctx, const Dims& d, ZLaunch& z);

// Codelets: the transform lengths each pass is compiled for (log2 of X's half length H, of GY, of GZ); any other
// length runs the runtime-plan kernel (K = 0).
#define ISCU_WF_CODELETS(logN, a, b, c, ...)                                                                            \
   switch (logN)                                                                                                       \
   {                                                                                                                   \
   case a: { constexpr int K = a; __VA_ARGS__; } break;                                                                \
   case b: { constexpr int K = b; __VA_ARGS__; } break;                                                                \
   case c: { constexpr int K = c; __VA_ARGS__; } break;                                                                \
   default: { constexpr int K = 0; __VA_ARGS__; } break;                                                               \
   }
#define ISCU_WF_X_CODELETS(logN, ...) ISCU_WF_CODELETS(logN, 8, 9, 10, __VA_ARGS__)
#define ISCU_WF_Y_CODELETS(logN, ...) ISCU_WF_CODELETS(logN, 9, 10, 11, __VA_ARGS__)
#define ISCU_WF_Z_CODELETS(logN, ...) ISCU_WF_CODELETS(logN, 6, 7, 8, __VA_ARGS__)

// The forward x and y passes of a (kzv x kyv x kxv) volume into A, B.
int ForwardXY(iscu_wf_plan* p, const float* in, const Dims& d, float2* A, float2* B, bool mark = false)
{
   iscu_ctx* ctx = p->ctx;
   const float2* tw = p->tw.as<float2>();
   const float2* twg = p->twg.as<float2>();
   const int BY = XLines(d.H);
   ISCU_WF_X_CODELETS(d.logH, (XForwardKernel<K><<<dim3((d.nyv + BY - 1) / BY, d.nzv), kThreads, XSmem(d.H, BY),
                                                 ctx->stream>>>(in, d, BY, Log2(BY), tw, twg, A)));
   ISCU_CK_LAUNCH(ctx, "XForwardKernel");
   if (mark)
      p->Mark(1);
   const int BK = YLines(d.py);
   ISCU_WF_Y_CODELETS(d.logGY, (YForwardKernel<K><<<dim3((d.NK + BK - 1) / BK, d.nzv), kThreads,
                                                    BK * RowBytes(d.py), ctx->stream>>>(A, d, BK, twg, B)));
   ISCU_CK_LAUNCH(ctx, "YForwardKernel");
   return ISCU_OK;
}

Dims MakeDims(const iscu_wf_plan* p, uint32_t nxv, uint32_t nyv, uint32_t nzv)
{
   Dims d;
   d.nxv = static_cast<int>(nxv);
   d.nyv = static_cast<int>(nyv);
   d.nzv = static_cast<int>(nzv);
   d.GX = static_cast<int>(p->GX);
   d.GY = static_cast<int>(p->GY);
   d.GZ = static_cast<int>(p->GZ);
   d.H = static_cast<int>(p->H);
   d.NK = static_cast<int>(p->NK);
   d.G = static_cast<int>(p->G);
   d.logH = p->logH;
   d.logGY = p->logGY;
   d.logGZ = p->logGZ;
   d.logG = Log2(p->G);
   d.logGX = Log2(p->GX);
   d.px = p->px;
   d.py = p->py;
   d.pz = p->pz;
   return d;
}

// The shared-memory ceiling of the kernels a plan of these lengths launches.
int SetFftSmem(int logH, int logGY, int logGZ)
{
   const int bytes = static_cast<int>(kSmemMax);
   const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
   ISCU_WF_X_CODELETS(logH, ISCU_CK(cudaFuncSetAttribute(XForwardKernel<K>, attr, bytes));
                      ISCU_CK(cudaFuncSetAttribute(XInverseKernel<K>, attr, bytes)));
   ISCU_WF_Y_CODELETS(logGY, ISCU_CK(cudaFuncSetAttribute(YForwardKernel<K>, attr, bytes));
                      ISCU_CK(cudaFuncSetAttribute(YInverseKernel<K>, attr, bytes)));
   ISCU_WF_Z_CODELETS(logGZ, ISCU_CK(cudaFuncSetAttribute(ZKernel<true, K>, attr, bytes));
                      ISCU_CK(cudaFuncSetAttribute(ZKernel<false, K>, attr, bytes)));
   return ISCU_OK;
}

template <bool kConvolve, int kLogN>
int ZPlan(const iscu_ctx* ctx, const Dims& d, ZLaunch& z)
{
   // 16 columns per block (8 when the buffers would pass the budget, ...), double-buffered where that fits
   z.BZ = ISCU_WF_Z_STAGES == 2 ? 16 : ISCU_WF_Z_COLUMNS;
   z.stages = ISCU_WF_Z_STAGES;
   while (z.BZ > 1 && ZSmem(d, z.BZ, z.stages, kConvolve) > kSmemBudget)
      z.BZ >>= 1;
   if (ZSmem(d, z.BZ, z.stages, kConvolve) > kSmemBudget)
      z.stages = 1;
   z.smem = ZSmem(d, z.BZ, z.stages, kConvolve);
   if (z.smem > kSmemMax)
      return Fail(ISCU_ERR_LIMIT, "widefield plan: a z column block does not fit in shared memory");
   z.logBZ = Log2(z.BZ);
   z.blocksPerK = (d.GY + z.BZ - 1) / z.BZ;
   z.nBlocks = z.blocksPerK * d.NK;
   int perSm = 0;
   ISCU_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, ZKernel<kConvolve, kLogN>, kThreads, z.smem));
   z.grid = z.stages == 2 ? std::max(1, std::min(z.nBlocks, std::max(1, perSm) * ctx->smCount)) : z.nBlocks;
   return ISCU_OK;
}

} // namespace

// The convolution of density_dev into the plan's A (cropped, before the x inverse) -- the passes up to YInverse.
static int ConvolveToA(iscu_wf_plan* p, const float* density)
{
   iscu_ctx* ctx = p->ctx;
   const Dims d = MakeDims(p, p->nx, p->ny, p->nz);
   const float2* twg = p->twg.as<float2>();
   p->Mark(0);
   int rc = ForwardXY(p, density, d, p->A.as<float2>(), p->B.as<float2>(), true);
   if (rc != ISCU_OK)
      return rc;
   p->Mark(2);
   int rc2 = ISCU_OK;
   ISCU_WF_Z_CODELETS(d.logGZ, ZLaunch zl; rc2 = ZPlan<true, K>(ctx, d, zl); if (rc2 != ISCU_OK) return rc2;
                      (ZKernel<true, K><<<zl.grid, kThreads, zl.smem, ctx->stream>>>(
                         p->B.as<float2>(), d, zl.BZ, zl.logBZ, zl.blocksPerK, zl.nBlocks, zl.stages,
                         static_cast<int>(p->kz / 2), twg, p->Kh.as<float2>())));
   ISCU_CK_LAUNCH(ctx, "ZKernel<convolve>");
   p->Mark(3);
   const int BK = YLines(d.py);
   ISCU_WF_Y_CODELETS(d.logGY, (YInverseKernel<K><<<dim3((d.NK + BK - 1) / BK, d.nzv), kThreads,
                                                    BK * RowBytes(d.py), ctx->stream>>>(
                                   p->B.as<float2>(), d, BK, static_cast<int>(p->ky / 2), twg, p->A.as<float2>())));
   ISCU_CK_LAUNCH(ctx, "YInverseKernel");
   p->Mark(4);
   return ISCU_OK;
}

static int FinishX(iscu_wf_plan* p, double background, const iscu_camera* cam, uint32_t seed, uint32_t frame0,
                   float* image, uint16_t* adu)
{
   iscu_ctx* ctx = p->ctx;
   const Dims d = MakeDims(p, p->nx, p->ny, p->nz);
   StaticView st;
   const uint32_t fw = p->FrameW(), fh = p->FrameH();
   if (ctx->haveStatic && ctx->width == fw && ctx->height == fh)
      st = ctx->Static();
   st.width = fw;
   st.height = fh;
   const float scale = static_cast<float>(1.0 / (static_cast<double>(p->GX) * p->GY * p->GZ));
   if (!image)
   {
      ISCU_CK(p->image.Reserve(p->FrameElems() * sizeof(float)));
      image = p->image.as<float>();
   }
   // a camera plan clamps the grid's cells first (no background) and bins its FOV window after
   float* xout = image;
   if (p->camera)
   {
      ISCU_CK(p->cells.Reserve(static_cast<size_t>(p->nx) * p->ny * p->nz * sizeof(float)));
      xout = p->cells.as<float>();
   }
   const int BY = XLines(d.H);
   ISCU_WF_X_CODELETS(d.logH, (XInverseKernel<K><<<dim3((d.nyv + BY - 1) / BY, d.nzv), kThreads, XSmem(d.H, BY),
                                                   ctx->stream>>>(
                                  p->A.as<float2>(), d, BY, Log2(BY), static_cast<int>(p->kx / 2), scale,
                                  p->camera ? 0.0f : static_cast<float>(background), 1, p->tw.as<float2>(),
                                  p->twg.as<float2>(), xout)));
   ISCU_CK_LAUNCH(ctx, "XInverseKernel");
   if (p->camera)
   {
      WfBinKernel<<<dim3((fw * fh + 255) / 256, p->nz), 256, 0, ctx->stream>>>(
         xout, p->nx, p->ny, p->fovX0, p->fovY0, fw, fh, p->up, static_cast<float>(background), image);
      ISCU_CK_LAUNCH(ctx, "WfBinKernel");
   }
   p->Mark(5);
   if (cam)
   {
      const CameraView cv = MakeCameraView(*cam);
      const uint32_t npix = fw * fh;
      WfNoiseKernel<<<dim3((npix + 255) / 256, p->nz), 256, 0, ctx->stream>>>(image, npix, st, cv, seed, frame0, adu);
      ISCU_CK_LAUNCH(ctx, "WfNoiseKernel");
   }
   p->Mark(6);
   return ISCU_OK;
}

} // namespace iscu

namespace iscu {
namespace {

// ------------------------------------------------------------------------ focus jobs (WidefieldAccelerator)
// Dense dye planes from a job's sparse ones: plane q's cell cells[i] (row-major in the nx x ny dye grid) += values[i]
// for i in [start[q], start[q+1]). dense: planes x ny x nx, zeroed before.
__global__ void JobScatterKernel(const uint32_t* __restrict__ cells, const float* __restrict__ values,
                                 const uint32_t* __restrict__ start, uint32_t nPlanes, size_t planeCells,
                                 float* __restrict__ dense)
{
   const uint32_t q = blockIdx.y;
   if (q >= nPlanes)
      return;
   for (uint32_t i = start[q] + blockIdx.x * blockDim.x + threadIdx.x; i < start[q + 1]; i += gridDim.x * blockDim.x)
      dense[q * planeCells + cells[i]] = values[i];
}

// A kernel spectrum in RealFft2d's layout (spec[ky W + kx], W = GX/2 + 1, ky natural) into the transforms' layout
// (out[kx GY + rev(ky)]).
__global__ void JobKernelLayoutKernel(const float2* __restrict__ spec, int NK, int GY, int logGY,
                                      float2* __restrict__ out)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= NK * GY)
      return;
   const int ky = i / NK, kx = i - ky * NK;
   out[static_cast<size_t>(kx) * GY + Rev(ky, logGY)] = spec[i];
}

// A job's channel spectra (ChannelImageStep, WidefieldRender.cpp:1790-1801): per frequency, channel c's
// S = sum over its deps d (in order) of plane P[d] x (w0 K[p0] + w1 K[p1]) in float (the blend and the product
// term by term, as the reference forms them), then the sub-cell shift (ApplyShiftRamp, DriftShift.cpp:24-48):
// S x (px[kx] py[ky]) formed in float64 and rounded to float, Nyquist terms their cosine only -- px and py
// tabulated on the host. Spectra in the transforms' layout (kx-major, ky bit-reversed); out: channels x NK x GY.
struct JobDep
{
   uint32_t plane, k0, k1;   // slots of the plane's spectrum and of its kernels (k1 only when two)
   float w0, w1;
   int32_t two;
};

__global__ void JobMacKernel(const float2* __restrict__ planes, const float2* __restrict__ kernels,
                             const JobDep* __restrict__ deps, const uint32_t* __restrict__ chanStart,
                             uint32_t nChannels, const double2* __restrict__ px, const double2* __restrict__ py,
                             int ramp, int NK, int GY, int logGY, float2* __restrict__ out)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   const size_t n = static_cast<size_t>(NK) * GY;
   if (i >= static_cast<int>(n))
      return;
   double2 r = make_double2(1.0, 0.0);
   if (ramp)
   {
      const int kx = i / GY, ky = Rev(i - kx * GY, logGY);
      const double2 a = px[kx], b = py[ky];
      r = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
   }
   for (uint32_t c = 0; c < nChannels; ++c)
   {
      float sr = 0.0f, si = 0.0f;
      for (uint32_t j = chanStart[c]; j < chanStart[c + 1]; ++j)
      {
         const JobDep d = deps[j];
         const float2 k0 = kernels[d.k0 * n + i];
         float kr = d.w0 * k0.x, ki = d.w0 * k0.y;
         if (d.two)
         {
            const float2 k1 = kernels[d.k1 * n + i];
            kr += d.w1 * k1.x;
            ki += d.w1 * k1.y;
         }
         const float2 a = planes[d.plane * n + i];
         sr += a.x * kr - a.y * ki;
         si += a.x * ki + a.y * kr;
      }
      float2 v = make_float2(sr, si);
      if (ramp)
      {
         const double vr = sr, vi = si;
         v = make_float2(static_cast<float>(vr * r.x - vi * r.y), static_cast<float>(vr * r.y + vi * r.x));
      }
      out[c * n + i] = v;
   }
}

} // namespace
} // namespace iscu

// A widefield focus-job engine (iscu_wf_job_*): one 2D transform geometry at a time; plane spectra resident by key and
// kernel spectra by plane index, both for the geometry value they were made in.
struct iscu_wf_job
{
   iscu_ctx* ctx = nullptr;
   size_t budget = 0;                     // device bytes the plane spectra may hold
   uint64_t geometry = 0;
   bool haveGeometry = false;
   std::unique_ptr<iscu_wf_plan> plan;    // the NX x NY transforms (GX = NX, GY = NY)
   std::vector<uint64_t> planeKeys;       // slot -> key
   std::vector<int32_t> kernelPs;         // slot -> plane index p
   iscu::DevBuf planes, kernels, dense, A, B, images, deps, starts, cells, values, rampX, rampY, stage;
   size_t planeCap = 0, kernelCap = 0;
   size_t Spec() const { return static_cast<size_t>(plan->NK) * plan->GY; }
};

namespace iscu {
namespace {

// The FFT length of one axis: a power of two that holds the kernel (k) and the volume's "same" window (n points from
// k/2 on) of the circular convolution with nothing wrapped into it -- n + k/2 points (the output point i + k/2 reads
// kernel taps i + k/2 - j for input points j < n: none of them wraps into [0, k) once the length passes n + k/2 - 1).
uint32_t AxisLength(uint32_t n, uint32_t k, uint32_t least)
{
   return Pow2AtLeast(std::max({n + k / 2, k, least}));
}

// The transforms' group plans, shared-memory ceilings and twiddle tables of a plan whose GX, GY and GZ are set.
int InitTables(iscu_wf_plan* p)
{
   iscu_ctx* ctx = p->ctx;
   p->H = p->GX / 2;
   p->NK = p->H + 1;
   p->G = std::max(p->GX, std::max(p->GY, p->GZ));
   p->logH = Log2(p->H);
   p->logGY = Log2(p->GY);
   p->logGZ = Log2(p->GZ);
   p->px = MakeLinePlan(p->logH, true);
   p->py = MakeLinePlan(p->logGY, false);
   p->pz = MakeZPlan(p->logGZ);
   int entries = PlaceTables(p->px, 0);
   entries += PlaceTables(p->py, entries);
   entries += PlaceTables(p->pz, entries);
   const int rc = SetFftSmem(p->logH, p->logGY, p->logGZ);
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(p->tw.Reserve(p->G * sizeof(float2)));
   ISCU_CK(p->twg.Reserve(std::max(entries, 1) * sizeof(float2)));
   TwiddleKernel<<<(p->G + 255) / 256, 256, 0, ctx->stream>>>(static_cast<int>(p->G), p->tw.as<float2>());
   ISCU_CK_LAUNCH(ctx, "TwiddleKernel");
   for (const LinePlan* P : {&p->px, &p->py, &p->pz})
      for (int g = 0; g < P->groups; ++g)
         if (P->tw[g] >= 0)
         {
            const int M = 1 << (LogQ(*P, g) + P->r[g]);
            GroupTwiddleKernel<<<(M + 255) / 256, 256, 0, ctx->stream>>>(LogQ(*P, g), P->r[g],
                                                                          p->twg.as<float2>() + P->tw[g]);
            ISCU_CK_LAUNCH(ctx, "GroupTwiddleKernel");
         }
   return ISCU_OK;
}

// A plan's geometry, tables and PSF spectrum; psf is a device pointer when psfOnDevice (kx*ky*kz floats).
int MakePlan(iscu_ctx* ctx, uint32_t nx, uint32_t ny, uint32_t nz, const float* psf, bool psfOnDevice, uint32_t kx,
             uint32_t ky, uint32_t kz, std::unique_ptr<iscu_wf_plan>& out)
{
   std::unique_ptr<iscu_wf_plan> p(new iscu_wf_plan());
   p->ctx = ctx;
   p->nx = nx;
   p->ny = ny;
   p->nz = nz;
   p->kx = kx;
   p->ky = ky;
   p->kz = kz;
   p->GX = AxisLength(nx, kx, 8u);
   p->GY = AxisLength(ny, ky, 4u);
   p->GZ = AxisLength(nz, kz, 4u);
   if (p->GX > 4096 || p->GY > 8192 || p->GZ > 8192)
      return Fail(ISCU_ERR_LIMIT, "widefield plan: padded grid beyond 4096 x 8192 x 8192");
   if (kx > p->GX || ky > p->GY)
      return Fail(ISCU_ERR_ARG, "widefield plan: PSF wider than the grid");
   int rc = InitTables(p.get());
   if (rc != ISCU_OK)
      return rc;
   const uint32_t nzA = std::max(nz, kz), nyA = std::max(ny, ky);
   ISCU_CK(p->A.Reserve(static_cast<size_t>(nzA) * p->NK * nyA * sizeof(float2)));
   ISCU_CK(p->B.Reserve(static_cast<size_t>(nzA) * p->NK * p->GY * sizeof(float2)));
   ISCU_CK(p->Kh.Reserve(static_cast<size_t>(p->GZ) * p->NK * p->GY * sizeof(float2)));
   // The PSF's spectrum: its own x and y passes (kx x ky x kz valid), then the forward z transform of all GZ planes.
   DevBuf dPsf;
   const size_t psfBytes = static_cast<size_t>(kx) * ky * kz * sizeof(float);
   if (!psfOnDevice)
   {
      ISCU_CK(dPsf.Reserve(psfBytes));
      ISCU_CK(cudaMemcpyAsync(dPsf.p, psf, psfBytes, cudaMemcpyHostToDevice, ctx->stream));
      psf = dPsf.as<float>();
   }
   const Dims dk = MakeDims(p.get(), kx, ky, kz);
   rc = ForwardXY(p.get(), psf, dk, p->A.as<float2>(), p->B.as<float2>());
   if (rc != ISCU_OK)
      return rc;
   ISCU_WF_Z_CODELETS(dk.logGZ, ZLaunch zl; rc = ZPlan<false, K>(ctx, dk, zl); if (rc != ISCU_OK) return rc;
                      (ZKernel<false, K><<<zl.grid, kThreads, zl.smem, ctx->stream>>>(
                         p->B.as<float2>(), dk, zl.BZ, zl.logBZ, zl.blocksPerK, zl.nBlocks, zl.stages, 0,
                         p->twg.as<float2>(), p->Kh.as<float2>())));
   ISCU_CK_LAUNCH(ctx, "ZKernel<spectrum>");
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   out = std::move(p);
   return ISCU_OK;
}

// KernelWidefieldPsf (WidefieldRender.cpp:263-330) of a kernel slot at `up` grid cells per camera pixel: r = os / up
// oversampled samples per cell, cell 0 from sample s0 = floor(kc - r / 2 + 1), the natural radius (the cells whose
// block meets the plane) capped at ceil(capUm / pitch - 1e-9) cells (WidefieldScene::SetupFft, :1315-1322).
void CellGeometry(const KernelSlot& k, int up, double pixelUm, double capUm, int& r, int& s0, int& R)
{
   const int n = k.size;
   r = std::max(1, k.os / up);
   const double kc = (n - 1) / 2.0;
   s0 = static_cast<int>(std::floor(kc - r / 2.0 + 1.0));
   const int dMin = static_cast<int>(std::ceil((-s0 - r + 1) / static_cast<double>(r)));
   const int dMax = static_cast<int>(std::floor((n - 1 - s0) / static_cast<double>(r)));
   const int natural = std::max(1, std::max(-dMin, dMax));
   const double pitch = pixelUm / up;
   const int cap = std::max(1, static_cast<int>(std::ceil(capUm / pitch - 1e-9)));
   R = std::max(1, std::min(cap, natural));
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_wf_plan_create(iscu_ctx* ctx, uint32_t nx, uint32_t ny, uint32_t nz, const float* psf, uint32_t kx,
                        uint32_t ky, uint32_t kz, iscu_wf_plan** out)
{
   if (!ctx || !psf || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   if (nx < 2 || ny < 1 || nz < 1 || kx < 1 || ky < 1 || kz < 1 || nx % 2 != 0)
      return Fail(ISCU_ERR_ARG, "widefield plan: nx even >= 2, all other sizes >= 1");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   std::unique_ptr<iscu_wf_plan> p;
   const int rc = MakePlan(ctx, nx, ny, nz, psf, false, kx, ky, kz, p);
   if (rc != ISCU_OK)
      return rc;
   *out = p.release();
   return ISCU_OK;
}

int iscu_wf_plan_from_kernel(iscu_ctx* ctx, int32_t slot, int32_t upscale, double pixel_um, double kernel_cap_um,
                             double plane_nm, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t fov_x0, uint32_t fov_y0,
                             uint32_t fov_w, uint32_t fov_h, iscu_wf_plan** out)
{
   if (!ctx || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   if (slot < 0 || slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (0..3)");
   if (nx < 1 || ny < 1 || nz < 1)
      return Fail(ISCU_ERR_ARG, "widefield plan: nx, ny and nz >= 1");
   if (!(pixel_um > 0.0) || !(kernel_cap_um > 0.0) || !(plane_nm > 0.0))
      return Fail(ISCU_ERR_ARG, "widefield plan: pixel size, kernel cap and plane thickness must be > 0");
   const uint64_t up = upscale < 1 ? 1u : static_cast<uint64_t>(upscale);
   if (fov_w == 0 || fov_h == 0 || fov_x0 + up * fov_w > nx || fov_y0 + up * fov_h > ny)
      return Fail(ISCU_ERR_ARG, "widefield plan: the camera window (fov_x0 + upscale fov_w, fov_y0 + upscale fov_h) "
                                "must lie inside the nx x ny grid");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const KernelSlot& k = ctx->kernels[slot];
   if (!k.valid)
      return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
   if (k.os % static_cast<int>(up) != 0)
      return Fail(ISCU_ERR_ARG, "widefield plan: upscale must divide the kernel's oversampling (" +
                                    std::to_string(k.os) + ")");
   int r = 1, s0 = 0, R = 1;
   CellGeometry(k, static_cast<int>(up), pixel_um, kernel_cap_um, r, s0, R);
   const int D = 2 * R + 1, D2 = D * D, nzk = k.nz;
   const uint32_t kz = 2 * nz - 1;
   // The kernel plane of each dye-plane offset d = nz - 1 - j (a dye plane d planes above the focus): PlanFocus
   // (WidefieldRender.cpp:1460-1522) with KernelWidefieldPsf::PlaneCoord (:282-287): t = defocus 1000 / zStep +
   // (nz - 1) / 2 clamped to the stack, p0 = floor(t), weights 1 - frac and frac as floats (the last plane: frac 0).
   std::vector<int2> planes(kz);
   std::vector<float2> weights(kz);
   for (uint32_t j = 0; j < kz; ++j)
   {
      const double defocusUm = (static_cast<double>(nz) - 1.0 - j) * (plane_nm / 1000.0);
      double t = (nzk <= 1 || !(k.zStepNm > 0.0)) ? 0.0 : defocusUm * 1000.0 / k.zStepNm + (nzk - 1) / 2.0;
      t = std::min<double>(nzk - 1, std::max(0.0, t));
      int p0 = static_cast<int>(std::floor(t));
      double frac = t - p0;
      if (p0 >= nzk - 1)
      {
         p0 = nzk - 1;
         frac = 0.0;
      }
      planes[j] = make_int2(p0, frac > 0.0 ? p0 + 1 : p0);
      weights[j] = make_float2(static_cast<float>(1.0 - frac), static_cast<float>(frac));
   }
   DevBuf dCells, dVol, dPlanes, dWeights;
   ISCU_CK(dCells.Reserve(static_cast<size_t>(nzk) * D2 * sizeof(float)));
   ISCU_CK(dVol.Reserve(static_cast<size_t>(kz) * D2 * sizeof(float)));
   ISCU_CK(dPlanes.Reserve(kz * sizeof(int2)));
   ISCU_CK(dWeights.Reserve(kz * sizeof(float2)));
   ISCU_CK(cudaMemcpyAsync(dPlanes.p, planes.data(), kz * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(dWeights.p, weights.data(), kz * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
   int rc = LaunchCellKernels(ctx, k.planes.as<float>(), k.size, nzk, r, s0, R, dCells.as<float>());
   if (rc != ISCU_OK)
      return rc;
   const size_t total = static_cast<size_t>(kz) * D2;
   WfKernelVolumeKernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, ctx->stream>>>(
      dCells.as<float>(), D2, dPlanes.as<int2>(), dWeights.as<float2>(), static_cast<int>(kz), dVol.as<float>());
   ISCU_CK_LAUNCH(ctx, "WfKernelVolumeKernel");
   std::unique_ptr<iscu_wf_plan> p;
   rc = MakePlan(ctx, nx, ny, nz, dVol.as<float>(), true, D, D, kz, p);
   if (rc != ISCU_OK)
      return rc;
   // a window that is the whole grid at one cell per pixel needs no binning pass: the frames are the grid's cells
   p->camera = !(fov_x0 == 0 && fov_y0 == 0 && fov_w == nx && fov_h == ny && up == 1);
   p->fovX0 = fov_x0;
   p->fovY0 = fov_y0;
   p->fovW = fov_w;
   p->fovH = fov_h;
   p->up = static_cast<uint32_t>(up);
   *out = p.release();
   return ISCU_OK;
}

int iscu_wf_job_create(iscu_ctx* ctx, uint64_t budget_bytes, iscu_wf_job** out)
{
   if (!ctx || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   std::unique_ptr<iscu_wf_job> j(new iscu_wf_job());
   j->ctx = ctx;
   size_t freeB = 0, total = 0;
   ISCU_CK(cudaMemGetInfo(&freeB, &total));
   j->budget = budget_bytes ? static_cast<size_t>(budget_bytes) : total / 4;
   *out = j.release();
   return ISCU_OK;
}

void iscu_wf_job_destroy(iscu_wf_job* job)
{
   if (!job)
      return;
   cudaStreamSynchronize(job->ctx->stream);
   delete job;
}

int iscu_wf_job_has_plane(iscu_wf_job* job, uint64_t geometry, uint64_t key)
{
   if (!job)
      return 0;
   std::lock_guard<std::recursive_mutex> lock(job->ctx->mu);
   if (!job->haveGeometry || job->geometry != geometry)
      return 0;
   return std::find(job->planeKeys.begin(), job->planeKeys.end(), key) != job->planeKeys.end() ? 1 : 0;
}

int iscu_wf_job_fits(iscu_wf_job* job, uint64_t geometry, uint32_t nx_fft, uint32_t ny_fft, uint64_t planes)
{
   (void)geometry;
   if (!job)
      return 0;
   const double per = (nx_fft / 2.0 + 1.0) * ny_fft * sizeof(float2);
   return per * static_cast<double>(planes) <= static_cast<double>(job->budget) ? 1 : 0;
}

int iscu_wf_job_images(iscu_wf_job* job, const iscu_wf_job_desc* d, float* const* images)
{
   if (!job || !d || (d->n_channels && (!images || !d->channel_start)))
      return Fail(ISCU_ERR_ARG, "null argument");
   const uint32_t NX = d->nx_fft, NY = d->ny_fft;
   if (NX < 16 || NY < 16 || NX > 2048 || NY > 2048 || (NX & (NX - 1)) || (NY & (NY - 1)))
      return Fail(ISCU_ERR_ARG, "widefield job: FFT sizes powers of two in 16..2048");
   if (d->nx == 0 || d->ny == 0 || d->nx > NX || d->ny > NY || d->cw == 0 || d->ch == 0 ||
       d->fov_x0 + d->cw > NX || d->fov_y0 + d->ch > NY)
      return Fail(ISCU_ERR_ARG, "widefield job: the dye grid and the FOV window must lie inside the FFT grid");
   iscu_ctx* ctx = job->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   // A new geometry (or transform size) drops every resident spectrum.
   if (!job->plan || job->plan->GX != NX || job->plan->GY != NY || !job->haveGeometry || job->geometry != d->geometry)
   {
      if (!job->plan || job->plan->GX != NX || job->plan->GY != NY)
      {
         std::unique_ptr<iscu_wf_plan> p(new iscu_wf_plan());
         p->ctx = ctx;
         p->GX = NX;
         p->GY = NY;
         p->GZ = 4;
         const int rc = InitTables(p.get());
         if (rc != ISCU_OK)
            return rc;
         job->plan = std::move(p);
         // the slots were sized for the old transform's spectra
         job->planes.Free();
         job->kernels.Free();
         job->planeCap = job->kernelCap = 0;
      }
      job->planeKeys.clear();
      job->kernelPs.clear();
      job->geometry = d->geometry;
      job->haveGeometry = true;
   }
   iscu_wf_plan* P = job->plan.get();
   const size_t spec = job->Spec(), specBytes = spec * sizeof(float2);
   auto growSlots = [&](DevBuf& buf, size_t& cap, size_t need) -> int {
      if (need <= cap)
         return ISCU_OK;
      size_t want = std::max(need, cap * 2 + 8);
      DevBuf grown;
      ISCU_CK(grown.Reserve(want * specBytes));
      if (cap)
         ISCU_CK(cudaMemcpyAsync(grown.p, buf.p, cap * specBytes, cudaMemcpyDeviceToDevice, ctx->stream));
      ISCU_CK(cudaStreamSynchronize(ctx->stream));
      std::swap(buf.p, grown.p);
      std::swap(buf.bytes, grown.bytes);
      cap = want;
      return ISCU_OK;
   };
   // Kernel spectra not yet resident: RealFft2d's layout in, the transforms' layout kept.
   for (uint32_t i = 0; i < d->n_kernels; ++i)
   {
      const iscu_wf_job_kernel& k = d->kernels[i];
      if (std::find(job->kernelPs.begin(), job->kernelPs.end(), k.p) != job->kernelPs.end())
         continue;
      if (!k.spec)
         return Fail(ISCU_ERR_ARG, "widefield job: a kernel without its spectrum");
      int rc = growSlots(job->kernels, job->kernelCap, job->kernelPs.size() + 1);
      if (rc != ISCU_OK)
         return rc;
      ISCU_CK(job->stage.Reserve(specBytes));
      ISCU_CK(cudaMemcpyAsync(job->stage.p, k.spec, specBytes, cudaMemcpyHostToDevice, ctx->stream));
      JobKernelLayoutKernel<<<static_cast<unsigned>((spec + 255) / 256), 256, 0, ctx->stream>>>(
         job->stage.as<float2>(), static_cast<int>(P->NK), static_cast<int>(NY), P->logGY,
         job->kernels.as<float2>() + job->kernelPs.size() * spec);
      ISCU_CK_LAUNCH(ctx, "JobKernelLayoutKernel");
      ISCU_CK(cudaStreamSynchronize(ctx->stream));   // the stage is reused by the next kernel
      job->kernelPs.push_back(k.p);
   }
   // New plane spectra: the sparse cells made dense, then the forward x and y passes straight into their slots.
   std::vector<uint32_t> starts(1, 0);
   std::vector<uint32_t> cellsH;
   std::vector<float> valuesH;
   std::vector<uint64_t> newKeys;
   for (uint32_t q = 0; q < d->n_planes; ++q)
   {
      const iscu_wf_job_plane& pl = d->planes[q];
      if (std::find(job->planeKeys.begin(), job->planeKeys.end(), pl.key) != job->planeKeys.end() ||
          std::find(newKeys.begin(), newKeys.end(), pl.key) != newKeys.end())
         continue;
      for (uint32_t i = 0; i < pl.count; ++i)
         if (pl.cells[i] >= static_cast<uint64_t>(d->nx) * d->ny)
            return Fail(ISCU_ERR_ARG, "widefield job: a plane cell outside the dye grid");
      cellsH.insert(cellsH.end(), pl.cells, pl.cells + pl.count);
      valuesH.insert(valuesH.end(), pl.values, pl.values + pl.count);
      starts.push_back(static_cast<uint32_t>(cellsH.size()));
      newKeys.push_back(pl.key);
   }
   const uint32_t nNew = static_cast<uint32_t>(newKeys.size());
   if (nNew)
   {
      const size_t base = job->planeKeys.size();
      if ((base + nNew) * specBytes > job->budget)
         return Fail(ISCU_ERR_LIMIT, "widefield job: the plane spectra pass the job's device budget");
      int rc = growSlots(job->planes, job->planeCap, base + nNew);
      if (rc != ISCU_OK)
         return rc;
      const size_t planeCells = static_cast<size_t>(d->nx) * d->ny;
      ISCU_CK(job->dense.Reserve(nNew * planeCells * sizeof(float)));
      ISCU_CK(cudaMemsetAsync(job->dense.p, 0, nNew * planeCells * sizeof(float), ctx->stream));
      ISCU_CK(job->cells.Reserve(std::max<size_t>(1, cellsH.size()) * sizeof(uint32_t)));
      ISCU_CK(job->values.Reserve(std::max<size_t>(1, valuesH.size()) * sizeof(float)));
      ISCU_CK(job->starts.Reserve(starts.size() * sizeof(uint32_t)));
      ISCU_CK(cudaMemcpyAsync(job->cells.p, cellsH.data(), cellsH.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              ctx->stream));
      ISCU_CK(cudaMemcpyAsync(job->values.p, valuesH.data(), valuesH.size() * sizeof(float), cudaMemcpyHostToDevice,
                              ctx->stream));
      ISCU_CK(cudaMemcpyAsync(job->starts.p, starts.data(), starts.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                              ctx->stream));
      JobScatterKernel<<<dim3(32, nNew), 256, 0, ctx->stream>>>(job->cells.as<uint32_t>(), job->values.as<float>(),
                                                               job->starts.as<uint32_t>(), nNew, planeCells,
                                                               job->dense.as<float>());
      ISCU_CK_LAUNCH(ctx, "JobScatterKernel");
      const Dims dp = MakeDims(P, d->nx, d->ny, nNew);
      ISCU_CK(job->A.Reserve(static_cast<size_t>(nNew) * P->NK * d->ny * sizeof(float2)));
      rc = ForwardXY(P, job->dense.as<float>(), dp, job->A.as<float2>(), job->planes.as<float2>() + base * spec);
      if (rc != ISCU_OK)
         return rc;
      ISCU_CK(cudaStreamSynchronize(ctx->stream));   // the host staging vectors go out of scope
      job->planeKeys.insert(job->planeKeys.end(), newKeys.begin(), newKeys.end());
   }
   const uint32_t nc = d->n_channels;
   if (nc == 0)
      return ISCU_OK;
   // The channels' deps as slots.
   std::vector<JobDep> deps;
   std::vector<uint32_t> chan(1, 0);
   for (uint32_t c = 0; c < nc; ++c)
   {
      for (uint32_t j = d->channel_start[c]; j < d->channel_start[c + 1]; ++j)
      {
         const iscu_wf_job_dep& e = d->deps[j];
         const auto pk = std::find(job->planeKeys.begin(), job->planeKeys.end(), e.key);
         const auto k0 = std::find(job->kernelPs.begin(), job->kernelPs.end(), e.p0);
         const auto k1 = std::find(job->kernelPs.begin(), job->kernelPs.end(), e.two ? e.p1 : e.p0);
         if (pk == job->planeKeys.end() || k0 == job->kernelPs.end() || k1 == job->kernelPs.end())
            return Fail(ISCU_ERR_STATE, "widefield job: a dep names a plane or kernel that is not resident");
         deps.push_back({static_cast<uint32_t>(pk - job->planeKeys.begin()),
                         static_cast<uint32_t>(k0 - job->kernelPs.begin()),
                         static_cast<uint32_t>(k1 - job->kernelPs.begin()), e.w0, e.two ? e.w1 : 0.0f,
                         e.two ? 1 : 0});
      }
      chan.push_back(static_cast<uint32_t>(deps.size()));
   }
   // ApplyShiftRamp's factors (DriftShift.cpp:24-48), tabulated as the reference tabulates them.
   const bool ramp = d->frac_x != 0.0 || d->frac_y != 0.0;
   const uint32_t W = NX / 2 + 1;
   std::vector<double2> px(W), py(NY);
   const double kPi = 3.14159265358979323846;
   for (uint32_t kx = 0; kx < W; ++kx)
   {
      const double a = 2.0 * kPi * kx * d->frac_x / NX;
      px[kx] = kx == NX / 2 ? make_double2(std::cos(a), 0.0) : make_double2(std::cos(a), std::sin(a));
   }
   for (uint32_t ky = 0; ky < NY; ++ky)
   {
      const long kys = ky <= NY / 2 ? static_cast<long>(ky) : static_cast<long>(ky) - static_cast<long>(NY);
      const double a = 2.0 * kPi * kys * d->frac_y / NY;
      py[ky] = ky == NY / 2 ? make_double2(std::cos(a), 0.0) : make_double2(std::cos(a), std::sin(a));
   }
   ISCU_CK(job->deps.Reserve(std::max<size_t>(1, deps.size()) * sizeof(JobDep)));
   ISCU_CK(job->starts.Reserve(chan.size() * sizeof(uint32_t)));
   ISCU_CK(job->rampX.Reserve(W * sizeof(double2)));
   ISCU_CK(job->rampY.Reserve(NY * sizeof(double2)));
   ISCU_CK(cudaMemcpyAsync(job->deps.p, deps.data(), deps.size() * sizeof(JobDep), cudaMemcpyHostToDevice,
                           ctx->stream));
   ISCU_CK(cudaMemcpyAsync(job->starts.p, chan.data(), chan.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                           ctx->stream));
   ISCU_CK(cudaMemcpyAsync(job->rampX.p, px.data(), W * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(job->rampY.p, py.data(), NY * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(job->B.Reserve(nc * specBytes));
   JobMacKernel<<<static_cast<unsigned>((spec + 255) / 256), 256, 0, ctx->stream>>>(
      job->planes.as<float2>(), job->kernels.as<float2>(), job->deps.as<JobDep>(), job->starts.as<uint32_t>(), nc,
      job->rampX.as<double2>(), job->rampY.as<double2>(), ramp ? 1 : 0, static_cast<int>(P->NK),
      static_cast<int>(NY), P->logGY, job->B.as<float2>());
   ISCU_CK_LAUNCH(ctx, "JobMacKernel");
   // The inverse: rows [fov_y0, + ch) then columns [fov_x0, + cw), scaled 1 / (NX NY) (RealFft2d::Inverse), no clamp.
   const Dims di = MakeDims(P, d->cw, d->ch, nc);
   ISCU_CK(job->A.Reserve(static_cast<size_t>(nc) * P->NK * d->ch * sizeof(float2)));
   const float2* twg = P->twg.as<float2>();
   const int BK = YLines(di.py);
   ISCU_WF_Y_CODELETS(di.logGY, (YInverseKernel<K><<<dim3((di.NK + BK - 1) / BK, di.nzv), kThreads,
                                                     BK * RowBytes(di.py), ctx->stream>>>(
                                    job->B.as<float2>(), di, BK, static_cast<int>(d->fov_y0), twg,
                                    job->A.as<float2>())));
   ISCU_CK_LAUNCH(ctx, "YInverseKernel");
   const size_t frame = static_cast<size_t>(d->cw) * d->ch;
   ISCU_CK(job->images.Reserve(nc * frame * sizeof(float)));
   const int BY = XLines(di.H);
   const float scale = static_cast<float>(1.0 / (static_cast<double>(NX) * NY));
   ISCU_WF_X_CODELETS(di.logH, (XInverseKernel<K><<<dim3((di.nyv + BY - 1) / BY, di.nzv), kThreads,
                                                    XSmem(di.H, BY), ctx->stream>>>(
                                   job->A.as<float2>(), di, BY, Log2(BY), static_cast<int>(d->fov_x0), scale, 0.0f,
                                   0, P->tw.as<float2>(), twg, job->images.as<float>())));
   ISCU_CK_LAUNCH(ctx, "XInverseKernel");
   for (uint32_t c = 0; c < nc; ++c)
      ISCU_CK(cudaMemcpyAsync(images[c], job->images.as<float>() + c * frame, frame * sizeof(float),
                              cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

int iscu_wf_plan_frame(iscu_wf_plan* plan, uint32_t* width, uint32_t* height, int32_t* kernel_radius)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   if (width)
      *width = plan->FrameW();
   if (height)
      *height = plan->FrameH();
   if (kernel_radius)
      *kernel_radius = static_cast<int32_t>(plan->kx / 2);
   return ISCU_OK;
}

int iscu_wf_set_timing(iscu_wf_plan* plan, int32_t on)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   if (on && !plan->ev[0])
      for (int i = 0; i <= ISCU_WF_PASSES; ++i)
         ISCU_CK(cudaEventCreate(&plan->ev[i]));
   plan->timing = on != 0;
   return ISCU_OK;
}

int iscu_wf_pass_times(iscu_wf_plan* plan, float* ms)
{
   if (!plan || !ms)
      return Fail(ISCU_ERR_ARG, "null argument");
   if (!plan->timing)
      return Fail(ISCU_ERR_STATE, "pass timing is off (iscu_wf_set_timing)");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   ISCU_CK(cudaEventSynchronize(plan->ev[ISCU_WF_PASSES]));
   for (int i = 0; i < ISCU_WF_PASSES; ++i)
      ISCU_CK(cudaEventElapsedTime(ms + i, plan->ev[i], plan->ev[i + 1]));
   return ISCU_OK;
}

void iscu_wf_plan_destroy(iscu_wf_plan* plan)
{
   if (!plan)
      return;
   cudaStreamSynchronize(plan->ctx->stream);
   for (auto& io : plan->io)
      for (cudaEvent_t e : {io.uploaded, io.rendered, io.downloaded})
         if (e)
         {
            cudaEventSynchronize(e);
            cudaEventDestroy(e);
         }
   for (int i = 0; i <= ISCU_WF_PASSES; ++i)
      if (plan->ev[i])
         cudaEventDestroy(plan->ev[i]);
   delete plan;
}

int iscu_wf_plan_grid(iscu_wf_plan* plan, uint32_t* gx, uint32_t* gy, uint32_t* gz)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   if (gx)
      *gx = plan->GX;
   if (gy)
      *gy = plan->GY;
   if (gz)
      *gz = plan->GZ;
   return ISCU_OK;
}

int iscu_wf_convolve_dev(iscu_wf_plan* plan, const float* density_dev, float* image_dev)
{
   if (!plan || !density_dev || !image_dev)
      return Fail(ISCU_ERR_ARG, "null argument");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   int rc = ConvolveToA(plan, density_dev);
   if (rc != ISCU_OK)
      return rc;
   return FinishX(plan, 0.0, nullptr, 0, 0, image_dev, nullptr);
}

int iscu_wf_render_dev(iscu_wf_plan* plan, const float* density_dev, double background, const iscu_camera* cam,
                       uint32_t seed, uint32_t frame0, float* image_dev, uint16_t* adu_dev)
{
   if (!plan || !density_dev || (cam && !adu_dev) || (!cam && !image_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   int rc = ConvolveToA(plan, density_dev);
   if (rc != ISCU_OK)
      return rc;
   return FinishX(plan, background, cam, seed, frame0, image_dev, adu_dev);
}

int iscu_wf_render_async(iscu_wf_plan* plan, int32_t io_slot, const float* density, double background,
                         const iscu_camera* cam, uint32_t seed, uint32_t frame0, float* image, uint16_t* adu)
{
   if (!plan || !density || (cam && !adu) || (!cam && !image))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (io_slot < 0 || io_slot >= ISCU_EVENT_IO_SLOTS)
      return Fail(ISCU_ERR_ARG, "I/O slot out of range (0..3)");
   iscu_ctx* ctx = plan->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   auto& io = plan->io[io_slot];
   if (io.busy)
      return Fail(ISCU_ERR_STATE, "the I/O slot's render has not been waited for");
   cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
   ISCU_CK(cudaStreamIsCapturing(ctx->stream, &capturing));
   if (capturing != cudaStreamCaptureStatusNone)
      return Fail(ISCU_ERR_STATE, "the pipelined render copies from host memory: not inside a stream capture");
   if (!ctx->upload)
      ISCU_CK(cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking));
   if (!ctx->download)
      ISCU_CK(cudaStreamCreateWithFlags(&ctx->download, cudaStreamNonBlocking));
   for (cudaEvent_t* e : {&io.uploaded, &io.rendered, &io.downloaded})
      if (!*e)
         ISCU_CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
   const size_t n = static_cast<size_t>(plan->nx) * plan->ny * plan->nz, nf = plan->FrameElems();
   ISCU_CK(io.density.Reserve(n * sizeof(float)));
   if (image)
      ISCU_CK(io.image.Reserve(nf * sizeof(float)));
   if (adu)
      ISCU_CK(io.adu.Reserve(nf * sizeof(uint16_t)));
   // the slot's buffers are free (its last render was waited for), so the upload waits on nothing
   ISCU_CK(cudaMemcpyAsync(io.density.p, density, n * sizeof(float), cudaMemcpyHostToDevice, ctx->upload));
   ISCU_CK(cudaEventRecord(io.uploaded, ctx->upload));
   ISCU_CK(cudaStreamWaitEvent(ctx->stream, io.uploaded, 0));
   int rc = ConvolveToA(plan, io.density.as<float>());
   if (rc != ISCU_OK)
      return rc;
   rc = FinishX(plan, background, cam, seed, frame0, image ? io.image.as<float>() : nullptr,
                adu ? io.adu.as<uint16_t>() : nullptr);
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(cudaEventRecord(io.rendered, ctx->stream));
   ISCU_CK(cudaStreamWaitEvent(ctx->download, io.rendered, 0));
   if (image)
      ISCU_CK(cudaMemcpyAsync(image, io.image.p, nf * sizeof(float), cudaMemcpyDeviceToHost, ctx->download));
   if (adu)
      ISCU_CK(cudaMemcpyAsync(adu, io.adu.p, nf * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->download));
   ISCU_CK(cudaEventRecord(io.downloaded, ctx->download));
   io.busy = true;
   return ISCU_OK;
}

int iscu_wf_render_wait(iscu_wf_plan* plan, int32_t io_slot)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   if (io_slot < 0 || io_slot >= ISCU_EVENT_IO_SLOTS)
      return Fail(ISCU_ERR_ARG, "I/O slot out of range (0..3)");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   auto& io = plan->io[io_slot];
   if (!io.busy)
      return Fail(ISCU_ERR_STATE, "no render in the I/O slot");
   io.busy = false;
   ISCU_CK(cudaEventSynchronize(io.downloaded));
   return ISCU_OK;
}

int iscu_wf_render(iscu_wf_plan* plan, const float* density, double background, const iscu_camera* cam,
                   uint32_t seed, uint32_t frame0, float* image, uint16_t* adu)
{
   if (!plan || !density || (cam && !adu) || (!cam && !image))
      return Fail(ISCU_ERR_ARG, "null argument");
   iscu_ctx* ctx = plan->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const size_t n = static_cast<size_t>(plan->nx) * plan->ny * plan->nz, nf = plan->FrameElems();
   ISCU_CK(ctx->dScratch.Reserve(n * sizeof(float)));
   if (image)
      ISCU_CK(plan->image.Reserve(nf * sizeof(float)));
   if (adu)
      ISCU_CK(plan->adu.Reserve(nf * sizeof(uint16_t)));
   ISCU_CK(cudaMemcpyAsync(ctx->dScratch.p, density, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
   int rc = ConvolveToA(plan, ctx->dScratch.as<float>());
   if (rc != ISCU_OK)
      return rc;
   rc = FinishX(plan, background, cam, seed, frame0, image ? plan->image.as<float>() : nullptr,
                adu ? plan->adu.as<uint16_t>() : nullptr);
   if (rc != ISCU_OK)
      return rc;
   if (image)
      ISCU_CK(cudaMemcpyAsync(image, plan->image.p, nf * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
   if (adu)
      ISCU_CK(cudaMemcpyAsync(adu, plan->adu.p, nf * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

int iscu_wf_shift_create(iscu_ctx* ctx, uint32_t nx, uint32_t ny, iscu_wf_shift** out)
{
   if (!ctx || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   if (nx < 8 || nx > 4096 || (nx & (nx - 1)) || ny < 4 || ny > 8192 || (ny & (ny - 1)))
      return Fail(ISCU_ERR_ARG, "drifting frames: nx a power of two in 8..4096, ny a power of two in 4..8192");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   std::unique_ptr<iscu_wf_shift> s(new iscu_wf_shift());
   s->ctx = ctx;
   s->nx = nx;
   s->ny = ny;
   s->H = nx / 2;
   s->W = nx / 2 + 1;
   s->G = std::max(nx, ny);
   s->px = MakeLinePlan(Log2(s->H), true);
   s->py = MakeLinePlan(Log2(ny), true);
   int entries = PlaceTables(s->px, 0);
   entries += PlaceTables(s->py, entries);
   const int bytes = static_cast<int>(kSmemMax);
   ISCU_CK(cudaFuncSetAttribute(ShiftColumnsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(cudaFuncSetAttribute(ShiftRowsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(s->tw.Reserve(s->G * sizeof(float2)));
   ISCU_CK(s->twg.Reserve(std::max(entries, 1) * sizeof(float2)));
   TwiddleKernel<<<(s->G + 255) / 256, 256, 0, ctx->stream>>>(static_cast<int>(s->G), s->tw.as<float2>());
   ISCU_CK_LAUNCH(ctx, "TwiddleKernel");
   for (const LinePlan* P : {&s->px, &s->py})
      for (int g = 0; g < P->groups; ++g)
         if (P->tw[g] >= 0)
         {
            const int M = 1 << (LogQ(*P, g) + P->r[g]);
            GroupTwiddleKernel<<<(M + 255) / 256, 256, 0, ctx->stream>>>(LogQ(*P, g), P->r[g],
                                                                          s->twg.as<float2>() + P->tw[g]);
            ISCU_CK_LAUNCH(ctx, "GroupTwiddleKernel");
         }
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   *out = s.release();
   return ISCU_OK;
}

void iscu_wf_shift_destroy(iscu_wf_shift* s)
{
   if (!s)
      return;
   cudaStreamSynchronize(s->ctx->stream);
   delete s;
}

int iscu_wf_shifted_frames_dev(iscu_wf_shift* s, const float* spectra_dev, uint32_t n_channels, const float* coef_dev,
                               const double* shift_dev, uint32_t n_frames, uint32_t x0, uint32_t y0, uint32_t cw,
                               uint32_t ch, uint32_t up, float scale, float* cam_dev)
{
   if (!s || (n_frames && (!spectra_dev || !coef_dev || !shift_dev || !cam_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   if (up < 1 || static_cast<uint64_t>(x0) + cw > s->nx || static_cast<uint64_t>(y0) + ch > s->ny)
      return Fail(ISCU_ERR_ARG, "the window must lie in the grid and up be >= 1");
   iscu_ctx* ctx = s->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const int camW = static_cast<int>(cw / up), camH = static_cast<int>(ch / up);
   if (!n_frames || !n_channels || camW == 0 || camH == 0)
      return ISCU_OK;
   const size_t budget = 200 * 1024;
   // column pass: BZ columns per CTA, with the row ramp table; the largest BZ <= 32 that lets two CTAs share an SM,
   // else the largest that fits one
   const size_t rampBytes = static_cast<size_t>(s->ny) * sizeof(double2);
   const auto colBytes = [&](int bz) { return rampBytes + static_cast<size_t>(s->ny) * bz * sizeof(float2); };
   int BZ = 1;
   while (BZ < 32 && colBytes(2 * BZ) <= kSmemPair)
      BZ *= 2;
   if (colBytes(BZ) > kSmemPair)   // (BZ = 1)
      while (BZ < 32 && colBytes(2 * BZ) <= budget)
         BZ *= 2;
   // row pass: BL lines (a power of two >= up), the staged rows and the transform's columns; the largest BL <= 16
   // that lets two CTAs share an SM, else the largest that fits one
   const auto rowBytes = [&](int bl) {
      return static_cast<size_t>(bl) * s->W * sizeof(float2) + static_cast<size_t>(s->H) * (bl + 1) * sizeof(float2);
   };
   int BL = 16;
   while (BL / 2 >= static_cast<int>(up) && rowBytes(BL) > kSmemPair)
      BL /= 2;
   if (rowBytes(BL) > kSmemPair)
      for (BL = 16; BL > 1 && rowBytes(BL) > budget; BL /= 2)
         ;
   if (BL < static_cast<int>(up))
      return Fail(ISCU_ERR_LIMIT, "drifting frames: " + std::to_string(up) + " cells per pixel need more rows in "
                                  "shared memory than this grid's width leaves");
   const int rowsPerCta = BL / static_cast<int>(up);
   ISCU_CK(s->T.Reserve(static_cast<size_t>(n_frames) * s->ny * s->W * sizeof(float2)));
   ShiftArgs a;
   a.spec = reinterpret_cast<const float2*>(spectra_dev);
   a.coef = coef_dev;
   a.shift = shift_dev;
   a.nChannels = static_cast<int>(n_channels);
   a.nx = static_cast<int>(s->nx);
   a.ny = static_cast<int>(s->ny);
   a.W = static_cast<int>(s->W);
   const size_t smemA = rampBytes + static_cast<size_t>(s->ny) * BZ * sizeof(float2);
   ShiftColumnsKernel<<<dim3((s->W + BZ - 1) / BZ, n_frames), kThreads, smemA, ctx->stream>>>(
      a, s->py, BZ, Log2(BZ), s->twg.as<float2>(), s->T.as<float2>());
   ISCU_CK_LAUNCH(ctx, "ShiftColumnsKernel");
   const size_t smemB = static_cast<size_t>(BL) * s->W * sizeof(float2) + static_cast<size_t>(s->H) * (BL + 1) *
                                                                             sizeof(float2);
   ShiftRowsKernel<<<dim3((camH + rowsPerCta - 1) / rowsPerCta, n_frames), kThreads, smemB, ctx->stream>>>(
      s->T.as<float2>(), s->px, static_cast<int>(s->nx), static_cast<int>(s->ny), static_cast<int>(s->W), BL,
      Log2(BL), rowsPerCta, static_cast<int>(up), static_cast<int>(x0), static_cast<int>(y0), camW, camH, scale,
      s->tw.as<float2>(), Log2(s->G) - Log2(s->nx), s->twg.as<float2>(), cam_dev);
   ISCU_CK_LAUNCH(ctx, "ShiftRowsKernel");
   return ISCU_OK;
}

} // extern "C"
