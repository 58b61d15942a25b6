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
// Passes (each a batch of 1D transforms in shared memory; the padded halves are never loaded, stored or
// transformed beyond the first butterfly stage that reads their zeros):
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
// are stored with ky and kz in bit-reversed order. Butterflies are fused in pairs (radix 4 per thread).
//
// Compiled with --fmad=false for the noise chain's exactness; the FFT arithmetic uses explicit __fmaf_rn.

#include "iscu_internal.h"
#include "noise_chain.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

struct iscu_wf_plan
{
   iscu_ctx* ctx = nullptr;
   uint32_t nx = 0, ny = 0, nz = 0, kx = 0, ky = 0, kz = 0;
   uint32_t GX = 0, GY = 0, GZ = 0, H = 0, NK = 0, G = 0;
   int logH = 0, logGY = 0, logGZ = 0;
   iscu::DevBuf A, B, Kh, tw, image, adu;
   // Pass timing (iscu_wf_set_timing): events before XForward and after each of the five passes.
   bool timing = false;
   cudaEvent_t ev[6] = {};
   void Mark(int i) const
   {
      if (timing)
         cudaEventRecord(ev[i], ctx->stream);
   }
};

namespace iscu {

namespace {

constexpr int kThreads = 256;
constexpr size_t kSmemLimit = 64 * 1024;

__device__ __forceinline__ float2 Cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 Csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 Cmul(float2 a, float2 b)
{
   return make_float2(__fmaf_rn(a.x, b.x, -(a.y * b.y)), __fmaf_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 Conj(float2 a) { return make_float2(a.x, -a.y); }

// W_M^j = exp(-2 pi i j / M) from the G-point table, M = 2^logM dividing G = 2^logG; conjugated for inverse
// transforms. Every size here is a power of two, so index arithmetic is shifts and masks.
__device__ __forceinline__ float2 Tw(const float2* __restrict__ tw, int logG, int logM, int j, bool inv)
{
   const float2 w = __ldg(tw + (j << (logG - logM)));
   return inv ? Conj(w) : w;
}

__device__ __forceinline__ int Rev(int n, int logN) { return static_cast<int>(__brev(static_cast<unsigned>(n)) >> (32 - logN)); }

// Lines in shared memory: element n of line b at s[b * ls + n * es]. kColumns: es > 1, ls = 1 (threads walk the
// lines fastest); else rows (es = 1, threads walk the elements fastest).
template <bool kColumns>
__device__ __forceinline__ void TupleOf(int t, int logTuples, int logNl, int& b, int& u)
{
   if (kColumns)
   {
      b = t & ((1 << logNl) - 1);
      u = t >> logNl;
   }
   else
   {
      b = t >> logTuples;
      u = t & ((1 << logTuples) - 1);
   }
}

// Decimation-in-frequency FFT of nl = 2^logNl lines of N = 2^logN points: natural order in, bit-reversed order out.
template <bool kColumns>
__device__ void DifLines(float2* s, int logN, int logNl, int ls, int es, const float2* __restrict__ tw, int logG,
                         bool inv)
{
   const int N = 1 << logN, total4 = (N >> 2) << logNl, total2 = (N >> 1) << logNl;
   int logQ = logN - 2;
   for (; logQ >= 0; logQ -= 2)
   {
      const int q = 1 << logQ;
      for (int t = threadIdx.x; t < total4; t += blockDim.x)
      {
         int b, u;
         TupleOf<kColumns>(t, logN - 2, logNl, b, u);
         const int j = u & (q - 1), i = ((u >> logQ) << (logQ + 2)) | j;
         float2* L = s + b * ls;
         const float2 e0 = L[i * es], e1 = L[(i + q) * es], e2 = L[(i + 2 * q) * es], e3 = L[(i + 3 * q) * es];
         const float2 a0 = Cadd(e0, e2), a1 = Cadd(e1, e3);
         const float2 a2 = Cmul(Csub(e0, e2), Tw(tw, logG, logQ + 2, j, inv));
         const float2 a3 = Cmul(Csub(e1, e3), Tw(tw, logG, logQ + 2, j + q, inv));
         const float2 w = Tw(tw, logG, logQ + 1, j, inv);
         L[i * es] = Cadd(a0, a1);
         L[(i + q) * es] = Cmul(Csub(a0, a1), w);
         L[(i + 2 * q) * es] = Cadd(a2, a3);
         L[(i + 3 * q) * es] = Cmul(Csub(a2, a3), w);
      }
      __syncthreads();
   }
   if (logQ == -1)   // logN odd: the last stage, span 1
   {
      for (int t = threadIdx.x; t < total2; t += blockDim.x)
      {
         int b, u;
         TupleOf<kColumns>(t, logN - 1, logNl, b, u);
         float2* L = s + b * ls;
         const float2 a = L[2 * u * es], c = L[(2 * u + 1) * es];
         L[2 * u * es] = Cadd(a, c);
         L[(2 * u + 1) * es] = Csub(a, c);
      }
      __syncthreads();
   }
}

// Decimation-in-time FFT: bit-reversed order in, natural order out.
template <bool kColumns>
__device__ void DitLines(float2* s, int logN, int logNl, int ls, int es, const float2* __restrict__ tw, int logG,
                         bool inv)
{
   const int N = 1 << logN, total4 = (N >> 2) << logNl, total2 = (N >> 1) << logNl;
   int logQ = 0;
   if (logN & 1)   // the first stage, span 1
   {
      for (int t = threadIdx.x; t < total2; t += blockDim.x)
      {
         int b, u;
         TupleOf<kColumns>(t, logN - 1, logNl, b, u);
         float2* L = s + b * ls;
         const float2 a = L[2 * u * es], c = L[(2 * u + 1) * es];
         L[2 * u * es] = Cadd(a, c);
         L[(2 * u + 1) * es] = Csub(a, c);
      }
      __syncthreads();
      logQ = 1;
   }
   for (; logQ < logN; logQ += 2)
   {
      const int q = 1 << logQ;
      for (int t = threadIdx.x; t < total4; t += blockDim.x)
      {
         int b, u;
         TupleOf<kColumns>(t, logN - 2, logNl, b, u);
         const int j = u & (q - 1), i = ((u >> logQ) << (logQ + 2)) | j;
         float2* L = s + b * ls;
         const float2 w = Tw(tw, logG, logQ + 1, j, inv);
         const float2 e0 = L[i * es], e1 = Cmul(L[(i + q) * es], w);
         const float2 e2 = L[(i + 2 * q) * es], e3 = Cmul(L[(i + 3 * q) * es], w);
         const float2 a0 = Cadd(e0, e1), a1 = Csub(e0, e1), a2 = Cadd(e2, e3), a3 = Csub(e2, e3);
         const float2 b2 = Cmul(a2, Tw(tw, logG, logQ + 2, j, inv)), b3 = Cmul(a3, Tw(tw, logG, logQ + 2, j + q, inv));
         L[i * es] = Cadd(a0, b2);
         L[(i + 2 * q) * es] = Csub(a0, b2);
         L[(i + q) * es] = Cadd(a1, b3);
         L[(i + 3 * q) * es] = Csub(a1, b3);
      }
      __syncthreads();
   }
}

// ------------------------------------------------------------------------------------------------ passes
struct Dims
{
   int nxv, nyv, nzv;   // valid extent of the input (volume or PSF)
   int GX, GY, GZ, H, NK, G, logH, logGY, logGZ, logG, logGX;
};

// Rows of `in` (nzv x nyv x nxv) -> A[z][k][y], k <= H, y < nyv. grid (ceil(nyv / BY), nzv); smem BY * H float2.
__global__ void __launch_bounds__(kThreads) XForwardKernel(const float* __restrict__ in, Dims d, int BY,
                                                           const float2* __restrict__ tw, float2* __restrict__ A)
{
   extern __shared__ float2 s[];
   const int z = blockIdx.y, y0 = blockIdx.x * BY;
   const int nb = min(BY, d.nyv - y0), H = d.H;
   const float* src = in + (static_cast<size_t>(z) * d.nyv + y0) * d.nxv;
   // packed pairs z[n] = x[2n] + i x[2n+1], natural order (the DIF input)
   for (int t = threadIdx.x; t < BY * H; t += blockDim.x)
   {
      const int b = t / H, n = t % H;
      float2 v = make_float2(0.f, 0.f);
      if (b < nb)
      {
         const float* row = src + static_cast<size_t>(b) * d.nxv;
         if (2 * n < d.nxv)
            v.x = row[2 * n];
         if (2 * n + 1 < d.nxv)
            v.y = row[2 * n + 1];
      }
      s[b * H + n] = v;
   }
   __syncthreads();
   DifLines<false>(s, d.logH, __ffs(BY) - 1, H, 1, tw, d.logG, false);
   // X[k] = ((Z[k] + conj Z[H-k]) - i W_GX^k (Z[k] - conj Z[H-k])) / 2, Z in bit-reversed order
   for (int t = threadIdx.x; t < (H + 1) * BY; t += blockDim.x)
   {
      const int k = t / BY, b = t % BY;
      if (b >= nb)
         continue;
      const float2 zk = s[b * H + Rev(k & (H - 1), d.logH)];
      const float2 zm = Conj(s[b * H + Rev((H - k) & (H - 1), d.logH)]);
      const float2 e = Cadd(zk, zm), o = Csub(zk, zm);
      const float2 w = Tw(tw, d.logG, d.logGX, k, false);
      const float2 wo = Cmul(w, o);   // then times -i: (x, y) -> (y, -x)
      const float2 X = make_float2(0.5f * (e.x + wo.y), 0.5f * (e.y - wo.x));
      A[(static_cast<size_t>(z) * d.NK + k) * d.nyv + y0 + b] = X;
   }
}

// A rows (nyv values per (z, k)) -> B[z][k][p], p = bit-reversed ky. grid (ceil(NK / BK), nzv).
__global__ void __launch_bounds__(kThreads) YForwardKernel(const float2* __restrict__ A, Dims d, int BK,
                                                           const float2* __restrict__ tw, float2* __restrict__ B)
{
   extern __shared__ float2 s[];
   const int z = blockIdx.y, k0 = blockIdx.x * BK, nb = min(BK, d.NK - k0), N = d.GY;
   for (int t = threadIdx.x; t < BK * N; t += blockDim.x)
   {
      const int b = t / N, n = t % N;
      float2 v = make_float2(0.f, 0.f);
      if (b < nb && n < d.nyv)
         v = A[(static_cast<size_t>(z) * d.NK + k0 + b) * d.nyv + n];
      s[b * N + n] = v;
   }
   __syncthreads();
   DifLines<false>(s, d.logGY, __ffs(BK) - 1, N, 1, tw, d.logG, false);
   for (int t = threadIdx.x; t < nb * N; t += blockDim.x)
   {
      const int b = t / N, p = t % N;
      B[(static_cast<size_t>(z) * d.NK + k0 + b) * N + p] = s[b * N + p];
   }
}

// Columns along z of B (nzv planes) -> GZ-point forward FFT -> either the PSF spectrum Kh[pz][k][p] (all GZ planes,
// forward only) or, times Kh, the inverse FFT cropped to planes [oz, oz + nzv) back into B.
// grid (ceil(GY / BZ), NK); smem GZ * BZ float2, column layout.
template <bool kConvolve>
__global__ void __launch_bounds__(kThreads) ZKernel(float2* __restrict__ B, Dims d, int BZ, int oz,
                                                    const float2* __restrict__ tw, float2* __restrict__ Kh)
{
   extern __shared__ float2 s[];
   const int k = blockIdx.y, p0 = blockIdx.x * BZ, nb = min(BZ, d.GY - p0), N = d.GZ;
   const size_t plane = static_cast<size_t>(d.NK) * d.GY;
   const size_t col = static_cast<size_t>(k) * d.GY + p0;
   for (int t = threadIdx.x; t < N * BZ; t += blockDim.x)
   {
      const int n = t / BZ, b = t % BZ;
      float2 v = make_float2(0.f, 0.f);
      if (b < nb && n < d.nzv)
         v = B[n * plane + col + b];
      s[n * BZ + b] = v;
   }
   __syncthreads();
   DifLines<true>(s, d.logGZ, __ffs(BZ) - 1, 1, BZ, tw, d.logG, false);
   if (!kConvolve)
   {
      for (int t = threadIdx.x; t < N * BZ; t += blockDim.x)
      {
         const int n = t / BZ, b = t % BZ;
         if (b < nb)
            Kh[n * plane + col + b] = s[n * BZ + b];
      }
      return;
   }
   for (int t = threadIdx.x; t < N * BZ; t += blockDim.x)
   {
      const int n = t / BZ, b = t % BZ;
      if (b < nb)
         s[n * BZ + b] = Cmul(s[n * BZ + b], Kh[n * plane + col + b]);
   }
   __syncthreads();
   DitLines<true>(s, d.logGZ, __ffs(BZ) - 1, 1, BZ, tw, d.logG, true);
   for (int t = threadIdx.x; t < d.nzv * BZ; t += blockDim.x)
   {
      const int n = t / BZ, b = t % BZ;
      if (b < nb)
         B[n * plane + col + b] = s[(n + oz) * BZ + b];
   }
}

// B rows (bit-reversed ky) -> inverse GY-point FFT -> rows [oy, oy + nyv) into A[z][k][y]. grid (ceil(NK / BK), nzv).
__global__ void __launch_bounds__(kThreads) YInverseKernel(const float2* __restrict__ B, Dims d, int BK, int oy,
                                                           const float2* __restrict__ tw, float2* __restrict__ A)
{
   extern __shared__ float2 s[];
   const int z = blockIdx.y, k0 = blockIdx.x * BK, nb = min(BK, d.NK - k0), N = d.GY;
   for (int t = threadIdx.x; t < BK * N; t += blockDim.x)
   {
      const int b = t / N, p = t % N;
      s[b * N + p] = b < nb ? B[(static_cast<size_t>(z) * d.NK + k0 + b) * N + p] : make_float2(0.f, 0.f);
   }
   __syncthreads();
   DitLines<false>(s, d.logGY, __ffs(BK) - 1, N, 1, tw, d.logG, true);
   for (int t = threadIdx.x; t < nb * d.nyv; t += blockDim.x)
   {
      const int b = t / d.nyv, y = t % d.nyv;
      A[(static_cast<size_t>(z) * d.NK + k0 + b) * d.nyv + y] = s[b * N + y + oy];
   }
}

// A (half spectrum along x, per (z, y)) -> GX reals -> columns [ox, ox + nxv), scaled, max(0, .) + background ->
// image and/or noise chain. grid (ceil(nyv / BY), nzv).
__global__ void __launch_bounds__(kThreads) XInverseKernel(const float2* __restrict__ A, Dims d, int BY, int ox,
                                                           float scale, float background, const float2* __restrict__ tw,
                                                           StaticView st, CameraView cam, int noise, uint32_t seed,
                                                           uint32_t frame0, float* __restrict__ image,
                                                           uint16_t* __restrict__ adu)
{
   extern __shared__ float2 s[];
   const int z = blockIdx.y, y0 = blockIdx.x * BY, nb = min(BY, d.nyv - y0), H = d.H;
   // Z'[k] = (X[k] + conj X[H-k]) + i W_GX^-k (X[k] - conj X[H-k]), k < H, into bit-reversed positions.
   for (int t = threadIdx.x; t < H * BY; t += blockDim.x)
   {
      const int k = t / BY, b = t % BY;
      float2 v = make_float2(0.f, 0.f);
      if (b < nb)
      {
         const float2 xk = A[(static_cast<size_t>(z) * d.NK + k) * d.nyv + y0 + b];
         const float2 xm = Conj(A[(static_cast<size_t>(z) * d.NK + (H - k)) * d.nyv + y0 + b]);
         const float2 e = Cadd(xk, xm), o = Cmul(Csub(xk, xm), Tw(tw, d.logG, d.logGX, k, true));
         v = make_float2(e.x - o.y, e.y + o.x);   // e + i o
      }
      s[b * H + Rev(k, d.logH)] = v;
   }
   __syncthreads();
   DitLines<false>(s, d.logH, __ffs(BY) - 1, H, 1, tw, d.logG, true);
   const uint32_t W = static_cast<uint32_t>(d.nxv);
   CounterRng u(seed, frame0 + static_cast<uint32_t>(z));
   for (int t = threadIdx.x; t < nb * d.nxv; t += blockDim.x)
   {
      const int b = t / d.nxv, x = t % d.nxv;
      const int m = x + ox;
      const float2 c = s[b * H + (m >> 1)];
      const float v = (m & 1 ? c.y : c.x) * scale;
      const float photons = (v > 0.f ? v : 0.f) + background;
      const uint32_t i = static_cast<uint32_t>(y0 + b) * W + static_cast<uint32_t>(x);
      const size_t o = static_cast<size_t>(z) * d.nyv * W + i;
      if (image)
         image[o] = photons;
      if (noise)
         adu[o] = NoisePixel(photons, i, cam, st, u);
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

int LinesPerCta(int N, int cap)
{
   int b = static_cast<int>(kSmemLimit / (static_cast<size_t>(N) * sizeof(float2)));
   return std::max(1, std::min(b, cap));
}

// The forward x and y passes of a (kzv x kyv x kxv) volume into A, B.
int ForwardXY(iscu_wf_plan* p, const float* in, const Dims& d, float2* A, float2* B, bool mark = false)
{
   iscu_ctx* ctx = p->ctx;
   const float2* tw = p->tw.as<float2>();
   const int BY = LinesPerCta(d.H, 16);
   XForwardKernel<<<dim3((d.nyv + BY - 1) / BY, d.nzv), kThreads, BY * d.H * sizeof(float2), ctx->stream>>>(
      in, d, BY, tw, A);
   ISCU_CK_LAUNCH(ctx, "XForwardKernel");
   if (mark)
      p->Mark(1);
   const int BK = LinesPerCta(d.GY, 16);
   YForwardKernel<<<dim3((d.NK + BK - 1) / BK, d.nzv), kThreads, BK * d.GY * sizeof(float2), ctx->stream>>>(
      A, d, BK, tw, B);
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
   return d;
}

int SetFftSmem()
{
   const int bytes = static_cast<int>(kSmemLimit);
   ISCU_CK(cudaFuncSetAttribute(XForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(cudaFuncSetAttribute(YForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(cudaFuncSetAttribute(ZKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(cudaFuncSetAttribute(ZKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(cudaFuncSetAttribute(YInverseKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   ISCU_CK(cudaFuncSetAttribute(XInverseKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   return ISCU_OK;
}

} // namespace

// The convolution of density_dev into the plan's A (cropped, before the x inverse) -- the passes up to YInverse.
static int ConvolveToA(iscu_wf_plan* p, const float* density)
{
   iscu_ctx* ctx = p->ctx;
   const Dims d = MakeDims(p, p->nx, p->ny, p->nz);
   const float2* tw = p->tw.as<float2>();
   p->Mark(0);
   int rc = ForwardXY(p, density, d, p->A.as<float2>(), p->B.as<float2>(), true);
   if (rc != ISCU_OK)
      return rc;
   p->Mark(2);
   const int BZ = LinesPerCta(d.GZ, 32);
   ZKernel<true><<<dim3((d.GY + BZ - 1) / BZ, d.NK), kThreads, d.GZ * BZ * sizeof(float2), ctx->stream>>>(
      p->B.as<float2>(), d, BZ, static_cast<int>(p->kz / 2), tw, p->Kh.as<float2>());
   ISCU_CK_LAUNCH(ctx, "ZKernel<convolve>");
   p->Mark(3);
   const int BK = LinesPerCta(d.GY, 16);
   YInverseKernel<<<dim3((d.NK + BK - 1) / BK, d.nzv), kThreads, BK * d.GY * sizeof(float2), ctx->stream>>>(
      p->B.as<float2>(), d, BK, static_cast<int>(p->ky / 2), tw, p->A.as<float2>());
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
   if (ctx->haveStatic && ctx->width == p->nx && ctx->height == p->ny)
      st = ctx->Static();
   st.width = p->nx;
   st.height = p->ny;
   const CameraView cv = cam ? MakeCameraView(*cam) : CameraView();
   const float scale = static_cast<float>(1.0 / (static_cast<double>(p->GX) * p->GY * p->GZ));
   // Few rows per CTA: the float64 noise chain that ends this pass wants occupancy more than row batching.
   const int BY = LinesPerCta(d.H, 4);
   XInverseKernel<<<dim3((d.nyv + BY - 1) / BY, d.nzv), kThreads, BY * d.H * sizeof(float2), ctx->stream>>>(
      p->A.as<float2>(), d, BY, static_cast<int>(p->kx / 2), scale, static_cast<float>(background),
      p->tw.as<float2>(), st, cv, cam ? 1 : 0, seed, frame0, image, adu);
   ISCU_CK_LAUNCH(ctx, "XInverseKernel");
   p->Mark(5);
   return ISCU_OK;
}

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
   std::unique_ptr<iscu_wf_plan> p(new iscu_wf_plan());
   p->ctx = ctx;
   p->nx = nx;
   p->ny = ny;
   p->nz = nz;
   p->kx = kx;
   p->ky = ky;
   p->kz = kz;
   p->GX = Pow2AtLeast(std::max(nx + kx - 1, 8u));
   p->GY = Pow2AtLeast(std::max(ny + ky - 1, 4u));
   p->GZ = Pow2AtLeast(std::max(nz + kz - 1, 4u));
   if (p->GX > 4096 || p->GY > 8192 || p->GZ > 8192)
      return Fail(ISCU_ERR_LIMIT, "widefield plan: padded grid beyond 4096 x 8192 x 8192");
   if (kx > p->GX || ky > p->GY)
      return Fail(ISCU_ERR_ARG, "widefield plan: PSF wider than the grid");
   p->H = p->GX / 2;
   p->NK = p->H + 1;
   p->G = std::max(p->GX, std::max(p->GY, p->GZ));
   p->logH = Log2(p->H);
   p->logGY = Log2(p->GY);
   p->logGZ = Log2(p->GZ);
   int rc = SetFftSmem();
   if (rc != ISCU_OK)
      return rc;
   const uint32_t nzA = std::max(nz, kz), nyA = std::max(ny, ky);
   ISCU_CK(p->tw.Reserve(p->G * sizeof(float2)));
   ISCU_CK(p->A.Reserve(static_cast<size_t>(nzA) * p->NK * nyA * sizeof(float2)));
   ISCU_CK(p->B.Reserve(static_cast<size_t>(nzA) * p->NK * p->GY * sizeof(float2)));
   ISCU_CK(p->Kh.Reserve(static_cast<size_t>(p->GZ) * p->NK * p->GY * sizeof(float2)));
   TwiddleKernel<<<(p->G + 255) / 256, 256, 0, ctx->stream>>>(static_cast<int>(p->G), p->tw.as<float2>());
   ISCU_CK_LAUNCH(ctx, "TwiddleKernel");
   // The PSF's spectrum: its own x and y passes (kx x ky x kz valid), then the forward z transform of all GZ planes.
   DevBuf dPsf;
   const size_t psfBytes = static_cast<size_t>(kx) * ky * kz * sizeof(float);
   ISCU_CK(dPsf.Reserve(psfBytes));
   ISCU_CK(cudaMemcpyAsync(dPsf.p, psf, psfBytes, cudaMemcpyHostToDevice, ctx->stream));
   const Dims dk = MakeDims(p.get(), kx, ky, kz);
   rc = ForwardXY(p.get(), dPsf.as<float>(), dk, p->A.as<float2>(), p->B.as<float2>());
   if (rc != ISCU_OK)
      return rc;
   const int BZ = LinesPerCta(dk.GZ, 32);
   ZKernel<false><<<dim3((dk.GY + BZ - 1) / BZ, dk.NK), kThreads, dk.GZ * BZ * sizeof(float2), ctx->stream>>>(
      p->B.as<float2>(), dk, BZ, 0, p->tw.as<float2>(), p->Kh.as<float2>());
   ISCU_CK_LAUNCH(ctx, "ZKernel<spectrum>");
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   *out = p.release();
   return ISCU_OK;
}

int iscu_wf_set_timing(iscu_wf_plan* plan, int32_t on)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   if (on && !plan->ev[0])
      for (int i = 0; i < 6; ++i)
         ISCU_CK(cudaEventCreate(&plan->ev[i]));
   plan->timing = on != 0;
   return ISCU_OK;
}

int iscu_wf_pass_times(iscu_wf_plan* plan, float* ms5)
{
   if (!plan || !ms5)
      return Fail(ISCU_ERR_ARG, "null argument");
   if (!plan->timing)
      return Fail(ISCU_ERR_STATE, "pass timing is off (iscu_wf_set_timing)");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   ISCU_CK(cudaEventSynchronize(plan->ev[5]));
   for (int i = 0; i < 5; ++i)
      ISCU_CK(cudaEventElapsedTime(ms5 + i, plan->ev[i], plan->ev[i + 1]));
   return ISCU_OK;
}

void iscu_wf_plan_destroy(iscu_wf_plan* plan)
{
   if (!plan)
      return;
   cudaStreamSynchronize(plan->ctx->stream);
   for (int i = 0; i < 6; ++i)
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

int iscu_wf_render(iscu_wf_plan* plan, const float* density, double background, const iscu_camera* cam,
                   uint32_t seed, uint32_t frame0, float* image, uint16_t* adu)
{
   if (!plan || !density || (cam && !adu) || (!cam && !image))
      return Fail(ISCU_ERR_ARG, "null argument");
   iscu_ctx* ctx = plan->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const size_t n = static_cast<size_t>(plan->nx) * plan->ny * plan->nz;
   ISCU_CK(ctx->dScratch.Reserve(n * sizeof(float)));
   if (image)
      ISCU_CK(plan->image.Reserve(n * sizeof(float)));
   if (adu)
      ISCU_CK(plan->adu.Reserve(n * sizeof(uint16_t)));
   ISCU_CK(cudaMemcpyAsync(ctx->dScratch.p, density, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
   int rc = ConvolveToA(plan, ctx->dScratch.as<float>());
   if (rc != ISCU_OK)
      return rc;
   rc = FinishX(plan, background, cam, seed, frame0, image ? plan->image.as<float>() : nullptr,
                adu ? plan->adu.as<uint16_t>() : nullptr);
   if (rc != ISCU_OK)
      return rc;
   if (image)
      ISCU_CK(cudaMemcpyAsync(image, plan->image.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
   if (adu)
      ISCU_CK(cudaMemcpyAsync(adu, plan->adu.p, n * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

} // extern "C"
