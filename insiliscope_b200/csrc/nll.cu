// Poisson negative log-likelihood of ROI images and its gradient on sm_100a (no reference counterpart: the
// reference has no gradient; its nearest relative is DescribePsfCramerRao's central-difference PSF derivatives,
// adapter/inSiliScope/Simulation/PsfGeneratorBridge.cpp:1554-1669).
//
// Model: the reference's Gibson-Lanni/Zernike pupil (ZernikePsf.cpp:188-248) at matched indices and depth 0,
// at a continuous defocus z and position (x, y) per emitter:
//   U[m] = a[m] exp(i phi[m]),  phi = z kz + 2 pi sum_j c_j Z_j - p (kx x + ky y)
//   E = A U A^T  (A[s][m] = exp(i k_m p u_s), u_s = (s + 0.5) / os: the separable DFT to the ROI's sub-pixel samples)
//   mu[i][j] = N kappa sum over pixel (i, j)'s os x os samples of |E|^2 + b_frame
//   NLL = sum mu - k log mu
// and its adjoint: w = 1 - k / mu, G = w N kappa, U_bar = A^H (G o E) conj(A), dNLL/dphi = -2 Im(conj(U_bar) U),
// then the chain through phi (x, y, z, Zernike), dNLL/dN = sum w PSF, dNLL/db = sum w.
//
// One CTA per emitter at a time (a persistent grid): the pupil phase in float64, reduced mod 2 pi, then float32
// sincos; the four complex matmuls (forward 32x32 -> 32x64 -> 64x64, adjoint back) in shared memory in float32; the
// per-emitter sums in float64. The gradient pass recomputes the field instead of storing per-emitter PSFs. The
// Zernike gradient accumulates per CTA in float64 across its emitters and is added once per CTA.

#include "iscu_internal.h"
#include "psf_common.cuh"

#include <cmath>
#include <memory>
#include <vector>

struct iscu_nll_model
{
   iscu_ctx* ctx = nullptr;
   iscu_nll_spec spec{};
   int M = 0, P = 0, J = 0;
   double kappa = 0.0;
   iscu::DevBuf samples;   // M*M x double4: (p kx, p ky, kz, a)
   iscu::DevBuf basis;     // J x M*M float64: 2 pi Z_j
   iscu::DevBuf A;         // P x M float2
   iscu::DevBuf zphase;    // M*M float64: 2 pi sum c_j Z_j of the current evaluation
   iscu::DevBuf zern;      // J float64
};

namespace iscu {

namespace {

constexpr int kM = 32, kP = 64, kThreads = 256, kMaxJ = 32;
constexpr int kPre = 4;   // observed counts a thread loads ahead (ROIs up to 32 x 32 pixels)

__device__ __forceinline__ float2 Cmul(float2 a, float2 b)
{
   return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ void Cfma(float2& acc, float2 a, float2 b)
{
   acc.x = fmaf(a.x, b.x, acc.x);
   acc.x = fmaf(-a.y, b.y, acc.x);
   acc.y = fmaf(a.x, b.y, acc.y);
   acc.y = fmaf(a.y, b.x, acc.y);
}

// C[r][c] = sum_k L(r, k) R(k, c) over a ROWS x COLS output, a TR x TC tile per thread (rows ty + 16 i, columns
// tx + 16 j); epi(r, c, value) stores.
template <int ROWS, int COLS, int K, class LF, class RF, class EF>
__device__ __forceinline__ void SmemGemm(LF L, RF R, EF epi)
{
   constexpr int TR = ROWS / 16, TC = COLS / 16;
   static_assert(TR * 16 == ROWS && TC * 16 == COLS, "16 x 16 threads");
   const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
   float2 acc[TR][TC];
#pragma unroll
   for (int i = 0; i < TR; ++i)
#pragma unroll
      for (int j = 0; j < TC; ++j)
         acc[i][j] = make_float2(0.f, 0.f);
#pragma unroll 4
   for (int k = 0; k < K; ++k)
   {
      float2 l[TR], r[TC];
#pragma unroll
      for (int i = 0; i < TR; ++i)
         l[i] = L(ty + 16 * i, k);
#pragma unroll
      for (int j = 0; j < TC; ++j)
         r[j] = R(k, tx + 16 * j);
#pragma unroll
      for (int i = 0; i < TR; ++i)
#pragma unroll
         for (int j = 0; j < TC; ++j)
            Cfma(acc[i][j], l[i], r[j]);
   }
#pragma unroll
   for (int i = 0; i < TR; ++i)
#pragma unroll
      for (int j = 0; j < TC; ++j)
         epi(ty + 16 * i, tx + 16 * j, acc[i][j]);
}

// Sums of NV float64 values over the CTA in one exchange, each in BlockSum's order (every thread calls it; every
// thread gets the sums). red: NV x (kThreads / 32) doubles.
template <int NV>
__device__ __forceinline__ void BlockSums(double (&v)[NV], double* red)
{
#pragma unroll
   for (int q = 0; q < NV; ++q)
#pragma unroll
      for (int d = 16; d > 0; d >>= 1)
         v[q] += __shfl_xor_sync(0xffffffffu, v[q], d);
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   __syncthreads();
   if (lane == 0)
#pragma unroll
      for (int q = 0; q < NV; ++q)
         red[q * (kThreads / 32) + warp] = v[q];
   __syncthreads();
#pragma unroll
   for (int q = 0; q < NV; ++q)
   {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w)
         t += red[q * (kThreads / 32) + w];
      v[q] = t;
   }
}

// Sum over the CTA in float64 (every thread calls it; the result is returned to every thread).
__device__ __forceinline__ double BlockSum(double v, double* red)
{
#pragma unroll
   for (int d = 16; d > 0; d >>= 1)
      v += __shfl_xor_sync(0xffffffffu, v, d);
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   __syncthreads();
   if (lane == 0)
      red[warp] = v;
   __syncthreads();
   double s = 0.0;
#pragma unroll
   for (int w = 0; w < kThreads / 32; ++w)
      s += red[w];
   return s;
}

__global__ void ZernPhaseKernel(const double* __restrict__ basis, const double* __restrict__ zern, int J, int MM,
                                double* __restrict__ zphase)
{
   const int m = blockIdx.x * blockDim.x + threadIdx.x;
   if (m >= MM)
      return;
   double s = 0.0;
   for (int j = 0; j < J; ++j)
      s += zern[j] * basis[static_cast<size_t>(j) * MM + m];
   zphase[m] = s;
}

struct NllArgs
{
   const double4* samples;
   const double* basis;
   const float2* A;
   const double* zphase;
   int J, R, os;
   double kappa;
   uint32_t n;
   const float4* params;     // x, y (ROI px), z (nm), N
   const int32_t* frame;
   uint32_t nFrames;
   const float* bg;
   const float* counts;      // n x R x R
   float* mu;                // nullable
   double* nll;              // accumulated
   float4* gParams;          // nullable: the gradient pass
   double* gBg;
   double* gZern;
   int* err;                 // 1: an emitter names a frame outside the batch
};

struct NllSmem
{
   float2 A[kP][kM];
   float2 At[kM][kP];     // A transposed: the first product reads it along rows (conflict-free) instead of down A's
                          // columns (16 lanes 256 bytes apart, one bank)
   float2 U[kM][kM];
   float2 T[kM][kP];
   float2 E[kP][kP];
   float dphi[kM * kM];
   double dphiSum[kM * kM];   // the CTA's emitters' dNLL/dphi, summed in float64, for the Zernike gradient
   double red[3 * (kThreads / 32)];
};

template <bool kGrad>
__global__ void __launch_bounds__(kThreads, 2) NllKernel(NllArgs a)
{
   extern __shared__ __align__(16) unsigned char smemRaw[];
   NllSmem& s = *reinterpret_cast<NllSmem*>(smemRaw);
   const int tid = threadIdx.x;
   for (int i = tid; i < kP * kM; i += kThreads)
   {
      s.A[i / kM][i % kM] = a.A[i];
      s.At[i % kM][i / kM] = a.A[i];
   }
   // the Zernike gradient is linear in dNLL/dphi: the CTA sums dphi over its emitters (float64, each sample by one
   // thread) and projects the sum onto the modes once, at the end
   for (int m = tid; m < kM * kM; m += kThreads)
      s.dphiSum[m] = 0.0;
   double nllAcc = 0.0;
   const int R = a.R, os = a.os, RR = R * R;
   __syncthreads();
   for (uint32_t e = blockIdx.x; e < a.n; e += gridDim.x)
   {
      const float4 pr = a.params[e];
      const int f = a.frame[e];
      const bool frameOk = f >= 0 && static_cast<uint32_t>(f) < a.nFrames;
      if (!frameOk && tid == 0)
         atomicExch(a.err, 1);
      const double b = frameOk ? static_cast<double>(a.bg[f]) : 0.0;
      const double x = pr.x, y = pr.y, z = pr.z, N = pr.w;
      // the observed counts of this thread's pixels p = tid + 256 q, loaded now so that their latency passes under
      // the pupil and the forward products (ROIs of up to 32 x 32 pixels: at most four a thread)
      const float* k = a.counts + static_cast<size_t>(e) * RR;
      const bool pre = RR <= kPre * kThreads;
      float kpre[kPre];
#pragma unroll
      for (int q = 0; q < kPre; ++q)
         kpre[q] = pre && tid + q * kThreads < RR ? k[tid + q * kThreads] : 0.f;
      // 1. the pupil
      for (int m = tid; m < kM * kM; m += kThreads)
      {
         const double4 sm = a.samples[m];
         const double ph = ReduceTwoPi(z * sm.z + a.zphase[m] - (sm.x * x + sm.y * y));
         float sn, cs;
         __sincosf(static_cast<float>(ph), &sn, &cs);
         const float amp = static_cast<float>(sm.w);
         s.U[m / kM][m % kM] = make_float2(amp * cs, amp * sn);
      }
      __syncthreads();
      // 2. T = U A^T (32 x 64), 3. E = A T (64 x 64)
      SmemGemm<kM, kP, kM>([&](int r, int k) { return s.U[r][k]; }, [&](int k, int c) { return s.At[k][c]; },
                           [&](int r, int c, float2 v) { s.T[r][c] = v; });
      __syncthreads();
      SmemGemm<kP, kP, kM>([&](int r, int k) { return s.A[r][k]; }, [&](int k, int c) { return s.T[k][c]; },
                           [&](int r, int c, float2 v) { s.E[r][c] = v; });
      __syncthreads();
      // 4. expected counts and the likelihood; the gradient weights into E
      double part = 0.0, gN = 0.0, gB = 0.0;
      auto pixel = [&](int p, float kf) {
         const int i = p / R, j = p % R;
         float sum = 0.f;
         for (int ty = 0; ty < os; ++ty)
            for (int tx = 0; tx < os; ++tx)
            {
               const float2 v = s.E[i * os + ty][j * os + tx];
               sum = fmaf(v.x, v.x, fmaf(v.y, v.y, sum));
            }
         const double psf = a.kappa * static_cast<double>(sum);
         const double mu = N * psf + b;
         const double kk = static_cast<double>(kf);
         part += mu - kk * log(mu);
         if (a.mu)
            a.mu[static_cast<size_t>(e) * RR + p] = static_cast<float>(mu);
         if (kGrad)
         {
            const double w = 1.0 - kk / mu;
            gN += w * psf;
            gB += w;
            const float G = static_cast<float>(w * N * a.kappa);
            for (int ty = 0; ty < os; ++ty)
               for (int tx = 0; tx < os; ++tx)
               {
                  float2& v = s.E[i * os + ty][j * os + tx];
                  v = make_float2(G * v.x, G * v.y);
               }
         }
      };
      if (RR == kPre * kThreads)
      {
         // Every thread has kPre pixels (32 x 32 ROIs): the same operations as `pixel`, in stages across its pixels so
         // that their float64 chains (the logarithm, the quotient) run side by side; each sum takes its terms in the
         // same order, so the results are the pixel-by-pixel form's.
         double psf[kPre], mu[kPre], lg[kPre], w[kPre];
#pragma unroll
         for (int q = 0; q < kPre; ++q)
         {
            const int p = tid + q * kThreads, i = p / R, j = p % R;
            float sum = 0.f;
            for (int ty = 0; ty < os; ++ty)
               for (int tx = 0; tx < os; ++tx)
               {
                  const float2 v = s.E[i * os + ty][j * os + tx];
                  sum = fmaf(v.x, v.x, fmaf(v.y, v.y, sum));
               }
            psf[q] = a.kappa * static_cast<double>(sum);
            mu[q] = N * psf[q] + b;
         }
#pragma unroll
         for (int q = 0; q < kPre; ++q)
            lg[q] = log(mu[q]);
#pragma unroll
         for (int q = 0; q < kPre; ++q)
            w[q] = 1.0 - static_cast<double>(kpre[q]) / mu[q];
#pragma unroll
         for (int q = 0; q < kPre; ++q)
         {
            const int p = tid + q * kThreads, i = p / R, j = p % R;
            part += mu[q] - static_cast<double>(kpre[q]) * lg[q];
            if (a.mu)
               a.mu[static_cast<size_t>(e) * RR + p] = static_cast<float>(mu[q]);
            if (kGrad)
            {
               gN += w[q] * psf[q];
               gB += w[q];
               const float G = static_cast<float>(w[q] * N * a.kappa);
               for (int ty = 0; ty < os; ++ty)
                  for (int tx = 0; tx < os; ++tx)
                  {
                     float2& v = s.E[i * os + ty][j * os + tx];
                     v = make_float2(G * v.x, G * v.y);
                  }
            }
         }
      }
      else if (pre)
      {
#pragma unroll
         for (int q = 0; q < kPre; ++q)
            if (tid + q * kThreads < RR)
               pixel(tid + q * kThreads, kpre[q]);
      }
      else
         for (int p = tid; p < RR; p += kThreads)
            pixel(p, k[p]);
      nllAcc += part;
      if (!kGrad)
      {
         __syncthreads();
         continue;
      }
      double nb[2] = {gN, gB};   // one exchange for both sums
      BlockSums<2>(nb, s.red);
      gN = nb[0];
      gB = nb[1];
      if (tid == 0 && frameOk)
         atomicAdd(&a.gBg[f], gB);
      __syncthreads();
      // 5. T_bar = A^H (G o E) (32 x 64), 6. U_bar = T_bar conj(A) (32 x 32) and dNLL/dphi
      SmemGemm<kM, kP, kP>([&](int r, int k) { const float2 v = s.A[k][r]; return make_float2(v.x, -v.y); },
                           [&](int k, int c) { return s.E[k][c]; },
                           [&](int r, int c, float2 v) { s.T[r][c] = v; });
      __syncthreads();
      SmemGemm<kM, kM, kP>([&](int r, int k) { return s.T[r][k]; },
                           [&](int k, int c) { const float2 v = s.A[k][c]; return make_float2(v.x, -v.y); },
                           [&](int r, int c, float2 v) {
                              const float2 u = s.U[r][c];
                              // -2 Im(conj(U_bar) U) = -2 (Ubar.x u.y - Ubar.y u.x)
                              s.dphi[r * kM + c] = -2.f * (v.x * u.y - v.y * u.x);
                           });
      __syncthreads();
      // 7. the chain through phi
      double gx = 0.0, gy = 0.0, gzd = 0.0;
      for (int m = tid; m < kM * kM; m += kThreads)
      {
         const double4 sm = a.samples[m];
         const double d = s.dphi[m];
         gx -= d * sm.x;
         gy -= d * sm.y;
         gzd += d * sm.z;
         s.dphiSum[m] += d;
      }
      double xyz[3] = {gx, gy, gzd};
      BlockSums<3>(xyz, s.red);
      gx = xyz[0];
      gy = xyz[1];
      gzd = xyz[2];
      if (tid == 0)
         a.gParams[e] = make_float4(static_cast<float>(gx), static_cast<float>(gy), static_cast<float>(gzd),
                                    static_cast<float>(gN));
      __syncthreads();
   }
   // the CTA's sums
   const double nllCta = BlockSum(nllAcc, s.red);
   if (tid == 0)
      atomicAdd(a.nll, nllCta);
   if (kGrad)
   {
      // warp w projects the summed dphi onto modes j = w, w + 8, ...
      __syncthreads();
      const int lane = tid & 31, warp = tid >> 5;
      for (int j = warp; j < a.J; j += kThreads / 32)
      {
         const double* Zj = a.basis + static_cast<size_t>(j) * kM * kM;
         double v = 0.0;
         for (int m = lane; m < kM * kM; m += 32)
            v += s.dphiSum[m] * Zj[m];
#pragma unroll
         for (int d = 16; d > 0; d >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, d);
         if (lane == 0)
            atomicAdd(&a.gZern[j], v);
      }
   }
}

// Noll's orthonormal Z_j (n, m from j) at (rho, theta).
void NollNm(int j, int& n, int& m)
{
   n = 0;
   int j1 = j - 1;
   while (j1 > n)
   {
      ++n;
      j1 -= n;
   }
   m = ((j % 2) ? -1 : 1) * ((n % 2) + 2 * ((j1 + ((n + 1) % 2)) / 2));
}

double Factorial(int k)
{
   double f = 1.0;
   for (int i = 2; i <= k; ++i)
      f *= i;
   return f;
}

double ZernikeNoll(int j, double rho, double theta)
{
   int n, m;
   NollNm(j, n, m);
   const int am = m < 0 ? -m : m;
   double r = 0.0;
   for (int s = 0; s <= (n - am) / 2; ++s)
   {
      const double c = ((s % 2) ? -1.0 : 1.0) * Factorial(n - s) /
                       (Factorial(s) * Factorial((n + am) / 2 - s) * Factorial((n - am) / 2 - s));
      r += c * std::pow(rho, n - 2 * s);
   }
   if (m == 0)
      return std::sqrt(n + 1.0) * r;
   return std::sqrt(2.0 * (n + 1)) * r * (m > 0 ? std::cos(am * theta) : std::sin(am * theta));
}

} // namespace

} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_nll_model_create(iscu_ctx* ctx, const iscu_nll_spec* spec, iscu_nll_model** out)
{
   if (!ctx || !spec || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   if (spec->pupil != kM || spec->roi * spec->os != kP || spec->roi < 1 || spec->os < 1)
      return Fail(ISCU_ERR_LIMIT, "the gradient model takes a 32 x 32 pupil and roi * os = 64 samples");
   if (spec->n_zern < 0 || spec->n_zern > kMaxJ)
      return Fail(ISCU_ERR_LIMIT, "at most 32 Zernike modes");
   if (!(spec->wavelength_nm > 0.0) || !(spec->na > 0.0) || !(spec->n_imm >= spec->na) || !(spec->pixel_nm > 0.0))
      return Fail(ISCU_ERR_ARG, "wavelength, NA, immersion index >= NA and pixel size must be positive");
   for (int j = 0; j < spec->n_zern; ++j)
      if (spec->noll[j] < 1 || spec->noll[j] > 66)
         return Fail(ISCU_ERR_ARG, "Noll indices 1..66");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   std::unique_ptr<iscu_nll_model> mdl(new iscu_nll_model());
   mdl->ctx = ctx;
   mdl->spec = *spec;
   const int M = kM, P = kP, J = spec->n_zern, MM = M * M;
   mdl->M = M;
   mdl->P = P;
   mdl->J = J;
   const double pi = 3.14159265358979323846;
   const double kmax = 2.0 * pi * spec->na / spec->wavelength_nm, dk = 2.0 * kmax / (M - 4);
   const double k0n = 2.0 * pi * spec->n_imm / spec->wavelength_nm;
   std::vector<double> samp(4 * static_cast<size_t>(MM)), basis(static_cast<size_t>(J) * MM, 0.0);
   double aSum = 0.0;
   for (int iy = 0; iy < M; ++iy)
      for (int ix = 0; ix < M; ++ix)
      {
         const int m = iy * M + ix;
         const double ky = (iy - M / 2) * dk, kx = (ix - M / 2) * dk, kr2 = kx * kx + ky * ky;
         const bool in = kr2 <= kmax * kmax;
         samp[4 * m + 0] = spec->pixel_nm * kx;
         samp[4 * m + 1] = spec->pixel_nm * ky;
         samp[4 * m + 2] = in ? std::sqrt(std::max(0.0, k0n * k0n - kr2)) : 0.0;
         samp[4 * m + 3] = in ? 1.0 : 0.0;
         aSum += in ? 1.0 : 0.0;
         if (in)
            for (int j = 0; j < J; ++j)
               basis[static_cast<size_t>(j) * MM + m] =
                  2.0 * pi * ZernikeNoll(spec->noll[j], std::sqrt(kr2) / kmax, std::atan2(ky, kx));
      }
   std::vector<float2> A(static_cast<size_t>(P) * M);
   for (int sIdx = 0; sIdx < P; ++sIdx)
      for (int m = 0; m < M; ++m)
      {
         const double u = (sIdx + 0.5) / spec->os;
         const double ph = (m - M / 2) * dk * spec->pixel_nm * u;
         A[static_cast<size_t>(sIdx) * M + m] = make_float2(static_cast<float>(std::cos(ph)),
                                                            static_cast<float>(std::sin(ph)));
      }
   const double L = 2.0 * pi / dk, px = spec->pixel_nm / spec->os;
   mdl->kappa = px * px / (L * L * aSum);
   ISCU_CK(mdl->samples.Reserve(samp.size() * sizeof(double)));
   ISCU_CK(mdl->basis.Reserve(std::max<size_t>(basis.size(), 1) * sizeof(double)));
   ISCU_CK(mdl->A.Reserve(A.size() * sizeof(float2)));
   ISCU_CK(mdl->zphase.Reserve(MM * sizeof(double)));
   ISCU_CK(mdl->zern.Reserve(kMaxJ * sizeof(double)));
   ISCU_CK(cudaMemcpyAsync(mdl->samples.p, samp.data(), samp.size() * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
   if (!basis.empty())
      ISCU_CK(cudaMemcpyAsync(mdl->basis.p, basis.data(), basis.size() * sizeof(double), cudaMemcpyHostToDevice,
                              ctx->stream));
   ISCU_CK(cudaMemcpyAsync(mdl->A.p, A.data(), A.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   ISCU_CK(cudaFuncSetAttribute(NllKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(NllSmem))));
   ISCU_CK(cudaFuncSetAttribute(NllKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(NllSmem))));
   *out = mdl.release();
   return ISCU_OK;
}

void iscu_nll_model_destroy(iscu_nll_model* model)
{
   if (!model)
      return;
   cudaStreamSynchronize(model->ctx->stream);
   delete model;
}

int iscu_nll_model_info(iscu_nll_model* model, double* kappa, int32_t* n_zern)
{
   if (!model)
      return Fail(ISCU_ERR_ARG, "null model");
   if (kappa)
      *kappa = model->kappa;
   if (n_zern)
      *n_zern = model->J;
   return ISCU_OK;
}

int iscu_nll_eval_dev(iscu_nll_model* model, uint32_t n_emitters, const float* params_dev, const int32_t* frame_dev,
                      uint32_t n_frames, const float* bg_dev, const double* zern, const float* counts_dev,
                      float* mu_dev, double* nll_dev, float* grad_params_dev, double* grad_bg_dev,
                      double* grad_zern_dev, int32_t* err_dev)
{
   if (!model || !nll_dev || !err_dev || (n_emitters && (!params_dev || !frame_dev || !counts_dev)) ||
       (n_frames && !bg_dev) || (model->J && !zern))
      return Fail(ISCU_ERR_ARG, "null argument");
   const bool grad = grad_params_dev != nullptr;
   if (grad && ((n_frames && !grad_bg_dev) || (model->J && !grad_zern_dev)))
      return Fail(ISCU_ERR_ARG, "the gradient needs every gradient output");
   iscu_ctx* ctx = model->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const int MM = model->M * model->M;
   if (model->J)
   {
      ISCU_CK(cudaMemcpyAsync(model->zern.p, zern, model->J * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      ZernPhaseKernel<<<(MM + 255) / 256, 256, 0, ctx->stream>>>(model->basis.as<double>(), model->zern.as<double>(),
                                                                  model->J, MM, model->zphase.as<double>());
      ISCU_CK_LAUNCH(ctx, "ZernPhaseKernel");
   }
   else
      ISCU_CK(cudaMemsetAsync(model->zphase.p, 0, MM * sizeof(double), ctx->stream));
   ISCU_CK(cudaMemsetAsync(nll_dev, 0, sizeof(double), ctx->stream));
   ISCU_CK(cudaMemsetAsync(err_dev, 0, sizeof(int32_t), ctx->stream));
   if (grad)
   {
      if (n_frames)
         ISCU_CK(cudaMemsetAsync(grad_bg_dev, 0, n_frames * sizeof(double), ctx->stream));
      if (model->J)
         ISCU_CK(cudaMemsetAsync(grad_zern_dev, 0, model->J * sizeof(double), ctx->stream));
   }
   if (n_emitters == 0)
      return ISCU_OK;
   NllArgs a;
   a.samples = model->samples.as<double4>();
   a.basis = model->basis.as<double>();
   a.A = model->A.as<float2>();
   a.zphase = model->zphase.as<double>();
   a.J = model->J;
   a.R = model->spec.roi;
   a.os = model->spec.os;
   a.kappa = model->kappa;
   a.n = n_emitters;
   a.params = reinterpret_cast<const float4*>(params_dev);
   a.frame = frame_dev;
   a.nFrames = n_frames;
   a.bg = bg_dev;
   a.counts = counts_dev;
   a.mu = mu_dev;
   a.nll = nll_dev;
   a.gParams = reinterpret_cast<float4*>(grad_params_dev);
   a.gBg = grad_bg_dev;
   a.gZern = grad_zern_dev;
   a.err = err_dev;
   const size_t smem = sizeof(NllSmem);
   int perSm = 0;
   if (grad)
      ISCU_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, NllKernel<true>, kThreads, smem));
   else
      ISCU_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, NllKernel<false>, kThreads, smem));
   const uint32_t grid = std::min<uint32_t>(n_emitters, static_cast<uint32_t>(std::max(1, perSm) * ctx->smCount));
   if (grad)
      NllKernel<true><<<grid, kThreads, smem, ctx->stream>>>(a);
   else
      NllKernel<false><<<grid, kThreads, smem, ctx->stream>>>(a);
   ISCU_CK_LAUNCH(ctx, "NllKernel");
   return ISCU_OK;
}

} // extern "C"
