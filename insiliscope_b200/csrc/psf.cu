// PSF stacks and libraries on sm_100a: the Gibson-Lanni + Zernike (+ double-helix) pupil and its chirp-Z image
// (ComputeZernikePsfPlanes, adapter/inSiliScope/Simulation/ZernikePsf.cpp:160-337).
//
// The reference evaluates out[p] = sum_m in[m] exp(i (kMin + m dk)(x0 + p dx)) per pupil line by Bluestein's
// chirp-Z in float64 (ChirpZ.h:28-142), rows then columns. Here the two passes are the dense products
// E = A U A^T with A[p][m] = exp(i (kMin + m dk)(x0 + p dx)) -- the DFT matrix the CZT factorizes -- so they run as
// matrix multiplications. Float64 is kept where the phases are large: the pupil's OPD phase
// k0 (opd1 + ni (ti - ti0) opd3) + zernike + mask, and the DFT exponent, are formed and reduced mod 2 pi in float64,
// then the unit phasors are rounded to float32.
//
// Kernels:
//  PupilTablesKernel  z-independent pupil tables per request set (aperture, opd1, the opd3 obliquity factor,
//                     Zernike + mask phase), float64 (ZernikePsf.cpp:188-231)
//  DftMatrixKernel    A (P x M) and A^T (M x P) per set, float32 phasors of float64 phases
//  CztFp32Kernel      the plain FP32 form: one CTA per PSF, pupil phasors into shared memory, T = A U and
//                     E = T A^T as register-tiled SIMT complex products, |E|^2, optional sum-1 normalization
// The tensor-core form (TF32 split products on tcgen05) is in psf_tc.cu.

#include "iscu_internal.h"
#include "psf_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace iscu {

namespace {

constexpr double kPi = 3.14159265358979323846;

// ------------------------------------------------------------------------------------------ Zernike (device, FP64)
__device__ double Binomial(int a, int b)
{
   if (b < 0 || b > a)
      return 0.0;
   double r = 1.0;
   for (int i = 0; i < b; ++i)
      r = r * (a - i) / (i + 1);
   return r;
}

// Unnormalized radial polynomial R_n^m, m >= 0 (ZernikePsf.cpp:58-67).
__device__ double ZernikeRadial(int n, int m, double rho)
{
   double r = 0.0;
   for (int k = 0; k <= (n - m) / 2; ++k)
   {
      const double coeff = (k % 2 == 0 ? 1.0 : -1.0) * Binomial(n - k, k) * Binomial(n - 2 * k, (n - m) / 2 - k);
      r += coeff * pow(rho, static_cast<double>(n - 2 * k));
   }
   return r;
}

// ZernikeValue (ZernikePsf.cpp:74-78).
__device__ double ZernikeValue(int n, int l, int m, double rho, double phi)
{
   const double radial = rho <= 1.0 ? ZernikeRadial(n, m, rho) : 0.0;
   return radial * (l >= 0 ? cos(m * phi) : sin(m * phi));
}

__device__ double LaguerreL(int p, int a, double x)
{
   double lm1 = 0.0, l = 1.0;
   for (int k = 0; k < p; ++k)
   {
      const double next = ((2 * k + 1 + a - x) * l - (k + a) * lm1) / (k + 1);
      lm1 = l;
      l = next;
   }
   return l;
}

// MaskPhase (ZernikePsf.cpp:93-110): the double-helix Gauss-Laguerre superposition's phase.
__device__ double MaskPhase(int maskModes, double maskWaist, double rhoNorm, double phi)
{
   const int n = maskModes > 2 ? maskModes : 2;
   const double w = maskWaist > 0.2 ? maskWaist : 0.2;
   const double u = fmax(0.0, fmin(1.0, rhoNorm)) / w;
   const double u2 = u * u;
   double re = 0.0, im = 0.0;
   for (int p = 0; p < n; ++p)
   {
      const int l = 2 * p + 1;
      const double amp = pow(u, static_cast<double>(l)) * exp(-u2) * LaguerreL(p, l, 2.0 * u2);
      re += amp * cos(l * phi);
      im += amp * sin(l * phi);
   }
   return (re == 0.0 && im == 0.0) ? 0.0 : atan2(im, re);
}

// ------------------------------------------------------------------------------------------ tables
// tables[s][idx] = (opd1, opd3Factor, zernike + mask phase); opd3Factor < 0 marks a sample outside the aperture.
__global__ void PupilTablesKernel(const SetParams* __restrict__ sets, int M, double3* __restrict__ tables)
{
   const int s = blockIdx.y;
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if (idx >= M * M)
      return;
   const SetParams& sp = sets[s];
   const int iy = idx / M, ix = idx % M, c0 = M / 2;
   const double ky = (iy - c0) * sp.dk, kx = (ix - c0) * sp.dk;
   // The aperture test decides samples that sit exactly on the circle (M = 64: (30, 0), (18, 24), ...): rounded
   // product by product, as the reference's uncontracted float64 does, so the same samples are in.
   const double kr2 = __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
   double3 out = make_double3(0.0, -1.0, 0.0);
   if (!(kr2 > __dmul_rn(sp.kMax, sp.kMax)))
   {
      const double kr = sqrt(kr2);
      const double rho = kr / (sp.k0 * sp.na);
      const double phi = atan2(ky, kx);
      const double s1 = sp.na * rho / sp.ns;
      const double s3 = sp.na * rho / sp.ni;
      out.x = sp.ns * sp.depthM * sqrt(fmax(0.0, 1.0 - s1 * s1));
      out.y = sqrt(fmax(0.0, 1.0 - s3 * s3));
      double zern = 0.0;
      for (int t = 0; t < sp.nModes; ++t)
         zern += sp.coeff[t] * ZernikeValue(sp.modeN[t], sp.modeL[t], sp.modeM[t], rho / sp.bMax, phi);
      zern *= 2.0 * kPi;
      const double mask = sp.doubleHelix ? MaskPhase(sp.maskModes, sp.maskWaist, rho / sp.bMax, phi) : 0.0;
      out.z = zern + mask;
   }
   tables[static_cast<size_t>(s) * M * M + idx] = out;
}

// ------------------------------------------------------------------------------------------ DFT matrices
// A[s][p][m] = exp(i (kMin + m dk)(x0 + p dx)); At[s][m][p] the same value. float64 phase reduced mod 2 pi first.
__global__ void DftMatrixKernel(const SetParams* __restrict__ sets, int M, int P, float2* __restrict__ A,
                                float2* __restrict__ At)
{
   const int s = blockIdx.y;
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if (idx >= P * M)
      return;
   const SetParams& sp = sets[s];
   const int p = idx / M, m = idx % M;
   const double ph = ReduceTwoPi((sp.kMin + m * sp.dk) * (sp.x0 + p * sp.dx));
   double sn, cs;
   sincos(ph, &sn, &cs);
   const float2 v = make_float2(static_cast<float>(cs), static_cast<float>(sn));
   A[static_cast<size_t>(s) * P * M + idx] = v;
   At[static_cast<size_t>(s) * P * M + static_cast<size_t>(m) * P + p] = v;
}

// ------------------------------------------------------------------------------------------ plain FP32 chirp-Z
constexpr int kCztThreads = 256;

__device__ __forceinline__ void Cmac(float2& acc, float2 a, float2 b)
{
   acc.x = fmaf(a.x, b.x, acc.x);
   acc.x = fmaf(-a.y, b.y, acc.x);
   acc.y = fmaf(a.x, b.y, acc.y);
   acc.y = fmaf(a.y, b.x, acc.y);
}

// C[r][c] = sum_k L[r][k] R[k][c], rows x cols, 64 x 64 output blocks, a 4 x 4 complex tile per thread (rows
// ty + 16 i, columns tx + 16 j: a warp reads R contiguously and L by broadcast). epi(r, c, value) stores.
template <class Epi>
__device__ __forceinline__ void CGemm(const float2* __restrict__ L, int ldl, const float2* __restrict__ R, int ldr,
                                      int rows, int cols, int K, Epi epi)
{
   const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
   for (int rb = 0; rb < rows; rb += 64)
      for (int cb = 0; cb < cols; cb += 64)
      {
         float2 acc[4][4];
#pragma unroll
         for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
               acc[i][j] = make_float2(0.f, 0.f);
         int ri[4], cj[4];
#pragma unroll
         for (int i = 0; i < 4; ++i)
         {
            ri[i] = min(rb + ty + 16 * i, rows - 1);
            cj[i] = min(cb + tx + 16 * i, cols - 1);
         }
#pragma unroll 4
         for (int k = 0; k < K; ++k)
         {
            float2 l[4], r[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
               l[i] = L[static_cast<size_t>(ri[i]) * ldl + k];
               r[i] = R[static_cast<size_t>(k) * ldr + cj[i]];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
               for (int j = 0; j < 4; ++j)
                  Cmac(acc[i][j], l[i], r[j]);
         }
#pragma unroll
         for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
               const int r = rb + ty + 16 * i, c = cb + tx + 16 * j;
               if (r < rows && c < cols)
                  epi(r, c, acc[i][j]);
            }
      }
}

__global__ void __launch_bounds__(kCztThreads) CztFp32Kernel(const SetParams* __restrict__ sets,
                                                               const double3* __restrict__ tables,
                                                               const float2* __restrict__ A,
                                                               const float2* __restrict__ At,
                                                               const PsfItem* __restrict__ items, int M, int P,
                                                               int normalize, float* __restrict__ out)
{
   extern __shared__ __align__(16) unsigned char smem[];
   float2* U = reinterpret_cast<float2*>(smem);                                  // M x M pupil phasors
   float2* T = U + static_cast<size_t>(M) * M;                                   // P x M
   __shared__ double sRed[kCztThreads / 32];
   const PsfItem it = items[blockIdx.x];
   const SetParams& sp = sets[it.set];
   const double3* tab = tables + static_cast<size_t>(it.set) * M * M;
   const float2* As = A + static_cast<size_t>(it.set) * P * M;
   const float2* Ats = At + static_cast<size_t>(it.set) * P * M;

   // Pupil: phase = k0 (opd1 + ni (ti - ti0) opd3F) + zernike + mask (ZernikePsf.cpp:240-248), float64 then reduced.
   for (int idx = threadIdx.x; idx < M * M; idx += blockDim.x)
      U[idx] = PupilPhasor(tab[idx], sp, it.dtiM);
   __syncthreads();
   // Row pass: T[y][m] = sum_n A[y][n] U[n][m].
   CGemm(As, M, U, M, P, M, M, [&](int r, int c, float2 v) { T[static_cast<size_t>(r) * M + c] = v; });
   __syncthreads();
   // Column pass: E[y][x] = sum_m T[y][m] A[x][m]; I = |E|^2.
   float* plane = out + static_cast<size_t>(blockIdx.x) * P * P;
   double local = 0.0;
   CGemm(T, M, Ats, P, P, P, M, [&](int r, int c, float2 v) {
      const float I = v.x * v.x + v.y * v.y;
      plane[static_cast<size_t>(r) * P + c] = I;
      local += static_cast<double>(I);
   });
   if (!normalize)
      return;
   const double sum = BlockSumDouble(local, sRed);
   __syncthreads();
   if (sum > 0.0)
      for (int idx = threadIdx.x; idx < P * P; idx += blockDim.x)
         plane[idx] = static_cast<float>(static_cast<double>(plane[idx]) / sum);
}

// ------------------------------------------------------------------------------------------ large pupils
// When the pupil and the row pass do not fit shared memory (M beyond ~128: a widefield kernel's 512-sample pupil),
// the same products go through global memory: the pupil phasors U (nPsf x M x M), then two batched complex GEMMs
// with 64 x 64 output tiles staged 16 deep in shared memory -- T = A U, E = T A^T -- the second one ending in |E|^2
// and the plane's float64 sum.
__global__ void PupilKernel(const SetParams* __restrict__ sets, const double3* __restrict__ tables,
                            const PsfItem* __restrict__ items, int M, float2* __restrict__ U)
{
   const int b = blockIdx.y;
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if (idx >= M * M)
      return;
   const PsfItem it = items[b];
   U[static_cast<size_t>(b) * M * M + idx] =
      PupilPhasor(tables[static_cast<size_t>(it.set) * M * M + idx], sets[it.set], it.dtiM);
}

// C[b] (rows x cols) = L (rows x K) R (K x cols), L = L0 + set * lSet + b * lBatch, R likewise. kIntensity: writes
// |C|^2 as float and adds the tile's float64 sum to sums[b].
template <bool kIntensity>
__global__ void __launch_bounds__(256) CGemmTiledKernel(const PsfItem* __restrict__ items, const float2* __restrict__ L0,
                                                       size_t lSet, size_t lBatch, const float2* __restrict__ R0,
                                                       size_t rSet, size_t rBatch, int rows, int cols, int K,
                                                       float2* __restrict__ C, float* __restrict__ I,
                                                       double* __restrict__ sums)
{
   __shared__ float2 sL[16][65];
   __shared__ float2 sR[16][64];
   __shared__ double sRed[8];
   const int b = blockIdx.z, set = items[b].set;
   const float2* L = L0 + set * lSet + b * lBatch;
   const float2* R = R0 + set * rSet + b * rBatch;
   const int rb = blockIdx.y * 64, cb = blockIdx.x * 64;
   const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
   float2 acc[4][4];
#pragma unroll
   for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
         acc[i][j] = make_float2(0.f, 0.f);
   for (int k0 = 0; k0 < K; k0 += 16)
   {
#pragma unroll
      for (int e4 = 0; e4 < 4; ++e4)
      {
         const int e = threadIdx.x + 256 * e4;
         const int r = e >> 4, kk = e & 15, kr = e >> 6, c = e & 63;
         sL[kk][r] = (rb + r < rows && k0 + kk < K) ? L[static_cast<size_t>(rb + r) * K + k0 + kk]
                                                    : make_float2(0.f, 0.f);
         sR[kr][c] = (k0 + kr < K && cb + c < cols) ? R[static_cast<size_t>(k0 + kr) * cols + cb + c]
                                                    : make_float2(0.f, 0.f);
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < 16; ++kk)
      {
         float2 l[4], r[4];
#pragma unroll
         for (int i = 0; i < 4; ++i)
         {
            l[i] = sL[kk][ty + 16 * i];
            r[i] = sR[kk][tx + 16 * i];
         }
#pragma unroll
         for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
               Cmac(acc[i][j], l[i], r[j]);
      }
      __syncthreads();
   }
   double local = 0.0;
#pragma unroll
   for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
      {
         const int r = rb + ty + 16 * i, c = cb + tx + 16 * j;
         if (r >= rows || c >= cols)
            continue;
         const size_t o = static_cast<size_t>(b) * rows * cols + static_cast<size_t>(r) * cols + c;
         if (kIntensity)
         {
            const float v = acc[i][j].x * acc[i][j].x + acc[i][j].y * acc[i][j].y;
            I[o] = v;
            local += static_cast<double>(v);
         }
         else
            C[o] = acc[i][j];
      }
   if (kIntensity)
   {
      const double t = BlockSumDouble(local, sRed);
      if (threadIdx.x == 0)
         atomicAdd(sums + b, t);
   }
}

__global__ void NormalizeKernel(float* __restrict__ planes, const double* __restrict__ sums, int planeElems)
{
   const int b = blockIdx.y;
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= planeElems)
      return;
   const double s = sums[b];
   if (s > 0.0)
   {
      float* p = planes + static_cast<size_t>(b) * planeElems;
      p[i] = static_cast<float>(static_cast<double>(p[i]) / s);
   }
}

} // namespace

// The large-pupil FP32 path (global-memory products); temporaries allocated here.
static int LaunchCztGlobalFp32(iscu_ctx* ctx, const SetParams* dSets, const double3* dTab, const float2* dA,
                               const float2* dAt, const PsfItem* dItems, uint32_t nPsf, int M, int P, int normalize,
                               float* out)
{
   DevBuf U, T, S;
   // in batches bounded to ~2 GB of temporaries
   const size_t perPsf = (static_cast<size_t>(M) * M + static_cast<size_t>(P) * M) * sizeof(float2);
   const uint32_t batch = static_cast<uint32_t>(std::max<size_t>(1, std::min<size_t>(nPsf, (2ull << 30) / perPsf)));
   ISCU_CK(U.Reserve(static_cast<size_t>(batch) * M * M * sizeof(float2)));
   ISCU_CK(T.Reserve(static_cast<size_t>(batch) * P * M * sizeof(float2)));
   ISCU_CK(S.Reserve(static_cast<size_t>(nPsf) * sizeof(double)));
   ISCU_CK(cudaMemsetAsync(S.p, 0, static_cast<size_t>(nPsf) * sizeof(double), ctx->stream));
   for (uint32_t b0 = 0; b0 < nPsf; b0 += batch)
   {
      const uint32_t nb = std::min(batch, nPsf - b0);
      PupilKernel<<<dim3((M * M + 255) / 256, nb), 256, 0, ctx->stream>>>(dSets, dTab, dItems + b0, M,
                                                                          U.as<float2>());
      ISCU_CK_LAUNCH(ctx, "PupilKernel");
      CGemmTiledKernel<false><<<dim3((M + 63) / 64, (P + 63) / 64, nb), 256, 0, ctx->stream>>>(
         dItems + b0, dA, static_cast<size_t>(P) * M, 0, U.as<float2>(), 0, static_cast<size_t>(M) * M, P, M, M,
         T.as<float2>(), nullptr, nullptr);
      ISCU_CK_LAUNCH(ctx, "CGemmTiledKernel<product>");
      CGemmTiledKernel<true><<<dim3((P + 63) / 64, (P + 63) / 64, nb), 256, 0, ctx->stream>>>(
         dItems + b0, T.as<float2>(), 0, static_cast<size_t>(P) * M, dAt, static_cast<size_t>(P) * M, 0, P, P, M,
         nullptr, out + static_cast<size_t>(b0) * P * P, S.as<double>() + b0);
      ISCU_CK_LAUNCH(ctx, "CGemmTiledKernel<intensity>");
   }
   if (normalize)
   {
      NormalizeKernel<<<dim3((P * P + 255) / 256, nPsf), 256, 0, ctx->stream>>>(out, S.as<double>(), P * P);
      ISCU_CK_LAUNCH(ctx, "NormalizeKernel");
   }
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

// ------------------------------------------------------------------------------------------ host side

// GeometryFor + ZernikePupilSamples (ZernikePsf.cpp:118-158).
bool GeometryFor(const iscu_psf_request& r, PsfGeometry& g, std::string& err)
{
   if (!(r.na > 0.0) || !(r.wavelength_nm > 0.0) || !(r.immersion_index > 0.0) || !(r.sample_index > 0.0) ||
       !(r.pixel_size_nm > 0.0) || !(r.z_step_nm > 0.0))
   {
      err = "GibsonLanniZernike PSF: NA, wavelength, refractive indices, pixel size and z step must be > 0.";
      return false;
   }
   g.os = std::max(1, r.oversampling);
   const int camHalf = std::max(1, r.kernel_half_width_px);
   g.halfOv = camHalf * g.os;
   g.size = 2 * g.halfOv + 1;
   const int nzWanted = std::max(3, r.nz);
   g.nz = (nzWanted % 2 == 1) ? nzWanted : nzWanted + 1;
   g.resLateralNm = r.pixel_size_nm / g.os;
   if (r.pupil_samples > 0)
      g.M = std::max(8, std::min(1024, static_cast<int>(r.pupil_samples)));
   else
   {
      const double diagonalUm = 2.0 * std::sqrt(2.0) * camHalf * r.pixel_size_nm / 1000.0;
      const double m = 4.0 + 2.0 * r.na * diagonalUm / (r.wavelength_nm / 1000.0);
      const int need = std::max(64, std::min(512, 4 * static_cast<int>(std::ceil(m / 4.0))));
      int fftLen = 1;
      while (fftLen < need + g.size - 1)
         fftLen <<= 1;
      g.M = std::max(need, std::min(512, (fftLen - g.size + 1) / 4 * 4));
   }
   return true;
}

// The set parameters of a request for planes of `size` samples (ZernikePsf.cpp:166-223's scalars).
static void MakeSetParams(const iscu_psf_request& r, int M, int size, double resLateralNm, SetParams& sp)
{
   std::memset(&sp, 0, sizeof(sp));
   const double NA = r.na;
   const double lambda = r.wavelength_nm * 1E-9;
   sp.na = NA;
   sp.ni = r.immersion_index;
   sp.ns = r.sample_index;
   sp.depthM = r.sample_depth_nm * 1E-9;
   sp.k0 = 2.0 * kPi / lambda;
   sp.bMax = std::min(1.0, sp.ns / NA);
   sp.kMax = sp.k0 * NA * sp.bMax;
   sp.dk = (2.0 * sp.kMax) / (M - 4);
   sp.kMin = -std::floor(M / 2.0) * sp.dk;
   sp.dx = resLateralNm * 1E-9;
   sp.x0 = -((size - 1) / 2.0) * sp.dx;
   sp.doubleHelix = r.mask_double_helix ? 1 : 0;
   sp.maskModes = r.mask_modes;
   sp.maskWaist = r.mask_waist;
   int n = 0;
   for (int j = 0; j < 28; ++j)
   {
      if (r.zernike[j] == 0.0)
         continue;
      // OSA/ANSI j -> (n, l): j = n(n+1)/2 + k, l = -n + 2k (ZernikePsf.cpp:34-44).
      int nn = 0;
      while ((nn + 1) * (nn + 2) / 2 <= j)
         ++nn;
      const int k = j - nn * (nn + 1) / 2;
      const int l = -nn + 2 * k;
      sp.coeff[n] = r.zernike[j];
      sp.modeN[n] = nn;
      sp.modeL[n] = l;
      sp.modeM[n] = std::abs(l);
      ++n;
   }
   sp.nModes = n;
   sp.ti0 = r.working_distance_um * 1E-6;
   sp.focalShift = sp.depthM * (sp.ni / sp.ns);
}

int BuildPsfLibrary(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t nSets, const uint32_t* setOfPsf,
                    const double* defocusM, uint32_t nPsf, int32_t size, int32_t normalize, int32_t method,
                    float* out)
{
   if (nSets == 0 || nPsf == 0)
      return ISCU_OK;
   std::string err;
   PsfGeometry g0;
   if (!GeometryFor(sets[0], g0, err))
      return Fail(ISCU_ERR_ARG, err);
   const int M = g0.M;
   const int P = size > 0 ? size : g0.size;
   std::vector<SetParams> hs(nSets);
   for (uint32_t s = 0; s < nSets; ++s)
   {
      PsfGeometry g;
      if (!GeometryFor(sets[s], g, err))
         return Fail(ISCU_ERR_ARG, err);
      if (g.M != M)
         return Fail(ISCU_ERR_ARG, "psf library: every set must have the same pupil samples");
      MakeSetParams(sets[s], M, P, g.resLateralNm, hs[s]);
   }
   std::vector<PsfItem> items(nPsf);
   for (uint32_t i = 0; i < nPsf; ++i)
   {
      if (setOfPsf[i] >= nSets)
         return Fail(ISCU_ERR_ARG, "psf library: set index out of range");
      const SetParams& sp = hs[setOfPsf[i]];
      items[i].set = static_cast<int>(setOfPsf[i]);
      // ti - ti0 = (ti0 - focalShift) + defocus - ti0 (ZernikePsf.cpp:237-243).
      const double ti = (sp.ti0 - sp.focalShift) + defocusM[i];
      items[i].dtiM = ti - sp.ti0;
   }
   const size_t tabBytes = static_cast<size_t>(nSets) * M * M * sizeof(double3);
   const size_t matBytes = static_cast<size_t>(nSets) * P * M * sizeof(float2);
   const size_t setBytes = nSets * sizeof(SetParams), itemBytes = nPsf * sizeof(PsfItem);
   DevBuf dSets, dItems, dTab, dA, dAt;
   ISCU_CK(dSets.Reserve(setBytes));
   ISCU_CK(dItems.Reserve(itemBytes));
   ISCU_CK(dTab.Reserve(tabBytes));
   ISCU_CK(dA.Reserve(matBytes));
   ISCU_CK(dAt.Reserve(matBytes));
   ISCU_CK(cudaMemcpyAsync(dSets.p, hs.data(), setBytes, cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(dItems.p, items.data(), itemBytes, cudaMemcpyHostToDevice, ctx->stream));
   PupilTablesKernel<<<dim3((M * M + 127) / 128, nSets), 128, 0, ctx->stream>>>(dSets.as<SetParams>(), M,
                                                                                 dTab.as<double3>());
   ISCU_CK_LAUNCH(ctx, "PupilTablesKernel");
   DftMatrixKernel<<<dim3((P * M + 255) / 256, nSets), 256, 0, ctx->stream>>>(dSets.as<SetParams>(), M, P,
                                                                              dA.as<float2>(), dAt.as<float2>());
   ISCU_CK_LAUNCH(ctx, "DftMatrixKernel");
   if (method == ISCU_CZT_TF32X3 || method == ISCU_CZT_F16X3)
   {
      const int rc = LaunchCztSplit(ctx, method, dSets.as<SetParams>(), dTab.as<double3>(), dA.as<float2>(), nSets,
                                    dItems.as<PsfItem>(), nPsf, M, P, normalize, out);
      if (rc != ISCU_OK)
         return rc;
   }
   else
   {
      const size_t smem = (static_cast<size_t>(M) * M + static_cast<size_t>(P) * M) * sizeof(float2);
      if (smem > 227 * 1024)
         return LaunchCztGlobalFp32(ctx, dSets.as<SetParams>(), dTab.as<double3>(), dA.as<float2>(),
                                    dAt.as<float2>(), dItems.as<PsfItem>(), nPsf, M, P, normalize, out);
      ISCU_CK(cudaFuncSetAttribute(CztFp32Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
      CztFp32Kernel<<<nPsf, kCztThreads, smem, ctx->stream>>>(dSets.as<SetParams>(), dTab.as<double3>(),
                                                               dA.as<float2>(), dAt.as<float2>(),
                                                               dItems.as<PsfItem>(), M, P, normalize, out);
      ISCU_CK_LAUNCH(ctx, "CztFp32Kernel");
   }
   // The temporaries are freed when this returns; the stream must finish with them first.
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

// The set parameters of up to maxSets requests into caller memory (no heap): the pupil samples M and plane size P
// they share. Used by the allocation-free entry point (psf_noalloc.cu).
int PrepareSetParams(const iscu_psf_request* sets, uint32_t nSets, int32_t size, uint32_t maxSets, SetParams* out,
                     int* M, int* P)
{
   if (nSets == 0 || nSets > maxSets)
      return Fail(ISCU_ERR_LIMIT, "psf library: 1.." + std::to_string(maxSets) + " request sets");
   std::string err;
   PsfGeometry g0;
   if (!GeometryFor(sets[0], g0, err))
      return Fail(ISCU_ERR_ARG, err);
   *M = g0.M;
   *P = size > 0 ? size : g0.size;
   for (uint32_t s = 0; s < nSets; ++s)
   {
      PsfGeometry g;
      if (!GeometryFor(sets[s], g, err))
         return Fail(ISCU_ERR_ARG, err);
      if (g.M != *M)
         return Fail(ISCU_ERR_ARG, "psf library: every set must have the same pupil samples");
      MakeSetParams(sets[s], *M, *P, g.resLateralNm, out[s]);
   }
   return ISCU_OK;
}

// The per-set tables and DFT matrices (once per set; a PSF plan keeps them).
int LaunchPsfTables(iscu_ctx* ctx, const SetParams* dSets, uint32_t nSets, int M, int P, double3* dTab, float2* dA,
                    float2* dAt)
{
   PupilTablesKernel<<<dim3((M * M + 127) / 128, nSets), 128, 0, ctx->stream>>>(dSets, M, dTab);
   ISCU_CK_LAUNCH(ctx, "PupilTablesKernel");
   DftMatrixKernel<<<dim3((P * M + 255) / 256, nSets), 256, 0, ctx->stream>>>(dSets, M, P, dA, dAt);
   ISCU_CK_LAUNCH(ctx, "DftMatrixKernel");
   return ISCU_OK;
}

// The plain FP32 chirp-Z of nPsf items over prepared tables (shared-memory form, or the global-memory form for
// pupils beyond shared memory).
int LaunchCztFp32(iscu_ctx* ctx, const SetParams* dSets, const double3* dTab, const float2* dA, const float2* dAt,
                  const PsfItem* dItems, uint32_t nPsf, int M, int P, int normalize, float* out)
{
   const size_t smem = (static_cast<size_t>(M) * M + static_cast<size_t>(P) * M) * sizeof(float2);
   if (smem > 227 * 1024)
      return LaunchCztGlobalFp32(ctx, dSets, dTab, dA, dAt, dItems, nPsf, M, P, normalize, out);
   ISCU_CK(cudaFuncSetAttribute(CztFp32Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
   CztFp32Kernel<<<nPsf, kCztThreads, smem, ctx->stream>>>(dSets, dTab, dA, dAt, dItems, M, P, normalize, out);
   ISCU_CK_LAUNCH(ctx, "CztFp32Kernel");
   return ISCU_OK;
}

int CheckFp32CztSmem(iscu_ctx* ctx, int M, int P, size_t* smem)
{
   *smem = (static_cast<size_t>(M) * M + static_cast<size_t>(P) * M) * sizeof(float2);
   cudaFuncAttributes fa;
   ISCU_CK(cudaFuncGetAttributes(&fa, CztFp32Kernel));
   int optin = 0;
   ISCU_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
   if (*smem + fa.sharedSizeBytes > static_cast<size_t>(optin))
      return Fail(ISCU_ERR_LIMIT, "psf library (fp32): the pupil and row pass need (M*M + P*M)*8 = " +
                                     std::to_string(*smem) + " bytes of shared memory beside the kernel's " +
                                     std::to_string(fa.sharedSizeBytes) + ", over the device's " +
                                     std::to_string(optin) + " per block (M = " + std::to_string(M) + ", P = " +
                                     std::to_string(P) + ")");
   return ISCU_OK;
}

// The plain FP32 pipeline (tables, DFT matrices, chirp-Z) on buffers the caller provides.
int LaunchPsfPipelineFp32(iscu_ctx* ctx, const SetParams* dSets, const PsfItem* dItems, double3* dTab, float2* dA,
                          float2* dAt, uint32_t nSets, uint32_t nPsf, int M, int P, int normalize, float* out)
{
   PupilTablesKernel<<<dim3((M * M + 127) / 128, nSets), 128, 0, ctx->stream>>>(dSets, M, dTab);
   ISCU_CK_LAUNCH(ctx, "PupilTablesKernel");
   DftMatrixKernel<<<dim3((P * M + 255) / 256, nSets), 256, 0, ctx->stream>>>(dSets, M, P, dA, dAt);
   ISCU_CK_LAUNCH(ctx, "DftMatrixKernel");
   size_t smem = 0;
   const int rc = CheckFp32CztSmem(ctx, M, P, &smem);
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(cudaFuncSetAttribute(CztFp32Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
   CztFp32Kernel<<<nPsf, kCztThreads, smem, ctx->stream>>>(dSets, dTab, dA, dAt, dItems, M, P, normalize, out);
   ISCU_CK_LAUNCH(ctx, "CztFp32Kernel");
   return ISCU_OK;
}

} // namespace iscu
