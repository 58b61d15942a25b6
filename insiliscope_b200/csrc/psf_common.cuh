// Shared by the PSF kernels (psf.cu: plain FP32 form; psf_tc.cu and psf_tc16.cu: the tensor-core TF32 and FP16
// split forms).
#pragma once

#include "iscu_internal.h"

#include <cstdint>

namespace iscu {

// One request set's scalars (ZernikePsf.cpp:166-223), in SI units.
struct SetParams
{
   double na, ni, ns, depthM, k0, bMax, kMax, dk, kMin, dx, x0, ti0, focalShift;
   double maskWaist;
   int doubleHelix, maskModes, nModes, pad;
   double coeff[28];
   int modeN[28], modeL[28], modeM[28];
};

// One PSF of a library: its set and ti - ti0 (metres).
struct PsfItem
{
   double dtiM;
   int set, pad;
};

// x - 2 pi n, n = rint(x / 2 pi), in float64 with a two-part 2 pi (Cody and Waite's additive reduction).
__device__ __forceinline__ double ReduceTwoPi(double x)
{
   const double kTwoPiHi = 6.283185307179586232;      // 2 pi rounded to float64
   const double kTwoPiLo = 2.4492935982947064e-16;    // 2 pi - kTwoPiHi
   const double n = rint(x * 0.15915494309189533577);
   double r = fma(-n, kTwoPiHi, x);
   r = fma(-n, kTwoPiLo, r);
   return r;
}

// The pupil phasor of one sample: phase = k0 (opd1 + ni (ti - ti0) opd3F) + (zernike + mask) in float64
// (ZernikePsf.cpp:240-248), reduced, then its float32 cosine and sine. Outside the aperture: 0.
__device__ __forceinline__ float2 PupilPhasor(double3 tab, const SetParams& sp, double dtiM)
{
   if (tab.y < 0.0)
      return make_float2(0.f, 0.f);
   const double opd3 = sp.ni * dtiM * tab.y;
   const double ph = ReduceTwoPi(sp.k0 * (tab.x + opd3) + tab.z);
   float s, c;
   sincosf(static_cast<float>(ph), &s, &c);
   return make_float2(c, s);
}

// Sum of one double per thread over the CTA (every thread gets the total). red: blockDim.x / 32 doubles.
__device__ __forceinline__ double BlockSumDouble(double v, double* red)
{
   for (int o = 16; o > 0; o >>= 1)
      v += __shfl_xor_sync(0xffffffffu, v, o);
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   __syncthreads();
   if (lane == 0)
      red[warp] = v;
   __syncthreads();
   double t = 0.0;
   for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
      t += red[w];
   return t;
}

// The split-precision chirp-Z (method ISCU_CZT_TF32X3 or ISCU_CZT_F16X3) for one library: builds the method's
// per-set data, runs, waits and reports a tensor-core wait that ran out.
int LaunchCztSplit(iscu_ctx* ctx, int method, const SetParams* sets, const double3* tables, const float2* A,
                   uint32_t nSets, const PsfItem* items, uint32_t nPsf, int M, int P, int normalize, float* out);
bool Tf32x3Supports(int M, int P);
bool F16x3Supports(int M, int P);
// The split-precision kernels' per-set data in one buffer: the DFT operand's K-block images in the method's layout
// (SplitImageBytes), then the pupil phase tables (TF32: float64 radians; FP16: float32 revolutions).
int BuildAhat(iscu_ctx* ctx, const float2* A, const SetParams* sets, const double3* tables, int nSets, int M, int P,
              int method, DevBuf& ahat);
size_t SplitImageBytes(int method, int nSets);
size_t AhatF16Bytes(int nSets);
int BuildAhatF16(iscu_ctx* ctx, const float2* A, const SetParams* sets, const double3* tables, int nSets, int M,
                 int P, unsigned char* out);
int LaunchCztTf32x3Core(iscu_ctx* ctx, const SetParams* sets, const float* ahat, int nSets, const PsfItem* items,
                        uint32_t nPsf, int M, int P, int normalize, float* out, int* dErr);
int LaunchCztF16x3Core(iscu_ctx* ctx, const SetParams* sets, const unsigned char* ahat, int nSets,
                       const PsfItem* items, uint32_t nPsf, int M, int P, int normalize, float* out, int* dErr);

int LaunchPsfTables(iscu_ctx* ctx, const SetParams* dSets, uint32_t nSets, int M, int P, double3* dTab, float2* dA,
                    float2* dAt);
int LaunchCztFp32(iscu_ctx* ctx, const SetParams* dSets, const double3* dTab, const float2* dA, const float2* dAt,
                  const PsfItem* dItems, uint32_t nPsf, int M, int P, int normalize, float* out);

int PrepareSetParams(const iscu_psf_request* sets, uint32_t nSets, int32_t size, uint32_t maxSets, SetParams* out,
                     int* M, int* P);
// ISCU_OK when the FP32 chirp-Z kernel's dynamic shared memory -- the pupil (M x M) and the row pass (P x M), complex
// float -- fits beside its static shared memory in one CTA of the context's device (the per-block opt-in limit);
// ISCU_ERR_LIMIT (naming the bytes) otherwise. *smem: the dynamic bytes.
int CheckFp32CztSmem(iscu_ctx* ctx, int M, int P, size_t* smem);
int LaunchPsfPipelineFp32(iscu_ctx* ctx, const SetParams* dSets, const PsfItem* dItems, double3* dTab, float2* dA,
                          float2* dAt, uint32_t nSets, uint32_t nPsf, int M, int P, int normalize, float* out);

} // namespace iscu
