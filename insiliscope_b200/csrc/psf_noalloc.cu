// A PSF library that allocates no device memory (iscu_psf_library_noalloc_dev).
//
// Who needs it: callers that cannot call cudaMalloc -- a plug-in whose process hands all device memory to another
// framework's caching allocator or to a fixed budget shared with other plug-ins, or a live loop that cannot take the
// device-wide synchronization a cudaFree brings. The allocating entry point (iscu_psf_library_dev) makes its
// temporaries with cudaMalloc per call; this one puts them in g_psfScratch below, a statically sized device array
// that exists on every GPU that loads libiscu.so, from load to exit.
//
// The host code never dereferences g_psfScratch: in host code that name is only a stand-in for the device symbol,
// not a device address. The address is looked up once per device (ScratchOn, cudaGetSymbolAddress, with that device
// current) and passed to the kernels. Every call shares the array and it keeps the last call's contents; nothing in
// it has to start at zero here (every region is written in full before it is read), and calls whose work overlaps on
// the GPU race on it.

#include "iscu_internal.h"
#include "psf_common.cuh"

#include <mutex>

namespace iscu {

namespace {

static __device__ __align__(256) unsigned char g_psfScratch[ISCU_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratchMu;
void* g_scratchAddr[kMaxDevices] = {};

// The device address of g_psfScratch on `device` (current): looked up on the first call, then remembered.
int ScratchOn(int device, unsigned char** out)
{
   if (device < 0 || device >= kMaxDevices)
      return Fail(ISCU_ERR_LIMIT, "psf library (no allocation): device index beyond 63");
   std::lock_guard<std::mutex> lock(g_scratchMu);
   if (!g_scratchAddr[device])
   {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_psfScratch);
      if (e != cudaSuccess)
         return CudaFail(e, "cudaGetSymbolAddress(g_psfScratch)");
      g_scratchAddr[device] = p;
   }
   *out = static_cast<unsigned char*>(g_scratchAddr[device]);
   return ISCU_OK;
}

size_t Align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

// items[i] = (ti - ti0, set) from the caller's set index and defocus (nm), with the allocating path's rounding
// ((ti0 - focalShift) + defocus * 1e-9, then - ti0; BuildPsfLibrary) spelled out so no contraction changes it.
__global__ void ItemsKernel(const SetParams* __restrict__ sets, const uint32_t* __restrict__ setOf,
                            const double* __restrict__ defocusNm, uint32_t n, PsfItem* __restrict__ items)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n)
      return;
   const uint32_t s = setOf[i];
   const SetParams& sp = sets[s];
   const double dM = __dmul_rn(defocusNm[i], 1E-9);
   const double ti = __dadd_rn(__dsub_rn(sp.ti0, sp.focalShift), dM);
   items[i].dtiM = __dsub_rn(ti, sp.ti0);
   items[i].set = static_cast<int>(s);
   items[i].pad = 0;
}

// Restores the caller's current device on scope exit.
struct DeviceScope
{
   int prev = -1;
   explicit DeviceScope(int dev)
   {
      if (cudaGetDevice(&prev) == cudaSuccess && prev != dev)
         cudaSetDevice(dev);
      else
         prev = -1;
   }
   ~DeviceScope()
   {
      if (prev >= 0)
         cudaSetDevice(prev);
   }
};

} // namespace

} // namespace iscu

using namespace iscu;

extern "C" int iscu_psf_library_noalloc_dev(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t n_sets,
                                            const uint32_t* set_of_psf, const double* defocus_nm, uint32_t n_psf,
                                            int32_t size, int32_t normalize, float* out_dev)
{
   if (!ctx || !sets || (n_psf && (!set_of_psf || !defocus_nm || !out_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (n_psf == 0)
      return ISCU_OK;
   if (n_psf > ISCU_NOALLOC_MAX_PSF)
      return Fail(ISCU_ERR_LIMIT, "psf library (no allocation): at most " + std::to_string(ISCU_NOALLOC_MAX_PSF) +
                                      " PSFs per call, asked for " + std::to_string(n_psf));
   if (size < 0 || size > 129)
      return Fail(ISCU_ERR_LIMIT, "psf library (no allocation): plane size at most 129");
   for (uint32_t i = 0; i < n_psf; ++i)
      if (set_of_psf[i] >= n_sets)
         return Fail(ISCU_ERR_ARG, "psf library: set index out of range");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   DeviceScope scope(ctx->device);
   SetParams hs[ISCU_NOALLOC_MAX_SETS];
   int M = 0, P = 0;
   int rc = PrepareSetParams(sets, n_sets, size, ISCU_NOALLOC_MAX_SETS, hs, &M, &P);
   if (rc != ISCU_OK)
      return rc;
   if (M > 128 || P > 129)
      return Fail(ISCU_ERR_LIMIT, "psf library (no allocation): pupil samples at most 128 and plane size at most "
                                  "129, asked for M = " + std::to_string(M) + ", P = " + std::to_string(P));
   // The FP32 chirp-Z kernel holds the pupil (M x M) and the row pass (P x M) complex in one CTA's shared memory.
   size_t smem = 0;
   rc = CheckFp32CztSmem(ctx, M, P, &smem);
   if (rc != ISCU_OK)
      return rc;
   // The layout inside the scratch array.
   const size_t oSets = 0;
   const size_t oSetOf = oSets + Align256(n_sets * sizeof(SetParams));
   const size_t oDefocus = oSetOf + Align256(n_psf * sizeof(uint32_t));
   const size_t oItems = oDefocus + Align256(n_psf * sizeof(double));
   const size_t oTab = oItems + Align256(n_psf * sizeof(PsfItem));
   const size_t oA = oTab + Align256(static_cast<size_t>(n_sets) * M * M * sizeof(double3));
   const size_t oAt = oA + Align256(static_cast<size_t>(n_sets) * P * M * sizeof(float2));
   const size_t end = oAt + Align256(static_cast<size_t>(n_sets) * P * M * sizeof(float2));
   if (end > ISCU_NOALLOC_SCRATCH_BYTES)
      return Fail(ISCU_ERR_LIMIT, "psf library (no allocation): needs " + std::to_string(end) +
                                      " bytes of scratch, the static array holds " +
                                      std::to_string(ISCU_NOALLOC_SCRATCH_BYTES));
   unsigned char* base = nullptr;
   rc = ScratchOn(ctx->device, &base);
   if (rc != ISCU_OK)
      return rc;
   SetParams* dSets = reinterpret_cast<SetParams*>(base + oSets);
   uint32_t* dSetOf = reinterpret_cast<uint32_t*>(base + oSetOf);
   double* dDefocus = reinterpret_cast<double*>(base + oDefocus);
   PsfItem* dItems = reinterpret_cast<PsfItem*>(base + oItems);
   ISCU_CK(cudaMemcpyAsync(dSets, hs, n_sets * sizeof(SetParams), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(dSetOf, set_of_psf, n_psf * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(dDefocus, defocus_nm, n_psf * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
   ItemsKernel<<<(n_psf + 127) / 128, 128, 0, ctx->stream>>>(dSets, dSetOf, dDefocus, n_psf, dItems);
   ISCU_CK_LAUNCH(ctx, "ItemsKernel");
   rc = LaunchPsfPipelineFp32(ctx, dSets, dItems, reinterpret_cast<double3*>(base + oTab),
                              reinterpret_cast<float2*>(base + oA), reinterpret_cast<float2*>(base + oAt), n_sets,
                              n_psf, M, P, normalize, out_dev);
   if (rc != ISCU_OK)
      return rc;
   // The host copies above read the caller's (and this frame's) memory; the call returns with the planes written.
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}
