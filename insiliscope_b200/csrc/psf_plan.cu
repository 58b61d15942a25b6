// A PSF library plan: the per-set work of ComputeZernikePsfPlanes (ZernikePsf.cpp:166-231 -- the aperture, OPD,
// Zernike and mask tables; the chirp-Z's DFT matrices) done once and kept resident, so a run is the per-PSF work
// only: pupil phasors at each PSF's defocus, the two chirp-Z products, |E|^2, normalization. The reference memoizes
// whole kernel stacks (ComputePsfKernelCache, PsfGeneratorBridge.h:317-364); a library of thousands of PSFs over a
// few request sets is this plan's shape.

#include "iscu_internal.h"
#include "psf_common.cuh"

#include <algorithm>
#include <vector>

struct iscu_psf_plan
{
   iscu_ctx* ctx = nullptr;
   int M = 0, P = 0, method = 0;
   uint32_t nSets = 0;
   iscu::DevBuf sets, tab, A, At, ahat, items, setOf, defocus, out, err;
};

namespace iscu {
namespace {

// items[i] = (ti - ti0, set) with the rounding of the host path ((ti0 - focalShift) + defocus * 1e-9, then - ti0).
__global__ void PlanItemsKernel(const SetParams* __restrict__ sets, const uint32_t* __restrict__ setOf,
                                const double* __restrict__ defocusNm, uint32_t n, uint32_t nSets,
                                PsfItem* __restrict__ items, int* __restrict__ err)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n)
      return;
   uint32_t s = setOf[i];
   if (s >= nSets)
   {
      atomicExch(err, 2);   // a set index out of range: reported by the run
      s = 0;
   }
   const SetParams& sp = sets[s];
   const double dM = __dmul_rn(defocusNm[i], 1E-9);
   const double ti = __dadd_rn(__dsub_rn(sp.ti0, sp.focalShift), dM);
   items[i].dtiM = __dsub_rn(ti, sp.ti0);
   items[i].set = static_cast<int>(s);
   items[i].pad = 0;
}

int RunDev(iscu_psf_plan* p, const uint32_t* setOf, const double* defocusNm, uint32_t n, int normalize, float* out,
           bool clearError = true)
{
   iscu_ctx* ctx = p->ctx;
   if (n == 0)
      return ISCU_OK;
   ISCU_CK(p->items.Reserve(static_cast<size_t>(n) * sizeof(PsfItem)));
   if (clearError)
      ISCU_CK(cudaMemsetAsync(p->err.p, 0, sizeof(int), ctx->stream));
   PlanItemsKernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(p->sets.as<SetParams>(), setOf, defocusNm, n, p->nSets,
                                                             p->items.as<PsfItem>(), p->err.as<int>());
   ISCU_CK_LAUNCH(ctx, "PlanItemsKernel");
   if (p->method == ISCU_CZT_F16X3)
      return LaunchCztF16x3Core(ctx, p->sets.as<SetParams>(), p->ahat.as<unsigned char>(), static_cast<int>(p->nSets),
                                p->items.as<PsfItem>(), n, p->M, p->P, normalize, out, p->err.as<int>());
   if (p->method == ISCU_CZT_TF32X3)
      return LaunchCztTf32x3Core(ctx, p->sets.as<SetParams>(), p->ahat.as<float>(), static_cast<int>(p->nSets),
                                 p->items.as<PsfItem>(), n, p->M, p->P, normalize, out, p->err.as<int>());
   return LaunchCztFp32(ctx, p->sets.as<SetParams>(), p->tab.as<double3>(), p->A.as<float2>(), p->At.as<float2>(),
                        p->items.as<PsfItem>(), n, p->M, p->P, normalize, out);
}

int Check(iscu_psf_plan* p)
{
   int err = 0;
   ISCU_CK(cudaMemcpyAsync(&err, p->err.p, sizeof(int), cudaMemcpyDeviceToHost, p->ctx->stream));
   ISCU_CK(cudaStreamSynchronize(p->ctx->stream));
   if (err == 1)
      return Fail(ISCU_ERR_TIMEOUT, "psf plan: a tensor-core completion wait ran out");
   if (err == 2)
      return Fail(ISCU_ERR_ARG, "psf plan: a set index out of range");
   return ISCU_OK;
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_psf_plan_create(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t n_sets, int32_t size, int32_t method,
                         iscu_psf_plan** out)
{
   if (!ctx || !sets || !out || n_sets == 0)
      return Fail(ISCU_ERR_ARG, "null argument or no sets");
   *out = nullptr;
   if (method != ISCU_CZT_FP32 && method != ISCU_CZT_TF32X3 && method != ISCU_CZT_F16X3)
      return Fail(ISCU_ERR_ARG, "unknown chirp-Z method");
   if (size < 0 || size > 1024)
      return Fail(ISCU_ERR_ARG, "plane size out of range (0..1024)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   std::unique_ptr<iscu_psf_plan> p(new iscu_psf_plan());
   p->ctx = ctx;
   p->method = method;
   p->nSets = n_sets;
   std::vector<SetParams> hs(n_sets);
   int rc = PrepareSetParams(sets, n_sets, size, n_sets, hs.data(), &p->M, &p->P);
   if (rc != ISCU_OK)
      return rc;
   if ((method == ISCU_CZT_TF32X3 && !Tf32x3Supports(p->M, p->P)) ||
       (method == ISCU_CZT_F16X3 && !F16x3Supports(p->M, p->P)))
      return Fail(ISCU_ERR_ARG, std::string(method == ISCU_CZT_F16X3 ? "f16x3" : "tf32x3") +
                                   " chirp-Z: needs pupil samples M <= 128 (a multiple of 16) and planes of at most "
                                   "64 x 64");
   const size_t M = p->M, P = p->P;
   ISCU_CK(p->sets.Reserve(n_sets * sizeof(SetParams)));
   ISCU_CK(p->tab.Reserve(n_sets * M * M * sizeof(double3)));
   ISCU_CK(p->A.Reserve(n_sets * P * M * sizeof(float2)));
   ISCU_CK(p->At.Reserve(n_sets * P * M * sizeof(float2)));
   ISCU_CK(p->err.Reserve(sizeof(int)));
   ISCU_CK(cudaMemcpyAsync(p->sets.p, hs.data(), n_sets * sizeof(SetParams), cudaMemcpyHostToDevice, ctx->stream));
   rc = LaunchPsfTables(ctx, p->sets.as<SetParams>(), n_sets, p->M, p->P, p->tab.as<double3>(), p->A.as<float2>(),
                        p->At.as<float2>());
   if (rc != ISCU_OK)
      return rc;
   if (method != ISCU_CZT_FP32 &&
       (rc = BuildAhat(ctx, p->A.as<float2>(), p->sets.as<SetParams>(), p->tab.as<double3>(),
                       static_cast<int>(n_sets), p->M, p->P, method, p->ahat)) != ISCU_OK)
      return rc;
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   *out = p.release();
   return ISCU_OK;
}

void iscu_psf_plan_destroy(iscu_psf_plan* plan)
{
   if (!plan)
      return;
   cudaStreamSynchronize(plan->ctx->stream);
   delete plan;
}

int iscu_psf_plan_info(iscu_psf_plan* plan, int32_t* size, int32_t* pupil_samples)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   if (size)
      *size = plan->P;
   if (pupil_samples)
      *pupil_samples = plan->M;
   return ISCU_OK;
}

int iscu_psf_plan_run_dev(iscu_psf_plan* plan, const uint32_t* set_of_psf_dev, const double* defocus_nm_dev,
                          uint32_t n_psf, int32_t normalize, float* out_dev)
{
   if (!plan || (n_psf && (!set_of_psf_dev || !defocus_nm_dev || !out_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   return RunDev(plan, set_of_psf_dev, defocus_nm_dev, n_psf, normalize, out_dev);
}

int iscu_psf_plan_check(iscu_psf_plan* plan)
{
   if (!plan)
      return Fail(ISCU_ERR_ARG, "null plan");
   std::lock_guard<std::recursive_mutex> lock(plan->ctx->mu);
   ClearError();
   return Check(plan);
}

int iscu_psf_plan_run(iscu_psf_plan* plan, const uint32_t* set_of_psf, const double* defocus_nm, uint32_t n_psf,
                      int32_t normalize, float* out)
{
   if (!plan || (n_psf && (!set_of_psf || !defocus_nm || !out)))
      return Fail(ISCU_ERR_ARG, "null argument");
   iscu_ctx* ctx = plan->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (n_psf == 0)
      return ISCU_OK;
   const size_t planeFloats = static_cast<size_t>(plan->P) * plan->P, planeBytes = planeFloats * sizeof(float);
   ISCU_CK(plan->setOf.Reserve(n_psf * sizeof(uint32_t)));
   ISCU_CK(plan->defocus.Reserve(n_psf * sizeof(double)));
   ISCU_CK(plan->out.Reserve(n_psf * planeBytes));
   ISCU_CK(cudaMemcpyAsync(plan->setOf.p, set_of_psf, n_psf * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(plan->defocus.p, defocus_nm, n_psf * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
   // A large library runs in kRunChunks launches, each chunk's planes copied back on the download stream while the
   // next chunk computes: the copy (PCIe) is the longer part, and a PSF's planes do not depend on the others'.
   constexpr uint32_t kRunChunks = 4, kChunkMin = 2048;
   const uint32_t chunks = n_psf >= kChunkMin ? kRunChunks : 1u;
   const uint32_t per = (n_psf + chunks - 1) / chunks;
   if (!ctx->download)
      ISCU_CK(cudaStreamCreateWithFlags(&ctx->download, cudaStreamNonBlocking));
   struct Events
   {
      cudaEvent_t e[kRunChunks] = {};
      ~Events()
      {
         for (cudaEvent_t x : e)
            if (x)
               cudaEventDestroy(x);
      }
   } ev;
   ISCU_CK(cudaMemsetAsync(plan->err.p, 0, sizeof(int), ctx->stream));
   for (uint32_t c = 0, c0 = 0; c0 < n_psf; ++c, c0 += per)
   {
      const uint32_t nc = std::min(per, n_psf - c0);
      const int rc = RunDev(plan, plan->setOf.as<uint32_t>() + c0, plan->defocus.as<double>() + c0, nc, normalize,
                            plan->out.as<float>() + c0 * planeFloats, false);
      if (rc != ISCU_OK)
      {
         cudaStreamSynchronize(ctx->download);
         return rc;
      }
      ISCU_CK(cudaEventCreateWithFlags(&ev.e[c], cudaEventDisableTiming));
      ISCU_CK(cudaEventRecord(ev.e[c], ctx->stream));
      ISCU_CK(cudaStreamWaitEvent(ctx->download, ev.e[c], 0));
      ISCU_CK(cudaMemcpyAsync(out + c0 * planeFloats, plan->out.as<float>() + c0 * planeFloats, nc * planeBytes,
                              cudaMemcpyDeviceToHost, ctx->download));
   }
   ISCU_CK(cudaStreamSynchronize(ctx->download));
   return Check(plan);
}

} // extern "C"
