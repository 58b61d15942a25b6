// Tensor-core (tcgen05) TF32 split-precision chirp-Z: filled in by the tensor-core build step.
#include "psf_common.cuh"

namespace iscu {

int LaunchCztTf32x3(iscu_ctx* ctx, const SetParams* sets, const double3* tables, const float2* A, const float2* At,
                    const PsfItem* items, uint32_t nPsf, int M, int P, int normalize, float* out)
{
   (void)ctx, (void)sets, (void)tables, (void)A, (void)At, (void)items, (void)nPsf, (void)M, (void)P, (void)normalize,
      (void)out;
   return Fail(ISCU_ERR_ARG, "the TF32 split chirp-Z is not in this build");
}

} // namespace iscu
