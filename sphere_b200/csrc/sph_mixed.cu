// sph_mixed.cu -- FP32-mixed step (SPH_PREC_MIXED).
//
// Same step as the FP64 form (sort, contact search with the exact FP64
// overlap test, so the contact lists are identical; walls; bonds; FP64 TY3
// integration) with the contact-law arithmetic in FP32
// (sph_mixed_laws.cuh).  Compiled with FMA contraction.
#include "sph_device.cuh"
#include "sph_internal.h"
#include "sph_step.cuh"

namespace sph {

static void interact_mixed(const StepArgs &A, cudaStream_t st, unsigned grid, bool fused, int lm,
                           int variant)
{
    launch_interact<true>(A, st, grid, fused, lm, variant);
}

static void contacts_mixed(const StepArgs &A, cudaStream_t st, unsigned grid, int lm, bool pdl)
{
    launch_contacts<true>(A, st, grid, lm, pdl);
}

int launch_step_mixed(const StepArgs &A, const StepConfig &cfg, cudaStream_t st,
                      uint64_t *launches, Prof *prof)
{
    if (!st && !launches) return SPH_OK;  // capability probe from sph_create
    return launch_step_with(A, cfg, st, launches, prof, interact_mixed, contacts_mixed);
}

}  // namespace sph
