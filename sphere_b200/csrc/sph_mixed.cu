// sph_mixed.cu -- FP32-mixed step (SPH_PREC_MIXED).
#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {

int launch_step_mixed(const StepArgs &, const StepConfig &, cudaStream_t, uint64_t *, Prof *)
{
    return SPH_ERR_UNSUPPORTED;
}

}  // namespace sph
