// rgc_fht_drift_wide.cu -- the fused FHT-path RGC with drift for tap boxes 22 .. 32 pixels wide
// (radius >= 10 magnified pixels), in a unit of its own so that the two halves of the
// instantiations compile in parallel.  See rgc_fht_drift.cu.
#include "esrrf_internal.h"
#include "fht_fused.cuh"

namespace esrrf {

cudaError_t fht_rgc_fused_drift_wide(int S, const fused::FusedParams& fp, const fused::DriftParams& dp,
                                     const FhtRgcArgs& a, cudaStream_t stream) {
    return fused::launch_fused_in<true, 22, 32>(S, fp.r0, fp.sens, fp, dp, a, stream);
}

}  // namespace esrrf
