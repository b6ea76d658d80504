// fused.cu -- the fused, batched form of the multislice step (register-resident FFT passes).
#include "engine.cuh"

namespace simk {

bool fused_supported(Context&, const GridGeom&) { return false; }

void scan_fused_batch(Context&, PotentialImpl&, const simk_probe&, const float2*, const double*, long long, int,
                      const DetectorPlan&, double* const*, double) {
    throw Error(SIMK_ERR_INVALID, "fused form not available for this grid");
}

}  // namespace simk
