// p2z_kern_v2_ref.cu -- instantiates the hot-path kernels of the reference's
// own FP32 evaluation (UPDK_V2_REF, selected by P2Z_FLAG_REFERENCE_ROUNDING).
// This translation unit is compiled with --fmad=false: like the reference
// built with -ffp-contract=off, every product and sum is rounded separately.
#include "p2z_kernels.cuh"

namespace p2z {
cudaError_t launch_v2_ref(const LaunchSpec &s, cudaStream_t st) { return Dispatch<UPDK_V2_REF, false>::launch(s, st); }
int occupancy_v2_ref(const LaunchSpec &s) { return Dispatch<UPDK_V2_REF, false>::occupancy(s); }
}  // namespace p2z
