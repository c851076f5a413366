// p2z_kern_3x3_f64.cu -- instantiates the hot-path kernels for one update kind
// (UPDK_3X3_F64); split per kind so the instances compile in parallel.
#include "p2z_kernels.cuh"

namespace p2z {
cudaError_t launch_3x3_f64(const LaunchSpec &s, cudaStream_t st) { return Dispatch<UPDK_3X3_F64, true>::launch(s, st); }
int occupancy_3x3_f64(const LaunchSpec &s) { return Dispatch<UPDK_3X3_F64, true>::occupancy(s); }
}  // namespace p2z
