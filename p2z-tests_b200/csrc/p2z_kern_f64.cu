// p2z_kern_f64.cu -- instantiates the hot-path kernels for one update kind
// (UPDK_F64); split per kind so the instances compile in parallel.
#include "p2z_kernels.cuh"

namespace p2z {
cudaError_t launch_f64(const LaunchSpec &s, cudaStream_t st) { return Dispatch<UPDK_F64, false>::launch(s, st); }
int occupancy_f64(const LaunchSpec &s) { return Dispatch<UPDK_F64, false>::occupancy(s); }
}  // namespace p2z
