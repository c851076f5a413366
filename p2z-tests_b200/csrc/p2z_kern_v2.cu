// p2z_kern_v2.cu -- instantiates the hot-path kernels for one update kind
// (UPDK_V2); split per kind so the instances compile in parallel.
#include "p2z_kernels.cuh"

namespace p2z {
cudaError_t launch_v2(const LaunchSpec &s, cudaStream_t st) { return Dispatch<UPDK_V2, true>::launch(s, st); }
int occupancy_v2(const LaunchSpec &s) { return Dispatch<UPDK_V2, true>::occupancy(s); }
}  // namespace p2z
