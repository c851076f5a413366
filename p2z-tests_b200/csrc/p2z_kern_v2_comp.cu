// p2z_kern_v2_comp.cu -- instantiates the hot-path kernels for one update kind
// (UPDK_V2_COMP); split per kind so the instances compile in parallel.
#include "p2z_kernels.cuh"

namespace p2z {
cudaError_t launch_v2_comp(const LaunchSpec &s, cudaStream_t st) { return Dispatch<UPDK_V2_COMP, true>::launch(s, st); }
int occupancy_v2_comp(const LaunchSpec &s) { return Dispatch<UPDK_V2_COMP, true>::occupancy(s); }
}  // namespace p2z
