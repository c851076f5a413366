// p2z_kern_3x3_comp.cu -- instantiates the hot-path kernels for one update kind
// (UPDK_3X3_COMP); split per kind so the instances compile in parallel.
#include "p2z_kernels.cuh"

namespace p2z {
cudaError_t launch_3x3_comp(const LaunchSpec &s, cudaStream_t st) { return Dispatch<UPDK_3X3_COMP, true>::launch(s, st); }
int occupancy_3x3_comp(const LaunchSpec &s) { return Dispatch<UPDK_3X3_COMP, true>::occupancy(s); }
}  // namespace p2z
