// Fused tile kernels: the backward pass at complex128 precision.
#include "fused_impl.cuh"

namespace mqb {
template cudaError_t launch_fused_bwd2<double>(const Bwd2Args<double> &, int, cudaStream_t);
}  // namespace mqb
