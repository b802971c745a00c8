// Fused tile kernels: the forward pass at complex128 precision.
#include "fused_impl.cuh"

namespace mqb {
template cudaError_t launch_fused_fwd2<double>(const Fwd2Args<double> &, int, cudaStream_t);
}  // namespace mqb
