// Fused tile kernels: the backward pass at complex64 precision.
#include "fused_impl.cuh"

namespace mqb {
template cudaError_t launch_fused_bwd2<float>(const Bwd2Args<float> &, int, cudaStream_t);
}  // namespace mqb
