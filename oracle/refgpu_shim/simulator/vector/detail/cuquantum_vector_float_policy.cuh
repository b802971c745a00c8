// Stand-in for the reference's cuQuantum float policy header, TEST INFRASTRUCTURE ONLY (oracle/Makefile,
// target _ref/libmqref_gpu.so).  The reference's thrust GPU sources instantiate their policy base
// for the cuStateVec-backed policy too; cuStateVec is not in this image, so the name is declared
// here as one more thrust policy and is never used by the harness.
#ifndef MQREF_GPU_SHIM_CUQUANTUM_FLOAT_POLICY
#define MQREF_GPU_SHIM_CUQUANTUM_FLOAT_POLICY
#include "simulator/vector/detail/gpu_vector_policy.cuh"
namespace mindquantum::sim::vector::detail {
struct CuQuantumVectorPolicyFloat : public GPUVectorPolicyBase<CuQuantumVectorPolicyFloat, float> {};
}  // namespace mindquantum::sim::vector::detail
#endif
