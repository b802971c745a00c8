// Stand-in for the reference's cuQuantum double policy header, TEST INFRASTRUCTURE ONLY (oracle/Makefile,
// target _ref/libmqref_gpu.so).  The reference's thrust GPU sources instantiate their policy base
// for the cuStateVec-backed policy too; cuStateVec is not in this image, so the name is declared
// here as one more thrust policy and is never used by the harness.
#ifndef MQREF_GPU_SHIM_CUQUANTUM_DOUBLE_POLICY
#define MQREF_GPU_SHIM_CUQUANTUM_DOUBLE_POLICY
#include "simulator/vector/detail/gpu_vector_policy.cuh"
namespace mindquantum::sim::vector::detail {
struct CuQuantumVectorPolicyDouble : public GPUVectorPolicyBase<CuQuantumVectorPolicyDouble, double> {};
}  // namespace mindquantum::sim::vector::detail
#endif
