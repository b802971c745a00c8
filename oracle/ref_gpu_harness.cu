// Driver of the reference's own thrust GPU state-vector simulator (`mqvector_gpu`), TEST
// INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile (target _ref/libmqref_gpu.so) with nvcc for sm_100a, together with the
// reference's GPU policy sources compiled in place from the reference tree
// (ccsrc/lib/simulator/vector/detail/gpu/gpu_vector_core_*.cu, ccsrc/include/simulator/vector/
// detail/gpu_vector_policy.cuh) and VectorState (vector_state.h/.tpp).  The reference's sources
// also instantiate their policy base for the cuStateVec policy; cuStateVec is not in this image,
// so refgpu_shim/ declares that name as one more thrust policy (never called here).  The circuits
// and Hamiltonians are built by ref_harness_common.h:
//
//   mqref_gpu_apply:    VectorState<GPUVectorPolicyDouble>::ApplyCircuit + GetQS;
//   mqref_gpu_grad:     GetExpectationWithGradMultiMulti, complex128 (GPUVectorPolicyDouble);
//   mqref_gpu_grad_c64: the same in complex64 (GPUVectorPolicyFloat).
//
// It is the second, external GPU comparison point of the measurements (the reference's own GPU
// path on the same B200); the product never loads it.
#include "ref_harness_common.h"
#include "simulator/vector/detail/gpu_vector_double_policy.cuh"
#include "simulator/vector/detail/gpu_vector_float_policy.cuh"

namespace {
using sim_d = mindquantum::sim::vector::detail::VectorState<mindquantum::sim::vector::detail::GPUVectorPolicyDouble>;
using sim_f = mindquantum::sim::vector::detail::VectorState<mindquantum::sim::vector::detail::GPUVectorPolicyFloat>;
}  // namespace

extern "C" {

int mqref_gpu_apply(MQREF_APPLY_ARGS) { return mqref::apply_impl<sim_d>(MQREF_APPLY_PASS); }

int mqref_gpu_grad(MQREF_GRAD_ARGS) { return mqref::grad_impl<sim_d, double>(MQREF_GRAD_PASS); }

int mqref_gpu_grad_c64(MQREF_GRAD_ARGS) { return mqref::grad_impl<sim_f, float>(MQREF_GRAD_PASS); }

}  // extern "C"
