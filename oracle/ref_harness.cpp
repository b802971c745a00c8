// Driver of the reference's own CPU state-vector simulator, TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile (target _ref/libmqref.so) together with the reference's C++ sources,
// compiled in place from the reference tree: VectorState<CPUVectorPolicyAvxDouble> and its CPU
// policy (ccsrc/include/simulator/vector/vector_state.h/.tpp, ccsrc/lib/simulator/vector/detail/
// cpu_common, cpu_avx_double), the gates and parameter resolvers it uses.  The circuits and
// Hamiltonians are built by ref_harness_common.h with the reference's classes:
//
//   mqref_apply:  VectorState::ApplyCircuit + GetQS (vector_state.tpp:949-960);
//   mqref_sample: SamplingMeasurementEndingWithoutNoise / Sampling (vector_state.tpp:1308-1373);
//   mqref_grad:  VectorState::GetExpectationWithGradMultiMulti (the adjoint gradient,
//                ccsrc/include/simulator/vector/gradient.h:100-197).
//
// Only tests/ and bench.py's CPU legs load it, to pin the oracle to the reference itself and to
// time the reference on the host; the product never does.
#include "ref_harness_common.h"
#include "simulator/vector/detail/cpu_vector_avx_double_policy.h"
#include "simulator/vector/detail/cpu_vector_avx_float_policy.h"

namespace {
using sim_d = mindquantum::sim::vector::detail::VectorState<mindquantum::sim::vector::detail::CPUVectorPolicyAvxDouble>;
using sim_f = mindquantum::sim::vector::detail::VectorState<mindquantum::sim::vector::detail::CPUVectorPolicyAvxFloat>;
}  // namespace

extern "C" {

int mqref_apply(MQREF_APPLY_ARGS) { return mqref::apply_impl<sim_d>(MQREF_APPLY_PASS); }

// complex128 (CPUVectorPolicyAvxDouble)
int mqref_sample(MQREF_SAMPLE_ARGS) { return mqref::sample_impl<sim_d>(MQREF_SAMPLE_PASS); }

// complex128 (CPUVectorPolicyAvxDouble)
int mqref_grad(MQREF_GRAD_ARGS) { return mqref::grad_impl<sim_d, double>(MQREF_GRAD_PASS); }

// complex64 (CPUVectorPolicyAvxFloat)
int mqref_grad_c64(MQREF_GRAD_ARGS) { return mqref::grad_impl<sim_f, float>(MQREF_GRAD_PASS); }

}  // extern "C"
