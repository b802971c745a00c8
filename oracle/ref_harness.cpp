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
//                ccsrc/include/simulator/vector/gradient.h:100-197);
//   mqref_dm_apply / mqref_dm_grad: the density-matrix simulator (DensityMatrixState, its CPU
//                policy under ccsrc/lib/simulator/densitymatrix/detail/cpu_common): rho after a
//                circuit with channels, and the expectation gradient with and without noise.
//
// Only tests/ and bench.py's CPU legs load it, to pin the oracle to the reference itself and to
// time the reference on the host; the product never does.
#include "ref_harness_common.h"
#include "simulator/densitymatrix/densitymatrix_state.h"
#include "simulator/densitymatrix/detail/cpu_densitymatrix_avx_double_policy.h"
#include "simulator/vector/detail/cpu_vector_avx_double_policy.h"
#include "simulator/vector/detail/cpu_vector_avx_float_policy.h"

namespace {
using sim_d = mindquantum::sim::vector::detail::VectorState<mindquantum::sim::vector::detail::CPUVectorPolicyAvxDouble>;
using sim_f = mindquantum::sim::vector::detail::VectorState<mindquantum::sim::vector::detail::CPUVectorPolicyAvxFloat>;
using dm_d = mindquantum::sim::densitymatrix::detail::DensityMatrixState<
    mindquantum::sim::densitymatrix::detail::CPUDensityMatrixPolicyAvxDouble>;
}  // namespace

extern "C" {

int mqref_apply(MQREF_APPLY_ARGS) { return mqref::apply_impl<sim_d>(MQREF_APPLY_PASS); }

// complex128 (CPUVectorPolicyAvxDouble)
int mqref_sample(MQREF_SAMPLE_ARGS) { return mqref::sample_impl<sim_d>(MQREF_SAMPLE_PASS); }

// complex128 (CPUVectorPolicyAvxDouble)
int mqref_grad(MQREF_GRAD_ARGS) { return mqref::grad_impl<sim_d, double>(MQREF_GRAD_PASS); }

// complex64 (CPUVectorPolicyAvxFloat)
int mqref_grad_c64(MQREF_GRAD_ARGS) { return mqref::grad_impl<sim_f, float>(MQREF_GRAD_PASS); }

// the parameter-shift gradient, complex128
int mqref_grad_pshift(MQREF_GRAD_ARGS) { return mqref::pshift_impl<sim_d, double>(MQREF_GRAD_PASS); }

// <H> and its gradient for a Hamiltonian given as a sparse matrix (mindquantum/core/operators/
// hamiltonian.py get_cpp_obj: the scipy CSR arrays as a CsrHdMatrix, Hamiltonian(csr, n); the
// simulator then takes ExpectationOfCsr / Csr_Dot_Vec), complex128, every parameter an encoder
// input: the CSR rows indptr[2^n + 1], indices[nnz], data[nnz] complex128 (re, im).
int mqref_grad_csr(int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl,
                   const int *param, const double *coeff, const double *cst, const double *ch, int64_t nnz,
                   const int64_t *indptr, const int64_t *indices, const double *data, int n_params, int n_samples,
                   const double *params, double *out) {
    try {
        const auto names = mqref::param_names(n_params);
        const auto c = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        const auto h = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, true, ch);
        if (int(c.size()) != n_gates || int(h.size()) != n_gates) return -1;
        const size_t d = size_t(1) << n;
        // the matrix owns malloc'd copies (CsrHdMatrix::FreeMemory frees them)
        auto *ip = static_cast<mindquantum::Index *>(malloc(sizeof(mindquantum::Index) * (d + 1)));
        auto *ix = static_cast<mindquantum::Index *>(malloc(sizeof(mindquantum::Index) * std::max<int64_t>(1, nnz)));
        auto *dt = static_cast<std::complex<double> *>(malloc(sizeof(std::complex<double>) * std::max<int64_t>(1, nnz)));
        if (!ip || !ix || !dt) {
            free(ip);
            free(ix);
            free(dt);
            return -3;
        }
        for (size_t i = 0; i <= d; ++i) ip[i] = mindquantum::Index(indptr[i]);
        for (int64_t k = 0; k < nnz; ++k) {
            ix[k] = mindquantum::Index(indices[k]);
            dt[k] = {data[2 * k], data[2 * k + 1]};
        }
        auto csr = std::make_shared<mindquantum::sparse::CsrHdMatrix<double>>(d, mindquantum::Index(nnz), ip, ix, dt);
        std::vector<std::shared_ptr<mindquantum::Hamiltonian<double>>> hams{
            std::make_shared<mindquantum::Hamiltonian<double>>(csr, static_cast<mindquantum::Index>(n))};
        std::vector<std::vector<double>> enc(n_samples, std::vector<double>(n_params));
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i < n_params; ++i) enc[s][i] = params[s * n_params + i];
        sim_d sim{static_cast<mindquantum::Index>(n)};
        const auto res = sim.GetExpectationWithGradMultiMulti(hams, c, h, enc, {}, names, {}, 1, 1);
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i <= n_params; ++i) {
                out[2 * (s * (n_params + 1) + i)] = res[s][0][i].real();
                out[2 * (s * (n_params + 1) + i) + 1] = res[s][0][i].imag();
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

// The QRAM gradient (QramExpectationWithGrad, vector_state.tpp:1010-1018; gradient.h
// QramHermitianAdjointGradient), complex128: one ansatz (every parameter an ansatz input, values
// params[n_params]) applied to n_samples initial states init[n_samples][2^n] complex128 (re, im).
// out: [n_samples][1 + n_params] complex128 (re, im).
int mqref_grad_qram(int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl,
                    const int *param, const double *coeff, const double *cst, const double *ch, int n_terms,
                    const int *term_len, const int *term_q, const char *term_p, const double *term_c, int n_params,
                    int n_samples, const double *params, const double *init, double *out) {
    try {
        const auto names = mqref::param_names(n_params);
        const auto c = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        const auto h = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, true, ch);
        if (int(c.size()) != n_gates || int(h.size()) != n_gates) return -1;
        std::vector<std::shared_ptr<mindquantum::Hamiltonian<double>>> hams{
            mqref::hamiltonian<double>(n_terms, term_len, term_q, term_p, term_c)};
        const size_t d = size_t(1) << n;
        std::vector<std::vector<std::complex<double>>> states(n_samples, std::vector<std::complex<double>>(d));
        for (int s = 0; s < n_samples; ++s)
            for (size_t i = 0; i < d; ++i) states[s][i] = {init[2 * (s * d + i)], init[2 * (s * d + i) + 1]};
        const std::vector<double> ans(params, params + n_params);
        sim_d sim{static_cast<mindquantum::Index>(n)};
        const auto res = sim.QramExpectationWithGrad(hams, c, h, states, ans, names, 1, 1);
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i <= n_params; ++i) {
                out[2 * (s * (n_params + 1) + i)] = res[s][0][i].real();
                out[2 * (s * (n_params + 1) + i) + 1] = res[s][0][i].imag();
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

// The non-Hermitian gradient <phi| U_l^dag H U_r(p) |psi> of MQSim.get_expectation_with_grad with
// circ_left and simulator_left (GetExpectationNonHermitianWithGradMultiMulti,
// vector_state.tpp:998-1008; gradient.h NonHermitianAdjointGradient), complex128: the right
// circuit is table r_*, the left one table l_* (both with channel-free gates, the left one's
// parameters fixed), psi and phi given as 2^n complex128 (re, im) amplitudes, every parameter of
// the right circuit an encoder input.  out: [n_samples][1 + n_params] complex128 (re, im).
int mqref_grad_nonherm(int n, int r_gates, const int *r_kind, const int *r_obj0, const int *r_obj1, const int *r_ctrl,
                       const int *r_param, const double *r_coeff, const double *r_cst, const double *r_ch, int l_gates,
                       const int *l_kind, const int *l_obj0, const int *l_obj1, const int *l_ctrl, const int *l_param,
                       const double *l_coeff, const double *l_cst, const double *l_ch, const double *psi,
                       const double *phi, int n_terms, const int *term_len, const int *term_q, const char *term_p,
                       const double *term_c, int n_params, int n_samples, const double *params, double *out) {
    try {
        const auto names = mqref::param_names(n_params);
        const std::vector<std::string> none;
        using mqref::build;
        const auto rc = build(r_gates, r_kind, r_obj0, r_obj1, r_ctrl, r_param, r_coeff, r_cst, names, false, r_ch);
        const auto rh = build(r_gates, r_kind, r_obj0, r_obj1, r_ctrl, r_param, r_coeff, r_cst, names, true, r_ch);
        const auto lc = build(l_gates, l_kind, l_obj0, l_obj1, l_ctrl, l_param, l_coeff, l_cst, none, false, l_ch);
        const auto lh = build(l_gates, l_kind, l_obj0, l_obj1, l_ctrl, l_param, l_coeff, l_cst, none, true, l_ch);
        if (int(rc.size()) != r_gates || int(lc.size()) != l_gates) return -1;
        std::vector<std::shared_ptr<mindquantum::Hamiltonian<double>>> hams{
            mqref::hamiltonian<double>(n_terms, term_len, term_q, term_p, term_c)};
        const size_t d = size_t(1) << n;
        std::vector<std::complex<double>> vpsi(d), vphi(d);
        for (size_t i = 0; i < d; ++i) {
            vpsi[i] = {psi[2 * i], psi[2 * i + 1]};
            vphi[i] = {phi[2 * i], phi[2 * i + 1]};
        }
        sim_d right{static_cast<mindquantum::Index>(n)};
        sim_d left{static_cast<mindquantum::Index>(n)};
        right.SetQS(vpsi);
        left.SetQS(vphi);
        std::vector<std::vector<double>> enc(n_samples, std::vector<double>(n_params));
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i < n_params; ++i) enc[s][i] = params[s * n_params + i];
        const auto res =
            right.GetExpectationNonHermitianWithGradMultiMulti(hams, hams, lc, lh, rc, rh, enc, {}, names, {}, left, 1, 1);
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i <= n_params; ++i) {
                out[2 * (s * (n_params + 1) + i)] = res[s][0][i].real();
                out[2 * (s * (n_params + 1) + i) + 1] = res[s][0][i].imag();
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

// The reference's density-matrix simulator (DensityMatrixState<CPUDensityMatrixPolicyAvxDouble>,
// ccsrc/include/simulator/densitymatrix/densitymatrix_state.tpp), complex128: the circuit (gates and
// channels, table as in mqref_sample, measurements not allowed) applied to |0><0|; out: rho as
// 2^n x 2^n complex128 (re, im), row-major.
int mqref_dm_apply(int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl,
                   const int *param, const double *coeff, const double *cst, const double *ch, int n_params,
                   const double *params, double *out) {
    try {
        const auto names = mqref::param_names(n_params);
        const mqref::circuit_t c = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        if (int(c.size()) != n_gates) return -1;
        parameter::ParameterResolver pr;
        for (int i = 0; i < n_params; ++i) pr.SetItem(names[i], params[i]);
        dm_d sim{static_cast<mindquantum::Index>(n)};
        sim.ApplyCircuit(c, pr);
        const auto rho = sim.GetQS();
        const size_t d = size_t(1) << n;
        for (size_t i = 0; i < d; ++i)
            for (size_t j = 0; j < d; ++j) {
                out[2 * (i * d + j)] = rho[i][j].real();
                out[2 * (i * d + j) + 1] = rho[i][j].imag();
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

// <H> and its gradient on the density-matrix simulator, as MQSim.get_expectation_with_grad calls it
// (mindquantum/simulator/mqsim.py:389-400): GetExpectationWithNoiseGradMultiMulti when the circuit
// holds a channel, else GetExpectationWithReversibleGradMultiMulti; every parameter an encoder
// input.  Arguments as mqref_grad plus the channel column ch.
int mqref_dm_grad(int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl,
                  const int *param, const double *coeff, const double *cst, const double *ch, int n_terms,
                  const int *term_len, const int *term_q, const char *term_p, const double *term_c, int n_params,
                  int n_samples, const double *params, double *out) {
    try {
        const auto names = mqref::param_names(n_params);
        const mqref::circuit_t c = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        const mqref::circuit_t h = mqref::build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, true, ch);
        if (int(c.size()) != n_gates || int(h.size()) != n_gates) return -1;
        bool noisy = false;
        for (int k = 0; k < n_gates; ++k) noisy = noisy || (kind[k] >= mqref::K_PC && kind[k] <= mqref::K_TR);
        std::vector<std::shared_ptr<mindquantum::Hamiltonian<double>>> hams{
            mqref::hamiltonian<double>(n_terms, term_len, term_q, term_p, term_c)};
        std::vector<std::vector<double>> enc(n_samples, std::vector<double>(n_params));
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i < n_params; ++i) enc[s][i] = params[s * n_params + i];
        dm_d sim{static_cast<mindquantum::Index>(n)};
        const auto res = noisy ? sim.GetExpectationWithNoiseGradMultiMulti(hams, c, h, enc, {}, names, {}, 1, 1)
                               : sim.GetExpectationWithReversibleGradMultiMulti(hams, c, h, enc, {}, names, {}, 1, 1);
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i <= n_params; ++i) {
                out[2 * (s * (n_params + 1) + i)] = res[s][0][i].real();
                out[2 * (s * (n_params + 1) + i) + 1] = res[s][0][i].imag();
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

}  // extern "C"
