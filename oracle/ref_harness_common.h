// Circuit and Hamiltonian builders shared by the drivers of the reference's own simulators,
// TEST INFRASTRUCTURE ONLY: ref_harness.cpp (the CPU simulator, _ref/libmqref.so) and
// ref_gpu_harness.cu (the thrust GPU simulator, _ref/libmqref_gpu.so).  Both are compiled with the
// reference's C++ sources by oracle/Makefile; this header only builds circuits and Hamiltonians
// with the reference's classes and calls its VectorState entry points:
//
//   apply_impl: VectorState::ApplyCircuit + GetQS (ccsrc/include/simulator/vector/vector_state.tpp:949-960);
//   sample_impl: VectorState::SamplingMeasurementEndingWithoutNoise / Sampling (vector_state.tpp:1308-1373),
//                the reference's seeded shot streams;
//   pshift_impl: GetExpectationWithGradParameterShiftMultiMulti (vector_state.tpp:1033-1305);
//   grad_impl:  VectorState::GetExpectationWithGradMultiMulti (the adjoint gradient,
//               ccsrc/include/simulator/vector/gradient.h:100-197), with the Hermitian circuit
//               built the way the reference's Python builds it (mindquantum/core/circuit/
//               circuit.py hermitian(): the daggers in reverse order, parameter expressions
//               negated).
#ifndef MQREF_HARNESS_COMMON_H
#define MQREF_HARNESS_COMMON_H
#include <omp.h>

#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "ops/basic_gate.h"
#include "ops/hamiltonian.h"
#include "simulator/vector/vector_state.h"

namespace mqref {

using mindquantum::Index;
using mindquantum::qbits_t;
using parameter::ParameterResolver;
using circuit_t = std::vector<std::shared_ptr<mindquantum::BasicGate>>;

// Gate kinds of the harness's gate table.  A measurement (K_M) takes its key from the param column:
// key "k<param>".  Each gate has six extra values ch[6 k .. 6 k + 5].  Channels take their arguments
// from the first three: Pauli (px, py, pz), depolarizing (p), amplitude damping (gamma, -,
// daggered), phase damping (gamma), thermal relaxation (t1, t2, gate time).  S, T, SX and ISWAP
// take a daggered flag from ch[6 k].  The multi-angle gates U3 (theta, phi, lambda), Rn (alpha,
// beta, gamma) and FSim (theta, phi) take angle i = ch[6 k + i] + ch[6 k + 3 + i] * p, p the
// gate's parameter (param column, -1 for none).
enum Kind {
    K_X = 0, K_H = 1, K_RX = 2, K_RY = 3, K_RZ = 4, K_Z = 5, K_RZZ = 6, K_Y = 7, K_PS = 8, K_M = 9,
    K_PC = 10, K_DEP = 11, K_AD = 12, K_PD = 13, K_TR = 14,
    K_S = 15, K_T = 16, K_SX = 17, K_SWAP = 18, K_ISWAP = 19, K_RXX = 20, K_RYY = 21, K_RXY = 22, K_RXZ = 23,
    K_RYZ = 24, K_GIVENS = 25, K_GP = 26, K_SWAPALPHA = 27, K_U3 = 28, K_RN = 29, K_FSIM = 30
};
constexpr int kCh = 6;   // extra values per gate

inline ParameterResolver angle(int param, double coeff, double cst, const std::vector<std::string> &names,
                               double sign) {
    if (param < 0) return ParameterResolver(sign * cst);
    return ParameterResolver(sign * cst, std::map<std::string, double>{{names[param], sign * coeff}});
}

// Angle i of a multi-angle gate: ch[i] + ch[3 + i] * p.
inline ParameterResolver angle_i(int param, const double *a, int i, const std::vector<std::string> &names,
                                 double sign) {
    return angle(param, a[3 + i], a[i], names, sign);
}

// The circuit of the table, or its Hermitian conjugate (reversed, parameter expressions negated).
inline circuit_t build(int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl,
                       const int *param, const double *coeff, const double *cst, const std::vector<std::string> &names,
                       bool herm, const double *ch = nullptr) {
    circuit_t c;
    for (int i = 0; i < n_gates; ++i) {
        const int k = herm ? n_gates - 1 - i : i;
        const double sign = herm ? -1.0 : 1.0;
        using q_t = qbits_t::value_type;
        qbits_t ctrls, obj1q{static_cast<q_t>(obj0[k])};
        if (ctrl[k] >= 0) ctrls.push_back(static_cast<q_t>(ctrl[k]));
        if (obj1[k] >= 0) obj1q.push_back(static_cast<q_t>(obj1[k]));
        switch (kind[k]) {
            case K_X: c.push_back(std::make_shared<mindquantum::XGate>(obj1q, ctrls)); break;
            case K_Y: c.push_back(std::make_shared<mindquantum::YGate>(obj1q, ctrls)); break;
            case K_Z: c.push_back(std::make_shared<mindquantum::ZGate>(obj1q, ctrls)); break;
            case K_H: c.push_back(std::make_shared<mindquantum::HGate>(obj1q, ctrls)); break;
            case K_RX:
                c.push_back(std::make_shared<mindquantum::RXGate>(angle(param[k], coeff[k], cst[k], names, sign), obj1q, ctrls));
                break;
            case K_RY:
                c.push_back(std::make_shared<mindquantum::RYGate>(angle(param[k], coeff[k], cst[k], names, sign), obj1q, ctrls));
                break;
            case K_RZ:
                c.push_back(std::make_shared<mindquantum::RZGate>(angle(param[k], coeff[k], cst[k], names, sign), obj1q, ctrls));
                break;
            case K_RZZ:
                c.push_back(std::make_shared<mindquantum::RzzGate>(angle(param[k], coeff[k], cst[k], names, sign), obj1q, ctrls));
                break;
            case K_PS:
                c.push_back(std::make_shared<mindquantum::PSGate>(angle(param[k], coeff[k], cst[k], names, sign), obj1q, ctrls));
                break;
            case K_M:
                c.push_back(std::make_shared<mindquantum::MeasureGate>("k" + std::to_string(param[k]), obj1q));
                break;
            case K_PC:
            case K_DEP:
            case K_AD:
            case K_PD:
            case K_TR: {
                if (!ch) return {};
                const double *a = ch + kCh * k;
                if (kind[k] == K_PC) c.push_back(std::make_shared<mindquantum::PauliChannel>(a[0], a[1], a[2], obj1q, ctrls));
                if (kind[k] == K_DEP) c.push_back(std::make_shared<mindquantum::DepolarizingChannel>(a[0], obj1q, ctrls));
                if (kind[k] == K_AD)   // the Hermitian circuit takes the daggered channel (basic.py hermitian())
                    c.push_back(
                        std::make_shared<mindquantum::AmplitudeDampingChannel>((a[2] != 0) != herm, a[0], obj1q, ctrls));
                if (kind[k] == K_PD) c.push_back(std::make_shared<mindquantum::PhaseDampingChannel>(a[0], obj1q, ctrls));
                if (kind[k] == K_TR)
                    c.push_back(std::make_shared<mindquantum::ThermalRelaxationChannel>(a[0], a[1], a[2], obj1q, ctrls));
                break;
            }
            case K_S:
            case K_T:
            case K_SX:
            case K_ISWAP: {   // the Hermitian circuit takes the other of the gate and its dagger
                const bool dag = ((ch && ch[kCh * k] != 0) != herm);
                if (kind[k] == K_S) {
                    if (dag) c.push_back(std::make_shared<mindquantum::SdagGate>(obj1q, ctrls));
                    else c.push_back(std::make_shared<mindquantum::SGate>(obj1q, ctrls));
                }
                if (kind[k] == K_T) {
                    if (dag) c.push_back(std::make_shared<mindquantum::TdagGate>(obj1q, ctrls));
                    else c.push_back(std::make_shared<mindquantum::TGate>(obj1q, ctrls));
                }
                if (kind[k] == K_SX) {
                    if (dag) c.push_back(std::make_shared<mindquantum::SXdagGate>(obj1q, ctrls));
                    else c.push_back(std::make_shared<mindquantum::SXGate>(obj1q, ctrls));
                }
                if (kind[k] == K_ISWAP) c.push_back(std::make_shared<mindquantum::ISWAPGate>(dag, obj1q, ctrls));
                break;
            }
            case K_SWAP: c.push_back(std::make_shared<mindquantum::SWAPGate>(obj1q, ctrls)); break;
            case K_RXX:
            case K_RYY:
            case K_RXY:
            case K_RXZ:
            case K_RYZ:
            case K_GIVENS:
            case K_GP:
            case K_SWAPALPHA: {
                const ParameterResolver a = angle(param[k], coeff[k], cst[k], names, sign);
                if (kind[k] == K_RXX) c.push_back(std::make_shared<mindquantum::RxxGate>(a, obj1q, ctrls));
                if (kind[k] == K_RYY) c.push_back(std::make_shared<mindquantum::RyyGate>(a, obj1q, ctrls));
                if (kind[k] == K_RXY) c.push_back(std::make_shared<mindquantum::RxyGate>(a, obj1q, ctrls));
                if (kind[k] == K_RXZ) c.push_back(std::make_shared<mindquantum::RxzGate>(a, obj1q, ctrls));
                if (kind[k] == K_RYZ) c.push_back(std::make_shared<mindquantum::RyzGate>(a, obj1q, ctrls));
                if (kind[k] == K_GIVENS) c.push_back(std::make_shared<mindquantum::GivensGate>(a, obj1q, ctrls));
                if (kind[k] == K_GP) c.push_back(std::make_shared<mindquantum::GPGate>(a, obj1q, ctrls));
                if (kind[k] == K_SWAPALPHA) c.push_back(std::make_shared<mindquantum::SWAPalphaGate>(a, obj1q, ctrls));
                break;
            }
            case K_U3:
            case K_RN:
            case K_FSIM: {
                if (!ch) return {};
                const double *a = ch + kCh * k;
                const ParameterResolver a0 = angle_i(param[k], a, 0, names, sign);
                const ParameterResolver a1 = angle_i(param[k], a, 1, names, sign);
                const ParameterResolver a2 = angle_i(param[k], a, 2, names, sign);
                // Hermitian forms (mindquantum/core/gates/basicgate.py): U3(-t, -l, -p), Rn(-a, -b, -g), FSim(-t, -p)
                if (kind[k] == K_U3) {
                    if (herm) c.push_back(std::make_shared<mindquantum::U3>(a0, a2, a1, obj1q, ctrls));
                    else c.push_back(std::make_shared<mindquantum::U3>(a0, a1, a2, obj1q, ctrls));
                }
                if (kind[k] == K_RN) c.push_back(std::make_shared<mindquantum::Rn>(a0, a1, a2, obj1q, ctrls));
                if (kind[k] == K_FSIM) c.push_back(std::make_shared<mindquantum::FSim>(a0, a1, obj1q, ctrls));
                break;
            }
            default:
                return {};
        }
    }
    return c;
}

inline std::vector<std::string> param_names(int n_params) {
    std::vector<std::string> v;
    for (int i = 0; i < n_params; ++i) v.push_back("p" + std::to_string(i));
    return v;
}

// Apply the circuit to |0...0> with parameter values params[n_params]; out: 2^n complex128 (re, im).
#define MQREF_APPLY_ARGS                                                                                            \
    int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl, const int *param,      \
        const double *coeff, const double *cst, const double *ch, int n_params, const double *params, int threads, \
        double *out
#define MQREF_APPLY_PASS n, n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, ch, n_params, params, threads, out

template <typename sim_t>
int apply_impl(MQREF_APPLY_ARGS) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        const auto names = param_names(n_params);
        const circuit_t c = build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        if (int(c.size()) != n_gates) return -1;
        ParameterResolver pr;
        for (int i = 0; i < n_params; ++i) pr.SetItem(names[i], params[i]);
        sim_t sim{static_cast<Index>(n)};
        sim.ApplyCircuit(c, pr);
        const auto qs = sim.GetQS();
        for (size_t i = 0; i < qs.size(); ++i) {
            out[2 * i] = double(qs[i].real());
            out[2 * i + 1] = double(qs[i].imag());
        }
        return 0;
    } catch (...) {
        return -2;
    }
}

// Shots of a circuit with measurements (and noise channels) from |0...0>: measurement-ending
// circuits by SamplingMeasurementEndingWithoutNoise (ending != 0), others by Sampling (one
// re-simulation per shot, channels drawing from the shot's stream, vector_state.tpp:465-709).  Measurement keys are "k<i>" for the M gates' param column i; out: [shots][n_keys] with
// column i the key "k<i>" (n_keys = the number of M gates).
#define MQREF_SAMPLE_ARGS                                                                                           \
    int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl, const int *param,      \
        const double *coeff, const double *cst, const double *ch, int n_params, const double *params, int shots,  \
        unsigned seed, int ending, int *out
#define MQREF_SAMPLE_PASS \
    n, n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, ch, n_params, params, shots, seed, ending, out

template <typename sim_t>
int sample_impl(MQREF_SAMPLE_ARGS) {
    try {
        const auto names = param_names(n_params);
        const circuit_t c = build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        if (int(c.size()) != n_gates) return -1;
        ParameterResolver pr;
        for (int i = 0; i < n_params; ++i) pr.SetItem(names[i], params[i]);
        mindquantum::MST<size_t> key_map;
        for (int k = 0; k < n_gates; ++k)
            if (kind[k] == K_M) key_map["k" + std::to_string(param[k])] = size_t(param[k]);
        sim_t sim{static_cast<Index>(n)};
        const auto res = ending ? sim.SamplingMeasurementEndingWithoutNoise(c, pr, size_t(shots), key_map, seed)
                                : sim.Sampling(c, pr, size_t(shots), key_map, seed);
        for (size_t i = 0; i < res.size(); ++i) out[i] = int(res[i]);
        return 0;
    } catch (...) {
        return -2;
    }
}

// <H> and its gradient for n_samples parameter rows (all parameters treated as encoder inputs, as
// get_expectation_with_grad does for an encoder circuit).  Hamiltonian: n_terms Pauli strings,
// term t has term_len[t] (qubit, 'X'|'Y'|'Z') pairs from term_q / term_p and coefficient term_c[t].
// out: [n_samples][1 + n_params] complex128 (re, im): f, then the gradient.
#define MQREF_GRAD_ARGS                                                                                             \
    int n, int n_gates, const int *kind, const int *obj0, const int *obj1, const int *ctrl, const int *param,      \
        const double *coeff, const double *cst, const double *ch, int n_terms, const int *term_len,                \
        const int *term_q, const char *term_p, const double *term_c, int n_params, int n_samples,                  \
        const double *params, int threads, double *out
#define MQREF_GRAD_PASS                                                                                               \
    n, n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, ch, n_terms, term_len, term_q, term_p, term_c, n_params, \
        n_samples, params, threads, out

// The Hamiltonian of a gradient call as the reference's type.
template <typename calc_t>
std::shared_ptr<mindquantum::Hamiltonian<calc_t>> hamiltonian(int n_terms, const int *term_len, const int *term_q,
                                                               const char *term_p, const double *term_c) {
    std::vector<mindquantum::PauliTerm<calc_t>> terms;
    for (int t = 0, o = 0; t < n_terms; ++t) {
        std::vector<mindquantum::PauliWord> w;
        for (int k = 0; k < term_len[t]; ++k, ++o) w.emplace_back(Index(term_q[o]), term_p[o]);
        terms.emplace_back(w, calc_t(term_c[t]));
    }
    return std::make_shared<mindquantum::Hamiltonian<calc_t>>(terms);
}

template <typename sim_t, typename calc_t>
int grad_impl(MQREF_GRAD_ARGS) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        const auto names = param_names(n_params);
        const circuit_t c = build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        const circuit_t h = build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, true, ch);
        if (int(c.size()) != n_gates || int(h.size()) != n_gates) return -1;
        std::vector<std::shared_ptr<mindquantum::Hamiltonian<calc_t>>> hams{
            hamiltonian<calc_t>(n_terms, term_len, term_q, term_p, term_c)};
        std::vector<std::vector<calc_t>> enc(n_samples, std::vector<calc_t>(n_params));
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i < n_params; ++i) enc[s][i] = calc_t(params[s * n_params + i]);
        sim_t sim{static_cast<Index>(n)};
        const auto res = sim.GetExpectationWithGradMultiMulti(hams, c, h, enc, {}, names, {}, 1, 1);
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i <= n_params; ++i) {
                out[2 * (s * (n_params + 1) + i)] = double(res[s][0][i].real());
                out[2 * (s * (n_params + 1) + i) + 1] = double(res[s][0][i].imag());
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

// The parameter-shift gradient, as MQSim.get_expectation_with_grad(..., pr_shift=True) calls it
// (GetExpectationWithGradParameterShiftMultiMulti, vector_state.tpp:1033-1305): same arguments and
// output as grad_impl; the simulator keeps the reference's default seed (42).
template <typename sim_t, typename calc_t>
int pshift_impl(MQREF_GRAD_ARGS) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        const auto names = param_names(n_params);
        const circuit_t c = build(n_gates, kind, obj0, obj1, ctrl, param, coeff, cst, names, false, ch);
        if (int(c.size()) != n_gates) return -1;
        std::vector<std::shared_ptr<mindquantum::Hamiltonian<calc_t>>> hams{
            hamiltonian<calc_t>(n_terms, term_len, term_q, term_p, term_c)};
        std::vector<std::vector<calc_t>> enc(n_samples, std::vector<calc_t>(n_params));
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i < n_params; ++i) enc[s][i] = calc_t(params[s * n_params + i]);
        sim_t sim{static_cast<Index>(n)};
        const auto res = sim.GetExpectationWithGradParameterShiftMultiMulti(hams, c, enc, {}, names, {}, 1, 1);
        for (int s = 0; s < n_samples; ++s)
            for (int i = 0; i <= n_params; ++i) {
                out[2 * (s * (n_params + 1) + i)] = double(res[s][0][i].real());
                out[2 * (s * (n_params + 1) + i) + 1] = double(res[s][0][i].imag());
            }
        return 0;
    } catch (...) {
        return -2;
    }
}

}  // namespace mqref

#endif
