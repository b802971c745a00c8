"""The reference's method checks of the state-vector simulator, run against `mqvector_b200` (GPU).

The cases follow tests/st/test_simulator/test_method_of_mqvector.py:53-280 of the reference:

* `get_expectation` of a random 10-term Pauli Hamiltonian, given as Pauli terms, as `.sparse(3)`
  and as a CSR matrix, after a 100-gate random circuit from a random initial state, in all four
  forms (circ_right only, with circ_left, with simulator_left, with both);
* the non-Hermitian gradient <phi| U_l^dag H U_r(a, b) |psi> with RX({'a': 1, 'b': 2}) between two
  random circuits, for the three Hamiltonian forms;
* parameter-shift gradients (`pr_shift=True`) of a circuit holding every one-parameter gate kind
  with two-parameter expressions and U3 gates, against the adjoint gradient; and of a circuit with
  controlled gates, FSim, a controlled U3 and a custom parameterized gate.

References are dense matrices made by the oracle (column j = the circuit applied to |j>), and the
Hamiltonian's matrix; tolerances are the reference test's.
"""
import numpy as np
import pytest
from scipy.sparse import csr_matrix

from mindquantum_b200 import complex64, complex128, workloads as W
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from mindquantum_b200.simulator import Simulator
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SINGLE_PARAMETER = [G.RX, G.RY, G.RZ, G.SWAPalpha, G.Givens, G.GlobalPhase, G.PhaseShift, G.Rxx, G.Rxy, G.Rxz,
                    G.Ryy, G.Ryz, G.Rzz]


def _random_fixed_circuit(rng, n, n_gates):
    """Random gates with numeric angles on n qubits (one, two and three-qubit kinds, controls)."""
    c = Circuit()
    for _ in range(n_gates):
        q = [int(x) for x in rng.permutation(n)[:3]]
        t = rng.uniform(0, 2 * np.pi, 3)
        k = int(rng.integers(14))
        c += [G.H.on(q[0]), G.X.on(q[0], q[1]), G.RX(t[0]).on(q[0]), G.RY(t[0]).on(q[0], q[1]),
              G.RZ(t[0]).on(q[0]), G.Rzz(t[0]).on([q[0], q[1]]), G.U3(*t).on(q[0]), G.SWAP.on([q[0], q[1]]),
              G.Z.on(q[0], q[1]), G.X.on(q[0], q[1:3]), G.FSim(t[0], t[1]).on([q[0], q[1]]),
              G.PhaseShift(t[0]).on(q[0]), G.Y.on(q[0]), G.T.on(q[0])][k]
    return c


def _dense(circ, n, prd=None):
    prd = prd or {}
    cols = []
    for j in range(1 << n):
        e = np.zeros(1 << n, dtype=np.complex128)
        e[j] = 1
        cols.append(O.OracleSim(n, np.complex128, e).apply_circuit(circ, prd).qs)
    return np.array(cols).T


def _state(rng, dim):
    v = rng.random(dim) + 1j * rng.random(dim)
    return v / np.linalg.norm(v)


def _hams(rng, n):
    ham0 = W.random_pauli_hamiltonian(n, 10, rng, max_weight=n)
    hm = O.ham_matrix(n, ham0)
    return ham0, hm, (ham0, ham0.sparse(n), Hamiltonian(csr_matrix(hm)))


@pytest.mark.parametrize("dtype", [complex64, complex128])
def test_get_expectation(dtype):
    rng = np.random.default_rng(61 if dtype == complex64 else 62)
    n = 3
    init, init_left = _state(rng, 8), _state(rng, 8)
    circ, circ_left = _random_fixed_circuit(rng, n, 100), _random_fixed_circuit(rng, n, 100)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim_left = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(init)
    sim_left.set_qs(init_left)
    _, hm, hams = _hams(rng, n)
    u, ul = _dense(circ, n), _dense(circ_left, n)
    for ham in hams:
        assert np.allclose(sim.get_expectation(ham, circ), init.conj() @ u.conj().T @ hm @ u @ init, atol=1e-6)
        assert np.allclose(sim.get_expectation(ham, circ, circ_left), init.conj() @ ul.conj().T @ hm @ u @ init,
                           atol=1e-6)
        assert np.allclose(sim.get_expectation(ham, circ, simulator_left=sim_left),
                           init_left.conj() @ u.conj().T @ hm @ u @ init, atol=1e-6)
        assert np.allclose(sim.get_expectation(ham, circ, circ_left, sim_left),
                           init_left.conj() @ ul.conj().T @ hm @ u @ init, atol=1e-6)


@pytest.mark.parametrize("dtype", [complex64, complex128])
def test_non_hermitian_get_expectation_with_grad(dtype):
    rng = np.random.default_rng(129 if dtype == complex64 else 130)
    n = 3
    init, init_left = _state(rng, 8), _state(rng, 8)
    circ0, circ1 = _random_fixed_circuit(rng, n, 100), _random_fixed_circuit(rng, n, 100)
    pr_gate = G.RX({'a': 1, 'b': 2}).on(0)
    circ = circ0 + pr_gate + circ1
    circ_left = _random_fixed_circuit(rng, n, 100)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim_left = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(init)
    sim_left.set_qs(init_left)
    pr = rng.random(2) * 2 * np.pi
    prd = {'a': pr[0], 'b': pr[1]}
    _, hm, hams = _hams(rng, n)
    u0, u1, ul = _dense(circ0, n), _dense(circ1, n), _dense(circ_left, n)
    ref_f = init_left.conj() @ ul.conj().T @ hm @ u1 @ np.kron(np.eye(4), pr_gate.matrix(prd)) @ u0 @ init
    ref_g = [init_left.conj() @ ul.conj().T @ hm @ u1 @ np.kron(np.eye(4), pr_gate.diff_matrix(prd, w)) @ u0 @ init
             for w in ('a', 'b')]
    for ham in hams:
        f, g = sim.get_expectation_with_grad(ham, circ, circ_left, sim_left)(pr)
        assert np.allclose(f, ref_f, atol=1e-6)
        assert np.allclose(g, ref_g, atol=1e-6)


@pytest.mark.parametrize("dtype", [complex64, complex128])
def test_parameter_shift_rule(dtype):
    rng = np.random.default_rng(206 if dtype == complex64 else 207)
    n = 3
    circ = _random_fixed_circuit(rng, n, 10)
    for i, gate in enumerate(SINGLE_PARAMETER):
        g = gate({f'pr0_{i}': 1, f'pr1_{i}': 2})
        circ += g.on(list(range(g.n_qubits)))
        circ += _random_fixed_circuit(rng, n, 10)
    circ += G.U3('u3_theta', 'u3_phi', 'u3_lamda').on(0)
    circ += _random_fixed_circuit(rng, n, 10)
    circ += G.U3('u3_theta_1', 'u3_phi_1', 1).on(0)
    circ += _random_fixed_circuit(rng, n, 10)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    ham = Hamiltonian(QubitOperator('X0') + QubitOperator('Z0'))
    pr = rng.random(len(circ.params_name)) * 2 * np.pi
    f, g = sim.get_expectation_with_grad(ham, circ, pr_shift=True)(pr)
    ref_f, ref_g = sim.get_expectation_with_grad(ham, circ)(pr)
    assert np.allclose(f, ref_f, atol=1e-4)
    assert np.allclose(g, ref_g, atol=1e-3)


def _custom_matrix(alpha):
    ep = 0.5 * (1 + np.exp(1j * np.pi * alpha))
    em = 0.5 * (1 - np.exp(1j * np.pi * alpha))
    return np.array([[ep, em], [em, ep]])


def _custom_diff_matrix(alpha):
    ep = 0.5 * 1j * np.pi * np.exp(1j * np.pi * alpha)
    em = -0.5 * 1j * np.pi * np.exp(1j * np.pi * alpha)
    return np.array([[ep, em], [em, ep]])


@pytest.mark.parametrize("dtype", [complex64, complex128])
def test_parameter_shift_rule_finite_diff_case(dtype):
    rng = np.random.default_rng(244 if dtype == complex64 else 245)
    n = 3
    custom_gate = G.gene_univ_parameterized_gate('custom', _custom_matrix, _custom_diff_matrix)
    circ = _random_fixed_circuit(rng, n, 10)
    for i, gate in enumerate(SINGLE_PARAMETER):
        g = gate({f'pr0_{i}': 1, f'pr1_{i}': 2})
        circ += g.on(list(range(g.n_qubits)), 2)
        circ += _random_fixed_circuit(rng, n, 10)
    circ += G.U3('u3_theta', 'u3_phi', 'u3_lamda').on(0, 1)
    circ += _random_fixed_circuit(rng, n, 10)
    circ += G.FSim('fsim_theta', 'fsim_phi').on([0, 1])
    circ += _random_fixed_circuit(rng, n, 10)
    circ += custom_gate('a').on(0)
    circ += _random_fixed_circuit(rng, n, 10)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    ham = Hamiltonian(QubitOperator('X0') + QubitOperator('Z0'))
    pr = rng.random(len(circ.params_name)) * 2 * np.pi
    f, g = sim.get_expectation_with_grad(ham, circ, pr_shift=True)(pr)
    ref_f, ref_g = sim.get_expectation_with_grad(ham, circ)(pr)
    assert np.allclose(f, ref_f, atol=1e-3)
    assert np.allclose(g, ref_g, atol=1e-2)
