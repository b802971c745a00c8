"""The reference's per-gate simulator checks, run against both B200 backends (GPU).

The cases follow tests/st/test_simulator/test_basic_gate_with_simulator.py:73-217 of the
reference, which loops over every registered simulator: every gate class without parameters
(H, I, ISWAP, S, SWAP, T, X, Y, Z, SX and the daggers of SX, T, S), with one parameter (RX, RY,
RZ, SWAPalpha, Givens, GlobalPhase, PhaseShift, Rxx, Rxy, Rxz, Ryy, Ryz, Rzz) and with several
(U3, FSim, Rn), applied on a random state of its own qubit count and, controlled by one more
qubit, on a random state one qubit larger; and for every one-parameter gate with the parameter
expression {'a': 1, 'b': 2}, <H> and the gradient with respect to a and b for a random
10-term Pauli Hamiltonian, uncontrolled and controlled.  References are dense: the gate's own
matrix and derivative matrix, the Hamiltonian's matrix.  The backends are `mqvector_b200` and the
density-matrix `mqmatrix_b200` (compared as rho = psi psi^dag), in complex128 and complex64.
Tolerances are the reference test's: 1e-8 default allclose for unparameterized gates, 1e-6 for
parameterized ones, 1e-4 / 1e-5 for expectations and gradients.
"""
import numpy as np
import pytest

from mindquantum_b200 import complex64, complex128, workloads as W
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.simulator import Simulator
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NONE_PARAMETER = [G.HGate, G.IGate, G.ISWAPGate, G.SGate, G.SWAPGate, G.TGate, G.XGate, G.YGate, G.ZGate,
                  G.SXGate, lambda: G.SXGate().hermitian(), lambda: G.TGate().hermitian(),
                  lambda: G.SGate().hermitian()]
NONE_IDS = ['H', 'I', 'ISWAP', 'S', 'SWAP', 'T', 'X', 'Y', 'Z', 'SX', 'SXdag', 'Tdag', 'Sdag']
SINGLE_PARAMETER = [G.RX, G.RY, G.RZ, G.SWAPalpha, G.Givens, G.GlobalPhase, G.PhaseShift, G.Rxx, G.Rxy, G.Rxz,
                    G.Ryy, G.Ryz, G.Rzz]
MULTI_PARAMETER = [(G.U3, 3), (G.FSim, 2), (G.Rn, 3)]
CONFIGS = [('mqvector_b200', complex128), ('mqvector_b200', complex64), ('mqmatrix_b200', complex128),
           ('mqmatrix_b200', complex64)]
CONFIG_IDS = ['vector-c128', 'vector-c64', 'matrix-c128', 'matrix-c64']


def _state(rng, dim):
    v = rng.random(dim) + 1j * rng.random(dim)
    return v


def _check_state(backend, sim, ref, atol):
    ref = ref / np.linalg.norm(ref)
    got = sim.get_qs()
    if backend.startswith('mqmatrix'):
        assert np.allclose(got, np.outer(ref, ref.conj()), atol=atol)
    else:
        assert np.allclose(got, ref, atol=atol)


def _controlled(m):
    dim = m.shape[0]
    z = np.zeros((dim, dim))
    return np.block([[np.eye(dim), z], [z, m]])


def _apply_and_check(backend, dtype, g, matrix, rng, atol):
    k = g.n_qubits
    dim = 1 << k
    init = _state(rng, dim)
    sim = Simulator(backend, k, dtype=dtype)
    sim.set_qs(init)
    sim.apply_gate(g.on(list(range(k))))
    _check_state(backend, sim, matrix @ (init / np.linalg.norm(init)), atol)
    c_init = _state(rng, 2 * dim)
    c_sim = Simulator(backend, k + 1, dtype=dtype)
    c_sim.set_qs(c_init)
    c_sim.apply_gate(g.on(list(range(k)), k))
    _check_state(backend, c_sim, _controlled(matrix) @ (c_init / np.linalg.norm(c_init)), max(atol, 1e-6))


@pytest.mark.parametrize("config", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("gate", NONE_PARAMETER, ids=NONE_IDS)
def test_none_parameter_gate(config, gate):
    backend, dtype = config
    rng = np.random.default_rng(CONFIGS.index(config) * 100 + NONE_PARAMETER.index(gate))
    g = gate()
    atol = 1e-8 if dtype == complex128 else 1e-6
    _apply_and_check(backend, dtype, g, g.matrix(), rng, atol)


@pytest.mark.parametrize("config", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("gate,n_pr", [(g, 1) for g in SINGLE_PARAMETER] + MULTI_PARAMETER,
                         ids=[g.__name__ for g in SINGLE_PARAMETER] + [g.__name__ for g, _ in MULTI_PARAMETER])
def test_parameter_gate(config, gate, n_pr):
    backend, dtype = config
    rng = np.random.default_rng(CONFIGS.index(config) * 100 + 50 + n_pr + len(gate.__name__))
    pr = rng.random(n_pr) * 2 * np.pi
    g = gate(*pr)
    _apply_and_check(backend, dtype, g, g.matrix(), rng, 1e-6)


def _dense_f_and_grad(g_on, n, ham, init, pr, extend=None):
    prd = {'a': pr[0], 'b': pr[1]}
    m = g_on.matrix(prd)
    dims = [m]
    diffs = [g_on.diff_matrix(prd, w) for w in ('a', 'b')]
    if extend is not None:
        dims = [extend(m)]
        diffs = [extend(d, zero=True) for d in diffs]
    hm = O.ham_matrix(n, ham)
    u = dims[0]
    f = init.conj() @ u.conj().T @ hm @ u @ init
    grad = [2 * (init.conj() @ u.conj().T @ hm @ d @ init).real for d in diffs]
    return f, np.array(grad)


@pytest.mark.parametrize("config", CONFIGS, ids=CONFIG_IDS)
@pytest.mark.parametrize("gate", SINGLE_PARAMETER, ids=[g.__name__ for g in SINGLE_PARAMETER])
def test_single_parameter_gate_expectation_with_grad(config, gate):
    backend, dtype = config
    rng = np.random.default_rng(1000 + CONFIGS.index(config) * 100 + SINGLE_PARAMETER.index(gate))
    g = gate({'a': 1, 'b': 2})
    k = g.n_qubits
    dim = 1 << k
    g = g.on(list(range(k)))
    init = _state(rng, dim)
    init = init / np.linalg.norm(init)
    ham = W.random_pauli_hamiltonian(k, 10, rng, max_weight=k)
    sim = Simulator(backend, k, dtype=dtype)
    sim.set_qs(init)
    pr = rng.random(2) * 2 * np.pi
    f, grad = sim.get_expectation_with_grad(ham, Circuit([g]))(pr)
    ref_f, ref_grad = _dense_f_and_grad(g, k, ham, init, pr)
    assert np.allclose(f, ref_f, atol=1e-4)
    assert np.allclose(grad, ref_grad, atol=1e-4)

    c_g = g.on(list(range(k)), k)
    c_init = _state(rng, 2 * dim)
    c_init = c_init / np.linalg.norm(c_init)
    c_ham = W.random_pauli_hamiltonian(k + 1, 10, rng, max_weight=k + 1)
    c_sim = Simulator(backend, k + 1, dtype=dtype)
    c_sim.set_qs(c_init)
    c_pr = rng.random(2) * 2 * np.pi
    c_f, c_grad = c_sim.get_expectation_with_grad(c_ham, Circuit([c_g]))(c_pr)

    def extend(m, zero=False):
        z = np.zeros((dim, dim))
        return np.block([[z if zero else np.eye(dim), z], [z, m]])

    ref_f, ref_grad = _dense_f_and_grad(g, k + 1, c_ham, c_init, c_pr, extend)
    assert np.allclose(c_f, ref_f, atol=1e-5)
    assert np.allclose(c_grad, ref_grad, atol=1e-5)
