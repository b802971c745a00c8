"""Parameter-shift gradients (vector_state.tpp:1033-1305; tests/st/test_simulator/test_method_of_mqvector.py:206-281).

Host: the oracle's restatement against its adjoint gradient (exact shift rules agree to 1e-6,
the central differences of controlled, Givens, FSim and custom gates to 1e-5), and the slot
plan (rows + combination) evaluated with the oracle against the oracle's own loop to 1e-12,
including the reference's value shift of U3/FSim parameters that other gates share.
GPU: ``get_expectation_with_grad(..., pr_shift=True)`` against the oracle's loop
(complex128 1e-9; complex64 1e-5 for f, 2e-3 for gradients: the central differences multiply
the complex64 expectation error by 500).
"""
import numpy as np
import pytest

from mindquantum_b200 import complex64, complex128
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from mindquantum_b200.simulator import Simulator
from mindquantum_b200.simulator.parameter_shift import ShiftPlan
from oracle import oracle as O
from test_host import _random_circuit

FIXED = ['h', 'x', 'cx', 'cz', 'swap', 'ccx', 'y']
SINGLE = [G.RX, G.RY, G.RZ, G.SWAPalpha, G.Givens, G.GlobalPhase, G.PhaseShift, G.Rxx, G.Rxy, G.Rxz, G.Ryy,
          G.Ryz, G.Rzz]


def _rot_custom():
    def m(a):
        c, s = np.cos(a / 2), np.sin(a / 2)
        return np.exp(0.3j * a) * np.array([[c, -1j * s], [-1j * s, c]])

    def dm(a):
        c, s = np.cos(a / 2), np.sin(a / 2)
        return 0.3j * m(a) + np.exp(0.3j * a) * 0.5 * np.array([[-s, -1j * c], [-1j * c, -s]])

    return G.gene_univ_parameterized_gate('rotc', m, dm)


def exact_circuit(seed=0):
    """Every single-parameter gate with a two-parameter expression, then two U3 gates."""
    rng = np.random.default_rng(seed)
    circ = _random_circuit(rng, 3, 6, FIXED)
    for i, gate in enumerate(SINGLE):
        g = gate({f'pr0_{i}': 1, f'pr1_{i}': 2})
        circ += g.on(list(range(g.n_qubits)))
        circ += _random_circuit(rng, 3, 4, FIXED)
    circ += G.U3('u3_theta', 'u3_phi', 'u3_lamda').on(0)
    circ += _random_circuit(rng, 3, 4, FIXED)
    circ += G.U3('u3_theta_1', 'u3_phi_1', 1).on(0)
    return Circuit(list(circ))


def difference_circuit(seed=1):
    """Controlled gates, FSim and a custom gate: central differences."""
    rng = np.random.default_rng(seed)
    circ = _random_circuit(rng, 3, 5, FIXED)
    for i, gate in enumerate(SINGLE):
        g = gate({f'pr0_{i}': 1, f'pr1_{i}': 2})
        circ += g.on(list(range(g.n_qubits)), 2)
        circ += _random_circuit(rng, 3, 3, FIXED)
    circ += G.U3('u3_theta', 'u3_phi', 'u3_lamda').on(0, 1)
    circ += G.FSim('fsim_theta', 'fsim_phi').on([0, 1])
    circ += _rot_custom()({'a': 1.5}).on(0)
    circ += _random_circuit(rng, 3, 3, FIXED)
    return Circuit(list(circ))


def shared_key_circuit():
    """A U3 angle and an FSim angle whose parameters other gates also use: the reference shifts the
    parameter value, so every gate using it moves."""
    c = Circuit([G.H.on(0), G.H.on(1), G.RX({'t': 1.0}).on(1), G.U3({'t': 2.0, 's': 0.5}, 'p', 0.3).on(0),
                 G.X.on(1, 0), G.FSim('p', {'t': -1.0}).on([0, 1]), G.RY('s').on(0), G.RZ({'p': 0.7}).on(1, 0)])
    return c


HAMS = [Hamiltonian(QubitOperator('X0') + QubitOperator('Z0')),
        Hamiltonian(QubitOperator('Y0 Z1', 0.6) + QubitOperator('X1 X2', -0.4))]


def _oracle_adjoint(circ, hams, p):
    return O.get_expectation_with_grad(3, hams, circ, np.zeros((1, 0)), p, [], circ.params_name)


def _oracle_shift(circ, hams, enc, ans, enc_names, ans_names, dtype=np.complex128):
    return O.get_expectation_with_grad_parameter_shift(3, hams, circ, enc, ans, enc_names, ans_names, dtype)


@pytest.mark.parametrize("make,tol", [(exact_circuit, 1e-6), (difference_circuit, 1e-5)])
def test_oracle_shift_matches_oracle_adjoint(make, tol):
    circ = make()
    p = np.random.default_rng(5).uniform(0, 2 * np.pi, len(circ.params_name))
    ref = _oracle_adjoint(circ, HAMS, p)
    got = _oracle_shift(circ, HAMS, np.zeros((1, 0)), p, [], circ.params_name)
    assert np.allclose(got[..., 0], ref[..., 0], atol=1e-12)
    assert np.allclose(got[..., 1:], ref[..., 1:], atol=tol)


def _plan_result(plan, circ_names, hams, P):
    rows = plan.rows(P)
    F = []
    for r in rows:
        qs = O.OracleSim(3, np.complex128).apply_circuit(plan.circuit, dict(zip(plan.slot_names, r))).qs
        F.append([O.expectation_of_terms(qs, qs, 3, h) for h in hams])
    return plan.combine(np.array(F))


@pytest.mark.parametrize("make", [exact_circuit, difference_circuit, shared_key_circuit])
def test_slot_plan_reproduces_the_oracle_loop(make):
    circ = make()
    names = circ.params_name
    rng = np.random.default_rng(9)
    P = rng.uniform(0, 2 * np.pi, (2, len(names)))
    f, g = _plan_result(ShiftPlan(circ, names), names, HAMS, P)
    for s in range(2):
        ref = _oracle_shift(circ, HAMS, np.zeros((1, 0)), P[s], [], names)
        assert np.allclose(f[s], ref[0, :, 0], atol=1e-12)
        assert np.allclose(g[s], ref[0, :, 1:], atol=1e-9)


def test_shared_key_shift_differs_from_the_adjoint():
    """The value shift is the reference's behaviour, not the derivative: pin that it is mirrored."""
    circ = shared_key_circuit()
    p = np.random.default_rng(2).uniform(0, 2 * np.pi, len(circ.params_name))
    ref = _oracle_adjoint(circ, HAMS[:1], p)
    got = _oracle_shift(circ, HAMS[:1], np.zeros((1, 0)), p, [], circ.params_name)
    assert np.max(np.abs(got[..., 1:] - ref[..., 1:])) > 1e-2


def test_plan_rows_and_jacobi():
    circ = Circuit([G.RX({'a': 2.0, 'b': -1.0}).on(0), G.RY(0.4).on(1), G.U3('a', 0.1, {'c': 3.0}).on(1),
                    G.RZ({'b': 1.0}, ).on(0, 1)])
    circ[0].coeff.no_grad_part('b')
    plan = ShiftPlan(circ, ['a', 'b', 'c'])
    assert plan.slot_names == ['_slot0', '_slot1', '_slot2', '_slot3']
    assert plan.n_shifts == 4
    rows = plan.rows(np.array([[0.5, 0.25, -1.0]]))
    assert rows.shape == (9, 4)
    assert np.allclose(rows[0], [0.75, 0.5, -3.0, 0.25])
    # RX slot shifted by pi/2; U3 theta shifts the value of 'a' (coefficient 1), which moves RX too
    assert np.allclose(rows[1] - rows[0], [-np.pi / 2, 0, 0, 0])
    assert np.allclose(rows[2] - rows[0], [-np.pi, -np.pi / 2, 0, 0])
    assert np.allclose(rows[3] - rows[0], [0, 0, -np.pi / 2, 0])      # U3 lambda: value of 'c' by pi/6
    assert np.allclose(rows[4] - rows[0], [0, 0, 0, -0.001])          # controlled RZ: difference
    assert np.allclose(plan.J[0], [2.0, 0.0, 0.0])                     # 'b' is no-grad in RX
    assert np.allclose(plan.coeff, [0.5, 0.5, 0.5, 500.0])


def test_unsupported_gate_raises():
    with pytest.raises(RuntimeError, match="not supported for parameter shift"):
        ShiftPlan(Circuit([G.Rn('a', 'b', 'c').on(0)]), ['a', 'b', 'c'])


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("make", [exact_circuit, difference_circuit, shared_key_circuit])
def test_parameter_shift_matches_oracle(dtype, make):
    circ = make()
    names = circ.params_name
    enc_names = names[:2]
    for g in circ:
        for p in getattr(g, 'prs', []):
            for k in p.params_name:
                if k in enc_names:
                    p.encoder_part(k)
    circ = Circuit(list(circ))
    rng = np.random.default_rng(11)
    enc = rng.uniform(0, 2 * np.pi, (3, len(circ.encoder_params_name)))
    ans = rng.uniform(0, 2 * np.pi, len(circ.ansatz_params_name))
    sim = Simulator('mqvector_b200', 3, dtype=dtype)
    f, ge, ga = sim.get_expectation_with_grad(HAMS, circ, pr_shift=True)(enc, ans)
    assert abs(sim.get_qs()[0] - 1) < 1e-6   # the simulator's own state is untouched
    ref = _oracle_shift(circ, HAMS, enc, ans, circ.encoder_params_name, circ.ansatz_params_name)
    ne = len(circ.encoder_params_name)
    ftol, gtol = (1e-9, 1e-9) if dtype == complex128 else (1e-5, 2e-3)
    assert np.allclose(f, ref[:, :, 0], atol=ftol, rtol=0)
    assert np.allclose(ge, ref[:, :, 1:1 + ne], atol=gtol, rtol=0)
    assert np.allclose(ga, ref[:, :, 1 + ne:], atol=gtol, rtol=0)


@pytest.mark.gpu
def test_parameter_shift_at_sixteen_qubits_matches_adjoint():
    """A 16-qubit hardware-efficient ansatz: exact shift rules equal the adjoint gradient."""
    from mindquantum_b200 import workloads as W

    circ, ham, params = W.hea(16, 2, 1, seed=4, encoder=False)
    sim = Simulator('mqvector_b200', 16, dtype=complex128)
    f, g = sim.get_expectation_with_grad(ham, circ, pr_shift=True)(params[0])
    f_ad, g_ad = sim.get_expectation_with_grad(ham, circ)(params[0])
    assert np.allclose(f, f_ad, atol=1e-10)
    assert np.allclose(g, g_ad, atol=1e-9)


@pytest.mark.parametrize("n_thread", [1, 2, 3])
def test_noiseless_stream_advance_matches_the_reference_loop(n_thread):
    """The noiseless batched path advances the simulator's stream by
    n_prs * (1 + groups + n_hams * (1 + 4 E)) draws: the count the reference's loop consumes."""
    circ = Circuit([G.RX('a').on(0), G.RY({'b': 2.0}).on(1), G.X.on(1, 0), G.U3('c', 0.3, 'd').on(0),
                    G.RZ('a').on(1, 0)])
    hams = [Hamiltonian(QubitOperator('Z0')), Hamiltonian(QubitOperator('X1')), Hamiltonian(QubitOperator('Y0 Y1'))]

    class Counting:
        def __init__(self):
            self.n, self.s = 0, O.UniformStream(5)

        def __call__(self):
            self.n += 1
            return self.s()

    draw = Counting()
    O.get_expectation_with_grad_parameter_shift_noisy(2, hams, circ, np.zeros((1, 0)), [0.1, 0.2, 0.3, 0.4], [],
                                                      circ.params_name, draw, n_thread=n_thread)
    E = ShiftPlan(circ, circ.params_name).n_shifts
    groups = -(-len(hams) // n_thread)
    assert draw.n == 1 + groups + len(hams) * (1 + 4 * E)
