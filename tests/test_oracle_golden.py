"""Pin the CPU oracle to the reference's own golden numbers (no GPU needed).

Each case reproduces a reference test or docstring (file:line in reference_goldens.json)
and checks the oracle's restatement of the reference algorithm against the numbers that
test asserts, at the tolerance that test uses.
"""
import numpy as np
import pytest

from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from oracle import oracle as O
from reference_circuits import generate_test_circuit, mul_qubit_circuit, multi_params_circuit


def _c(a):
    a = np.asarray(a, dtype=float)
    return a[..., 0] + 1j * a[..., 1]


@pytest.mark.parametrize("dtype,atol", [(np.complex128, 1e-7), (np.complex64, 1e-6)])
def test_all_gate_state(goldens, dtype, atol):
    g = goldens['all_gate_qs']
    sim = O.OracleSim(3, dtype).apply_circuit(generate_test_circuit(), g['pr'])
    assert np.allclose(sim.qs, _c(g['qs']), atol=atol)


def test_multi_params_state_and_grad(goldens):
    g = goldens['multi_params']
    circ = multi_params_circuit()
    prd = dict(zip(circ.params_name, g['p0']))
    sim = O.OracleSim(2).apply_circuit(circ, prd)
    assert np.allclose(sim.qs, _c(g['qs']), atol=1e-7)
    ham = Hamiltonian(QubitOperator('X0 Y1'))
    res = O.get_expectation_with_grad(2, [ham], circ, np.zeros((1, 0)), g['p0'], [], circ.params_name)
    assert np.allclose(res[:, :, 0], _c(g['f']), atol=1e-6)
    assert np.allclose(res[:, :, 1:], _c(g['g']), atol=1e-6)


def test_custom_gate_in_parallel(goldens):
    g = goldens['custom_gate_in_parallel']
    circ = generate_test_circuit().as_encoder()
    hams = [Hamiltonian(QubitOperator('Y0')), Hamiltonian(QubitOperator('X2'))]
    np.random.seed(g['seed'])
    p0 = np.random.uniform(0, 1, size=(2, len(circ.params_name)))
    res = O.get_expectation_with_grad(3, hams, circ, p0, [], circ.encoder_params_name, [])
    assert np.allclose(np.sum(res[:, :, 0]), g['f_sum'], atol=1e-6)
    assert np.allclose(np.sum(res[:, :, 1:]), g['g_sum'], atol=1e-6)


def test_mul_qubit_gate(goldens):
    g = goldens['mul_qubit_gate']
    circ = mul_qubit_circuit()
    ham = Hamiltonian(QubitOperator('X0'))
    res = O.get_expectation_with_grad(3, [ham], circ, np.zeros((1, 0)), [g['p']], [], circ.params_name)
    assert np.allclose(res[0, 0, 0], g['f1'])
    assert np.allclose(res[0, 0, 1], g['g1'])


def test_apply_circuit_docstring(goldens):
    g = goldens['apply_circuit_doc']
    sim = O.OracleSim(2)
    sim.apply_circuit(Circuit().un(G.H, 2))
    sim.apply_circuit(Circuit().ry('a', 0).ry('b', 1), dict(zip(['a', 'b'], g['pr'])))
    assert np.allclose(sim.qs, _c(g['qs']), atol=1e-12)


def test_grad_docstring(goldens):
    g = goldens['grad_doc']
    circ = Circuit().ry('a', 0)
    res = O.get_expectation_with_grad(1, [Hamiltonian(QubitOperator('Z0'))], circ, np.zeros((1, 0)), [g['p']],
                                      [], ['a'])
    assert np.allclose(res[0, 0, 0], g['f'], atol=1e-8)
    assert np.allclose(res[0, 0, 1], g['g'], atol=1e-8)


def test_sampling_docstring_distribution(goldens):
    """Non-measure-ending circuit: per-shot re-simulation with the reference's mt19937 streams.

    The docstring's exact counts (simulator.py:484) are not reproduced by the restated random
    streams (the docstring is not executed by the reference's tests); the counts are checked
    against the exact outcome probabilities instead, and the generator itself is pinned by
    test_mt19937_known_answer.
    """
    g = goldens['sampling_doc']
    circ = Circuit().ry('a', 0).ry('b', 1)
    circ += G.Measure('q0_0').on(0)
    circ += G.Measure('q0_1').on(0)
    circ += G.Measure('q1').on(1)
    assert not circ.is_measure_end
    shots = 4000
    keys, samples = O.sampling_general(2, circ, g['pr'], shots, g['seed'])
    assert keys == ['q0_0', 'q0_1', 'q1']
    assert np.all(samples[:, 0] == samples[:, 1])
    p0 = np.sin(g['pr']['a'] / 2) ** 2
    p1 = np.sin(g['pr']['b'] / 2) ** 2
    assert abs(samples[:, 0].mean() - p0) < 4 * np.sqrt(p0 * (1 - p0) / shots)
    assert abs(samples[:, 2].mean() - p1) < 4 * np.sqrt(p1 * (1 - p1) / shots)


def test_mt19937_known_answer():
    """The 10000th output of std::mt19937 seeded with 5489 is 4123659995 (C++ standard, [rand.predef])."""
    eng = O._Mt19937(5489)  # pylint: disable=protected-access
    for _ in range(9999):
        eng()
    assert eng() == 4123659995


def test_oracle_matches_dense_matrices():
    """Every gate kind of the oracle against the dense matrix of this package's gate classes."""
    rng = np.random.default_rng(7)
    n = 4
    gates = [G.X.on(1), G.Y.on(2, 0), G.Z.on(3, [0, 1]), G.H.on(0), G.S.on(2), G.S.on(1).hermitian(), G.T.on(3),
             G.SX.on(1, 3), G.SWAP.on([0, 3], 2), G.ISWAP.on([1, 2]), G.ISWAP.on([2, 0]).hermitian(),
             G.RX(0.3).on(2, 1), G.RY(1.1).on(0), G.RZ(-0.4).on(3, 2), G.PhaseShift(0.7).on(1, 0),
             G.GlobalPhase(0.9).on(2), G.Rxx(0.5).on([0, 2]), G.Ryy(0.6).on([3, 1], 0), G.Rzz(0.7).on([1, 3]),
             G.Rxy(0.8).on([2, 0]), G.Rxz(0.9).on([0, 3], 1), G.Ryz(1.0).on([3, 2]), G.Givens(0.4).on([1, 2], 3),
             G.SWAPalpha(0.3).on([0, 1]), G.U3(0.1, 0.2, 0.3).on(2, 3), G.Rn(0.2, -0.5, 0.7).on(1),
             G.FSim(0.6, 0.8).on([2, 3], 0), G.RotPauliString('XYZ', 0.9).on([0, 2, 3], 1)]
    for g in gates:
        v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        v /= np.linalg.norm(v)
        sim = O.OracleSim(n, state=v).apply_circuit(Circuit([g]))
        full = _full_matrix(g, n)
        assert np.allclose(sim.qs, full @ v, atol=1e-12), str(g)


def _full_matrix(g, n):
    m = g.matrix()
    objs, ctrls = g.obj_qubits, g.ctrl_qubits
    k = len(objs)
    dim = 1 << n
    out = np.zeros((dim, dim), dtype=complex)
    for col in range(dim):
        if any(not (col >> c) & 1 for c in ctrls):
            out[col, col] = 1
            continue
        sub = sum(((col >> q) & 1) << b for b, q in enumerate(objs))
        base = col & ~sum(1 << q for q in objs)
        for r in range(1 << k):
            row = base | sum(((r >> b) & 1) << q for b, q in enumerate(objs))
            out[row, col] += m[r, sub]
    return out
