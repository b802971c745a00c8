"""The density-matrix backend ``mqmatrix_b200`` against dense density-matrix evolution.

The oracle is the dense restatement in oracle/oracle.py (dm_*): U rho U^dag with the oracle's own
gate kernels, the reference's density-matrix channel maps (cpu_densitymatrix_core_channel.cpp),
Tr(H rho), and the exact derivative of the map's output at every gate holding a parameter, the
quantity the reference's tests check for mqmatrix (tests/st/test_simulator/
test_method_of_mqmatrix.py builds the same dense products).  On pure states without channels the
density-matrix oracle equals the state-vector oracle (checked here), which is pinned to the
reference's own simulator.

Host: the conjugation rules of every parameterized gate, and the channels' superoperators.
GPU: states, channels, expectations and gradients (with and without noise, several Hamiltonians,
encoder batches), apply_hamiltonian, purity / partial trace, sampling; complex128 within 1e-10,
complex64 within 1e-5.
"""
import numpy as np
import pytest

from mindquantum_b200 import complex64, complex128
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from mindquantum_b200.simulator import mqmatrix_b200 as M
from oracle import oracle as O

TOL = {complex128: 1e-10, complex64: 1e-5}


def _rx(x):
    return np.array([[np.cos(x / 2), -1j * np.sin(x / 2)], [-1j * np.sin(x / 2), np.cos(x / 2)]])


def _drx(x):
    return np.array([[np.sin(x / 2), 1j * np.cos(x / 2)], [1j * np.cos(x / 2), np.sin(x / 2)]]) / -2


def _param_gates():
    custom = G.gene_univ_parameterized_gate('crx', _rx, _drx)
    return [G.RX('a'), G.RY('a'), G.RZ('a'), G.PhaseShift('a'), G.GlobalPhase('a'), G.Rxx('a'), G.Ryy('a'),
            G.Rzz('a'), G.Rxy('a'), G.Rxz('a'), G.Ryz('a'), G.Givens('a'), G.SWAPalpha('a'),
            G.U3('a', 'b', 'c'), G.Rn('a', 'b', 'c'), G.FSim('a', 'b'), G.RotPauliString('XYZ', 'a'),
            G.RotPauliString('XZ', 'a'), custom('a')]


@pytest.mark.parametrize("g", _param_gates(), ids=lambda g: g.name)
def test_conjugated_gate_has_the_conjugate_matrix(g):
    pr = {'a': 0.37, 'b': -1.21, 'c': 2.05}
    assert np.allclose(M.conj_gate(g).matrix(pr), np.conj(g.matrix(pr)), atol=1e-14)


def _vec_apply(vec, n2, objs, S):
    """Apply matrix S (index bit b <-> objs[b]) to a 2^n2 vector, in numpy."""
    k = len(objs)
    out = np.zeros_like(vec)
    for i in range(1 << n2):
        r = 0
        for b, q in enumerate(objs):
            r |= ((i >> q) & 1) << b
        base = i
        for q in objs:
            base &= ~(1 << q)
        for c in range(1 << k):
            j = base
            for b, q in enumerate(objs):
                j |= ((c >> b) & 1) << q
            out[i] += S[r, c] * vec[j]
    return out


def _random_dm(n, rng, rank=3):
    vs = rng.normal(size=(rank, 1 << n)) + 1j * rng.normal(size=(rank, 1 << n))
    rho = sum(np.outer(v, v.conj()) for v in vs)
    return rho / np.trace(rho)


def _channels(n, rng):
    kraus = [np.array([[1, 0], [0, np.sqrt(0.7)]]), np.array([[0, np.sqrt(0.3)], [0, 0]])]
    return [G.PauliChannel(0.1, 0.05, 0.2).on(1), G.BitFlipChannel(0.2).on(0), G.PhaseFlipChannel(0.3).on(n - 1),
            G.BitPhaseFlipChannel(0.15).on(1), G.DepolarizingChannel(0.4).on(0),
            G.DepolarizingChannel(0.3, 2).on([1, 0]), G.AmplitudeDampingChannel(0.35).on(1),
            G.AmplitudeDampingChannel(0.35).on(0).hermitian(), G.PhaseDampingChannel(0.45).on(n - 1),
            G.KrausChannel('k', kraus).on(0), G.ThermalRelaxationChannel(100.0, 80.0, 30.0).on(1),
            G.GroupedPauliChannel(np.array([[0.1, 0.0, 0.2], [0.05, 0.1, 0.0]])).on([0, 1])]


def test_channel_superoperators_match_the_density_matrix_maps():
    n = 3
    rng = np.random.default_rng(3)
    for ch in _channels(n, rng):
        rho = _random_dm(n, rng)
        ref = O.dm_apply_channel(rho, n, ch)
        vec = rho.reshape(-1)
        for S, objs in M._superops(ch, n):   # pylint: disable=protected-access
            vec = _vec_apply(vec, 2 * n, objs, S)
        assert np.allclose(vec.reshape(1 << n, 1 << n), ref, atol=1e-12), ch.name


def test_dm_oracle_equals_state_vector_oracle_on_pure_states():
    n = 4
    rng = np.random.default_rng(4)
    circ = _random_circuit(n, 30, rng)
    ham = Hamiltonian(QubitOperator('X0 Z2', 0.6) + QubitOperator('Y1 Y3', -0.8) + QubitOperator('Z0'))
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    p = rng.uniform(0, 2 * np.pi, size=(2, len(circ.params_name)))
    dm = O.dm_expectation_with_grad(n, [ham], circ, p, circ.params_name, np.outer(psi, psi.conj()))
    vec = O.get_expectation_with_grad(n, [ham], circ, p, np.zeros(0), circ.params_name, [], np.complex128, psi)
    assert np.max(np.abs(dm - vec)) <= 1e-12


def _random_circuit(n, n_gates, rng, noise=False):
    names = ['a', 'b', 'c', 'd']
    gates = []
    for _ in range(n_gates):
        k = int(rng.integers(0, 9))
        q = [int(x) for x in rng.permutation(n)[:3]]
        if k == 0:
            gates.append(G.RX(names[int(rng.integers(4))]).on(q[0]))
        elif k == 1:
            gates.append(G.RY({names[int(rng.integers(4))]: float(rng.normal())}).on(q[0], q[1]))
        elif k == 2:
            gates.append(G.RZ(names[int(rng.integers(4))]).on(q[0]))
        elif k == 3:
            gates.append(G.X.on(q[0], q[1]))
        elif k == 4:
            gates.append(G.H.on(q[0]))
        elif k == 5:
            gates.append(G.Rzz(names[int(rng.integers(4))]).on([q[0], q[1]]))
        elif k == 6:
            gates.append(G.U3('a', 'b', float(rng.normal())).on(q[0]))
        elif k == 7:
            gates.append(G.Y.on(q[0]))
        else:
            gates.append(G.S.on(q[0], q[1]))
        if noise and rng.random() < 0.3:
            gates.append(G.DepolarizingChannel(0.05).on(q[0]))
            gates.append(G.AmplitudeDampingChannel(0.1).on(q[1]))
    return Circuit(gates)


# ------------------------------------------------------------------------------------------ GPU
def _dm_sim(n, dtype, rho=None):
    from mindquantum_b200.simulator import Simulator

    sim = Simulator('mqmatrix_b200', n, dtype=dtype, seed=11)
    if rho is not None:
        sim.set_qs(rho)
    return sim


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_apply_circuit_and_channels_against_dense_evolution(dtype):
    n = 4
    rng = np.random.default_rng(10)
    rho0 = _random_dm(n, rng)
    circ = _random_circuit(n, 40, rng)
    prd = {k: float(rng.uniform(0, 2 * np.pi)) for k in circ.params_name}
    sim = _dm_sim(n, dtype, rho0)
    sim.apply_circuit(circ, prd)
    ref = O.dm_apply_circuit(n, circ, prd, rho0)
    assert np.max(np.abs(sim.get_qs() - ref)) <= TOL[dtype]
    for ch in _channels(n, rng):
        sim.apply_circuit(Circuit([ch]))
        ref = O.dm_apply_channel(ref, n, ch)
        assert np.max(np.abs(sim.get_qs() - ref)) <= TOL[dtype] * 10, ch.name
    assert abs(sim.backend.purity() - np.real(np.trace(ref @ ref))) <= TOL[dtype] * 10


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("noise", [False, True])
def test_expectation_with_grad_against_dense_evolution(dtype, noise):
    n = 4
    rng = np.random.default_rng(20 + int(noise))
    rho0 = _random_dm(n, rng)
    circ = _random_circuit(n, 40, rng, noise=noise)
    hams = [Hamiltonian(QubitOperator('X0 Z2', 0.6) + QubitOperator('Y1 Y3', -0.8) + QubitOperator('Z0', 0.3)),
            Hamiltonian(QubitOperator('Y0', 1.1) + QubitOperator('Z1 Z2 X3', 0.4))]
    p = rng.uniform(0, 2 * np.pi, size=len(circ.params_name))
    sim = _dm_sim(n, dtype, rho0)
    f, g = sim.get_expectation_with_grad(hams, circ)(p)
    ref = O.dm_expectation_with_grad(n, hams, circ, p[None, :], circ.params_name, rho0)
    assert np.max(np.abs(f - ref[:, :, 0])) <= TOL[dtype]
    assert np.max(np.abs(g - ref[:, :, 1:].real)) <= TOL[dtype] * 10
    # and the expectation alone
    e = sim.get_expectation(hams[1], circ, pr=dict(zip(circ.params_name, p)))
    assert abs(e - ref[0, 1, 0]) <= TOL[dtype]


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_encoder_batch_gradient(dtype):
    n = 3
    rng = np.random.default_rng(30)
    circ = Circuit([G.RX('x0').on(0), G.RX('x1').on(1), G.RY('w0').on(2), G.X.on(1, 0), G.RZ('w1').on(2, 1),
                    G.DepolarizingChannel(0.1).on(2), G.RY('w0').on(0)])
    circ = Circuit([g for g in circ])
    for g in circ:
        for pr in getattr(g, 'prs', []):
            for k in pr.params_name:
                if k.startswith('x'):
                    pr.encoder_part(k)
    circ = Circuit(list(circ))
    ham = Hamiltonian(QubitOperator('Z0 Z1', 0.5) + QubitOperator('X2', -0.7))
    enc = rng.uniform(0, np.pi, size=(4, 2))
    ans = rng.uniform(0, 2 * np.pi, size=2)
    sim = _dm_sim(n, dtype)
    f, ge, ga = sim.get_expectation_with_grad(ham, circ)(enc, ans)
    rho0 = np.zeros((8, 8), dtype=complex)
    rho0[0, 0] = 1
    names = circ.encoder_params_name + circ.ansatz_params_name
    params = np.concatenate([enc, np.broadcast_to(ans, (4, 2))], axis=1)
    ref = O.dm_expectation_with_grad(n, [ham], circ, params, names, rho0)
    assert np.max(np.abs(f - ref[:, :, 0])) <= TOL[dtype]
    assert np.max(np.abs(ge - ref[:, :, 1:3].real)) <= TOL[dtype] * 10
    assert np.max(np.abs(ga - ref[:, :, 3:].real)) <= TOL[dtype] * 10


@pytest.mark.gpu
def test_apply_hamiltonian_is_h_rho_h():
    n = 3
    rng = np.random.default_rng(40)
    rho0 = _random_dm(n, rng)
    sim = _dm_sim(n, complex128, rho0)
    ham = Hamiltonian(QubitOperator('X0 Y1', 1.0))
    sim.apply_hamiltonian(ham)
    Hm = O.ham_matrix(n, ham)
    assert np.allclose(sim.get_qs(), Hm @ rho0 @ Hm.conj().T, atol=1e-12)


@pytest.mark.gpu
def test_pure_state_utilities_and_sampling():
    n = 3
    sim = _dm_sim(n, complex128)
    circ = Circuit([G.H.on(0), G.X.on(1, 0), G.RY(0.7).on(2)])
    sim.apply_circuit(circ)
    psi = O.OracleSim(n).apply_circuit(circ, {}).qs
    rho = np.outer(psi, psi.conj())
    assert np.allclose(sim.get_qs(), rho, atol=1e-12)
    assert abs(sim.backend.purity() - 1) < 1e-12
    v = sim.backend.get_pure_state_vector()
    assert abs(abs(np.vdot(v, psi)) - 1) < 1e-10
    pt = sim.backend.get_partial_trace([2])
    rt = rho.reshape(2, 2, 2, 2, 2, 2)   # (q2, q1, q0) x (q2, q1, q0)
    assert np.allclose(pt, np.einsum('aijakl->ijkl', rt).reshape(4, 4), atol=1e-12)
    mcirc = Circuit([G.Measure('q0').on(0), G.Measure('q1').on(1), G.Measure('q2').on(2)])
    res = sim.sampling(mcirc, shots=4000, seed=5)
    probs = np.abs(psi) ** 2
    counts = np.zeros(8)
    km = res.keys_map
    for row in res.samples:
        counts[int(row[km['q0']]) | (int(row[km['q1']]) << 1) | (int(row[km['q2']]) << 2)] += 1
    assert np.max(np.abs(counts / 4000 - probs)) < 0.03


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_ten_qubit_pure_gradient_on_the_generated_kernels(dtype):
    """n = 10: the doubled register has 20 qubits, so the default path runs the generated pass
    kernels; on a pure state the density-matrix gradient equals the state-vector oracle's."""
    from mindquantum_b200 import workloads as W

    n = 10
    circ, ham, params = W.hea(n, 2, 2, seed=5, encoder=True)
    sim = _dm_sim(n, dtype)
    f, g = sim.get_expectation_with_grad(ham, circ)(params)
    ref = O.get_expectation_with_grad(n, [ham], circ, params, np.zeros(0), circ.params_name, [])
    assert np.max(np.abs(f - ref[:, :, 0])) <= TOL[dtype]
    assert np.max(np.abs(g - ref[:, :, 1:].real)) <= TOL[dtype] * 10
