"""The oracle against the reference's own CPU simulator, built from its sources (oracle/_ref).

The reference (VectorState<CPUVectorPolicyAvxDouble>, its adjoint GetExpectationWithGradMultiMulti
and ApplyCircuit) runs here on the host through oracle/refbin.py; these tests pin the oracle's
restatement to it on the benchmark circuit families at full size where the host finishes in
seconds: config 1 exactly (16 qubits x 8 layers), the QNN encoder/ansatz, QAOA MaxCut and random
Pauli Hamiltonians with Y terms.  Tolerance: 1e-12 (both FP64), complex64 reference within 1e-5.
Both samplers (measurement-ending and mid-circuit) and the noise channels' trajectories are pinned
shot for shot for the same seed; random circuits of every gate kind pin the gate formulas,
Hermitian conjugates and Jacobians; the parameter-shift loop, the QRAM gradient, sparse-matrix
Hamiltonians and the non-Hermitian gradient's convention are pinned to the reference's own entry
points; the dense
density-matrix oracle is pinned to the reference's DensityMatrixState.
Skipped where the reference checkout was not available to build the library.

The reference's thrust GPU simulator (`mqvector_gpu`, VectorState<GPUVectorPolicyDouble/Float>,
built from its sources for sm_100a into oracle/_ref/libmqref_gpu.so) is pinned the same way on a
B200 (marked gpu): FP64 within 1e-10 (its reductions run in another order), complex64 within 1e-5.
"""
import numpy as np
import pytest

from mindquantum_b200 import workloads as W
from oracle import oracle as O
from oracle import refbin as R

pytestmark = pytest.mark.skipif(not R.available(), reason="the reference simulator is not built (oracle/_ref)")


def _oracle(n, circ, ham, params):
    return O.get_expectation_with_grad(n, [ham], circ, params, np.zeros(0), circ.params_name, [])[:, 0]


def test_config1_oracle_equals_reference():
    n, layers = 16, 8
    circ, ham, params = W.hea(n, layers, 1, seed=0, encoder=False)
    ref = R.grad(n, circ, ham, params)
    orc = _oracle(n, circ, ham, params)
    assert np.max(np.abs(ref - orc)) <= 1e-12
    qs = R.apply(n, circ, params[0])
    oqs = O.OracleSim(n).apply_circuit(circ, dict(zip(circ.params_name, params[0].tolist()))).qs
    assert np.max(np.abs(qs - oqs)) <= 1e-12
    ref64 = R.grad(n, circ, ham, params, complex64=True)
    assert np.max(np.abs(ref64 - orc)) <= 1e-5


def test_qnn_oracle_equals_reference():
    n = 12
    circ, hams, enc, ans = W.qnn(n, 3, 3, n_obs=2, seed=11)
    params = np.concatenate([enc, np.broadcast_to(ans, (enc.shape[0], ans.size))], axis=1)
    for ham in hams:
        assert np.max(np.abs(R.grad(n, circ, ham, params) - _oracle(n, circ, ham, params))) <= 1e-12


def test_qaoa_oracle_equals_reference():
    n, p = 12, 3
    circ, ham, pr, _ = W.qaoa_maxcut(n, p, seed=5)
    assert np.max(np.abs(R.grad(n, circ, ham, pr[None, :]) - _oracle(n, circ, ham, pr[None, :]))) <= 1e-12


def test_random_pauli_hamiltonians_oracle_equals_reference():
    n = 12
    rng = np.random.default_rng(21)
    circ, _, params = W.hea(n, 3, 2, seed=3, encoder=True)
    ham = W.random_pauli_hamiltonian(n, 25, rng)
    assert np.max(np.abs(R.grad(n, circ, ham, params) - _oracle(n, circ, ham, params))) <= 1e-12


def test_sampling_oracle_equals_reference():
    """Both samplers shot for shot against the reference's own (its std::mt19937 streams, compiled
    with this image's C++ library): a measurement-ending circuit through
    SamplingMeasurementEndingWithoutNoise, and circuits with mid-circuit and repeated measurements
    through Sampling (one re-simulation per shot)."""
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit

    n = 6
    circ = Circuit().un(G.H, n).rx(0.7, 2).x(3, 1).ry(1.3, 4)
    for q in range(n):
        circ.measure(f'q{q}', q)
    keys, ref = R.sample(n, circ, [], 500, 17, ending=True)
    okeys, orc = O.sampling_measure_ending(n, circ, {}, 500, 17)
    assert keys == okeys and np.array_equal(ref, orc)

    n = 5
    circ = Circuit().un(G.H, n).rx('t', 2).x(3, 1).ry(1.3, 4).rz('u', 0)
    circ.measure('m0', 2)
    circ += G.RX(0.4).on(2)
    circ.measure('m1', 2)
    circ.measure('m2', 0)
    circ += G.H.on(0)
    circ.measure('m3', 0)
    prd = {'t': 0.9, 'u': 1.7}
    keys, ref = R.sample(n, circ, [prd[k] for k in circ.params_name], 300, 1234, ending=False)
    okeys, orc = O.sampling_general(n, circ, prd, 300, 1234)
    assert keys == okeys and np.array_equal(ref, orc)

    # the sampling example of mindquantum/simulator/simulator.py:470-484 (RY(a), RY(b), q0 measured
    # twice): the compiled reference and the oracle agree shot for shot; neither reproduces the
    # docstring's printed counts, which the reference's tests never execute
    circ = Circuit().ry('a', 0).ry('b', 1)
    circ += G.Measure('q0_0').on(0)
    circ += G.Measure('q0_1').on(0)
    circ += G.Measure('q1').on(1)
    keys, ref = R.sample(2, circ, [1.1, 2.2], 100, 42, ending=False)
    okeys, orc = O.sampling_general(2, circ, {'a': 1.1, 'b': 2.2}, 100, 42)
    assert keys == okeys and np.array_equal(ref, orc)


def test_noise_channels_oracle_equals_reference():
    """Noisy trajectories shot for shot against the reference's Sampling, whose shots apply each
    channel with a draw from the shot's stream (ApplyChannel, vector_state.tpp:465-709): one- and
    two-qubit depolarizing, amplitude damping, Pauli, phase damping, thermal relaxation and
    bit-flip channels between gates, then measurements."""
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit

    n = 4
    circ = Circuit().un(G.H, n).rx('t', 2).x(3, 1)
    circ += G.DepolarizingChannel(0.1).on(0)
    circ += G.AmplitudeDampingChannel(0.3).on(1)
    circ += G.PauliChannel(0.05, 0.1, 0.15).on(2)
    circ += G.PhaseDampingChannel(0.2).on(3)
    circ += G.ThermalRelaxationChannel(10.0, 15.0, 3.0).on(1)
    circ += G.BitFlipChannel(0.2).on(3)
    circ += G.DepolarizingChannel(0.3, 2).on([0, 2])
    circ += G.RY(0.8).on(1)
    for q in range(n):
        circ.measure(f'q{q}', q)
    prd = {'t': 0.9}
    keys, ref = R.sample(n, circ, [prd[k] for k in circ.params_name], 400, 99, ending=False)
    okeys, orc = O.sampling_general(n, circ, prd, 400, 99)
    assert keys == okeys and np.array_equal(ref, orc)


@pytest.mark.gpu
@pytest.mark.skipif(not R.available('gpu'), reason="the reference GPU simulator is not built (oracle/_ref)")
def test_reference_gpu_simulator_equals_oracle():
    """Config 1 exactly (16 qubits x 8 layers, T = 31) and a random Pauli Hamiltonian with Y terms on
    the reference's own thrust GPU simulator, against the oracle."""
    n, layers = 16, 8
    circ, ham, params = W.hea(n, layers, 1, seed=0, encoder=False)
    orc = _oracle(n, circ, ham, params)
    assert np.max(np.abs(R.grad(n, circ, ham, params, device='gpu') - orc)) <= 1e-10
    assert np.max(np.abs(R.grad(n, circ, ham, params, complex64=True, device='gpu') - orc)) <= 1e-5
    qs = R.apply(n, circ, params[0], device='gpu')
    oqs = O.OracleSim(n).apply_circuit(circ, dict(zip(circ.params_name, params[0].tolist()))).qs
    assert np.max(np.abs(qs - oqs)) <= 1e-12
    n = 12
    rng = np.random.default_rng(21)
    circ, _, params = W.hea(n, 3, 2, seed=3, encoder=True)
    ham = W.random_pauli_hamiltonian(n, 25, rng)
    assert np.max(np.abs(R.grad(n, circ, ham, params, device='gpu') - _oracle(n, circ, ham, params))) <= 1e-10


def _noisy_dm_circuit(with_tr=True):
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit

    circ = Circuit().un(G.H, 4).rx('t', 2).x(3, 1).ry('u', 0)
    circ += G.DepolarizingChannel(0.1).on(0)
    circ += G.AmplitudeDampingChannel(0.3).on(1)
    circ += G.PauliChannel(0.05, 0.1, 0.15).on(2)
    circ += G.RZ('t').on(1)
    circ += G.PhaseDampingChannel(0.2).on(3)
    if with_tr:
        circ += G.ThermalRelaxationChannel(10.0, 15.0, 3.0).on(1)
    circ += G.BitFlipChannel(0.2).on(3)
    circ += G.DepolarizingChannel(0.3, 2).on([0, 2])
    circ += G.RY('v').on(1)
    circ += G.X.on(2, 0)
    return circ


def test_density_matrix_oracle_equals_reference():
    """The dense density-matrix oracle against the reference's DensityMatrixState compiled from its
    sources: rho after gates and every channel kind (1e-12), the reversible gradient of a noiseless
    circuit and the noise gradient (GetExpectationWithNoiseGrad) with depolarizing, amplitude
    damping (daggered in the Hermitian circuit), Pauli, phase damping and bit-flip channels
    (1e-12)."""
    from mindquantum_b200.core.operators import Hamiltonian, QubitOperator

    n = 4
    ham = Hamiltonian(QubitOperator('Z0 Z1', 0.7) + QubitOperator('X2', -0.4) + QubitOperator('Y3 Y1', 0.25))
    rho0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rho0[0, 0] = 1
    prd = {'t': 0.9, 'u': -0.4, 'v': 1.3}
    circ = _noisy_dm_circuit(with_tr=True)
    names = list(circ.params_name)
    p = np.array([[prd[k] for k in names]])
    assert np.max(np.abs(R.dm_apply(n, circ, p[0]) - O.dm_apply_circuit(n, circ, prd, rho0))) <= 1e-12
    for c in (_noisy_dm_circuit(with_tr=False), type(circ)([g for g in circ if not O.is_channel(g)])):
        ref = R.dm_grad(n, c, ham, p)
        orc = O.dm_expectation_with_grad(n, [ham], c, p, names, rho0)[:, 0]
        assert np.max(np.abs(ref - orc)) <= 1e-12


def test_density_matrix_thermal_relaxation_gradient_is_the_derivative():
    """With a thermal-relaxation channel after a parameterized gate, the reference's noise gradient
    is not the derivative of its own expectation: its Hermitian circuit keeps the channel itself
    where the backward sweep needs the channel's adjoint (the C++ channel has no daggered form,
    unlike amplitude damping).  The oracle, which the B200 backend follows, returns the
    derivative: it matches central finite differences of the reference's own f."""
    from mindquantum_b200.core.operators import Hamiltonian, QubitOperator

    n = 4
    ham = Hamiltonian(QubitOperator('Z0 Z1', 0.7) + QubitOperator('X2', -0.4) + QubitOperator('Y3 Y1', 0.25))
    rho0 = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rho0[0, 0] = 1
    circ = _noisy_dm_circuit(with_tr=True)
    names = list(circ.params_name)
    prd = {'t': 0.9, 'u': -0.4, 'v': 1.3}
    p = np.array([[prd[k] for k in names]])
    ref = R.dm_grad(n, circ, ham, p)[0, 1:].real
    orc = O.dm_expectation_with_grad(n, [ham], circ, p, names, rho0)[0, 0, 1:].real
    h = 1e-5
    fd = np.array([(R.dm_grad(n, circ, ham, p + h * e)[0, 0] - R.dm_grad(n, circ, ham, p - h * e)[0, 0]).real / (2 * h)
                   for e in np.eye(len(names))[:, None, :]])
    assert np.max(np.abs(orc - fd)) <= 1e-8
    assert np.max(np.abs(ref - fd)) > 1e-3     # the reference's divergence (0.028 on 'u' here)


def _every_gate_circuit(n, n_gates, seed, with_rn=True, fixed=False):
    """Random gates of every kind the reference's VectorState applies: fixed one- and two-qubit
    gates and their daggers, one-parameter rotations, U3 / Rn / FSim with angles sharing a
    parameter, controls on a third of them; angles coeff * p + const."""
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit
    from mindquantum_b200.core.parameterresolver import ParameterResolver

    rng = np.random.default_rng(seed)
    names = [f'p{i}' for i in range(6)]

    def pr(k):
        if fixed:   # numeric angles only
            return float(rng.uniform(-3, 3))
        return ParameterResolver({k: float(rng.uniform(0.5, 2))}, const=float(rng.uniform(-1, 1)))

    one = [G.X, G.Y, G.Z, G.H, G.S, G.T, G.SX]
    p1 = [G.RX, G.RY, G.RZ, G.PhaseShift, G.GlobalPhase]
    p2 = [G.Rxx, G.Ryy, G.Rzz, G.Rxy, G.Rxz, G.Ryz, G.Givens, G.SWAPalpha]
    circ = Circuit()
    for _ in range(n_gates):
        q = [int(x) for x in rng.permutation(n)[:3]]
        kind = int(rng.integers(7))
        if kind == 5 and not with_rn:
            kind = 4
        ctrl = [q[2]] if rng.random() < 0.3 else []
        k = names[int(rng.integers(len(names)))]
        if kind == 0:
            g = one[int(rng.integers(len(one)))]
            circ += (g.hermitian() if rng.random() < 0.5 else g).on(q[0], ctrl)
        elif kind == 1:
            g = (G.SWAP, G.ISWAP)[int(rng.integers(2))]
            circ += (g.hermitian() if rng.random() < 0.5 else g).on(q[:2], ctrl)
        elif kind == 2:
            circ += p1[int(rng.integers(len(p1)))](pr(k)).on(q[0], ctrl)
        elif kind == 3:
            circ += p2[int(rng.integers(len(p2)))](pr(k)).on(q[:2], ctrl)
        elif kind == 4:
            circ += G.U3(pr(k), pr(k), pr(k)).on(q[0], ctrl)
        elif kind == 5:
            circ += G.Rn(pr(k), pr(k), pr(k)).on(q[0], ctrl)
        else:
            circ += G.FSim(pr(k), pr(k)).on(q[:2], ctrl)
    return circ


@pytest.mark.parametrize("seed", [5, 6])
def test_every_gate_kind_oracle_equals_reference(seed):
    """The oracle's gate formulas, Hermitian conjugates and Jacobians against the reference's own
    ApplyCircuit and adjoint gradient on a random 120-gate circuit of every gate kind at 8 qubits
    (amplitudes 1e-12, f and gradients 1e-12)."""
    n = 8
    circ = _every_gate_circuit(n, 120, seed)
    names = list(circ.params_name)
    vals = np.random.default_rng(seed).uniform(0, 2 * np.pi, len(names))
    qs = R.apply(n, circ, vals)
    oqs = O.OracleSim(n).apply_circuit(circ, dict(zip(names, vals.tolist()))).qs
    assert np.max(np.abs(qs - oqs)) <= 1e-12
    ham = W.random_pauli_hamiltonian(n, 12, np.random.default_rng(seed + 100))
    ref = R.grad(n, circ, ham, vals[None, :])
    orc = O.get_expectation_with_grad(n, [ham], circ, vals[None, :], np.zeros(0), names, [])[:, 0]
    assert np.max(np.abs(ref - orc)) <= 1e-12


def test_parameter_shift_oracle_equals_reference():
    """The oracle's parameter-shift loop against the reference's own
    GetExpectationWithGradParameterShiftMultiMulti on random circuits of every gate kind that rule
    supports (Rn is refused there), two parameter rows, angles sharing parameters (where the
    reference's shift rule departs from the derivative, the oracle follows it): 1e-11."""
    n = 6
    circ = _every_gate_circuit(n, 40, 9, with_rn=False)
    names = list(circ.params_name)
    vals = np.random.default_rng(1).uniform(0, 2 * np.pi, (2, len(names)))
    ham = W.random_pauli_hamiltonian(n, 8, np.random.default_rng(2))
    ref = R.grad_pshift(n, circ, ham, vals)
    orc = O.get_expectation_with_grad_parameter_shift(n, [ham], circ, vals, [], names, [])[:, 0]
    assert np.max(np.abs(ref - orc)) <= 1e-11


def test_non_hermitian_gradient_convention_of_the_reference():
    """<phi| U_l^dag H U_r(p) |psi> with circ_left and simulator_left: the reference's own
    GetExpectationNonHermitianWithGradMultiMulti returns f (complex, equal to the oracle's states
    and Hamiltonian within 1e-12) and the complex derivative df/dp (central differences of the
    oracle's f, 1e-7), the quantity the B200 backend's non-Hermitian GPU tests expect."""
    n = 5
    rng = np.random.default_rng(3)
    circ = _every_gate_circuit(n, 30, 11)
    left = _every_gate_circuit(n, 20, 12, fixed=True)
    names = list(circ.params_name)
    vals = rng.uniform(0, 2 * np.pi, (1, len(names)))
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    phi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi, phi = psi / np.linalg.norm(psi), phi / np.linalg.norm(phi)
    ham = W.random_pauli_hamiltonian(n, 8, np.random.default_rng(4))
    ref = R.grad_nonherm(n, circ, left, ham, vals, psi, phi)[0]
    bra = O.OracleSim(n, state=phi).apply_circuit(left, {}).qs

    def f(p):
        ket = O.OracleSim(n, state=psi).apply_circuit(circ, dict(zip(names, p.tolist()))).qs
        return np.vdot(bra, O.apply_terms(ket, n, ham))

    assert abs(ref[0] - f(vals[0])) <= 1e-12
    h = 1e-6
    fd = np.array([(f(vals[0] + h * e) - f(vals[0] - h * e)) / (2 * h) for e in np.eye(len(names))])
    assert np.max(np.abs(ref[1:] - fd)) <= 1e-7


def test_qram_oracle_equals_reference():
    """Per-sample initial states through one ansatz: the oracle's driver with an initial state
    against the reference's own QramExpectationWithGrad (1e-12), on a circuit of every gate kind."""
    n = 5
    rng = np.random.default_rng(23)
    circ = _every_gate_circuit(n, 30, 13)
    names = list(circ.params_name)
    ans = rng.uniform(0, 2 * np.pi, len(names))
    qs = rng.normal(size=(3, 1 << n)) + 1j * rng.normal(size=(3, 1 << n))
    qs /= np.linalg.norm(qs, axis=1, keepdims=True)
    ham = W.random_pauli_hamiltonian(n, 8, np.random.default_rng(24))
    ref = R.grad_qram(n, circ, ham, ans, qs)
    for s in range(3):
        orc = O.get_expectation_with_grad(n, [ham], circ, np.zeros((1, 0)), ans, [], names, np.complex128, qs[s])
        assert np.max(np.abs(ref[s] - orc[0, 0])) <= 1e-12


def test_sparse_matrix_hamiltonian_oracle_equals_reference():
    """A Hamiltonian given as a scipy CSR matrix (Hermitian, random rows of 0..20 entries, and the
    CSR form of a Pauli sum): the oracle's Csr_Dot_Vec / ExpectationOfCsr path against the
    reference's own gradient with its CsrHdMatrix Hamiltonian (1e-12)."""
    import scipy.sparse as sp

    from mindquantum_b200.core.operators import Hamiltonian

    n = 6
    rng = np.random.default_rng(31)
    dim = 1 << n
    lens = rng.integers(0, 21, size=dim)
    rows = np.repeat(np.arange(dim), lens)
    cols = np.concatenate([np.sort(rng.choice(dim, size=k, replace=False)) for k in lens])
    m = sp.csr_matrix((rng.normal(size=rows.size) + 1j * rng.normal(size=rows.size), (rows, cols)), shape=(dim, dim))
    circ = _every_gate_circuit(n, 30, 17)
    names = list(circ.params_name)
    vals = rng.uniform(0, 2 * np.pi, (2, len(names)))
    for mat in ((m + m.conj().T).tocsr(), W.pauli_csr(W.random_pauli_hamiltonian(n, 10, rng), n)):
        ref = R.grad_csr(n, circ, mat, vals)
        orc = O.get_expectation_with_grad(n, [Hamiltonian(mat)], circ, vals, np.zeros(0), names, [])[:, 0]
        assert np.max(np.abs(ref - orc)) <= 1e-12


def test_hea22_fixture_equals_reference():
    """The committed FP64 fixture of the 22-qubit x 6-layer HEA workload (made by the oracle, used
    by the GPU tests) against the reference's own adjoint gradient, both parameter rows (1e-12)."""
    import json
    import os

    with open(os.path.join(os.path.dirname(__file__), 'golden', 'hea22_oracle.json'), encoding='utf8') as f:
        fx = json.load(f)
    circ, ham, params = W.hea(fx['n_qubits'], fx['layers'], fx['batch'], seed=0, encoder=True)
    ref = R.grad(fx['n_qubits'], circ, ham, params)
    for row in fx['samples']:
        s = row['sample']
        assert abs(ref[s, 0].real - row['f']) <= 1e-12
        assert np.max(np.abs(ref[s, 1:].real - np.array(row['grad']))) <= 1e-12
