"""Noise channels as stochastic trajectories (vector_state.tpp:465-709; channel.py).

Host: the oracle's trajectories average to the channel's Kraus map (written here from the
channel definitions, independent of the oracle), within the statistical error of the sample;
channel argument validation.  GPU: one trajectory on the device equals the oracle's trajectory
with the same seed, draw for draw (complex128 1e-10, complex64 1e-5), over many seeds so every
branch runs; sampling frequencies of noisy circuits against the Kraus map; the noisy
parameter-shift gradient against the oracle's loop with the same simulator stream.
Reference tests: tests/st/test_simulator/test_channel_with_simulator.py:40-230.
"""
import math

import numpy as np
import pytest

from mindquantum_b200 import complex64, complex128
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from mindquantum_b200.simulator import Simulator
from oracle import oracle as O

X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]])
Z = np.diag([1.0 + 0j, -1.0])
I2 = np.eye(2, dtype=complex)


def kraus_of(g):
    """Kraus operators of a single-qubit channel, from its definition."""
    if isinstance(g, G.PauliChannel):
        return [math.sqrt(1 - g.px - g.py - g.pz) * I2, math.sqrt(g.px) * X, math.sqrt(g.py) * Y,
                math.sqrt(g.pz) * Z]
    if isinstance(g, G.DepolarizingChannel):
        return [math.sqrt(1 - 3 * g.p / 4) * I2] + [math.sqrt(g.p / 4) * P for P in (X, Y, Z)]
    if isinstance(g, G.AmplitudeDampingChannel):
        return [np.array([[1, 0], [0, math.sqrt(1 - g.gamma)]]), np.array([[0, math.sqrt(g.gamma)], [0, 0]])]
    if isinstance(g, G.PhaseDampingChannel):
        return [np.array([[1, 0], [0, math.sqrt(1 - g.gamma)]]), np.array([[0, 0], [0, math.sqrt(g.gamma)]])]
    if isinstance(g, G.KrausChannel):
        return list(np.asarray(g.kraus_op, dtype=complex))
    raise TypeError(g)


def _kraus_ops():
    a, b = 0.3, 0.5
    k0 = np.array([[1, 0], [0, math.sqrt(1 - a)]])
    k1 = np.array([[0, math.sqrt(a) * math.sqrt(b)], [0, 0]])
    k2 = np.array([[0, math.sqrt(a) * math.sqrt(1 - b)], [0, 0]])
    return [k0, k1, k2]


CHANNELS = [G.BitFlipChannel(0.3), G.PhaseFlipChannel(0.2), G.BitPhaseFlipChannel(0.4),
            G.PauliChannel(0.1, 0.15, 0.2), G.DepolarizingChannel(0.6), G.AmplitudeDampingChannel(0.35),
            G.PhaseDampingChannel(0.45), G.KrausChannel('k3', _kraus_ops())]


def _rho_avg(g, psi, trajectories, seed0):
    rho = np.zeros((2, 2), dtype=complex)
    for t in range(trajectories):
        qs = O.OracleSim(1, np.complex128, psi).apply_circuit(Circuit([g.on(0)]), {},
                                                               O.UniformStream(seed0 + t)).qs
        rho += np.outer(qs, qs.conj())
    return rho / trajectories


@pytest.mark.parametrize("g", CHANNELS, ids=lambda g: g.name)
def test_oracle_trajectories_average_to_the_kraus_map(g):
    rng = np.random.default_rng(3)
    psi = rng.normal(size=2) + 1j * rng.normal(size=2)
    psi /= np.linalg.norm(psi)
    T = 4000
    rho = _rho_avg(g, psi, T, 100)
    ref = sum(k @ np.outer(psi, psi.conj()) @ k.conj().T for k in kraus_of(g))
    assert np.allclose(np.trace(ref), 1)
    assert np.max(np.abs(rho - ref)) < 5 / math.sqrt(T)


def test_thermal_relaxation_preserves_trace_and_decays():
    psi = np.array([0, 1], dtype=complex)
    g = G.ThermalRelaxationChannel(2.0, 1.5, 0.5)
    rho = _rho_avg(g, psi, 3000, 7)
    assert abs(np.trace(rho) - 1) < 1e-12
    # excited population decays as exp(-t / T1)
    assert abs(rho[1, 1].real - math.exp(-0.5 / 2.0)) < 5 / math.sqrt(3000)


def test_channel_argument_checks():
    with pytest.raises(ValueError):
        G.PauliChannel(0.5, 0.4, 0.3)
    with pytest.raises(ValueError):
        G.AmplitudeDampingChannel(1.5)
    with pytest.raises(TypeError):
        G.PhaseDampingChannel('a')
    with pytest.raises(ValueError):
        G.DepolarizingChannel(1.4)
    with pytest.raises(ValueError, match="completeness"):
        G.KrausChannel('bad', [np.eye(2), np.eye(2)])
    with pytest.raises(ValueError):
        G.ThermalRelaxationChannel(1.0, 2.5, 0.1)
    with pytest.raises(ValueError):
        G.GroupedPauliChannel(np.array([[0.5, 0.4, 0.3]]))
    assert Circuit([G.H.on(0), G.AmplitudeDampingChannel(0.1).on(0)]).is_noise_circuit
    assert not Circuit([G.H.on(0)]).is_noise_circuit


@pytest.mark.parametrize("case", ['qubit', 'ctrl_on_target', 'ctrl_outside', 'batch'])
def test_matrix_abi_rejects_invalid_arguments(case):
    import ctypes
    from mindquantum_b200 import _native as N

    m = np.eye(2, dtype=np.complex128).reshape(4).view(np.float64)
    q, ctrl, batch = 1, 0, 1
    if case == 'qubit':
        q = 3
    elif case == 'ctrl_on_target':
        ctrl = 1 << q
    elif case == 'ctrl_outside':
        ctrl = 1 << 5
    else:
        batch = 0
    with pytest.raises(RuntimeError):
        N.call('mqb_apply_matrix1', 3, N.MQB_PREC_C128, ctypes.c_void_p(16), batch, q, ctrl,
               m.ctypes.data_as(ctypes.c_void_p), None)


@pytest.mark.parametrize("case", ['duplicate_rows', 'row', 'qubit', 'ctrl_on_target', 'ctrl_outside', 'null'])
def test_row_matrix_abi_rejects_invalid_arguments(case):
    """mqb_rows_apply_matrix1 / mqb_rows_matrix1_norm check every request on the host."""
    import ctypes
    from mindquantum_b200 import _native as N

    rows = np.array([0, 2], dtype=np.int64)
    qubits = np.array([1, 0], dtype=np.int32)
    masks = np.zeros(2, dtype=np.uint64)
    mats = np.tile(np.eye(2, dtype=np.complex128).reshape(4), 2).view(np.float64)
    fn = 'mqb_rows_apply_matrix1'
    if case == 'duplicate_rows':
        rows[1] = 0
    elif case == 'row':
        rows[1] = 3
    elif case == 'qubit':
        qubits[0] = 3
    elif case == 'ctrl_on_target':
        masks[0] = 1 << 1
    elif case == 'ctrl_outside':
        masks[1] = 1 << 4
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)   # noqa: E731
    args = [3, N.MQB_PREC_C128, ctypes.c_void_p(16), 3, 2, vp(rows), vp(qubits), vp(masks), vp(mats)]
    if case == 'null':
        args[5] = None
    with pytest.raises(RuntimeError):
        N.call(fn, *args, None)
    if case not in ('duplicate_rows',):   # the norm only reads: one row may be asked twice
        with pytest.raises(RuntimeError):
            N.call('mqb_rows_matrix1_norm', *args, ctypes.c_void_p(64), None)


def test_state_pointers_must_be_16_byte_aligned():
    """Misaligned state buffers are refused on the host, before any device work."""
    import ctypes
    from mindquantum_b200 import _native as N

    with pytest.raises(RuntimeError, match="16-byte aligned"):
        N.call('mqb_vdot', 3, N.MQB_PREC_C128, ctypes.c_void_p(8), ctypes.c_void_p(32), 1, ctypes.c_void_p(64), None)


def noisy_circuit():
    c = Circuit([G.H.on(0), G.RX('a').on(1), G.X.on(2, 0), G.BitFlipChannel(0.3).on(1),
                 G.RY({'b': 2.0}).on(2), G.DepolarizingChannel(0.5, 2).on([0, 2]), G.RZ('a').on(0, 1),
                 G.AmplitudeDampingChannel(0.4).on(1), G.PhaseDampingChannel(0.3).on(2, 0),
                 G.PauliChannel(0.1, 0.2, 0.3).on(0), G.KrausChannel('k3', _kraus_ops()).on(2),
                 G.ThermalRelaxationChannel(2.0, 1.5, 0.7).on(0), G.ThermalRelaxationChannel(1.0, 1.5, 0.4).on(1),
                 G.GroupedPauliChannel(np.array([[0.2, 0.1, 0.1], [0.0, 0.3, 0.2]])).on([1, 2]), G.H.on(1),
                 G.Rzz('c').on([0, 1])])
    return c


class _NumpyRows:
    """MQVectorB200's trajectory driver with its device calls (row-wise 2x2 applies and norms,
    unitary segments) served by numpy and the oracle, so the channel logic runs on the host."""

    def __new__(cls, n):
        from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

        class Host(MQVectorB200):
            def __init__(self):   # pylint: disable=super-init-not-called
                self.n_qubits = n

            def _rows_apply(self, states, rows, mats, q, mask=0):
                mats = np.broadcast_to(np.asarray(mats, dtype=complex), (len(rows), 2, 2))
                for r, m in zip(rows, mats):
                    states[r] = _on(states[r], n, m, q, mask)

            def _rows_norm(self, states, rows, mats, q, mask=0):
                mats = np.broadcast_to(np.asarray(mats, dtype=complex), (len(rows), 2, 2))
                return np.array([float(np.vdot(t, t).real) for t in
                                 (_on(states[r], n, m, q, mask) for r, m in zip(rows, mats))])

            def _apply_segment(self, states, circuit, pr, batch=1):
                for r in range(batch):
                    for g in circuit:
                        O.apply_gate(states[r], n, g, pr)

        return Host()


def _on(psi, n, m, q, mask):
    idx = np.arange(1 << n)
    out = psi.copy()
    i0 = idx[(((idx >> q) & 1) == 0) & ((idx & mask) == mask)]
    i1 = i0 | (1 << q)
    out[i0] = m[0, 0] * psi[i0] + m[0, 1] * psi[i1]
    out[i1] = m[1, 0] * psi[i0] + m[1, 1] * psi[i1]
    return out


@pytest.mark.parametrize("batched", [True, False])
def test_trajectory_driver_follows_the_oracle_draw_for_draw(batched):
    """The trajectory logic of the device driver (every channel and measurement step vectorised
    over the trajectories, its device calls served here by numpy) equals the oracle's shots one by
    one: 200 shots of a circuit with every channel kind and measurements in the middle, all at
    once from read-ahead streams, or one at a time from exact streams.  A controlled damping
    channel leaves the state unnormalised (the reference renormalises by the uncontrolled
    population), so the thermal-relaxation channel after it must take P(q = 0) as the reference
    does, not 1 - P(q = 1)."""
    from mindquantum_b200.simulator.rng import Mt19937Uniform, UniformBlocks, UniformStreams

    circ = _measured_noisy_circuit()
    pr = {'a': 0.7, 'b': -1.3, 'c': 2.1}
    n, shots = 3, 200
    keys, ref = O.sampling_general(n, circ, pr, shots, 29)
    rng = Mt19937Uniform(29)
    seeds = [int(rng.draw(low=1.0, high=float(1 << 20))) for _ in range(shots)]
    host = _NumpyRows(n)
    if batched:
        states = np.zeros((shots, 1 << n), dtype=np.complex128)
        states[:, 0] = 1
        out = host._run_batch(states, circ, pr, UniformBlocks(seeds, block=7))   # pylint: disable=protected-access
        got = np.stack([out[k] for k in keys], axis=1)
    else:
        got = np.zeros_like(ref)
        for s in range(shots):
            states = np.zeros((1, 1 << n), dtype=np.complex128)
            states[0, 0] = 1
            out = host._run_batch(states, circ, pr, UniformStreams([Mt19937Uniform(seeds[s])]))  # pylint: disable=W0212
            got[s] = [out[k][0] for k in keys]
    assert np.array_equal(got, ref), np.where(np.any(got != ref, axis=1))[0]


def test_uniform_blocks_equal_the_streams():
    from mindquantum_b200.simulator.rng import Mt19937Uniform, UniformBlocks

    seeds = [3, 99, 12345]
    blocks = UniformBlocks(seeds, block=5)
    ref = [Mt19937Uniform(x).draw(40) for x in seeds]
    cur = [0, 0, 0]
    rng = np.random.default_rng(0)
    for _ in range(60):
        rows = np.flatnonzero(rng.random(3) < 0.6)
        got = blocks.take(rows)
        for r, v in zip(rows, got):
            if cur[r] < 40:
                assert v == ref[r][cur[r]]
            cur[r] += 1


# ------------------------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_trajectories_match_the_oracle_draw_for_draw(dtype):
    circ = noisy_circuit()
    pr = {'a': 0.7, 'b': -1.3, 'c': 2.1}
    rng = np.random.default_rng(5)
    psi = rng.normal(size=8) + 1j * rng.normal(size=8)
    psi /= np.linalg.norm(psi)
    tol = 1e-10 if dtype == complex128 else 1e-5
    for seed in range(1, 41):
        sim = Simulator('mqvector_b200', 3, dtype=dtype, seed=seed)
        sim.set_qs(psi)
        sim.apply_circuit(circ, pr)
        ref = O.OracleSim(3, np.complex128, psi).apply_circuit(circ, pr, O.UniformStream(seed)).qs
        assert np.allclose(sim.get_qs(), ref, atol=tol, rtol=0), seed


@pytest.mark.gpu
@pytest.mark.parametrize("g", CHANNELS[3:], ids=lambda g: g.name)
def test_noisy_sampling_frequencies(g):
    """test_channel_with_simulator.py: outcome frequencies of channel + measurement."""
    rng = np.random.default_rng(9)
    psi = rng.normal(size=2) + 1j * rng.normal(size=2)
    psi /= np.linalg.norm(psi)
    sim = Simulator('mqvector_b200', 1, dtype=complex128, seed=11)
    sim.set_qs(psi)
    shots = 4000
    res = sim.sampling(Circuit([g.on(0), G.Measure().on(0)]), shots=shots, seed=17)
    p1 = res.data.get('1', 0) / shots
    ref = sum(k @ np.outer(psi, psi.conj()) @ k.conj().T for k in kraus_of(g))
    assert abs(p1 - ref[1, 1].real) < 5 * math.sqrt(0.25 / shots)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_noisy_parameter_shift_matches_the_oracle_loop(dtype):
    circ = Circuit([G.RX('a').on(0), G.AmplitudeDampingChannel(0.3).on(0), G.RY({'b': 2.0}).on(1),
                    G.X.on(1, 0), G.DepolarizingChannel(0.2).on(1), G.RZ('a').on(1), G.U3('c', 0.3, 'd').on(0)])
    hams = [Hamiltonian(QubitOperator('Z0')), Hamiltonian(QubitOperator('X1 Y0', 0.5))]
    p = np.array([0.4, 1.1, -0.7, 2.0])
    sim = Simulator('mqvector_b200', 2, dtype=dtype, seed=23)
    f, g = sim.get_expectation_with_grad(hams, circ)(p)
    ref = O.get_expectation_with_grad_parameter_shift_noisy(2, hams, circ, np.zeros((1, 0)), p, [],
                                                            circ.params_name, O.UniformStream(23))
    tol = 1e-10 if dtype == complex128 else 2e-3
    assert np.allclose(f, ref[:, :, 0], atol=tol, rtol=0)
    assert np.allclose(g, ref[:, :, 1:], atol=tol * (1 if dtype == complex128 else 10), rtol=0)
    with pytest.raises(ValueError, match="noise circuit"):
        sim.get_expectation_with_grad(hams, circ, Circuit([G.H.on(0)]))


def _row_requests(rng, n, batch, count):
    rows = rng.choice(batch, size=count, replace=False)
    qubits = rng.integers(0, n, size=count)
    masks = []
    for q in qubits:
        others = [c for c in range(n) if c != q]
        picked = rng.choice(others, size=int(rng.integers(0, 3)), replace=False)
        masks.append(sum(1 << int(c) for c in picked))
    mats = rng.normal(size=(count, 2, 2)) + 1j * rng.normal(size=(count, 2, 2))
    return rows, qubits, masks, mats


def _numpy_matrix1(psi, n, m, q, mask):
    out = psi.copy()
    idx = np.arange(1 << n)
    sel = ((idx >> q) & 1 == 0) & ((idx & mask) == mask)
    i0 = idx[sel]
    i1 = i0 | (1 << q)
    a, c = psi[i0], psi[i1]
    out[i0] = m[0, 0] * a + m[0, 1] * c
    out[i1] = m[1, 0] * a + m[1, 1] * c
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n,batch,count", [(6, 9, 7), (17, 3, 3), (4, 600, 300)])
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_row_matrix_ops_against_numpy(n, batch, count, dtype):
    """Per-row 2x2 operators (one launch per 256 requests) and their norms against numpy."""
    import ctypes
    import torch
    from mindquantum_b200 import _native as N

    rng = np.random.default_rng(n * 1000 + count)
    psi = rng.normal(size=(batch, 1 << n)) + 1j * rng.normal(size=(batch, 1 << n))
    rows, qubits, masks, mats = _row_requests(rng, n, batch, count)
    prec = N.MQB_PREC_C128 if dtype == complex128 else N.MQB_PREC_C64
    tdt = torch.complex128 if dtype == complex128 else torch.complex64
    st = torch.as_tensor(psi, dtype=tdt, device='cuda').contiguous()
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)   # noqa: E731
    r64 = np.ascontiguousarray(rows, dtype=np.int64)
    q32 = np.ascontiguousarray(qubits, dtype=np.int32)
    m64 = np.ascontiguousarray(masks, dtype=np.uint64)
    mv = np.ascontiguousarray(mats.reshape(count, 4)).view(np.float64)
    args = [n, prec, ctypes.c_void_p(st.data_ptr()), batch, count, vp(r64), vp(q32), vp(m64), vp(mv)]
    out = torch.empty(count, dtype=torch.float64, device='cuda')
    N.call('mqb_rows_matrix1_norm', *args, ctypes.c_void_p(out.data_ptr()), None)
    N.call('mqb_rows_apply_matrix1', *args, None)
    got_norm = out.cpu().numpy()
    got = st.cpu().numpy()
    ref = psi.copy()
    tol = 1e-10 if dtype == complex128 else 2e-4
    for i in range(count):
        ref[rows[i]] = _numpy_matrix1(psi[rows[i]], n, mats[i], qubits[i], masks[i])
        expect = float(np.sum(np.abs(ref[rows[i]]) ** 2))
        assert abs(got_norm[i] - expect) <= tol * expect, i
    assert np.max(np.abs(got - ref)) <= tol * max(1.0, np.max(np.abs(ref)))


def _measured_noisy_circuit():
    c = noisy_circuit()
    c += G.Measure('m0').on(0)
    c += G.AmplitudeDampingChannel(0.2).on(0)
    c += G.Measure('m1').on(1)
    c += G.Measure('m2').on(2)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_noisy_sampling_matches_the_oracle_shot_by_shot(dtype):
    """Every shot of a noisy circuit with measurements in the middle is one trajectory; the shots
    run as one batch, each on its own stream, and equal the oracle's shots one by one."""
    circ = _measured_noisy_circuit()
    pr = {'a': 0.7, 'b': -1.3, 'c': 2.1}
    sim = Simulator('mqvector_b200', 3, dtype=dtype, seed=3)
    res = sim.sampling(circ, pr, shots=80, seed=29)
    keys, ref = O.sampling_general(3, circ, pr, 80, 29)
    got = np.array(res.samples)
    cols = [res.keys_map[k] for k in keys]
    assert np.array_equal(got[:, cols], ref)


@pytest.mark.gpu
def test_batched_trajectories_equal_one_at_a_time(monkeypatch):
    """12 qubits, 200 shots of a layered circuit with a channel on every qubit: the batched run
    (all shots at once) and the run one trajectory at a time give the same outcomes."""
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    n = 12
    c = Circuit()
    for layer in range(2):
        for q in range(n):
            c += G.RY(f'y{layer}_{q}').on(q)
        for q in range(n - 1):
            c += G.X.on(q + 1, q)
        for q in range(n):
            c += G.DepolarizingChannel(0.05).on(q)
            c += G.AmplitudeDampingChannel(0.1).on(q)
        c += G.Measure(f'mid{layer}').on(layer)
    for q in range(n):
        c += G.Measure(f'q{q}').on(q)
    rng = np.random.default_rng(4)
    pr = {k: float(v) for k, v in zip(c.params_name, rng.uniform(-2, 2, len(c.params_name)))}
    a = Simulator('mqvector_b200', n, dtype=complex64, seed=1).sampling(c, pr, shots=200, seed=5)
    monkeypatch.setattr(MQVectorB200, '_trajectory_chunk', lambda self, count: 1)
    b = Simulator('mqvector_b200', n, dtype=complex64, seed=1).sampling(c, pr, shots=200, seed=5)
    assert np.array_equal(np.array(a.samples), np.array(b.samples))
