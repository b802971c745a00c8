"""Parity of the B200 kernels (through the C ABI) with the CPU oracle and the reference goldens.

Tolerances: complex128 amplitudes within 1e-12 (the bar for complex128), expectations and
gradients within 1e-10; complex64 (FP32 state, FP64 reductions) within 2e-6 for amplitudes of
small circuits and 1e-4 for gradients.
"""
import numpy as np
import pytest
import torch

from mindquantum_b200 import complex64, complex128
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from mindquantum_b200.simulator import Simulator, inner_product
from oracle import oracle as O
from reference_circuits import (generate_test_circuit, hea_circuit, hea_hamiltonian, mul_qubit_circuit,
                                multi_params_circuit)

pytestmark = pytest.mark.gpu

TOL = {complex128: 1e-12, complex64: 2e-6}
NP = {complex128: np.complex128, complex64: np.complex64}


def _c(a):
    a = np.asarray(a, dtype=float)
    return a[..., 0] + 1j * a[..., 1]


def _all_gates(n, rng):
    """Every gate kind, with and without controls, on random qubits."""
    q = lambda k: [int(x) for x in rng.permutation(n)[:k]]  # noqa: E731
    out = []
    for fuse_ctrl in (False, True):
        def on(g, k):
            qs = q(k + (1 if fuse_ctrl else 0))
            return g.on(qs[:k] if k > 1 else qs[0], qs[k:] if fuse_ctrl else None)
        out += [on(G.X, 1), on(G.Y, 1), on(G.Z, 1), on(G.H, 1), on(G.S, 1), on(G.S, 1).hermitian(), on(G.T, 1),
                on(G.T, 1).hermitian(), on(G.SX, 1), on(G.SX, 1).hermitian(), on(G.SWAP, 2), on(G.ISWAP, 2),
                on(G.ISWAP, 2).hermitian(), on(G.RX(0.3), 1), on(G.RY(1.1), 1), on(G.RZ(-0.4), 1),
                on(G.PhaseShift(0.7), 1), on(G.GlobalPhase(0.9), 1), on(G.Rxx(0.5), 2), on(G.Ryy(0.6), 2),
                on(G.Rzz(0.7), 2), on(G.Rxy(0.8), 2), on(G.Rxz(0.9), 2), on(G.Ryz(1.0), 2), on(G.Givens(0.4), 2),
                on(G.SWAPalpha(0.3), 2), on(G.U3(0.1, 0.2, 0.3), 1), on(G.Rn(0.2, -0.5, 0.7), 1),
                on(G.FSim(0.6, 0.8), 2), on(G.UnivMathGate('u3q', np.linalg.qr(rng.normal(size=(8, 8)) + 1j *
                                                                             rng.normal(size=(8, 8)))[0]), 3),
                on(G.Power(G.X, 0.3), 1)]
        qs = q(4)
        out.append(G.RotPauliString('XZY', 0.9).on(qs[:3], qs[3:] if fuse_ctrl else None))
    return out


@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("fuse", [True, False])
@pytest.mark.parametrize("n", [3, 7, 11])
def test_every_gate_against_oracle(dtype, fuse, n):
    rng = np.random.default_rng(n)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    for g in _all_gates(n, rng):
        sim = Simulator('mqvector_b200', n, dtype=dtype, fuse=fuse)
        sim.set_qs(v)
        sim.apply_circuit(Circuit([g]))
        ref = O.OracleSim(n, np.complex128, v).apply_circuit(Circuit([g])).qs
        assert np.allclose(sim.get_qs(), ref, atol=TOL[dtype], rtol=0), str(g)


@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("n,tile", [(9, 0), (13, 6), (14, 0), (16, 8)])
def test_random_deep_circuit_fused_passes(dtype, n, tile):
    """Many passes with small tiles: qubits move in and out of the tile between passes."""
    from test_host import _random_circuit

    rng = np.random.default_rng(100 + n)
    c = _random_circuit(rng, n, 300)
    prd = {k: float(x) for k, x in zip(c.params_name, rng.uniform(0, 2 * np.pi, len(c.params_name)))}
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    be = MQVectorB200('mqvector_b200', n, dtype=dtype)
    if tile:
        from mindquantum_b200.simulator import lowering

        prog = lowering.lowered(c, n, be.precision, c.params_name, None, True, tile)
        assert prog.info.n_passes > 3
        params = torch.tensor([[prd[k] for k in c.params_name]], dtype=torch.float64, device='cuda')
        st = be.state
        import ctypes

        from mindquantum_b200 import _native as N

        ws_b = ctypes.c_size_t()
        N.call('mqb_apply_workspace_size', prog.handle, 1, ctypes.byref(ws_b))
        ws = torch.empty(ws_b.value, dtype=torch.uint8, device='cuda')
        N.call('mqb_apply', prog.handle, ctypes.c_void_p(st.data_ptr()), 1, ctypes.c_void_p(params.data_ptr()), 0,
               None, ctypes.c_void_p(ws.data_ptr()), ws_b.value, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    else:
        be.apply_circuit(c, prd)
    ref = O.OracleSim(n).apply_circuit(c, prd).qs
    tol = 1e-11 if dtype == complex128 else 5e-6
    assert np.allclose(be.get_qs(), ref, atol=tol, rtol=0)


@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_reference_goldens_through_the_product(goldens, dtype):
    atol = 1e-7 if dtype == complex128 else 1e-5
    g = goldens['all_gate_qs']
    sim = Simulator('mqvector_b200', 3, dtype=dtype)
    sim.apply_circuit(generate_test_circuit(), g['pr'])
    assert np.allclose(sim.get_qs(), _c(g['qs']), atol=atol)

    g = goldens['multi_params']
    circ = multi_params_circuit()
    sim = Simulator('mqvector_b200', 2, dtype=dtype)
    sim.apply_circuit(circ, dict(zip(circ.params_name, g['p0'])))
    assert np.allclose(sim.get_qs(), _c(g['qs']), atol=atol)
    sim.reset()
    ops = sim.get_expectation_with_grad(Hamiltonian(QubitOperator('X0 Y1')), circ)
    f, gr = ops(np.array(g['p0']))
    assert np.allclose(f, _c(g['f']), atol=1e-6)
    assert np.allclose(gr, _c(g['g']), atol=1e-6)

    g = goldens['custom_gate_in_parallel']
    circ = generate_test_circuit().as_encoder()
    hams = [Hamiltonian(QubitOperator('Y0')), Hamiltonian(QubitOperator('X2'))]
    np.random.seed(g['seed'])
    p0 = np.random.uniform(0, 1, size=(2, len(circ.params_name)))
    sim = Simulator('mqvector_b200', 3, dtype=dtype)
    f, gr = sim.get_expectation_with_grad(hams, circ, parallel_worker=4)(p0)
    assert np.allclose(np.sum(f), g['f_sum'], atol=1e-6 if dtype == complex128 else 1e-5)
    assert np.allclose(np.sum(gr), g['g_sum'], atol=1e-6 if dtype == complex128 else 1e-5)

    g = goldens['mul_qubit_gate']
    sim = Simulator('mqvector_b200', 3, dtype=dtype)
    f, gr = sim.get_expectation_with_grad(Hamiltonian(QubitOperator('X0')), mul_qubit_circuit())(np.array([g['p']]))
    assert np.allclose(f, g['f1'], atol=1e-6) and np.allclose(gr, g['g1'], atol=1e-5)

    g = goldens['apply_circuit_doc']
    sim = Simulator('mqvector_b200', 2, dtype=dtype)
    sim.apply_circuit(Circuit().un(G.H, 2))
    sim.apply_circuit(Circuit().ry('a', 0).ry('b', 1), np.array(g['pr']))
    assert np.allclose(sim.get_qs(), _c(g['qs']), atol=1e-12 if dtype == complex128 else 1e-6)

    g = goldens['grad_doc']
    sim = Simulator('mqvector_b200', 1, dtype=dtype)
    f, gr = sim.get_expectation_with_grad(Hamiltonian(QubitOperator('Z0')), Circuit().ry('a', 0))(np.array([g['p']]))
    assert np.allclose(f, g['f'], atol=1e-8) and np.allclose(gr, g['g'], atol=1e-7)


def _oracle_grad(n, hams, circ, enc, ans, dtype=np.complex128, init=None):
    return O.get_expectation_with_grad(n, hams, circ, enc, ans, circ.encoder_params_name, circ.ansatz_params_name,
                                       dtype, init)


@pytest.mark.parametrize("dtype,tol", [(complex128, 1e-10), (complex64, 1e-4)])
@pytest.mark.parametrize("fuse", [True, False])
def test_gradient_against_oracle(dtype, tol, fuse):
    from test_host import _random_circuit

    n = 10
    rng = np.random.default_rng(5)
    circ = _random_circuit(rng, n, 160)
    enc_names = circ.params_name[:7]
    for g in circ:
        for p in g.get_parameters():
            for k in p.params_name:
                if k in enc_names:
                    p.encoder_part(k)
    circ = Circuit(list(circ))
    hams = [Hamiltonian(hea_hamiltonian(n, rng)), Hamiltonian(QubitOperator('Y3 Z5', 0.7) + QubitOperator('X0 X9'))]
    enc = rng.uniform(0, 2 * np.pi, size=(3, len(circ.encoder_params_name)))
    ans = rng.uniform(0, 2 * np.pi, size=len(circ.ansatz_params_name))
    sim = Simulator('mqvector_b200', n, dtype=dtype, fuse=fuse)
    f, ge, ga = sim.get_expectation_with_grad(hams, circ)(enc, ans)
    ref = _oracle_grad(n, hams, circ, enc, ans)
    assert np.allclose(f, ref[:, :, 0], atol=tol, rtol=0)
    ne = len(circ.encoder_params_name)
    assert np.allclose(ge, ref[:, :, 1:1 + ne], atol=tol, rtol=0)
    assert np.allclose(ga, ref[:, :, 1 + ne:], atol=tol, rtol=0)


@pytest.mark.parametrize("stride", [1, 2, 3, 0])
def test_checkpoint_strides_agree(stride):
    n = 14
    rng = np.random.default_rng(9)
    circ = hea_circuit(n, 4).as_encoder()
    ham = Hamiltonian(hea_hamiltonian(n, rng))
    enc = rng.uniform(0, 2 * np.pi, size=(2, len(circ.params_name)))
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    be = MQVectorB200('mqvector_b200', n, dtype=complex128)
    p = torch.as_tensor(enc, device='cuda')
    f, g = be.expectation_with_grad_tensor([ham], circ, p, circ.params_name, ckpt_stride=stride)
    ref = _oracle_grad(n, [ham], circ, enc, np.zeros(0))
    assert np.allclose(f[..., 0].cpu().numpy(), ref[:, :, 0].real, atol=1e-10)
    assert np.allclose(g.cpu().numpy(), ref[:, :, 1:].real, atol=1e-10)


@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_expectation_hamiltonian_and_vdot(dtype):
    n = 12
    rng = np.random.default_rng(3)
    circ = hea_circuit(n, 2)
    prd = dict(zip(circ.params_name, rng.uniform(0, 2 * np.pi, len(circ.params_name))))
    op = hea_hamiltonian(n, rng) + QubitOperator('Y2 X7 Z11', 0.3) + QubitOperator('', 1.5)
    ham = Hamiltonian(op)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    e = sim.get_expectation(ham, circ, pr=prd)
    psi = O.OracleSim(n).apply_circuit(circ, prd).qs
    e_ref = O.expectation_of_terms(psi, psi, n, ham)
    tol = 1e-10 if dtype == complex128 else 1e-5
    assert abs(e - e_ref) < tol
    sim.apply_circuit(circ, prd)
    sim2 = sim.copy()
    sim.apply_hamiltonian(ham)
    lam_ref = O.apply_terms(psi, n, ham)
    assert np.allclose(sim.get_qs(), lam_ref, atol=1e-11 if dtype == complex128 else 1e-5)
    v = inner_product(sim2, sim)
    assert abs(v - np.vdot(psi, lam_ref)) < tol


@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("n", [10, 14, 17])
def test_random_pauli_hamiltonians(dtype, n):
    """Many terms per flip class, Y factors, masks across tile and outside qubits."""
    rng = np.random.default_rng(40 + n)
    op = QubitOperator('', 0.25)
    for _ in range(120):
        w = int(rng.integers(1, 7))
        qs = rng.permutation(n)[:w]
        op += QubitOperator(' '.join(f"{'XYZ'[int(p)]}{int(q)}" for p, q in zip(rng.integers(0, 3, w), qs)),
                            float(rng.normal()))
    for _ in range(60):   # diagonal terms: one large class
        w = int(rng.integers(1, 5))
        op += QubitOperator(' '.join(f'Z{int(q)}' for q in rng.permutation(n)[:w]), float(rng.normal()))
    ham = Hamiltonian(op)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(psi)
    e = sim.get_expectation(ham)
    lam_ref = O.apply_terms(psi, n, ham)
    tol = 1e-10 if dtype == complex128 else 2e-5
    assert abs(e - np.vdot(psi, lam_ref)) < tol
    sim.apply_hamiltonian(ham)
    assert np.allclose(sim.get_qs(), lam_ref, atol=1e-11 if dtype == complex128 else 2e-5, rtol=0)


def test_sampling_matches_reference_algorithm():
    """Measure-ending circuits: same shots as the reference's sampler for the same seed."""
    n = 6
    circ = Circuit().un(G.H, n).rx(0.7, 2).x(3, 1).ry(1.3, 4)
    for q in range(n):
        circ.measure(f'q{q}', q)
    sim = Simulator('mqvector_b200', n, dtype=complex128)
    res = sim.sampling(circ, shots=500, seed=17)
    keys, samples = O.sampling_measure_ending(n, circ, {}, 500, 17)
    order = [keys.index(k) for k in res.keys]
    ref = samples[:, order]
    assert np.array_equal(res.samples, ref)


def test_mid_circuit_measurement_sampling_matches_oracle(goldens):
    g = goldens['sampling_doc']
    circ = Circuit().ry('a', 0).ry('b', 1)
    circ += G.Measure('q0_0').on(0)
    circ += G.Measure('q0_1').on(0)
    circ += G.Measure('q1').on(1)
    sim = Simulator('mqvector_b200', 2)
    res = sim.sampling(circ, g['pr'], shots=200, seed=g['seed'])
    keys, samples = O.sampling_general(2, circ, g['pr'], 200, g['seed'])
    order = [keys.index(k) for k in res.keys]
    assert np.array_equal(res.samples, samples[:, order])


def test_torch_autograd_against_finite_differences():
    from mindquantum_b200.framework import MQOps

    n = 6
    rng = np.random.default_rng(11)
    enc_c = Circuit([G.RX(f'x{i}').on(i) for i in range(n)]).as_encoder()
    ans_c = hea_circuit(n, 2, prefix='w')
    circ = enc_c + ans_c
    hams = [Hamiltonian(QubitOperator(f'Z{i}')) for i in range(3)]
    sim = Simulator('mqvector_b200', n, dtype=complex128)
    op = MQOps(sim.get_expectation_with_grad(hams, circ))
    enc = torch.tensor(rng.uniform(0, np.pi, (4, n)), dtype=torch.float64, requires_grad=True)
    ans = torch.tensor(rng.uniform(0, 2 * np.pi, len(circ.ansatz_params_name)), dtype=torch.float64,
                       requires_grad=True)
    w = torch.tensor(rng.normal(size=(4, 3)), dtype=torch.float64)
    out = op(enc, ans)
    (out * w.to(out.device)).sum().backward()
    eps = 1e-6
    for idx in [(0, 1), (3, 5)]:
        e2 = enc.detach().clone()
        e2[idx] += eps
        e1 = enc.detach().clone()
        e1[idx] -= eps
        fd = ((op(e2, ans.detach()) - op(e1, ans.detach())).cpu() * w).sum() / (2 * eps)
        assert abs(fd.item() - enc.grad[idx].item()) < 1e-6
    for k in [0, 7, len(circ.ansatz_params_name) - 1]:
        a2 = ans.detach().clone()
        a2[k] += eps
        a1 = ans.detach().clone()
        a1[k] -= eps
        fd = ((op(enc.detach(), a2) - op(enc.detach(), a1)).cpu() * w).sum() / (2 * eps)
        assert abs(fd.item() - ans.grad[k].item()) < 1e-6


@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_large_register_properties(dtype):
    """22 qubits (beyond the oracle's comfortable size): norm, U then U^dag, gradient vs finite differences."""
    n = 22
    rng = np.random.default_rng(21)
    circ = hea_circuit(n, 3)
    prd = dict(zip(circ.params_name, rng.uniform(0, 2 * np.pi, len(circ.params_name))))
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.apply_circuit(circ, prd)
    qs = sim.get_qs()
    assert abs(np.linalg.norm(qs) - 1) < (1e-12 if dtype == complex128 else 1e-5)
    sim.apply_circuit(circ.hermitian(), prd)
    back = sim.get_qs()
    assert abs(back[0] - 1) < (1e-11 if dtype == complex128 else 1e-4)
    sim.reset()
    ham = Hamiltonian(hea_hamiltonian(n, rng))
    ops = sim.get_expectation_with_grad(ham, circ)
    p0 = np.array([prd[k] for k in circ.params_name])
    f, g = ops(p0)
    for k in [0, 30, len(p0) - 1]:
        d = np.zeros_like(p0)
        d[k] = 1e-4
        fd = (ops(p0 + d)[0] - ops(p0 - d)[0]).real / 2e-4
        assert abs(fd[0, 0] - g[0, 0, k].real) < (1e-6 if dtype == complex128 else 2e-2)


@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_non_hermitian_gradient_against_dense_matrices(dtype):
    """<phi| U_l^dag H U_r |psi> and its gradient over the parameters of both circuits
    (tests/st/test_simulator/test_method_of_mqvector.py:130-172), against dense matrices built with
    the oracle and central finite differences."""
    from test_host import _random_circuit

    n = 3
    rng = np.random.default_rng(17)
    psi0 = rng.normal(size=8) + 1j * rng.normal(size=8)
    psi0 /= np.linalg.norm(psi0)
    phi0 = rng.normal(size=8) + 1j * rng.normal(size=8)
    phi0 /= np.linalg.norm(phi0)
    fixed = ['h', 'x', 'cx', 'cz', 'swap', 'ccx', 'y']
    circ0 = _random_circuit(rng, n, 40, fixed)
    circ1 = _random_circuit(rng, n, 40, fixed)
    circ_r = circ0 + G.RX({'a': 1, 'b': 2}).on(0) + circ1 + G.RZ('c').on(2, 1)
    circ_l = _random_circuit(rng, n, 30, fixed) + G.RY('c').on(1) + G.Rzz({'d': 0.5}).on([0, 2])
    ham = Hamiltonian(QubitOperator('X0 Y1', 0.3) + QubitOperator('Z2', -1.1) + QubitOperator('Y0 Z1 X2', 0.7))

    def unitary(circ, pr):
        cols = []
        for k in range(8):
            e = np.zeros(8, dtype=np.complex128)
            e[k] = 1
            cols.append(O.OracleSim(n, np.complex128, e).apply_circuit(circ, pr).qs)
        return np.array(cols).T

    eye = np.eye(8, dtype=np.complex128)
    hmat = np.array([O.apply_terms(eye[k].copy(), n, ham) for k in range(8)]).T

    def f_of(pr):
        return phi0.conj() @ unitary(circ_l, pr).conj().T @ hmat @ unitary(circ_r, pr) @ psi0

    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(psi0)
    sim_left = Simulator('mqvector_b200', n, dtype=dtype)
    sim_left.set_qs(phi0)
    ops = sim.get_expectation_with_grad(ham, circ_r, circ_l, sim_left)
    names = ops.ansatz_params_name
    p = rng.uniform(0, 2 * np.pi, len(names))
    f, g = ops(p)
    # the operator leaves both simulators' states as they were
    assert np.allclose(sim.get_qs(), psi0, atol=1e-6) and np.allclose(sim_left.get_qs(), phi0, atol=1e-6)
    pr = dict(zip(names, p))
    tol = 1e-10 if dtype == complex128 else 2e-5
    assert abs(f[0, 0] - f_of(pr)) < tol
    eps = 1e-6
    for k, name in enumerate(names):
        pp, pm = dict(pr), dict(pr)
        pp[name] += eps
        pm[name] -= eps
        fd = (f_of(pp) - f_of(pm)) / (2 * eps)
        assert abs(g[0, 0, k] - fd) < (1e-7 if dtype == complex128 else 5e-5), (name, g[0, 0, k], fd)


def test_qram_operator_matches_oracle():
    """QRamVecOps: a batch of initial states through one ansatz (operations.py:539-664)."""
    from mindquantum_b200.framework import QRamVecOps

    n = 6
    rng = np.random.default_rng(23)
    circ = hea_circuit(n, 2, prefix='w')
    hams = [Hamiltonian(QubitOperator('Z0 Z1')), Hamiltonian(QubitOperator('X3', 0.4) + QubitOperator('Y5'))]
    qs = rng.normal(size=(5, 1 << n)) + 1j * rng.normal(size=(5, 1 << n))
    qs /= np.linalg.norm(qs, axis=1, keepdims=True)
    ans = torch.tensor(rng.uniform(0, 2 * np.pi, len(circ.params_name)), dtype=torch.float64, requires_grad=True)
    sim = Simulator('mqvector_b200', n, dtype=complex128)
    op = QRamVecOps(hams, circ, sim)
    out = op(torch.tensor(qs.real), torch.tensor(qs.imag), ans)
    w = torch.tensor(rng.normal(size=(5, 2)), dtype=torch.float64)
    (out * w).sum().backward()
    g_ref = np.zeros(len(circ.params_name))
    for s in range(5):
        ref = O.get_expectation_with_grad(n, hams, circ, np.zeros((1, 0)), ans.detach().numpy(), [],
                                          circ.params_name, np.complex128, qs[s])
        assert np.allclose(out[s].detach().numpy(), ref[0, :, 0].real, atol=1e-10)
        g_ref += np.einsum('mp,m->p', ref[0, :, 1:].real, w[s].numpy())
    assert np.allclose(ans.grad.numpy(), g_ref, atol=1e-9)


@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_non_hermitian_gradient_batched_encoder(dtype):
    """Three encoder samples through the batched lambda-injection sweeps, each against central
    finite differences of <phi|U_l^dag H U_r|psi> computed with the oracle."""
    n = 3
    rng = np.random.default_rng(29)
    psi0 = rng.normal(size=8) + 1j * rng.normal(size=8)
    psi0 /= np.linalg.norm(psi0)
    circ_r = Circuit([G.RX('x0').on(0), G.RY('x1').on(1), G.X.on(2, 0), G.RZ({'w0': 1.0, 'x0': 0.5}).on(2),
                      G.H.on(1), G.Ryy('w1').on([0, 2])]).as_encoder()
    for g in circ_r:
        for p in g.get_parameters():
            for k in p.params_name:
                if k.startswith('w'):
                    p.ansatz_part(k)
    circ_r = Circuit(list(circ_r))
    circ_l = Circuit([G.H.on(0), G.RX('w1').on(2), G.X.on(1, 2)])
    ham = Hamiltonian(QubitOperator('X0 Z2', 0.6) + QubitOperator('Y1', -0.8))
    hmat = np.array([O.apply_terms(np.eye(8, dtype=np.complex128)[k].copy(), n, ham) for k in range(8)]).T

    def f_of(pr):
        r = O.OracleSim(n, np.complex128, psi0).apply_circuit(circ_r, pr).qs
        l = O.OracleSim(n, np.complex128, psi0).apply_circuit(circ_l, pr).qs
        return np.vdot(l, hmat @ r)

    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(psi0)
    ops = sim.get_expectation_with_grad(ham, circ_r, circ_l)
    enc_names, ans_names = ops.encoder_params_name, ops.ansatz_params_name
    enc = rng.uniform(0, 2 * np.pi, (3, len(enc_names)))
    ans = rng.uniform(0, 2 * np.pi, len(ans_names))
    f, ge, ga = ops(enc, ans)
    tol = 1e-7 if dtype == complex128 else 5e-5
    for s in range(3):
        pr = dict(zip(enc_names, enc[s]))
        pr.update(zip(ans_names, ans))
        assert abs(f[s, 0] - f_of(pr)) < tol
        for k, name in enumerate(enc_names + ans_names):
            pp, pm = dict(pr), dict(pr)
            pp[name] += 1e-6
            pm[name] -= 1e-6
            fd = (f_of(pp) - f_of(pm)) / 2e-6
            got = ge[s, 0, k] if k < len(enc_names) else ga[s, 0, k - len(enc_names)]
            assert abs(got - fd) < (1e-7 if dtype == complex128 else 1e-4), (s, name, got, fd)
