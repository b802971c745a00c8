"""Hamiltonians given as sparse matrices (HowTo.FRONTEND) and ``.sparse(n)`` (HowTo.BACKEND).

Reference behaviour: mindquantum/core/operators/hamiltonian.py:35-245, ``Csr_Dot_Vec`` /
``ExpectationOfCsr`` (ccsrc/include/core/sparse/algo.h:160-200) and the tests
tests/st/test_simulator/test_method_of_mqvector.py:60-172, test_simulator.py:390-440.

Host: the oracle's CSR restatement equals its Pauli kernels on the same operator (1e-12), the
Hamiltonian modes and their errors, and the C ABI's CSR validation (rejected before any device
work).  GPU: expectations, ``apply_hamiltonian``, Hermitian and non-Hermitian gradients with
CSR Hamiltonians against the oracle and the Pauli path (complex128 1e-10, complex64 1e-5 for
amplitudes and expectations, 1e-4 for gradients), batches above the kernel's four states per
matrix pass, and row lengths that select every lane count of the kernel.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from mindquantum_b200 import _native as N, complex64, complex128, workloads as W
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import Circuit
from mindquantum_b200.core.operators import Hamiltonian, HowTo, QubitOperator
from mindquantum_b200.simulator import Simulator
from oracle import oracle as O
from test_host import _random_circuit

TOL = {complex128: 1e-10, complex64: 1e-5}


def _pauli_and_csr(n, n_terms, seed):
    ham0 = W.random_pauli_hamiltonian(n, n_terms, np.random.default_rng(seed))
    return ham0, Hamiltonian(sp.csr_matrix(ham0.hamiltonian.matrix(n)))


def _random_csr(n, seed, max_row=70):
    """A random complex matrix whose row lengths range over 0..max_row (every lane count)."""
    rng = np.random.default_rng(seed)
    dim = 1 << n
    lens = rng.integers(0, max_row + 1, size=dim)
    lens[rng.integers(dim)] = 0
    rows = np.repeat(np.arange(dim), lens)
    cols = np.concatenate([np.sort(rng.choice(dim, size=k, replace=False)) for k in lens])
    vals = rng.normal(size=rows.size) + 1j * rng.normal(size=rows.size)
    return sp.csr_matrix((vals, (rows, cols)), shape=(dim, dim))


def test_oracle_csr_equals_pauli_kernels():
    n = 6
    ham0, ham2 = _pauli_and_csr(n, 12, 1)
    rng = np.random.default_rng(2)
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    b = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    assert np.allclose(O.apply_terms(a, n, ham2), O.apply_terms(a, n, ham0), atol=1e-12)
    assert abs(O.expectation_of_terms(b, a, n, ham2) - O.expectation_of_terms(b, a, n, ham0)) < 1e-12
    m = _random_csr(n, 3, 20)
    hm = Hamiltonian(m)
    assert np.allclose(O.apply_terms(a, n, hm), m @ a, atol=1e-12)
    assert abs(O.expectation_of_terms(b, a, n, hm) - np.vdot(b, m @ a)) < 1e-12


def test_pauli_csr_builder_matches_dense_matrix():
    for n, seed in ((4, 1), (7, 2)):
        h = W.random_pauli_hamiltonian(n, 15, np.random.default_rng(seed))
        m = W.pauli_csr(h, n)
        assert np.array_equal(m.indptr, np.sort(m.indptr))
        assert np.allclose(m.toarray(), h.hamiltonian.matrix(n), atol=1e-14)


def test_hamiltonian_modes():
    qo = QubitOperator('X0 Y2', 0.5) + QubitOperator('Z1')
    h = Hamiltonian(qo)
    assert h.how_to == HowTo.ORIGIN and h.n_qubits == 3
    assert h.sparse(4) is h and h.how_to == HowTo.BACKEND and h.n_qubits == 4
    with pytest.raises(ValueError, match="Already a sparse"):
        h.sparse(4)
    with pytest.raises(ValueError, match="Can not sparse"):
        Hamiltonian(qo).sparse(2)
    hc = Hamiltonian(sp.csr_matrix(np.eye(8)))
    assert hc.how_to == HowTo.FRONTEND and hc.n_qubits == 3 and hc.dtype == complex128
    assert Hamiltonian(sp.csr_matrix(np.eye(4, dtype=np.complex64))).dtype == complex64
    with pytest.raises(ValueError, match="Pauli term list"):
        _ = hc.ham_termlist
    with pytest.raises(ValueError, match="QubitOperator"):
        _ = hc.hamiltonian
    with pytest.raises(ValueError, match="power of 2"):
        Hamiltonian(sp.csr_matrix(np.eye(6)))
    with pytest.raises(ValueError, match="square"):
        Hamiltonian(sp.csr_matrix(np.ones((4, 8))))
    with pytest.raises(TypeError):
        Hamiltonian(np.eye(4))


def test_sparse_hamiltonian_must_match_the_register():
    sim_err = None
    try:
        sim = Simulator('mqvector_b200', 3)
    except RuntimeError as e:   # no device here: check the qubit rule through the backend class
        sim_err = e
    if sim_err is None:
        with pytest.raises(ValueError, match="not match"):
            sim.get_expectation(Hamiltonian(sp.csr_matrix(np.eye(4))))
        with pytest.raises(ValueError, match="not match"):
            sim.get_expectation(Hamiltonian(QubitOperator('Z0')).sparse(2))


@pytest.mark.parametrize("case", ['indptr_start', 'indptr_end', 'decreasing', 'column', 'qubits'])
def test_csr_abi_rejects_invalid_matrices(case):
    n = 2
    indptr = np.array([0, 1, 2, 3, 4], dtype=np.int64)
    indices = np.array([0, 1, 2, 3], dtype=np.int64)
    data = np.ones(4, dtype=np.complex128)
    nq = n
    if case == 'indptr_start':
        indptr[0] = 1
    elif case == 'indptr_end':
        indptr[-1] = 3
    elif case == 'decreasing':
        indptr[2] = 0
    elif case == 'column':
        indices[2] = 4
    else:
        nq = 0
    h = ctypes.c_void_p()
    with pytest.raises(RuntimeError):
        N.call('mqb_ham_create_csr', nq, N.MQB_PREC_C128, 4, indptr.ctypes.data_as(ctypes.c_void_p),
               indices.ctypes.data_as(ctypes.c_void_p), data.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
    assert not h.value


# ------------------------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_expectation_of_all_three_modes(dtype):
    """test_method_of_mqvector.py:60-113 with the oracle as the reference."""
    n = 3
    rng = np.random.default_rng(4)
    init = rng.normal(size=8) + 1j * rng.normal(size=8)
    init /= np.linalg.norm(init)
    init_l = rng.normal(size=8) + 1j * rng.normal(size=8)
    init_l /= np.linalg.norm(init_l)
    circ = _random_circuit(rng, n, 60, ['h', 'x', 'cx', 'cz', 'swap', 'ccx', 'y'])
    circ_l = _random_circuit(rng, n, 60, ['h', 'x', 'cx', 'cz', 'swap', 'y'])
    ham0, ham2 = _pauli_and_csr(n, 10, 5)
    ham1 = W.random_pauli_hamiltonian(n, 10, np.random.default_rng(5)).sparse(3)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim_l = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(init)
    sim_l.set_qs(init_l)
    psi = O.OracleSim(n, np.complex128, init).apply_circuit(circ).qs
    for left_circ, left_state in ((None, None), (circ_l, None), (None, init_l), (circ_l, init_l)):
        phi = O.OracleSim(n, np.complex128, init if left_state is None else left_state).apply_circuit(
            circ if left_circ is None else left_circ).qs
        ref = np.vdot(phi, O.apply_terms(psi, n, ham0))
        for ham in (ham0, ham1, ham2):
            f = sim.get_expectation(ham, circ, left_circ, sim_l if left_state is not None else None)
            assert abs(f - ref) < TOL[dtype]


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_csr_gradient_and_apply_on_one_qubit(dtype):
    """test_simulator.py:390-440: a 2x2 CSR Hamiltonian, Hermitian and not."""
    circ = Circuit([G.RX('a').on(0), G.RY('b').on(0)])
    ham = Hamiltonian(sp.csr_matrix([[1.0, 2.0], [2.0, 4.0]]), dtype=dtype)
    sim = Simulator('mqvector_b200', 1, dtype=dtype)
    f, g = sim.get_expectation_with_grad(ham, circ)(np.array([1.0, 2.0]))
    ref = O.get_expectation_with_grad(1, [ham], circ, np.zeros((1, 0)), [1.0, 2.0], [], ['a', 'b'])
    assert abs(f[0, 0] - ref[0, 0, 0]) < TOL[dtype]
    assert np.allclose(g[0, 0], ref[0, 0, 1:], atol=10 * TOL[dtype])
    sim.apply_circuit(circ, np.array([1.0, 2.0]))
    sim.apply_hamiltonian(ham)
    u = O.OracleSim(1).apply_circuit(circ, {'a': 1.0, 'b': 2.0}).qs
    assert np.allclose(sim.get_qs(), np.array([[1.0, 2.0], [2.0, 4.0]]) @ u, atol=TOL[dtype])
    # non-Hermitian matrix, left circuit on the same simulator (test_non_hermitian_grad_ops2)
    ham_nh = Hamiltonian(sp.csr_matrix([[1.0, 2.0], [3.0, 4.0]]), dtype=dtype)
    sim2 = Simulator('mqvector_b200', 1, dtype=dtype)
    f, _ = sim2.get_expectation_with_grad(ham_nh, Circuit([G.RY('b').on(0)]), Circuit([G.RX('a').on(0)]))(
        np.array([1.0, 2.0]))
    rx = O.OracleSim(1).apply_circuit(Circuit([G.RX(2.0).on(0)])).qs
    ry = O.OracleSim(1).apply_circuit(Circuit([G.RY(1.0).on(0)])).qs
    assert abs(f[0, 0] - np.vdot(rx, np.array([[1.0, 2.0], [3.0, 4.0]]) @ ry)) < TOL[dtype]


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_non_hermitian_gradient_with_csr(dtype):
    """<phi|U_l^dag A U_r|psi> for a non-Hermitian A: the right sweep uses A^dag."""
    n = 3
    rng = np.random.default_rng(8)
    psi0 = rng.normal(size=8) + 1j * rng.normal(size=8)
    psi0 /= np.linalg.norm(psi0)
    phi0 = rng.normal(size=8) + 1j * rng.normal(size=8)
    phi0 /= np.linalg.norm(phi0)
    circ_r = Circuit([G.H.on(0), G.RX({'a': 1, 'b': 2}).on(0), G.X.on(1, 0), G.RZ('c').on(2, 1), G.RY('a').on(1)])
    circ_l = Circuit([G.H.on(2), G.RY('c').on(1), G.Rzz({'d': 0.5}).on([0, 2])])
    A = _random_csr(n, 6, 5)
    ham = Hamiltonian(A)

    def f_of(pr):
        r = O.OracleSim(n, np.complex128, psi0).apply_circuit(circ_r, pr).qs
        l = O.OracleSim(n, np.complex128, phi0).apply_circuit(circ_l, pr).qs
        return np.vdot(l, A @ r)

    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(psi0)
    sim_l = Simulator('mqvector_b200', n, dtype=dtype)
    sim_l.set_qs(phi0)
    ops = sim.get_expectation_with_grad(ham, circ_r, circ_l, sim_l)
    names = ops.ansatz_params_name
    p = rng.uniform(0, 2 * np.pi, len(names))
    f, g = ops(p)
    pr = dict(zip(names, p))
    assert abs(f[0, 0] - f_of(pr)) < 10 * TOL[dtype]
    for k, name in enumerate(names):
        pp, pm = dict(pr), dict(pr)
        pp[name] += 1e-6
        pm[name] -= 1e-6
        fd = (f_of(pp) - f_of(pm)) / 2e-6
        assert abs(g[0, 0, k] - fd) < (1e-6 if dtype == complex128 else 1e-4), (name, g[0, 0, k], fd)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_csr_gradient_matches_pauli_path_batched(dtype):
    """The same Hamiltonian as Pauli terms and as a CSR matrix: f and gradients of 6 samples (two
    matrix passes of the kernel) agree."""
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200
    import torch

    n = 11
    circ, _, params = W.hea(n, 2, 6, seed=2, encoder=False)
    rng = np.random.default_rng(3)
    ham0 = W.random_pauli_hamiltonian(n, 20, rng)
    ham2 = Hamiltonian(sp.csr_matrix(ham0.hamiltonian.matrix(n)))
    be = MQVectorB200('mqvector_b200', n, dtype=dtype)
    p = torch.as_tensor(params, device='cuda')
    f0, g0 = be.expectation_with_grad_tensor([ham0], circ, p, circ.params_name)
    f2, g2 = be.expectation_with_grad_tensor([ham2], circ, p, circ.params_name)
    assert torch.allclose(f0, f2, atol=TOL[dtype], rtol=0)
    assert torch.allclose(g0, g2, atol=10 * TOL[dtype], rtol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_random_csr_apply_and_expectation_against_oracle(dtype):
    """Row lengths 0..70 (lane counts 1..32), 14 qubits: A psi and <psi|A|psi>."""
    n = 14
    A = _random_csr(n, 10)
    ham = Hamiltonian(A)
    rng = np.random.default_rng(12)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.set_qs(psi)
    f = sim.get_expectation(ham)
    ref = O.expectation_of_terms(psi, psi, n, ham)
    assert abs(f - ref) < 100 * TOL[dtype] * max(1.0, abs(ref))
    sim.apply_hamiltonian(ham)
    out = sim.get_qs()
    ref_v = O.apply_terms(psi, n, ham)
    assert np.allclose(out, ref_v, atol=100 * TOL[dtype], rtol=0)


@pytest.mark.gpu
def test_circuit_batch_with_sparse_matrix_hamiltonians():
    """Graph-captured CircuitBatch members whose Hamiltonians are CSR matrices."""
    from mindquantum_b200.simulator.batch import CircuitBatch

    members = W.uneven_u3(4, 8, 11, layers=2, n_terms=8, seed=3)
    batch = CircuitBatch([(n, c, Hamiltonian(W.pauli_csr(h, n))) for n, c, h, _ in members], dtype=complex128,
                         graph=True, streams=2)
    params = [p for _, _, _, p in members]
    fs, gs = batch(params)
    for (n, c, h, _), p, f, g in zip(members, params, fs, gs):
        ref = O.get_expectation_with_grad(n, [h], c, np.zeros((1, 0)), p, [], c.params_name)
        assert abs(f[0].item() - ref[0, 0, 0]) < 1e-10
        assert np.allclose(g[0].cpu().numpy(), ref[0, 0, 1:].real, atol=1e-10, rtol=0)
