"""Precision checks and failure handling of the engine.

Host (no GPU): invalid Hamiltonian tables and invalid arguments of the entry points that take a
bare state are refused with MQB_ERR_INVALID before any device work, and an injected allocation
failure surfaces as MQB_ERR_ALLOC with its message.

GPU:
* the periodic FP64 norm check of the complex64 state (every ceil(sqrt(P)) passes): present for
  every checkpoint stride, within 1e-5 of 1 on a 20-qubit HEA, absent for complex128;
* a deep complex64 circuit whose backward sweep rebuilds every state by reverse application
  (stride 0) against the FP64 oracle (gradients within 1e-4, norm drift within 1e-4);
* determinism: two identical calls agree within 1e-12 (the FP64 gradient slots are summed with
  atomics, so bit equality is not promised);
* a workspace one byte short is refused with MQB_ERR_WORKSPACE; an injected allocation failure
  in the middle of building a program leaves the engine usable.
"""
import ctypes
import math

import numpy as np
import pytest

from mindquantum_b200 import _native as N
from mindquantum_b200 import workloads as W

U64 = ctypes.c_uint64
MQB_ERR_INVALID, MQB_ERR_WORKSPACE, MQB_ERR_ALLOC = -1, -4, -5


def _ham_call(n, prec, mx, my, mz, ny, cf, n_terms):
    L = N.lib()
    out = ctypes.c_void_p()
    arr = lambda t, v: None if v is None else (t * max(1, len(v)))(*v)  # noqa: E731
    st = L.mqb_ham_create(n, prec, arr(U64, mx), arr(U64, my), arr(U64, mz), arr(ctypes.c_int32, ny),
                          arr(ctypes.c_double, cf), n_terms, ctypes.byref(out))
    return st, out, L.mqb_last_error().decode()


def test_ham_create_rejects_bad_tables_on_the_host():
    st, _, msg = _ham_call(4, N.MQB_PREC_C64, [1], [0], [0], [0], [1.0], -1)
    assert st == MQB_ERR_INVALID and 'n_terms' in msg
    st, _, msg = _ham_call(4, N.MQB_PREC_C64, None, [0], [0], [0], [1.0], 1)
    assert st == MQB_ERR_INVALID and 'null' in msg
    st, _, msg = _ham_call(4, 7, [1], [0], [0], [0], [1.0], 1)
    assert st == MQB_ERR_INVALID and 'precision' in msg
    st, _, msg = _ham_call(4, N.MQB_PREC_C64, [1], [1], [0], [1], [1.0], 1)
    assert st == MQB_ERR_INVALID and 'overlapping' in msg
    st, _, msg = _ham_call(4, N.MQB_PREC_C64, [1 << 5], [0], [0], [0], [1.0], 1)
    assert st == MQB_ERR_INVALID and 'outside' in msg


def test_state_entry_points_reject_bad_arguments_on_the_host():
    """The entry points that take a bare state check their arguments before any device work: the
    register (1..40 qubits, a known precision), null pointers, batch and shot counts, qubit and
    outcome ranges.  The pointers below are never dereferenced."""
    L = N.lib()
    p = ctypes.c_void_p(4096)
    sz = ctypes.c_size_t()
    i1, i2 = ctypes.c_int(), ctypes.c_int()
    C64 = N.MQB_PREC_C64

    def err(st, what):
        msg = L.mqb_last_error().decode()
        assert st == MQB_ERR_INVALID and what in msg, (st, msg)

    err(L.mqb_vdot(0, C64, p, p, 1, p, None), 'n_qubits')
    err(L.mqb_vdot(41, C64, p, p, 1, p, None), 'n_qubits')
    err(L.mqb_vdot(3, 7, p, p, 1, p, None), 'precision')
    err(L.mqb_vdot(3, C64, p, p, -1, p, None), 'batch')
    err(L.mqb_sample_scratch_size(0, ctypes.byref(sz)), 'n_qubits')
    err(L.mqb_sample_scratch_size(3, None), 'null')
    err(L.mqb_sample_indices(3, C64, None, p, 1, p, p, 1 << 20, None), 'null')
    err(L.mqb_sample_indices(3, C64, p, p, -1, p, p, 1 << 20, None), 'shots')
    err(L.mqb_sample_indices(3, 9, p, p, 1, p, p, 1 << 20, None), 'precision')
    err(L.mqb_qubit_one_probability(3, C64, p, 3, p, None), 'qubit')
    err(L.mqb_qubit_one_probability(3, C64, None, 0, p, None), 'null')
    err(L.mqb_collapse(3, C64, p, 0, 2, 1.0, None), 'outcome')
    err(L.mqb_collapse(3, C64, None, 0, 1, 1.0, None), 'null')
    err(L.mqb_apply_workspace_size(None, 1, ctypes.byref(sz)), 'null')
    err(L.mqb_grad_workspace_size(None, 1, 1, 1, ctypes.byref(sz)), 'null')
    err(L.mqb_program_grad_passes(None, 1, ctypes.byref(i1), ctypes.byref(i2)), 'null')


def test_injected_allocation_failure_is_reported():
    L = N.lib()
    assert L.mqb_inject_alloc_failure(0) == 0   # the next device allocation fails
    try:
        st, out, msg = _ham_call(4, N.MQB_PREC_C64, [1, 0], [0, 0], [0, 2], [0, 0], [1.0, 0.5], 2)
    finally:
        L.mqb_inject_alloc_failure(-1)
    assert st == MQB_ERR_ALLOC, (st, msg)
    assert 'out of device memory' in msg and not out.value


# ------------------------------------------------------------------------------------------ GPU
def _sim(n, dtype):
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    return MQVectorB200('mqvector_b200', n, dtype=dtype)


@pytest.mark.gpu
def test_norm_checks_of_complex64_for_every_stride():
    import torch

    from mindquantum_b200 import complex64, complex128
    from mindquantum_b200.simulator import lowering

    n, layers = 20, 4
    circ, ham, params = W.hea(n, layers, 2, seed=4, encoder=True)
    prog = lowering.lowered(circ, n, N.MQB_PREC_C64, circ.params_name, None, True)
    P = prog.grad_passes(1)[0]
    sn = max(1, math.ceil(math.sqrt(P)))
    n_fwd = len([q for q in range(1, P + 1) if q % sn == 0 or q == P])
    p = torch.as_tensor(params, device='cuda')
    for stride in (1, max(2, sn), 0):
        sim = _sim(n, complex64)
        sim.expectation_with_grad_tensor([ham], circ, p, circ.params_name, ckpt_stride=stride)
        checks = sim.norm_checks()
        stored = [q for q in range(1, P + 1) if q == P or (stride > 0 and q % stride == 0)]
        n_bwd = len([q for q in range(1, P) if q not in stored and q % sn == 0])
        assert checks.shape == (n_fwd + n_bwd, 2), (stride, checks.shape)
        assert np.max(np.abs(checks - 1.0)) <= 1e-5, (stride, checks)
    sim = _sim(n, complex128)
    sim.expectation_with_grad_tensor([ham], circ, p, circ.params_name, ckpt_stride=0)
    assert sim.norm_checks().shape[0] == 0


@pytest.mark.gpu
def test_deep_complex64_reverse_application_against_oracle():
    import torch

    from mindquantum_b200 import complex64
    from oracle import oracle as O

    n, layers = 16, 24
    circ, ham, params = W.hea(n, layers, 1, seed=6, encoder=True)
    sim = _sim(n, complex64)
    f, g = sim.expectation_with_grad_tensor([ham], circ, torch.as_tensor(params, device='cuda'), circ.params_name,
                                            ckpt_stride=0)
    ref = O.get_expectation_with_grad(n, [ham], circ, params, np.zeros(0), circ.params_name, [])
    assert abs(f[0, 0, 0].item() - ref[0, 0, 0].real) <= 1e-5
    assert np.max(np.abs(g[0, 0].cpu().numpy() - ref[0, 0, 1:].real)) <= 1e-4
    assert sim.norm_drift() <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("dtype_name", ["complex64", "complex128"])
def test_two_identical_calls_agree(dtype_name):
    import torch

    import mindquantum_b200 as M

    dtype = getattr(M, dtype_name)
    n, layers = 18, 3
    circ, ham, params = W.hea(n, layers, 3, seed=8, encoder=True)
    p = torch.as_tensor(params, device='cuda')
    sim = _sim(n, dtype)
    f1, g1 = sim.expectation_with_grad_tensor([ham], circ, p, circ.params_name)
    f2, g2 = sim.expectation_with_grad_tensor([ham], circ, p, circ.params_name)
    assert (f1 - f2).abs().max().item() <= 1e-12
    assert (g1 - g2).abs().max().item() <= 1e-12


@pytest.mark.gpu
def test_workspace_one_byte_short_is_refused():
    import torch

    from mindquantum_b200.core.operators import Hamiltonian  # noqa: F401
    from mindquantum_b200.simulator import lowering

    n = 12
    circ, ham, params = W.hea(n, 2, 2, seed=1, encoder=True)
    prog = lowering.lowered(circ, n, N.MQB_PREC_C64, circ.params_name, None, True)
    h = lowering.native_ham(ham, n, N.MQB_PREC_C64)
    need = ctypes.c_size_t()
    N.call('mqb_grad_workspace_size', prog.handle, 2, 1, 1, ctypes.byref(need))
    ws = torch.empty(need.value, dtype=torch.uint8, device='cuda')
    p = torch.as_tensor(params, device='cuda')
    f = torch.empty((2, 1, 2), dtype=torch.float64, device='cuda')
    g = torch.empty((2, 1, len(circ.params_name)), dtype=torch.float64, device='cuda')
    hams = (ctypes.c_void_p * 1)(h.handle.value)
    L = N.lib()
    st = L.mqb_expectation_with_grad(prog.handle, hams, 1, None, 0, 2, ctypes.c_void_p(p.data_ptr()), p.shape[1],
                                     None, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(g.data_ptr()), 1,
                                     ctypes.c_void_p(ws.data_ptr()), need.value - 1,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == MQB_ERR_WORKSPACE
    assert b'workspace too small' in L.mqb_last_error()


@pytest.mark.gpu
def test_allocation_failure_mid_program_leaves_the_engine_usable():
    from mindquantum_b200.simulator import lowering

    n = 10
    circ, _, _ = W.hea(n, 2, 1, seed=2, encoder=True)
    L = N.lib()
    L.mqb_inject_alloc_failure(2)   # two table uploads succeed, the third fails
    try:
        with pytest.raises(N.NativeError, match='out of device memory'):
            lowering.Program(circ, n, N.MQB_PREC_C64, circ.params_name)
    finally:
        L.mqb_inject_alloc_failure(-1)
    prog = lowering.Program(circ, n, N.MQB_PREC_C64, circ.params_name)
    assert prog.n_gates == len(circ)
