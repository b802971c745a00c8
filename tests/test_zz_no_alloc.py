"""The allocation-free entry point mqb_apply_static against mqb_apply (GPU).

mqb_apply_static serves callers that cannot allocate device memory when they apply a circuit
(a runtime whose device memory is a fixed pool, a binding that only owns the state buffers): it
keeps the per-sample gate matrices in a fixed 4 MiB array inside the library instead of a caller
workspace, and runs the precompiled tile kernels only.  At 18 qubits and more mqb_apply runs the
generated pass kernels instead, so that case compares two kernel families.  This file is collected last so a failure here does not stop the
other tests; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

from mindquantum_b200 import _native as N
from mindquantum_b200.simulator import lowering

pytestmark = pytest.mark.gpu


def _lib():
    L = N.lib()
    L.mqb_apply_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                   ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    L.mqb_apply_static.restype = ctypes.c_int
    return L


STATIC_SCRATCH_BYTES = 4 << 20   # the fixed scratch size stated in include/mqb200.h


def _circuit(n, layers):
    from reference_circuits import hea_circuit

    return hea_circuit(n, layers)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


@pytest.mark.parametrize("n", [14, 18])
@pytest.mark.parametrize("precision,tol", [(N.MQB_PREC_C64, 1e-6), (N.MQB_PREC_C128, 1e-12)])
def test_static_scratch_matches_workspace_path(precision, tol, n):
    L = _lib()
    batch = 3
    circ = _circuit(n, 3)
    names = circ.params_name
    prog = lowering.Program(circ, n, precision, names)
    dt = torch.complex64 if precision == N.MQB_PREC_C64 else torch.complex128
    rng = np.random.default_rng(1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):   # two calls in a row share (and overwrite) the static scratch
        params = torch.as_tensor(rng.uniform(0, 2 * np.pi, (batch, len(names))), device='cuda')
        init = torch.randn(batch, 1 << n, dtype=dt, device='cuda')
        init /= init.abs().pow(2).sum(dim=1, keepdim=True).sqrt()
        ref = init.clone()
        ws_b = ctypes.c_size_t()
        N.call('mqb_apply_workspace_size', prog.handle, batch, ctypes.byref(ws_b))
        ws = torch.empty(ws_b.value, dtype=torch.uint8, device='cuda')
        N.call('mqb_apply', prog.handle, _ptr(ref), batch, _ptr(params), len(names), None, _ptr(ws), ws_b.value,
               stream)
        got = init.clone()
        st = L.mqb_apply_static(prog.handle, _ptr(got), batch, _ptr(params), len(names), None, stream)
        assert st == 0, L.mqb_last_error()
        torch.cuda.synchronize()
        err = (got - ref).abs().max().item()
        assert err <= tol, (call, err)


def test_static_scratch_rejects_oversized_batches():
    L = _lib()
    n = 12
    circ = _circuit(n, 2)
    prog = lowering.Program(circ, n, N.MQB_PREC_C128, circ.params_name)
    need = ctypes.c_size_t()
    N.call('mqb_apply_workspace_size', prog.handle, 1, ctypes.byref(need))
    batch = int(STATIC_SCRATCH_BYTES // max(1, need.value)) + 2
    states = torch.zeros(1, dtype=torch.complex128, device='cuda')   # never touched: rejected on the host
    params = torch.zeros(1, dtype=torch.float64, device='cuda')
    st = L.mqb_apply_static(prog.handle, _ptr(states), batch, _ptr(params), 0, None,
                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == -4
    assert b'exceed the fixed scratch' in L.mqb_last_error()
