"""Generated pass kernels: compile checks on the host, parity with the oracle on the GPU.

The generated kernels (one per fused pass, compiled with NVRTC) must give the results of the
precompiled tile kernels: complex128 amplitudes within 1e-11 of the oracle, complex64 within
5e-6; gradients within 1e-10 (complex128) and 1e-4 (complex64).
"""
import numpy as np
import pytest
import torch

from mindquantum_b200 import _native as N, complex64, complex128
from mindquantum_b200.simulator import Simulator, lowering
from oracle import oracle as O
from reference_circuits import hea_circuit, hea_hamiltonian
from test_host import _random_circuit


@pytest.mark.parametrize("n,prec,tile,n_hams", [(10, N.MQB_PREC_C64, 0, 0), (11, N.MQB_PREC_C128, 8, 1),
                                               (12, N.MQB_PREC_C64, 9, 2), (10, N.MQB_PREC_C64, 0, 4),
                                               (12, N.MQB_PREC_C64, 0, 1), (11, N.MQB_PREC_C64, 9, 1)])
def test_generated_kernels_compile(n, prec, tile, n_hams):
    rng = np.random.default_rng(n + 10 * n_hams)
    c = _random_circuit(rng, n, 60)
    count = lowering.jit_check(c, n, prec, tile_bits=tile, n_hams=n_hams)
    assert count >= 1


def test_hea_kernels_repeat_across_layers():
    """Layers of the same structure reuse one generated kernel per distinct pass."""
    c = hea_circuit(20, 6)
    count = lowering.jit_check(c, 20, N.MQB_PREC_C64, n_hams=0)
    _, _, qmask, fused = lowering.plan_schedule(c, 20, N.MQB_PREC_C64)
    assert 1 <= count <= int(np.sum(fused))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("n,tile", [(11, 0), (13, 8), (14, 0)])
def test_generated_apply_matches_oracle(dtype, n, tile):
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    rng = np.random.default_rng(200 + n)
    c = _random_circuit(rng, n, 250)
    prd = {k: float(x) for k, x in zip(c.params_name, rng.uniform(0, 2 * np.pi, len(c.params_name)))}
    be = MQVectorB200('mqvector_b200', n, dtype=dtype, jit=True)
    if tile:
        import ctypes

        prog = lowering.lowered(c, n, be.precision, c.params_name, None, True, tile, jit=True)
        params = torch.tensor([[prd[k] for k in c.params_name]], dtype=torch.float64, device='cuda')
        ws_b = ctypes.c_size_t()
        N.call('mqb_apply_workspace_size', prog.handle, 1, ctypes.byref(ws_b))
        ws = torch.empty(max(256, ws_b.value), dtype=torch.uint8, device='cuda')
        N.call('mqb_apply', prog.handle, ctypes.c_void_p(be.state.data_ptr()), 1, ctypes.c_void_p(params.data_ptr()),
               0, None, ctypes.c_void_p(ws.data_ptr()), ws_b.value,
               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    else:
        be.apply_circuit(c, prd)
    ref = O.OracleSim(n).apply_circuit(c, prd).qs
    assert np.allclose(be.get_qs(), ref, atol=1e-11 if dtype == complex128 else 5e-6, rtol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,tol", [(complex128, 1e-10), (complex64, 1e-4)])
@pytest.mark.parametrize("n_hams", [1, 2, 4])
def test_generated_gradient_matches_oracle(dtype, tol, n_hams):
    from mindquantum_b200.core.circuit import Circuit
    from mindquantum_b200.core.operators import Hamiltonian, QubitOperator

    n = 11
    rng = np.random.default_rng(7 + n_hams)
    circ = _random_circuit(rng, n, 150)
    enc_names = circ.params_name[:5]
    for g in circ:
        for p in g.get_parameters():
            for k in p.params_name:
                if k in enc_names:
                    p.encoder_part(k)
    circ = Circuit(list(circ))
    pool = [Hamiltonian(hea_hamiltonian(n, rng)), Hamiltonian(QubitOperator('Y3 Z5', 0.7) + QubitOperator('X0 X9')),
            Hamiltonian(QubitOperator('Z2')), Hamiltonian(QubitOperator('X1 Y4 Z7', -0.3))]
    hams = pool[:n_hams]
    enc = rng.uniform(0, 2 * np.pi, size=(2, len(circ.encoder_params_name)))
    ans = rng.uniform(0, 2 * np.pi, size=len(circ.ansatz_params_name))
    sim = Simulator('mqvector_b200', n, dtype=dtype, jit=True)
    f, ge, ga = sim.get_expectation_with_grad(hams, circ)(enc, ans)
    ref = O.get_expectation_with_grad(n, hams, circ, enc, ans, circ.encoder_params_name, circ.ansatz_params_name,
                                      np.complex128, None)
    ne = len(circ.encoder_params_name)
    assert np.allclose(f, ref[:, :, 0], atol=tol, rtol=0)
    assert np.allclose(ge, ref[:, :, 1:1 + ne], atol=tol, rtol=0)
    assert np.allclose(ga, ref[:, :, 1 + ne:], atol=tol, rtol=0)


@pytest.mark.gpu
def test_generated_and_precompiled_kernels_agree_on_hea():
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200
    from mindquantum_b200.core.operators import Hamiltonian

    n = 18
    rng = np.random.default_rng(3)
    circ = hea_circuit(n, 4)
    ham = Hamiltonian(hea_hamiltonian(n, rng))
    p = torch.as_tensor(rng.uniform(0, 2 * np.pi, size=(2, len(circ.params_name))), device='cuda')
    out = {}
    for jit in (True, False):
        be = MQVectorB200('mqvector_b200', n, dtype=complex64, jit=jit)
        out[jit] = be.expectation_with_grad_tensor([ham], circ, p, circ.params_name)
    assert torch.allclose(out[True][0], out[False][0], atol=1e-5, rtol=0)
    assert torch.allclose(out[True][1], out[False][1], atol=1e-4, rtol=0)
