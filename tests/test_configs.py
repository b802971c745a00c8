"""The benchmark workload families at reduced sizes, against the CPU oracle (GPU).

* QNN: RX encoder + RY/RZ/CZ-ring ansatz, several Z_i observables, many samples, gradients of
  the encoder inputs and the shared ansatz weights through torch.autograd.
* QAOA MaxCut on a 3-regular graph: complex64 against complex128, the oracle and central finite
  differences, with every checkpoint stride (all passes, every sqrt(passes), none).
* Uneven batch: circuits of different qubit counts (U3 layers + brick CNOTs, each with its own
  random Pauli Hamiltonian) through one graph-captured CircuitBatch with autotuned tile widths.

Tolerances: complex128 1e-10, complex64 1e-4 (gradients), 1e-5 (expectations).
"""
import numpy as np
import pytest
import torch

from mindquantum_b200 import complex64, complex128, workloads as W
from mindquantum_b200.simulator import Simulator
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GTOL = {complex128: 1e-10, complex64: 1e-4}


def _oracle(n, hams, circ, enc, ans):
    return O.get_expectation_with_grad(n, hams, circ, enc, ans, circ.encoder_params_name, circ.ansatz_params_name,
                                       np.complex128, None)


@pytest.mark.parametrize("dtype", [complex128, complex64])
def test_qnn_autograd_matches_oracle(dtype):
    from mindquantum_b200.framework import MQLayer

    n, layers, samples = 10, 2, 12
    circ, hams, enc, ans = W.qnn(n, layers, samples, n_obs=4, seed=3)
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    layer = MQLayer(sim.get_expectation_with_grad(hams, circ), weight=torch.tensor(ans, dtype=torch.float64))
    x = torch.tensor(enc, dtype=torch.float64, requires_grad=True)
    out = layer(x)
    w = torch.tensor(np.random.default_rng(4).normal(size=(samples, len(hams))), dtype=torch.float64)
    (out * w.to(out.device)).sum().backward()
    ref = _oracle(n, hams, circ, enc, ans)
    assert np.allclose(out.detach().cpu().numpy(), ref[:, :, 0].real, atol=GTOL[dtype], rtol=0)
    ne = len(circ.encoder_params_name)
    g_enc = np.einsum('smp,sm->sp', ref[:, :, 1:1 + ne].real, w.numpy())
    g_ans = np.einsum('smp,sm->p', ref[:, :, 1 + ne:].real, w.numpy())
    assert np.allclose(x.grad.cpu().numpy(), g_enc, atol=GTOL[dtype] * 10, rtol=0)
    assert np.allclose(layer.weight.grad.cpu().numpy(), g_ans, atol=GTOL[dtype] * 10 * samples, rtol=0)


@pytest.mark.parametrize("stride", [1, 2, 0])
def test_qaoa_complex64_against_complex128_oracle_and_fd(stride):
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    n, p = 14, 3
    circ, ham, params, edges = W.qaoa_maxcut(n, p, seed=5)
    assert len(edges) == 3 * n // 2
    names = circ.params_name
    res = {}
    for dt in (complex64, complex128):
        be = MQVectorB200('mqvector_b200', n, dtype=dt)
        f, g = be.expectation_with_grad_tensor([ham], circ, torch.tensor(params[None, :]), names, ckpt_stride=stride)
        res[dt] = (f[0, 0, 0].item(), g[0, 0].cpu().numpy())
    ref = _oracle(n, [ham], circ, np.zeros((1, 0)), params)
    assert abs(res[complex128][0] - ref[0, 0, 0].real) < 1e-10
    assert np.allclose(res[complex128][1], ref[0, 0, 1:].real, atol=1e-10)
    assert abs(res[complex64][0] - res[complex128][0]) < 1e-5
    assert np.max(np.abs(res[complex64][1] - res[complex128][1])) < 1e-4
    # central finite differences of the complex128 expectation
    be = MQVectorB200('mqvector_b200', n, dtype=complex128)
    eps = 1e-5
    for k in (0, len(names) - 1):
        pp, pm = params.copy(), params.copy()
        pp[k] += eps
        pm[k] -= eps
        fp = be.expectation_with_grad_tensor([ham], circ, torch.tensor(pp[None, :]), names)[0][0, 0, 0].item()
        fm = be.expectation_with_grad_tensor([ham], circ, torch.tensor(pm[None, :]), names)[0][0, 0, 0].item()
        assert abs((fp - fm) / (2 * eps) - res[complex128][1][k]) < 1e-6


@pytest.mark.parametrize("dtype", [complex128, complex64])
@pytest.mark.parametrize("graph", [True, False])
def test_uneven_batch_matches_oracle(dtype, graph):
    from mindquantum_b200.simulator.batch import CircuitBatch

    members = W.uneven_u3(6, 6, 11, layers=3, n_terms=10, seed=7)
    batch = CircuitBatch([(n, c, h) for n, c, h, _ in members], dtype=dtype, graph=graph, streams=3)
    for rep in range(2):   # two replays with different parameters
        rng = np.random.default_rng(rep)
        params = [rng.uniform(0, 2 * np.pi, size=len(c.params_name)) for _, c, _, _ in members]
        if rep == 0:   # device tensors out
            fs, gs = batch(params)
            torch.cuda.synchronize()
            fs = [f.cpu().numpy() for f in fs]
            gs = [g.cpu().numpy() for g in gs]
        else:          # host in, host out: one copy each way for the whole batch
            fs, gs = batch.evaluate(params)
        for (n, c, h, _), p, f, g in zip(members, params, fs, gs):
            ref = _oracle(n, [h], c, np.zeros((1, 0)), p)
            assert abs(f[0] - ref[0, 0, 0]) < (1e-10 if dtype == complex128 else 1e-5)
            assert np.allclose(g[0], ref[0, 0, 1:].real, atol=GTOL[dtype], rtol=0)
