"""Parity of the benchmark configurations themselves with the FP64 oracle (GPU).

* Config 1 exactly: HEA 16 qubits x 8 layers (RY, RZ on every qubit, CNOT ladder), 256
  parameters, the 31-term ZZ + X Hamiltonian, seed 0, complex128: amplitudes within 1e-12,
  <H> and the gradient within 1e-10 of the oracle, through every kernel family (the default
  precompiled tiles, the generated pass kernels and the plain per-gate path).
* The default path of 20 and 22 qubits (generated pass kernels on 12/13-qubit tiles with many
  outside qubits): amplitudes and gradients against the oracle in complex128 (1e-12 / 1e-10)
  and complex64 (2e-6 amplitudes, 1e-5 gradients), for every checkpoint stride in complex64.
* The headline 26-qubit workload (12 layers, 624 parameters, 51 terms): parameter set 0 against
  the oracle's result committed in tests/golden/hea26_oracle.json (made by
  tests/golden/make_oracle_fixtures.py): complex128 within 1e-10, complex64 within 1e-5.
"""
import json
import math
import os

import numpy as np
import pytest
import torch

from mindquantum_b200 import complex64, complex128, workloads as W
from mindquantum_b200.simulator import Simulator
from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _grad(n, dtype, circ, ham, params, stride=None, **kw):
    be = MQVectorB200('mqvector_b200', n, dtype=dtype, **kw)
    f, g = be.expectation_with_grad_tensor([ham], circ, torch.as_tensor(params, device='cuda'), circ.params_name,
                                           ckpt_stride=stride)
    return f[:, 0, 0].cpu().numpy(), g[:, 0].cpu().numpy()


@pytest.mark.parametrize("kernels", [dict(), dict(jit=True), dict(fuse=False)])
def test_config1_exactly_against_oracle(kernels):
    n, layers = 16, 8
    circ, ham, params = W.hea(n, layers, 1, seed=0, encoder=False)
    assert len(circ.params_name) == 256 and len(circ) == 376
    assert len(ham.ham_termlist) == 31
    prd = dict(zip(circ.params_name, params[0].tolist()))
    sim = Simulator('mqvector_b200', n, dtype=complex128, **kernels)
    sim.apply_circuit(circ, prd)
    ref_qs = O.OracleSim(n).apply_circuit(circ, prd).qs
    assert np.max(np.abs(sim.get_qs() - ref_qs)) <= 1e-12
    grad_ops = Simulator('mqvector_b200', n, dtype=complex128, **kernels).get_expectation_with_grad(ham, circ)
    f, g = grad_ops(params[0])
    ref = O.get_expectation_with_grad(n, [ham], circ, np.zeros((1, 0)), params[0], [], circ.params_name)
    assert abs(f[0, 0] - ref[0, 0, 0]) <= 1e-10
    assert np.max(np.abs(g[0, 0] - ref[0, 0, 1:].real)) <= 1e-10


@pytest.mark.parametrize("dtype,atol", [(complex128, 1e-12), (complex64, 2e-6)])
def test_default_generated_path_amplitudes_at_20_qubits(dtype, atol):
    n, layers = 20, 4
    circ, _, params = W.hea(n, layers, 1, seed=1, encoder=False)
    prd = dict(zip(circ.params_name, params[0].tolist()))
    sim = Simulator('mqvector_b200', n, dtype=dtype)
    sim.apply_circuit(circ, prd)
    ref = O.OracleSim(n).apply_circuit(circ, prd).qs
    assert np.max(np.abs(sim.get_qs() - ref)) <= atol


def _strides(n, circ):
    from mindquantum_b200.simulator import lowering

    prog = lowering.lowered(circ, n, 0, circ.params_name, None, True)
    passes = prog.grad_passes(1)[0]
    return [1, max(2, int(math.ceil(math.sqrt(passes)))), 0]


@pytest.mark.parametrize("dtype,tol", [(complex128, 1e-10), (complex64, 1e-5)])
def test_default_generated_path_gradient_at_20_qubits(dtype, tol):
    n, layers = 20, 4
    circ, ham, params = W.hea(n, layers, 2, seed=2, encoder=True)
    ref = O.get_expectation_with_grad(n, [ham], circ, params, np.zeros(0), circ.params_name, [])
    strides = _strides(n, circ) if dtype == complex64 else [None]
    for stride in strides:
        f, g = _grad(n, dtype, circ, ham, params, stride)
        assert np.max(np.abs(f - ref[:, 0, 0].real)) <= tol, stride
        assert np.max(np.abs(g - ref[:, 0, 1:].real)) <= tol, stride


def _fixture(name):
    with open(os.path.join(GOLDEN, name), encoding='utf8') as f:
        return json.load(f)


def _fixture_workload(fx):
    circ, ham, params = W.hea(fx['n_qubits'], fx['layers'], fx['batch'], seed=0, encoder=True)
    assert np.allclose([c for _, c in ham.ham_termlist[:6]], fx['ham_coeff_head'], atol=0, rtol=0)
    for row in fx['samples']:
        assert np.allclose(params[row['sample'], :8], row['params_head'], atol=0, rtol=0)
    return circ, ham, params


@pytest.mark.parametrize("dtype,tol", [(complex128, 1e-10), (complex64, 1e-5)])
def test_hea22_against_oracle_fixture(dtype, tol):
    fx = _fixture('hea22_oracle.json')
    circ, ham, params = _fixture_workload(fx)
    f, g = _grad(fx['n_qubits'], dtype, circ, ham, params)
    for row in fx['samples']:
        s = row['sample']
        assert abs(f[s] - row['f']) <= tol
        assert np.max(np.abs(g[s] - np.array(row['grad']))) <= tol


@pytest.mark.parametrize("dtype,tol", [(complex128, 1e-10), (complex64, 1e-5)])
def test_headline_26_qubits_against_oracle_fixture(dtype, tol):
    fx = _fixture('hea26_oracle.json')
    circ, ham, params = _fixture_workload(fx)
    assert len(circ.params_name) == fx['n_params'] == 624
    row = fx['samples'][0]
    f, g = _grad(fx['n_qubits'], dtype, circ, ham, params[:1])
    assert abs(f[0] - row['f']) <= tol
    assert np.max(np.abs(g[0] - np.array(row['grad']))) <= tol


def _refbin():
    from oracle import refbin as R

    if not R.available():
        pytest.skip("the reference simulator is not built (oracle/_ref)")
    return R


@pytest.mark.parametrize("dtype,tol", [(complex128, 1e-10), (complex64, 1e-5)])
def test_cuda_path_against_the_reference_binary(dtype, tol):
    """The default (generated-kernel) path at 20 qubits against the reference's own CPU simulator
    (built from its sources), HEA and QAOA MaxCut."""
    R = _refbin()
    n = 20
    circ, ham, params = W.hea(n, 4, 2, seed=12, encoder=True)
    ref = R.grad(n, circ, ham, params)
    f, g = _grad(n, dtype, circ, ham, params)
    assert np.max(np.abs(f - ref[:, 0].real)) <= tol
    assert np.max(np.abs(g - ref[:, 1:].real)) <= tol
    circ, ham, pr, _ = W.qaoa_maxcut(n, 2, seed=13)
    ref = R.grad(n, circ, ham, pr[None, :])
    f, g = _grad(n, dtype, circ, ham, pr[None, :])
    scale = max(1.0, float(np.max(np.abs(ref))))   # QAOA values and gradients are O(10): relative bound
    assert abs(f[0] - ref[0, 0].real) <= tol * scale
    assert np.max(np.abs(g[0] - ref[0, 1:].real)) <= tol * scale
