"""The autograd operators and layers (mindquantum_b200.framework) on the host, with stand-in
grad operators whose expectations and gradients are known in closed form.

* The callable path (non-Hermitian, parameter-shift and density-matrix operators): the operator
  returns the reference's layout, f[s][m] complex and its complex derivatives, for
  f[s][m] = sum_p A[m][p] exp(i x_p) with x = (encoder row s, ansatz); MQ*Ops give Re f and the
  MQN2*Ops |f|^2 (mindquantum/framework/operations.py), checked with torch.autograd.gradcheck in
  the encoder + ansatz, encoder-only and ansatz-only forms.
* The device path (``device_grad``, the Hermitian adjoint operator of the state-vector backend):
  f = sum_p A[m][p] cos(x_p) as (re, im) pairs and its real gradient, checked the same way.
* The layers hold the ansatz weights and reject weights of the wrong shape.
"""
import numpy as np
import pytest
import torch

from mindquantum_b200.framework import (MQAnsatzOnlyLayer, MQAnsatzOnlyOps, MQEncoderOnlyOps, MQLayer,
                                        MQN2AnsatzOnlyLayer, MQN2AnsatzOnlyOps, MQN2EncoderOnlyOps, MQN2Layer,
                                        MQN2Ops, MQOps)


class _StandIn:
    """A grad operator with the reference's call forms: (enc, ans) -> (f, g_enc, g_ans), (enc) ->
    (f, g) or (ans) -> (f, g)."""

    def __init__(self, n_enc, n_ans, n_hams=2, seed=0, device_path=False):
        rng = np.random.default_rng(seed)
        self.A = rng.normal(size=(n_hams, n_enc + n_ans)) + (0 if device_path else 1j) * rng.normal(
            size=(n_hams, n_enc + n_ans))
        self.encoder_params_name = [f'e{i}' for i in range(n_enc)]
        self.ansatz_params_name = [f'a{i}' for i in range(n_ans)]
        self.device_grad = self._device if device_path else None
        self.sim = type('Sim', (), {'device': torch.device('cpu')})()
        self.calls = 0

    def _x(self, enc, ans):
        n_enc = len(self.encoder_params_name)
        enc = np.zeros((1, 0)) if enc is None else np.asarray(enc, dtype=np.float64).reshape(-1, n_enc)
        ans = np.zeros(0) if ans is None else np.asarray(ans, dtype=np.float64).reshape(-1)
        return np.concatenate([enc, np.broadcast_to(ans, (enc.shape[0], ans.size))], axis=1)

    def __call__(self, *inputs):
        self.calls += 1
        n_enc, n_ans = len(self.encoder_params_name), len(self.ansatz_params_name)
        if n_enc and n_ans:
            x = self._x(inputs[0], inputs[1])
        elif n_enc:
            x = self._x(inputs[0], None)
        else:
            x = self._x(None, inputs[0])
        f = np.einsum('mp,sp->sm', self.A, np.exp(1j * x))
        g = 1j * self.A[None, :, :] * np.exp(1j * x)[:, None, :]
        if n_enc and n_ans:
            return f, g[:, :, :n_enc], g[:, :, n_enc:]
        return f, g

    def _device(self, params):
        self.calls += 1
        x = params.numpy()
        f = np.einsum('mp,sp->sm', self.A.real, np.cos(x))
        g = -self.A.real[None, :, :] * np.sin(x)[:, None, :]
        return torch.as_tensor(np.stack([f, np.zeros_like(f)], axis=-1)), torch.as_tensor(g)


def _inputs(n_enc, n_ans, seed=1):
    rng = np.random.default_rng(seed)
    enc = torch.tensor(rng.uniform(0, 6, (3, n_enc)), dtype=torch.float64, requires_grad=True)
    ans = torch.tensor(rng.uniform(0, 6, n_ans), dtype=torch.float64, requires_grad=True)
    return enc, ans


@pytest.mark.parametrize("device_path", [False, True])
@pytest.mark.parametrize("ops_cls,square", [(MQOps, False), (MQN2Ops, True)])
def test_encoder_ansatz_ops(device_path, ops_cls, square):
    op = _StandIn(3, 4, device_path=device_path)
    enc, ans = _inputs(3, 4)
    net = ops_cls(op)
    out = net(enc, ans)
    x = op._x(enc.detach().numpy(), ans.detach().numpy())  # pylint: disable=protected-access
    f = np.einsum('mp,sp->sm', op.A.real if device_path else op.A, np.cos(x) if device_path else np.exp(1j * x))
    ref = np.abs(f) ** 2 if square else f.real
    assert out.shape == (3, 2) and np.allclose(out.detach().numpy(), ref, atol=1e-12)
    assert torch.autograd.gradcheck(lambda e, a: ops_cls(op)(e, a), (enc, ans), eps=1e-6, atol=1e-7)


@pytest.mark.parametrize("ops_cls", [MQEncoderOnlyOps, MQN2EncoderOnlyOps])
def test_encoder_only_ops(ops_cls):
    op = _StandIn(4, 0)
    enc, _ = _inputs(4, 0)
    assert torch.autograd.gradcheck(lambda e: ops_cls(op)(e), (enc,), eps=1e-6, atol=1e-7)


@pytest.mark.parametrize("ops_cls", [MQAnsatzOnlyOps, MQN2AnsatzOnlyOps])
def test_ansatz_only_ops(ops_cls):
    op = _StandIn(0, 5)
    _, ans = _inputs(0, 5)
    out = ops_cls(op)(ans)
    assert out.shape == (1, 2)
    assert torch.autograd.gradcheck(lambda a: ops_cls(op)(a), (ans,), eps=1e-6, atol=1e-7)


def test_layers_train_their_weights():
    op = _StandIn(3, 4)
    enc, _ = _inputs(3, 4)
    for cls in (MQLayer, MQN2Layer):
        layer = cls(op, weight=torch.zeros(4, dtype=torch.float64))
        layer(enc.detach()).sum().backward()
        assert layer.weight.grad is not None and layer.weight.grad.shape == (4,)
    op2 = _StandIn(0, 4)
    for cls in (MQAnsatzOnlyLayer, MQN2AnsatzOnlyLayer):
        layer = cls(op2, weight=torch.ones(4, dtype=torch.float64))
        layer().sum().backward()
        assert layer.weight.grad.shape == (4,)
    with pytest.raises(ValueError, match="Weight init shape"):
        MQLayer(op, weight=torch.zeros(5))


@pytest.mark.gpu
def test_operators_over_non_hermitian_and_density_matrix_grad_ops():
    """On the B200 backends: MQOps / MQN2Ops over a non-Hermitian operator
    <phi| U_l^dag H U_r(enc, ans) |psi> (circ_left and simulator_left) give Re f and |f|^2 of the
    operator's own values and pass gradcheck; MQAnsatzOnlyOps over a noisy density-matrix operator
    passes gradcheck."""
    from mindquantum_b200 import complex128
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit
    from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
    from mindquantum_b200.simulator import Simulator

    n = 3
    rng = np.random.default_rng(3)
    enc = Circuit([G.RX(f'x{i}').on(i) for i in range(n)]).as_encoder()
    ans = Circuit([G.RY(f'w{i}').on(i) for i in range(n)] + [G.X.on(1, 0), G.RZ('w9').on(2)])
    circ = enc + ans
    left = Circuit([G.H.on(0), G.RX(0.3).on(1), G.X.on(2, 1)])
    ham = Hamiltonian(QubitOperator('Z0 X1', 0.7) + QubitOperator('Y2', 0.2))
    sim = Simulator('mqvector_b200', n, dtype=complex128)
    sim_left = Simulator('mqvector_b200', n, dtype=complex128)
    sim_left.set_qs(rng.normal(size=8) + 1j * rng.normal(size=8))
    ops = sim.get_expectation_with_grad(ham, circ, left, sim_left)
    e = torch.tensor(rng.uniform(0, 3, (2, n)), dtype=torch.float64, requires_grad=True)
    a = torch.tensor(rng.uniform(0, 3, len(circ.ansatz_params_name)), dtype=torch.float64, requires_grad=True)
    f, _, _ = ops(e.detach().numpy(), a.detach().numpy())
    for cls, ref in ((MQOps, f.real), (MQN2Ops, np.abs(f) ** 2)):
        assert np.max(np.abs(cls(ops)(e, a).detach().cpu().numpy() - ref)) <= 1e-12
        assert torch.autograd.gradcheck(lambda x, y, c=cls: c(ops)(x, y), (e, a), eps=1e-6, atol=1e-6)
    dm = Simulator('mqmatrix_b200', n, dtype=complex128)
    c2 = ans + G.DepolarizingChannel(0.1).on(0)
    ops2 = dm.get_expectation_with_grad(ham, c2)
    a2 = torch.tensor(rng.uniform(0, 3, len(c2.params_name)), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda y: MQAnsatzOnlyOps(ops2)(y), (a2,), eps=1e-6, atol=1e-6)
