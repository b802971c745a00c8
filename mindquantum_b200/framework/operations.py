"""torch.autograd.Function wrappers of ``get_expectation_with_grad``.

The forward returns real(f) with shape [n_samples][n_hams]; the backward contracts the
gradients computed in the same adjoint sweep with the incoming gradient, as the reference's
MindSpore operators do (mindquantum/framework/operations.py:132-146, 295-306, 446-457):
encoder gradient einsum('smp,sm->sp'), ansatz gradient einsum('smp,sm->p').  Everything stays
on the device: parameters, expectations and gradients are CUDA tensors.
"""
import torch


class _ExpectationFunction(torch.autograd.Function):
    """f = Re <psi(enc, ans)| H_m |psi(enc, ans)> for every sample s and Hamiltonian m."""

    @staticmethod
    def forward(ctx, enc, ans, grad_ops):  # pylint: disable=arguments-differ
        sim = grad_ops.sim
        n_enc = len(grad_ops.encoder_params_name)
        n_ans = len(grad_ops.ansatz_params_name)
        enc2 = enc.detach().to(torch.float64).reshape(-1, n_enc) if n_enc else None
        batch = enc2.shape[0] if enc2 is not None else 1
        ans2 = ans.detach().to(torch.float64).reshape(1, n_ans).expand(batch, n_ans) if n_ans else None
        parts = [p for p in (enc2, ans2) if p is not None]
        params = torch.cat([p.to(sim.device) for p in parts], dim=1) if parts else torch.zeros(
            (batch, 0), dtype=torch.float64, device=sim.device)
        names = grad_ops.encoder_params_name + grad_ops.ansatz_params_name
        f, g = sim.expectation_with_grad_tensor(grad_ops.hams, grad_ops.circ_right, params, names,
                                                init_state=sim._state)  # pylint: disable=protected-access
        ctx.n_enc = n_enc
        ctx.save_for_backward(g)
        ctx.enc_dtype, ctx.enc_device = enc.dtype, enc.device
        ctx.ans_dtype, ctx.ans_device = ans.dtype, ans.device
        ref = enc if n_enc else ans
        return f[..., 0].to(device=ref.device, dtype=ref.dtype)

    @staticmethod
    def backward(ctx, dout):  # pylint: disable=arguments-differ
        (g,) = ctx.saved_tensors
        dout = dout.to(g.dtype).to(g.device)
        g_enc = g[:, :, :ctx.n_enc]
        g_ans = g[:, :, ctx.n_enc:]
        enc_grad = (torch.einsum('smp,sm->sp', g_enc, dout).to(device=ctx.enc_device, dtype=ctx.enc_dtype)
                    if ctx.n_enc else None)
        ans_grad = (torch.einsum('smp,sm->p', g_ans, dout).to(device=ctx.ans_device, dtype=ctx.ans_dtype)
                    if g_ans.shape[2] else None)
        return enc_grad, ans_grad, None


def mq_expectation(enc, ans, grad_ops):
    """Differentiable expectation: enc [n_samples][n_enc] (or None), ans [n_ans] (or None)."""
    if enc is None:
        enc = torch.zeros((1, 0), dtype=ans.dtype, device=ans.device)
    if ans is None:
        ans = torch.zeros((0,), dtype=enc.dtype, device=enc.device)
    return _ExpectationFunction.apply(enc, ans, grad_ops)


class MQOps(torch.nn.Module):
    """Encoder + ansatz operator: forward(enc_data, ans_data) -> [n_samples][n_hams]."""

    def __init__(self, expectation_with_grad):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad

    def forward(self, enc_data, ans_data):
        return mq_expectation(enc_data, ans_data, self.expectation_with_grad)


class MQAnsatzOnlyOps(torch.nn.Module):
    """Ansatz-only operator: forward(ans_data) -> [1][n_hams]."""

    def __init__(self, expectation_with_grad):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad

    def forward(self, ans_data):
        return mq_expectation(None, ans_data, self.expectation_with_grad)


class MQEncoderOnlyOps(torch.nn.Module):
    """Encoder-only operator: forward(enc_data) -> [n_samples][n_hams]."""

    def __init__(self, expectation_with_grad):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad

    def forward(self, enc_data):
        return mq_expectation(enc_data, None, self.expectation_with_grad)


class _QRamFunction(torch.autograd.Function):
    """f[s][m] = Re <psi_s| U^dag H_m U |psi_s> for given initial states psi_s (QRamVecOps)."""

    @staticmethod
    def forward(ctx, qs_r, qs_i, ans, hams, circ, sim):  # pylint: disable=arguments-differ,too-many-arguments
        names = circ.params_name
        init = torch.complex(qs_r.detach().to(torch.float64), qs_i.detach().to(torch.float64)).to(
            device=sim.device, dtype=sim.torch_dtype).contiguous()
        batch = init.shape[0]
        params = ans.detach().to(torch.float64).reshape(1, -1).expand(batch, -1).to(sim.device).contiguous()
        f, g = sim.expectation_with_grad_tensor(hams, circ, params, names, init_state=init)
        ctx.save_for_backward(g)
        ctx.meta = (qs_r.shape, qs_r.dtype, qs_r.device, ans.dtype, ans.device)
        return f[..., 0].to(device=qs_r.device, dtype=qs_r.dtype)

    @staticmethod
    def backward(ctx, dout):  # pylint: disable=arguments-differ
        (g,) = ctx.saved_tensors
        shape, dt, dev, adt, adev = ctx.meta
        ans_grad = torch.einsum('smp,sm->p', g, dout.to(g.dtype).to(g.device)).to(device=adev, dtype=adt)
        zero = torch.zeros(shape, dtype=dt, device=dev)   # no gradient with respect to the amplitudes
        return zero, zero.clone(), ans_grad, None, None, None


class QRamVecOps(torch.nn.Module):
    """Initial states as input (mindquantum/framework/operations.py:539-664): forward(qs_r, qs_i,
    ans_data) -> [n_states][n_hams] for states [n_states][2^n] given as real and imaginary parts;
    the gradient flows to the ansatz parameters only, as in the reference."""

    def __init__(self, hams, circ, sim, n_thread=None):  # pylint: disable=unused-argument
        super().__init__()
        from ..core.operators import Hamiltonian  # pylint: disable=import-outside-toplevel

        self.hams = [hams] if isinstance(hams, Hamiltonian) else list(hams)
        if circ.encoder_params_name:
            raise ValueError("circ can not have encoder parameters.")
        self.circ = circ
        self.sim = getattr(sim, 'backend', sim)

    def forward(self, qs_r, qs_i, ans_data):
        dim = 1 << self.sim.n_qubits
        if qs_r.shape != qs_i.shape or qs_r.dim() != 2 or qs_r.shape[1] != dim:
            raise ValueError(f"quantum states need shape (N, {dim}), got {tuple(qs_r.shape)} and {tuple(qs_i.shape)}")
        if ans_data.numel() != len(self.circ.params_name):
            raise ValueError(f"ansatz data requires {len(self.circ.params_name)} values, got {ans_data.numel()}")
        return _QRamFunction.apply(qs_r, qs_i, ans_data, self.hams, self.circ, self.sim)
