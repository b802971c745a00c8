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
