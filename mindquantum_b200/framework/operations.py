"""torch.autograd.Function wrappers of ``get_expectation_with_grad``.

The forward returns real(f) with shape [n_samples][n_hams] (the MQ*Ops) or |f|^2 (the MQN2*Ops);
the backward contracts the gradients computed in the same sweep with the incoming gradient, as
the reference's MindSpore operators do (mindquantum/framework/operations.py:132-146, 221-236,
295-306, 370-383, 446-457, 524-538): encoder gradient einsum('smp,sm->sp'), ansatz gradient
einsum('smp,sm->p'), and for |f|^2 the same with the weight 2 conj(f) dout, real part taken.

A Hermitian adjoint operator of the state-vector backend carries ``device_grad`` and stays on
the device: parameters, expectations and gradients are CUDA tensors.  Every other operator (the
non-Hermitian <phi|U_l^dag H U_r|psi>, parameter-shift gradients, the density-matrix backend) is
evaluated through its own call with numpy inputs, like the reference operators evaluate it.
"""
import numpy as np
import torch


def _versioned_call(grad_ops, enc, ans):
    """(f, g_enc, g_ans) of a grad operator as complex numpy arrays [s][m], [s][m][n_enc],
    [s][m][n_ans], whatever its encoder / ansatz form (mindquantum/simulator/mqsim.py:341-380)."""
    n_enc = len(grad_ops.encoder_params_name)
    n_ans = len(grad_ops.ansatz_params_name)
    enc_np = enc.detach().to(torch.float64).reshape(-1, n_enc).cpu().numpy() if n_enc else None
    ans_np = ans.detach().to(torch.float64).reshape(n_ans).cpu().numpy() if n_ans else None
    if n_enc and n_ans:
        f, g_enc, g_ans = grad_ops(enc_np, ans_np)
    elif n_enc:
        f, g_enc = grad_ops(enc_np)
        g_ans = np.zeros(g_enc.shape[:2] + (0,), dtype=g_enc.dtype)
    else:
        f, g_ans = grad_ops(ans_np if ans_np is not None else np.zeros(0))
        g_enc = np.zeros(g_ans.shape[:2] + (0,), dtype=g_ans.dtype)
    return np.asarray(f), np.asarray(g_enc), np.asarray(g_ans)


def _device_call(grad_ops, enc, ans):
    """The same on the device through ``grad_ops.device_grad(params)``: f [s][m] and the
    gradient [s][m][n_enc + n_ans], complex128 tensors."""
    n_enc = len(grad_ops.encoder_params_name)
    n_ans = len(grad_ops.ansatz_params_name)
    device = grad_ops.sim.device
    enc2 = enc.detach().to(torch.float64).reshape(-1, n_enc) if n_enc else None
    batch = enc2.shape[0] if enc2 is not None else 1
    ans2 = ans.detach().to(torch.float64).reshape(1, n_ans).expand(batch, n_ans) if n_ans else None
    parts = [p.to(device) for p in (enc2, ans2) if p is not None]
    params = torch.cat(parts, dim=1) if parts else torch.zeros((batch, 0), dtype=torch.float64, device=device)
    f, g = grad_ops.device_grad(params)
    return torch.complex(f[..., 0], f[..., 1]), g.to(torch.complex128)


class _ExpectationFunction(torch.autograd.Function):
    """f[s][m] = Re <H_m> (square=False) or |<H_m>|^2 (square=True) for every sample s."""

    @staticmethod
    def forward(ctx, enc, ans, grad_ops, square):  # pylint: disable=arguments-differ
        n_enc = len(grad_ops.encoder_params_name)
        ref = enc if n_enc else ans
        if getattr(grad_ops, 'device_grad', None) is not None:
            f, g = _device_call(grad_ops, enc, ans)
        else:
            f_np, ge, ga = _versioned_call(grad_ops, enc, ans)
            f = torch.as_tensor(f_np, dtype=torch.complex128)
            g = torch.as_tensor(np.concatenate([ge, ga], axis=2), dtype=torch.complex128)
        ctx.n_enc = n_enc
        ctx.square = square
        ctx.save_for_backward(f, g)
        ctx.enc_dtype, ctx.enc_device = enc.dtype, enc.device
        ctx.ans_dtype, ctx.ans_device = ans.dtype, ans.device
        out = f.real ** 2 + f.imag ** 2 if square else f.real
        return out.to(device=ref.device, dtype=ref.dtype)

    @staticmethod
    def backward(ctx, dout):  # pylint: disable=arguments-differ
        f, g = ctx.saved_tensors
        w = dout.to(device=g.device, dtype=torch.float64).to(torch.complex128)
        if ctx.square:   # d|f|^2 = 2 Re(conj(f) df)
            w = 2 * f.conj() * w
        g_enc = g[:, :, :ctx.n_enc]
        g_ans = g[:, :, ctx.n_enc:]
        enc_grad = (torch.einsum('smp,sm->sp', g_enc, w).real.to(device=ctx.enc_device, dtype=ctx.enc_dtype)
                    if ctx.n_enc else None)
        ans_grad = (torch.einsum('smp,sm->p', g_ans, w).real.to(device=ctx.ans_device, dtype=ctx.ans_dtype)
                    if g_ans.shape[2] else None)
        return enc_grad, ans_grad, None, None


def mq_expectation(enc, ans, grad_ops, square=False):
    """Differentiable expectation: enc [n_samples][n_enc] (or None), ans [n_ans] (or None);
    Re <H> per sample and Hamiltonian, or |<H>|^2 with ``square``."""
    if enc is None:
        enc = torch.zeros((1, 0), dtype=ans.dtype, device=ans.device)
    if ans is None:
        ans = torch.zeros((0,), dtype=enc.dtype, device=enc.device)
    return _ExpectationFunction.apply(enc, ans, grad_ops, square)


class MQOps(torch.nn.Module):
    """Encoder + ansatz operator: forward(enc_data, ans_data) -> Re <H>, [n_samples][n_hams]."""

    square = False

    def __init__(self, expectation_with_grad):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad

    def forward(self, enc_data, ans_data):
        return mq_expectation(enc_data, ans_data, self.expectation_with_grad, self.square)


class MQAnsatzOnlyOps(torch.nn.Module):
    """Ansatz-only operator: forward(ans_data) -> Re <H>, [1][n_hams]."""

    square = False

    def __init__(self, expectation_with_grad):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad

    def forward(self, ans_data):
        return mq_expectation(None, ans_data, self.expectation_with_grad, self.square)


class MQEncoderOnlyOps(torch.nn.Module):
    """Encoder-only operator: forward(enc_data) -> Re <H>, [n_samples][n_hams]."""

    square = False

    def __init__(self, expectation_with_grad):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad

    def forward(self, enc_data):
        return mq_expectation(enc_data, None, self.expectation_with_grad, self.square)


class MQN2Ops(MQOps):
    """|<phi| U_l^dag H U_r |psi>|^2 of an encoder + ansatz operator (operations.py:149-236)."""

    square = True


class MQN2AnsatzOnlyOps(MQAnsatzOnlyOps):
    """|<H>|^2 of an ansatz-only operator (operations.py:309-383)."""

    square = True


class MQN2EncoderOnlyOps(MQEncoderOnlyOps):
    """|<H>|^2 of an encoder-only operator (operations.py:460-538)."""

    square = True


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
