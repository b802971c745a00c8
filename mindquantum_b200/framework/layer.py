"""Trainable layers (mindquantum/framework/layer.py): the ansatz parameters are an nn.Parameter."""
import torch

from .operations import QRamVecOps, mq_expectation


def _ansatz_weight(n_ans, weight):
    w = torch.randn(n_ans, dtype=torch.float32) if weight is None else torch.as_tensor(weight)
    if w.dim() != 1 or w.shape[0] != n_ans:
        raise ValueError(f"Weight init shape error, required ({n_ans}, ), but get {tuple(w.shape)}.")
    return torch.nn.Parameter(w)


class MQLayer(torch.nn.Module):
    """Encoder data in, ansatz weights trained: forward(enc_data) -> Re <H>, [n_samples][n_hams]."""

    square = False

    def __init__(self, expectation_with_grad, weight=None):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad
        self.weight = _ansatz_weight(len(expectation_with_grad.ansatz_params_name), weight)

    def forward(self, enc_data):
        return mq_expectation(enc_data, self.weight, self.expectation_with_grad, self.square)


class MQAnsatzOnlyLayer(torch.nn.Module):
    """Ansatz weights trained, no encoder: forward() -> Re <H>, [1][n_hams]."""

    square = False

    def __init__(self, expectation_with_grad, weight=None):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad
        self.weight = _ansatz_weight(len(expectation_with_grad.ansatz_params_name), weight)

    def forward(self):
        return mq_expectation(None, self.weight, self.expectation_with_grad, self.square)


class MQN2Layer(MQLayer):
    """|<H>|^2 with encoder data in and ansatz weights trained (layer.py:97-170)."""

    square = True


class MQN2AnsatzOnlyLayer(MQAnsatzOnlyLayer):
    """|<H>|^2 with ansatz weights trained, no encoder (layer.py:239-307)."""

    square = True


class QRamVecLayer(torch.nn.Module):
    """Initial states in, ansatz weights trained (layer.py:310-397): forward(qs_r, qs_i) ->
    Re <psi_s| U^dag H_m U |psi_s>, [n_states][n_hams]."""

    def __init__(self, hams, circ, sim, n_thread=None, weight=None):  # pylint: disable=too-many-arguments
        super().__init__()
        self.evolution = QRamVecOps(hams, circ, sim, n_thread)
        self.weight = _ansatz_weight(len(circ.params_name), weight)

    def forward(self, qs_r, qs_i):
        return self.evolution(qs_r, qs_i, self.weight)
