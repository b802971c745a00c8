"""Trainable layers (mindquantum/framework/layer.py): the ansatz parameters are an nn.Parameter."""
import torch

from .operations import mq_expectation


class MQLayer(torch.nn.Module):
    """Encoder data in, ansatz weights trained: forward(enc_data) -> [n_samples][n_hams]."""

    def __init__(self, expectation_with_grad, weight=None):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad
        n_ans = len(expectation_with_grad.ansatz_params_name)
        w = torch.randn(n_ans, dtype=torch.float32) if weight is None else torch.as_tensor(weight)
        self.weight = torch.nn.Parameter(w.reshape(n_ans))

    def forward(self, enc_data):
        return mq_expectation(enc_data, self.weight, self.expectation_with_grad)


class MQAnsatzOnlyLayer(torch.nn.Module):
    """Ansatz weights trained, no encoder: forward() -> [1][n_hams]."""

    def __init__(self, expectation_with_grad, weight=None):
        super().__init__()
        self.expectation_with_grad = expectation_with_grad
        n_ans = len(expectation_with_grad.ansatz_params_name)
        w = torch.randn(n_ans, dtype=torch.float32) if weight is None else torch.as_tensor(weight)
        self.weight = torch.nn.Parameter(w.reshape(n_ans))

    def forward(self):
        return mq_expectation(None, self.weight, self.expectation_with_grad)
