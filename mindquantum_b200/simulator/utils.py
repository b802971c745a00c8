"""GradOpsWrapper: the callable returned by get_expectation_with_grad (mindquantum/simulator/utils.py)."""


def _thread_balance(n_prs, n_meas, parallel_worker):
    """(batch_threads, mea_threads) the reference derives from ``parallel_worker``
    (mindquantum/simulator/utils.py:18-32); here it fixes the order of the random draws of a
    noisy parameter-shift gradient."""
    if parallel_worker is None:
        parallel_worker = n_meas * n_prs
    if n_meas * n_prs <= parallel_worker:
        return n_prs, n_meas
    if n_meas < n_prs:
        batch = min(n_prs, parallel_worker)
        return batch, min(n_meas, max(1, parallel_worker // batch))
    mea = min(n_meas, parallel_worker)
    return min(n_prs, max(1, parallel_worker // mea)), mea


class GradOpsWrapper:
    """Wrap a grad operator with the data it was built from.

    Args:
        grad_ops: callable ``grad_ops(*inputs) -> (f, g...)``.
        hams, circ_right, circ_left: the Hamiltonians and circuits.
        encoder_params_name, ansatz_params_name: parameter names in gradient order.
        parallel_worker: accepted for interface compatibility (the device runs the whole batch).
        sim: the backend that built the operator.
    """

    def __init__(self, grad_ops, hams, circ_right, circ_left, encoder_params_name, ansatz_params_name,
                 parallel_worker, sim=None):
        self.grad_ops = grad_ops
        self.hams = hams
        self.circ_right = circ_right
        self.circ_left = circ_left
        self.encoder_params_name = encoder_params_name
        self.ansatz_params_name = ansatz_params_name
        self.parallel_worker = parallel_worker
        self.sim = sim
        self.str = ''

    def __call__(self, *args):
        return self.grad_ops(*args)

    def set_str(self, s):
        self.str = s

    def __str__(self):
        return self.str

    __repr__ = __str__
