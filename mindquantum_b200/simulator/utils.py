"""GradOpsWrapper: the callable returned by get_expectation_with_grad (mindquantum/simulator/utils.py),
and the reduced-state helpers the backends share (mindquantum/simulator/mqsim.py:559-626)."""
import numpy as np


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
        # set by the Hermitian adjoint operator of the state-vector backend: device_grad(params
        # [batch][n_enc + n_ans] float64 tensor) -> (f [batch][n_hams][2], g [batch][n_hams][P])
        # tensors on the device, the path the autograd operators take
        self.device_grad = None

    def __call__(self, *args):
        return self.grad_ops(*args)

    def set_str(self, s):
        self.str = s

    def __str__(self):
        return self.str

    __repr__ = __str__


def check_kept_qubits(kept_qubits, n_qubits):
    """The checks of MQSim.get_reduced_density_matrix (mindquantum/simulator/mqsim.py:559-570);
    returns the kept qubits as a sorted list."""
    if isinstance(kept_qubits, int):
        kept_qubits = [kept_qubits]
    kept = [int(q) for q in kept_qubits]
    if len(set(kept)) != len(kept):
        raise ValueError("kept_qubits cannot contain repeated indices.")
    if len(kept) >= n_qubits:
        raise ValueError("Number of kept qubits must be less than total number of qubits.")
    if kept and max(kept) >= n_qubits:
        raise ValueError(f"Qubit index {max(kept)} is out of range for a {n_qubits}-qubit system.")
    if kept and min(kept) < 0:
        raise ValueError(f"Qubit index {min(kept)} is out of range for a {n_qubits}-qubit system.")
    return sorted(kept)


def reduced_density_matrix(state, n_qubits, kept):
    """rho of the sorted qubits ``kept`` of a 2^n state tensor, the others traced out: rho[i][j] =
    sum over the traced bits of psi_i conj(psi_j), bit k of a row or column index being qubit
    kept[k] (GetReducedDensityMatrix, ccsrc/lib/simulator/vector/detail/cpu_common/
    cpu_vector_core_policy.cpp:335-383).  Computed where the tensor lives as M M^H, with M the state
    viewed as [kept bits][traced bits], in the state's precision; returned as numpy complex128."""
    psi = state.reshape([2] * n_qubits)          # axis a of the view is qubit n - 1 - a
    kept_axes = [n_qubits - 1 - q for q in reversed(kept)]
    traced_axes = [a for a in range(n_qubits) if a not in kept_axes]
    m = psi.permute(kept_axes + traced_axes).reshape(1 << len(kept), -1)
    rho = m @ m.conj().transpose(0, 1)
    return rho.cpu().numpy().astype(np.complex128)


def _ket_terms(vec, n):
    return [f"{v}¦{format(i, f'0{n}b')}⟩" for i, v in enumerate(vec) if abs(v) > 1e-12]


def qs_of_qubits(backend, qubits, ket=False):
    """Reduced state of ``qubits`` (MQSim.get_qs_of_qubits, mindquantum/simulator/mqsim.py:598-626):
    the whole state when every qubit is kept; else the reduced density matrix, or, when it is pure
    (|Tr rho^2 - 1| < 1e-6), its eigenvector of the largest eigenvalue with the first nonzero
    amplitude's real part made non-negative.  ``ket=True`` returns the state as a ket string
    (a probability-weighted sum of eigenvectors for a mixed state)."""
    if isinstance(qubits, int):
        qubits = [qubits]
    if not isinstance(qubits, (list, tuple)):
        raise TypeError(f"qubits requires an int or a list/tuple of ints, but get {type(qubits)}")
    if not all(isinstance(q, (int, np.integer)) for q in qubits):
        raise TypeError("all elements in qubits must be integers")
    n = backend.n_qubits
    if not all(0 <= q < n for q in qubits):
        raise ValueError(f"qubit indices must be between 0 and {n - 1}")
    if len(set(qubits)) == n:
        return backend.get_qs(ket=ket)
    rho = backend.get_reduced_density_matrix(list(qubits))
    k = int(round(np.log2(rho.shape[0])))
    w, v = np.linalg.eigh(rho)
    pure = abs(float(np.real(np.trace(rho @ rho))) - 1.0) < 1e-6
    if pure:
        vec = v[:, int(np.argmax(w))]
        first = np.nonzero(np.abs(vec) > 1e-12)[0][0]
        if vec[first].real < 0:
            vec = -vec
        return ' + '.join(_ket_terms(vec, k)) if ket else vec
    if not ket:
        return rho
    order = np.argsort(w)[::-1]
    terms = [f"{float(w[i]):.8g}¦[{' + '.join(_ket_terms(v[:, i], k))}]" for i in order if abs(w[i]) > 1e-6]
    return ' + '.join(terms) + ' (mixed state)'
