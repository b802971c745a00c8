"""Simulator facade (mindquantum/simulator/simulator.py:43-560) and inner_product."""
import numpy as np

from ..dtype import to_mq_type
from .backend_base import BackendBase

SUPPORTED_SIMULATOR = ('mqvector_b200', 'mqvector_gpu', 'mqmatrix_b200', 'mqmatrix_gpu')


def _make_backend(name, n_qubits, seed, dtype, **kwargs):
    # pylint: disable=import-outside-toplevel
    from .mqmatrix_b200 import MQMatrixB200
    from .mqvector_b200 import MQVectorB200

    if name not in SUPPORTED_SIMULATOR:
        raise ValueError(f"backend {name} not supported, supported backends: {SUPPORTED_SIMULATOR}")
    if name.startswith('mqmatrix'):
        return MQMatrixB200(name, n_qubits, seed, dtype, **kwargs)
    return MQVectorB200(name, n_qubits, seed, dtype, **kwargs)


class Simulator:
    """Quantum simulator.

    Args:
        backend (Union[str, BackendBase]): ``'mqvector_b200'`` (alias ``'mqvector_gpu'``), the density-matrix
            ``'mqmatrix_b200'`` (alias ``'mqmatrix_gpu'``) or a backend object.
        n_qubits (int): number of qubits.
        seed (int): random seed of measurements and sampling.
        dtype: ``complex128`` (default) or ``complex64``.
        kwargs: ``fuse`` (bool) selects fused tile passes (default) or one kernel per gate.
    """

    def __init__(self, backend, n_qubits=None, seed=None, dtype=None, **kwargs):
        if isinstance(backend, BackendBase):
            self.backend = backend
        else:
            if not isinstance(n_qubits, int) or n_qubits < 1:
                raise ValueError(f"n_qubits should be a positive integer, but get {n_qubits}")
            if seed is None:
                seed = int(np.random.randint(1, 2**23))
            self.backend = _make_backend(backend, n_qubits, seed, to_mq_type(dtype), **kwargs)

    @property
    def n_qubits(self):
        return self.backend.n_qubits

    @property
    def seed(self):
        return self.backend.seed

    @property
    def dtype(self):
        return self.backend.dtype

    def astype(self, dtype, seed=None):
        return Simulator(self.backend.astype(dtype, seed))

    def copy(self):
        return Simulator(self.backend.copy())

    def apply_circuit(self, circuit, pr=None):
        return self.backend.apply_circuit(circuit, pr)

    def apply_gate(self, gate, pr=None, diff=False):
        return self.backend.apply_gate(gate, pr, diff)

    def apply_hamiltonian(self, hamiltonian):
        return self.backend.apply_hamiltonian(hamiltonian)

    def get_expectation(self, hamiltonian, circ_right=None, circ_left=None, simulator_left=None, pr=None):
        if isinstance(simulator_left, Simulator):
            simulator_left = simulator_left.backend
        return self.backend.get_expectation(hamiltonian, circ_right, circ_left, simulator_left, pr)

    def get_expectation_with_grad(self, hams, circ_right, circ_left=None, simulator_left=None, parallel_worker=None,
                                  pr_shift=False):
        if isinstance(simulator_left, Simulator):
            simulator_left = simulator_left.backend
        return self.backend.get_expectation_with_grad(hams, circ_right, circ_left, simulator_left, parallel_worker,
                                                      pr_shift)

    def get_qs(self, ket=False):
        return self.backend.get_qs(ket)

    def set_qs(self, quantum_state):
        return self.backend.set_qs(quantum_state)

    def reset(self):
        return self.backend.reset()

    def sampling(self, circuit, pr=None, shots=1, seed=None):
        return self.backend.sampling(circuit, pr, shots, seed)

    def __str__(self):
        return f"{self.backend.device_name()}"

    __repr__ = __str__

    # density-matrix methods (mqsim.py:546-600); a state vector is pure
    def purity(self):
        fn = getattr(self.backend, 'purity', None)
        return fn() if fn else 1.0

    def entropy(self):
        fn = getattr(self.backend, 'entropy', None)
        return fn() if fn else 0.0

    def get_partial_trace(self, qubits_to_trace):
        """Trace out ``qubits_to_trace`` (simulator.py:516; density-matrix backends only)."""
        if isinstance(qubits_to_trace, int):
            qubits_to_trace = [qubits_to_trace]
        if not hasattr(self.backend, 'get_partial_trace'):
            raise ValueError(f"{self.backend.name} simulator not support partial trace method.")
        return self.backend.get_partial_trace(list(qubits_to_trace))

    def get_reduced_density_matrix(self, kept_qubits):
        if isinstance(kept_qubits, int):
            kept_qubits = [kept_qubits]
        if not hasattr(self.backend, 'get_reduced_density_matrix'):
            raise ValueError(f"{self.backend.name} simulator not support reduced density matrices.")
        return self.backend.get_reduced_density_matrix(list(kept_qubits))

    def get_pure_state_vector(self):
        fn = getattr(self.backend, 'get_pure_state_vector', None)
        return fn() if fn else self.get_qs()

    def get_qs_of_qubits(self, qubits, ket=False):
        """Reduced state of ``qubits``: a vector when pure, else a density matrix (simulator.py:641)."""
        return self.backend.get_qs_of_qubits(qubits, ket)

    def set_threads_number(self, number):
        """Forwarded to the backend (simulator.py:507); the B200 backends, like the reference's
        MQSim, do not implement it (BackendBase raises NotImplementedError)."""
        return self.backend.set_threads_number(number)


def inner_product(bra_simulator, ket_simulator):
    """<bra|ket> of two simulators (mindquantum/simulator/simulator.py inner_product; Vdot)."""
    import ctypes  # pylint: disable=import-outside-toplevel

    import torch  # pylint: disable=import-outside-toplevel

    from .. import _native as N  # pylint: disable=import-outside-toplevel

    bra = bra_simulator.backend if isinstance(bra_simulator, Simulator) else bra_simulator
    ket = ket_simulator.backend if isinstance(ket_simulator, Simulator) else ket_simulator
    if bra.n_qubits != ket.n_qubits or bra.dtype != ket.dtype:
        raise ValueError("inner_product needs simulators of the same qubits and dtype")
    out = torch.zeros(2, dtype=torch.float64, device=ket.device)
    N.call('mqb_vdot', ket.n_qubits, ket.precision, ctypes.c_void_p(bra.state.data_ptr()),
           ctypes.c_void_p(ket.state.data_ptr()), 1, ctypes.c_void_p(out.data_ptr()),
           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    o = out.cpu().numpy()
    return complex(o[0], o[1])
