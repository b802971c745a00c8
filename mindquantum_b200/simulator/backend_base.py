"""BackendBase: the plugin interface a simulator backend implements.

Mirrors mindquantum/simulator/backend_base.py:28-130: the ``Simulator`` facade forwards every
call to an object of this interface, so a backend can be passed to ``Simulator`` directly.
"""
from ..dtype import to_mq_type


class BackendBase:
    """Abstract simulator backend."""

    def __init__(self, name: str, n_qubits: int, seed=None, dtype=None):
        self.name = name
        self.n_qubits = n_qubits
        self.seed = seed
        self.arithmetic_type = to_mq_type(dtype)

    def apply_circuit(self, circuit, pr=None):
        raise NotImplementedError(f"apply_circuit not implemented for {self.device_name()}")

    def apply_gate(self, gate, pr=None, diff=False):
        raise NotImplementedError(f"apply_gate not implemented for {self.device_name()}")

    def apply_hamiltonian(self, hamiltonian):
        raise NotImplementedError(f"apply_hamiltonian not implemented for {self.device_name()}")

    def astype(self, dtype, seed=None):
        raise NotImplementedError(f"astype not implemented for {self.device_name()}")

    def copy(self):
        raise NotImplementedError(f"copy not implemented for {self.device_name()}")

    def device_name(self):
        return self.name

    @property
    def dtype(self):
        return self.arithmetic_type

    def get_expectation(self, hamiltonian, circ_right=None, circ_left=None, simulator_left=None, pr=None):
        raise NotImplementedError(f"get_expectation not implemented for {self.device_name()}")

    def get_expectation_with_grad(self, hams, circ_right, circ_left=None, simulator_left=None, parallel_worker=None,
                                  pr_shift=False):
        raise NotImplementedError(f"get_expectation_with_grad not implemented for {self.device_name()}")

    def get_qs(self, ket=False):
        raise NotImplementedError(f"get_qs not implemented for {self.device_name()}")

    def reset(self):
        raise NotImplementedError(f"reset not implemented for {self.device_name()}")

    def sampling(self, circuit, pr=None, shots=1, seed=None):
        raise NotImplementedError(f"sampling not implemented for {self.device_name()}")

    def set_qs(self, quantum_state):
        raise NotImplementedError(f"set_qs not implemented for {self.device_name()}")

    def set_threads_number(self, number):
        raise NotImplementedError(f"set_threads_number not implemented for {self.device_name()}")
