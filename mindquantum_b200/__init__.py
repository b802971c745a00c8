"""mindquantum_b200: MindQuantum's state-vector path (gate application, Pauli expectation and the
adjoint gradient) as hand-written CUDA kernels for the NVIDIA B200 (sm_100a).

Drop-in surface: ``Simulator('mqvector_b200', n_qubits)`` with ``apply_circuit``, ``get_qs``,
``set_qs``, ``get_expectation``, ``get_expectation_with_grad`` and ``sampling``, built from the
``Circuit`` / gate / ``Hamiltonian`` / ``ParameterResolver`` classes of ``mindquantum_b200.core``.
"""
from . import core, dtype
from .core import *  # noqa: F401,F403
from .dtype import complex64, complex128
from .simulator import MeasureResult, Simulator, inner_product

__version__ = '0.1.0'
