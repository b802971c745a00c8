"""Circuits of the reference's own tests, rebuilt with this package's API.

Each builder names the reference test it reproduces so the golden numbers in
tests/golden/reference_goldens.json apply to it.
"""
import numpy as np

from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import UN, Circuit, qft


def rx_matrix_generator(x):
    return np.array([[np.cos(x / 2), -1j * np.sin(x / 2)], [-1j * np.sin(x / 2), np.cos(x / 2)]])


def rx_diff_matrix_generator(x):
    return np.array([[np.sin(x / 2), 1j * np.cos(x / 2)], [1j * np.cos(x / 2), np.sin(x / 2)]]) / -2


def generate_test_circuit():
    """tests/st/test_simulator/test_simulator.py:230-257 (every gate kind, with controls)."""
    circuit = Circuit()
    circuit += UN(G.H, 3)
    circuit.x(0).y(1).z(2)
    circuit += G.SWAP.on([0, 2], 1)
    circuit += UN(G.X, 3)
    circuit += G.ISWAP.on([0, 1], 2)
    circuit.rx(1.2, 0).ry(2.3, 1).rz(3.4, 2)
    circuit.x(0, 1).x(1, 2).x(0, 2)
    circuit += G.PhaseShift(1.3).on(0, [1, 2])
    circuit += UN(G.H, 3)
    circuit += UN(G.S, 3)
    circuit += qft(range(3))
    circuit += G.gene_univ_parameterized_gate('fake_x', rx_matrix_generator, rx_diff_matrix_generator)('a').on(0)
    circuit += G.RX('b').on(1, 2)
    circuit += G.RX('c').on(2, 0)
    circuit += UN(G.H, 3)
    circuit += UN(G.T, 3)
    circuit += G.UnivMathGate('fake_Rxx', G.Rxx(2.4).matrix()).on([0, 1])
    circuit += G.Ryy(4.6).on([1, 2])
    circuit += G.Rzz(6.8).on([0, 2])
    circuit += G.UnivMathGate('myX', G.X.matrix()).on(0)
    circuit += G.Power(G.X, 1.2).on(1)
    return circuit


def multi_params_circuit():
    """tests/st/test_simulator/test_simulator.py:528-532 (U3 and FSim with parameters)."""
    circ = Circuit() + G.U3('a', 'b', 1.0).on(0) + G.U3('c', 'd', 2.0).on(1) + G.X.on(0, 1)
    circ += G.FSim('e', -3.0).on([0, 1])
    return circ


def custom_matrix(x):
    return np.diag([np.exp(1j * 2 * k * x) for k in range(1, 9)])


def custom_diff_matrix(x):
    return np.diag([2 * k * np.exp(1j * 2 * k * x) for k in range(1, 9)]) * 1j


def mul_qubit_circuit():
    """tests/st/test_simulator/test_simulator.py:661-672 (3-qubit parameterized custom gate)."""
    q = G.gene_univ_parameterized_gate('q', custom_matrix, custom_diff_matrix)
    return UN(G.H, 3) + q('a').on([0, 1, 2])


def hea_circuit(n_qubits, n_layers, prefix='p'):
    """Hardware-efficient ansatz: per layer RY then RZ on every qubit, then CNOT q_i -> q_{i+1}."""
    circ = Circuit()
    k = 0
    for _ in range(n_layers):
        for q in range(n_qubits):
            circ += G.RY(f'{prefix}{k}').on(q)
            k += 1
        for q in range(n_qubits):
            circ += G.RZ(f'{prefix}{k}').on(q)
            k += 1
        for q in range(n_qubits - 1):
            circ += G.X.on(q + 1, q)
    return circ


def hea_hamiltonian(n_qubits, rng):
    """H = sum a_i Z_i Z_{i+1} + sum b_i X_i with a, b ~ N(0, 1)."""
    from mindquantum_b200.core.operators import QubitOperator

    a = rng.normal(size=n_qubits - 1)
    b = rng.normal(size=n_qubits)
    op = QubitOperator()
    for i in range(n_qubits - 1):
        op += QubitOperator(f'Z{i} Z{i + 1}', float(a[i]))
    for i in range(n_qubits):
        op += QubitOperator(f'X{i}', float(b[i]))
    return op
