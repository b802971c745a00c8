"""Circuit: an ordered list of gates with parameter bookkeeping.

Mirrors the reference ``mindquantum.core.circuit.Circuit`` (mindquantum/core/circuit/circuit.py)
for the state-vector path: construction, fluent gate helpers, parameter-name collections
(encoder / ansatz, in first-appearance order), ``hermitian`` (reversed daggers,
circuit.py:831-845), measurement bookkeeping and ``get_qs`` / ``matrix`` through a simulator.
"""
from __future__ import annotations

import copy
from typing import Iterable

import numpy as np

from . import gates as G
from .parameterresolver import ParameterResolver


class CollectionMap:
    """Insertion-ordered counter of names (circuit.py:140-240)."""

    def __init__(self):
        self.map = {}

    def collect(self, keys):
        if isinstance(keys, (str, int)):
            keys = [keys]
        for k in keys:
            self.map[k] = self.map.get(k, 0) + 1

    def keys(self):
        return list(self.map.keys())

    def merge(self, other):
        for k, v in other.map.items():
            self.map[k] = self.map.get(k, 0) + v

    def __len__(self):
        return len(self.map)

    def __contains__(self, k):
        return k in self.map


class Circuit(list):
    """An ordered list of gates."""

    def __init__(self, gates=None):
        super().__init__()
        self.all_qubits = CollectionMap()
        self.all_paras = CollectionMap()
        self.all_measures = CollectionMap()
        self.all_encoder = CollectionMap()
        self.all_ansatz = CollectionMap()
        self._measure_gates = {}
        if gates is not None:
            if isinstance(gates, Iterable):
                self.extend(gates)
            else:
                self.append(gates)

    # ------------------------------------------------------------------ building
    def _collect(self, gate):
        if isinstance(gate, G.Measure):
            if gate.key in self.all_measures:
                raise ValueError(f"measure key {gate.key} already exist.")
            self.all_measures.collect(gate.key)
            self._measure_gates[gate.key] = gate
        self.all_qubits.collect(gate.obj_qubits)
        self.all_qubits.collect(gate.ctrl_qubits)
        if gate.parameterized:
            keys, ansatz, encoder = gate.__params_prop__()
            for k in ansatz:
                if k in self.all_encoder:
                    raise RuntimeError(f"Parameter '{k}' already set to encoder parameter.")
            for k in encoder:
                if k in self.all_ansatz:
                    raise RuntimeError(f"Parameter '{k}' already set to ansatz parameters.")
            self.all_paras.collect(keys)
            self.all_ansatz.collect(ansatz)
            self.all_encoder.collect(encoder)

    def append(self, gate):
        if not isinstance(gate, G.BasicGate):
            raise TypeError(f"Expect a quantum gate, but get {type(gate)}.")
        if not gate.obj_qubits and not isinstance(gate, G.BarrierGate):
            raise ValueError(f"Gate {gate} has no object qubits; call .on(...) first.")
        self._collect(gate)
        super().append(gate)

    def extend(self, gates):
        if isinstance(gates, Circuit):
            gates = list(gates)
        for g in gates:
            self.append(g)

    def __add__(self, other):
        out = copy.deepcopy(self)
        out += other
        return out

    def __radd__(self, other):
        return Circuit(other) + self

    def __iadd__(self, other):
        if isinstance(other, G.BasicGate):
            self.append(other)
        elif isinstance(other, Iterable):
            self.extend(other)
        else:
            raise TypeError(f"Cannot add {type(other)} to a circuit.")
        return self

    def __mul__(self, num):
        out = Circuit()
        for _ in range(num):
            out += copy.deepcopy(self)
        return out

    __rmul__ = __mul__

    def __deepcopy__(self, memo):
        return Circuit([copy.deepcopy(g) for g in self])

    def copy(self):
        return copy.deepcopy(self)

    def __getitem__(self, sliced):
        if isinstance(sliced, slice):
            return Circuit(super().__getitem__(sliced))
        return super().__getitem__(sliced)

    # ------------------------------------------------------------------ properties
    @property
    def n_qubits(self):
        qs = self.all_qubits.keys()
        return max(qs) + 1 if qs else 0

    @property
    def params_name(self):
        return self.all_paras.keys()

    @property
    def encoder_params_name(self):
        return self.all_encoder.keys()

    @property
    def ansatz_params_name(self):
        return self.all_ansatz.keys()

    @property
    def parameterized(self):
        return any(g.parameterized for g in self)

    @property
    def has_measure_gate(self):
        return len(self.all_measures) > 0

    @property
    def is_noise_circuit(self):
        return any(isinstance(g, G.NoiseGate) for g in self)

    @property
    def is_measure_end(self):
        """All measurements last on their qubits, each qubit at most once (circuit.py:920-944)."""
        circ = self.remove_barrier()
        n = self.n_qubits
        high = [0] * n
        measure_num = [0] * n
        for gate in circ:
            for idx in set(gate.obj_qubits + gate.ctrl_qubits):
                high[idx] += 1
            if isinstance(gate, G.Measure):
                m_idx = gate.obj_qubits[0]
                measure_num[m_idx] += 1
                if high[m_idx] != circ.all_qubits.map[m_idx]:
                    return False
        return sum(measure_num) > 0 and max(measure_num) == 1

    def get_measure_gate(self, key):
        return self._measure_gates[key]

    # ------------------------------------------------------------------ transforms
    def hermitian(self):
        """Reversed circuit of daggered gates (circuit.py:831-845)."""
        return Circuit([g.hermitian() for g in reversed(self)])

    def as_encoder(self, inplace=True):
        circ = self if inplace else copy.deepcopy(self)
        for gate in circ:
            if gate.parameterized:
                for p in gate.get_parameters():
                    p.as_encoder()
        circ.all_encoder.merge(circ.all_ansatz)
        circ.all_ansatz.map = {}
        return circ

    def as_ansatz(self, inplace=True):
        circ = self if inplace else copy.deepcopy(self)
        for gate in circ:
            if gate.parameterized:
                for p in gate.get_parameters():
                    p.as_ansatz()
        circ.all_ansatz.merge(circ.all_encoder)
        circ.all_encoder.map = {}
        return circ

    def no_grad(self):
        for gate in self:
            for p in gate.get_parameters():
                p.no_grad()
        return self

    def requires_grad(self):
        for gate in self:
            for p in gate.get_parameters():
                p.requires_grad()
        return self

    def remove_barrier(self):
        return Circuit([g for g in self if not isinstance(g, G.BarrierGate)])

    def remove_measure(self):
        return Circuit([g for g in self if not isinstance(g, G.Measure)])

    def parameter_resolver(self):
        return ParameterResolver({k: 1.0 for k in self.params_name})

    # ------------------------------------------------------------------ fluent helpers
    def h(self, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.H.on(obj_qubits, ctrl_qubits))

    def x(self, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.X.on(obj_qubits, ctrl_qubits))

    def y(self, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Y.on(obj_qubits, ctrl_qubits))

    def z(self, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Z.on(obj_qubits, ctrl_qubits))

    def s(self, obj_qubits, ctrl_qubits=None, hermitian=False):
        g = G.S.on(obj_qubits, ctrl_qubits)
        return self.__iadd__(g.hermitian() if hermitian else g)

    def t(self, obj_qubits, ctrl_qubits=None, hermitian=False):
        g = G.T.on(obj_qubits, ctrl_qubits)
        return self.__iadd__(g.hermitian() if hermitian else g)

    def sx(self, obj_qubits, ctrl_qubits=None, hermitian=False):
        g = G.SX.on(obj_qubits, ctrl_qubits)
        return self.__iadd__(g.hermitian() if hermitian else g)

    def swap(self, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.SWAP.on(obj_qubits, ctrl_qubits))

    def iswap(self, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.ISWAP.on(obj_qubits, ctrl_qubits))

    def swap_alpha(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.SWAPalpha(para).on(obj_qubits, ctrl_qubits))

    def rx(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.RX(para).on(obj_qubits, ctrl_qubits))

    def ry(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.RY(para).on(obj_qubits, ctrl_qubits))

    def rz(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.RZ(para).on(obj_qubits, ctrl_qubits))

    def phase_shift(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.PhaseShift(para).on(obj_qubits, ctrl_qubits))

    def global_phase(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.GlobalPhase(para).on(obj_qubits, ctrl_qubits))

    def givens(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Givens(para).on(obj_qubits, ctrl_qubits))

    def rxx(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Rxx(para).on(obj_qubits, ctrl_qubits))

    def rxy(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Rxy(para).on(obj_qubits, ctrl_qubits))

    def rxz(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Rxz(para).on(obj_qubits, ctrl_qubits))

    def ryy(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Ryy(para).on(obj_qubits, ctrl_qubits))

    def ryz(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Ryz(para).on(obj_qubits, ctrl_qubits))

    def rzz(self, para, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.Rzz(para).on(obj_qubits, ctrl_qubits))

    def fsim(self, theta, phi, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.FSim(theta, phi).on(obj_qubits, ctrl_qubits))

    def u3(self, theta, phi, lam, obj_qubits, ctrl_qubits=None):
        return self.__iadd__(G.U3(theta, phi, lam).on(obj_qubits, ctrl_qubits))

    def measure(self, key, obj_qubit=None, reset_to=None):
        if obj_qubit is None:
            if not isinstance(key, int):
                raise ValueError("Need an object qubit for the measure gate.")
            obj_qubit, key = key, f"q{key}"
        return self.__iadd__(G.Measure(key, reset_to).on(obj_qubit))

    def measure_all(self, suffix=None, up_to: int = -1):
        n = self.n_qubits if up_to == -1 else up_to + 1
        for i in range(n):
            self.measure(f"q{i}" + (f"_{suffix}" if suffix else ""), i)
        return self

    def barrier(self, show=True):
        super().append(G.BarrierGate(show))
        return self

    def un(self, gate, maps_obj, maps_ctrl=None):
        return self.__iadd__(UN(gate, maps_obj, maps_ctrl))

    # ------------------------------------------------------------------ evaluation
    def get_qs(self, backend='mqvector_b200', pr=None, ket=False, seed=None, dtype=None):
        """Final state of this circuit from |0...0> on ``backend`` (circuit.py:1598-1616)."""
        from ..simulator import Simulator  # pylint: disable=import-outside-toplevel

        sim = Simulator(backend, self.n_qubits, seed=seed, dtype=dtype)
        sim.apply_circuit(self, pr)
        return sim.get_qs(ket)

    def matrix(self, pr=None, big_end=False, backend='mqvector_b200', seed=None, dtype=None):
        """Unitary of this circuit, column j = circuit applied to |j> (circuit.py:946-992)."""
        from ..simulator import Simulator  # pylint: disable=import-outside-toplevel

        n = self.n_qubits
        cols = []
        for j in range(1 << n):
            sim = Simulator(backend, n, seed=seed, dtype=dtype)
            v = np.zeros(1 << n, dtype=complex)
            v[j] = 1
            sim.set_qs(v)
            sim.apply_circuit(self.remove_measure(), pr)
            cols.append(sim.get_qs())
        m = np.array(cols).T
        if big_end:
            perm = [int(format(i, f'0{n}b')[::-1], 2) for i in range(1 << n)]
            m = m[np.ix_(perm, perm)]
        return m

    def __str__(self):
        return "\n".join(str(g) for g in self)

    __repr__ = __str__


def UN(gate, maps_obj, maps_ctrl=None):  # pylint: disable=invalid-name
    """Map a gate onto many qubits (mindquantum/core/circuit/module_circuit.py UN)."""
    if isinstance(maps_obj, int):
        maps_obj = list(range(maps_obj))
    maps_obj = list(maps_obj)
    if maps_ctrl is None:
        maps_ctrl = [None] * len(maps_obj)
    elif isinstance(maps_ctrl, int):
        maps_ctrl = [maps_ctrl] * len(maps_obj)
    return Circuit([gate.on(o, c) for o, c in zip(maps_obj, maps_ctrl)])


def SwapParts(a, b, maps_ctrl=None):  # pylint: disable=invalid-name
    """Swap qubits a[i] <-> b[i] (module_circuit.py SwapParts)."""
    return Circuit([G.SWAP.on([i, j], maps_ctrl) for i, j in zip(a, b)])


def qft(qubits):
    """Quantum Fourier transform: H, controlled phase shifts 2pi/2^k, then qubit reversal.

    Same gate sequence as mindquantum/algorithm/library/quantum_fourier.py:19-66.
    """
    qubits = list(qubits)
    circuit = Circuit()
    n = len(qubits)
    for i in range(n):
        sub = qubits[i:]
        circuit += G.H.on(sub[0])
        for index, ctrl_qubit in enumerate(sub[1:]):
            circuit += G.PhaseShift(2 * np.pi / 2 ** (index + 2)).on(sub[0], ctrl_qubit)
    if n > 1:
        part1 = [qubits[j] for j in range(n // 2)]
        part2 = [qubits[n - 1 - j] for j in range(n // 2)]
        circuit += SwapParts(part1, part2)
    return circuit
