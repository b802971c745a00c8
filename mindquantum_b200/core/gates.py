"""Quantum gates of the state-vector path.

Mirrors the reference gate classes (mindquantum/core/gates/basicgate.py, basic.py,
measurement.py) for the gates that ``VectorState::ApplyGate`` dispatches
(ccsrc/include/simulator/vector/vector_state.tpp:166-437): Pauli/Clifford/T gates,
single- and two-qubit Pauli rotations, phase gates, SWAP-like gates, U3 / Rn / FSim,
rotations about a Pauli string, constant and parameterized custom matrix gates,
measurement and barriers.

Each gate knows:
  * ``matrix(pr)`` / ``diff_matrix(pr, about_what)`` in numpy (dense references);
  * ``hermitian()`` with the reference semantics (parameterized rotations negate
    their coefficient, basic.py:510-515; U3(-t,-l,-p), basicgate.py:2445-2454;
    non-Hermitian constant gates toggle ``hermitianed``);
  * its device lowering: a gate id from ``mindquantum_b200/csrc/mqb_gate_ids.h``
    plus up to three angle expressions, or a constant matrix.
"""
from __future__ import annotations

import copy
import numbers
from typing import List

import numpy as np
from scipy.linalg import fractional_matrix_power

from .parameterresolver import ParameterResolver

# Device gate ids: keep in sync with mindquantum_b200/csrc/mqb_gate_ids.h
GID_MATRIX = 0
GID_RX, GID_RY, GID_RZ, GID_PS, GID_GP = 1, 2, 3, 4, 5
GID_RXX, GID_RYY, GID_RZZ, GID_RXY, GID_RXZ, GID_RYZ = 6, 7, 8, 9, 10, 11
GID_GIVENS, GID_SWAPALPHA, GID_U3, GID_RN, GID_FSIM, GID_RPS = 12, 13, 14, 15, 16, 17
GID_CUSTOM = 18

_SQ2 = 1 / np.sqrt(2)
MAT = {
    'X': np.array([[0, 1], [1, 0]], dtype=complex),
    'Y': np.array([[0, -1j], [1j, 0]], dtype=complex),
    'Z': np.array([[1, 0], [0, -1]], dtype=complex),
    'I': np.array([[1, 0], [0, 1]], dtype=complex),
    'H': np.array([[1, 1], [1, -1]], dtype=complex) * _SQ2,
    'S': np.array([[1, 0], [0, 1j]], dtype=complex),
    'T': np.array([[1, 0], [0, (1 + 1j) * _SQ2]], dtype=complex),
    'SX': np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]], dtype=complex) / 2,
    'ISWAP': np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=complex),
    'SWAP': np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex),
    'CNOT': np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex),
}


def _qubit_list(q) -> List[int]:
    if q is None:
        return []
    if isinstance(q, numbers.Integral):
        return [int(q)]
    return [int(i) for i in q]


def pauli_string_matrix(pauli: str) -> np.ndarray:
    """Matrix of a Pauli string whose i-th letter acts on the i-th object qubit (little endian)."""
    m = np.array([[1]], dtype=complex)
    for p in pauli:
        m = np.kron(MAT[p.upper()], m)
    return m


def two_qubit_rotation_matrix(pauli: str, val: float, diff: bool = False) -> np.ndarray:
    """exp(-i val/2 P) (or its val-derivative) with P = pauli[0] on obj0 (x) pauli[1] on obj1."""
    mp = pauli_string_matrix(pauli)
    mi = np.identity(len(mp), dtype=complex)
    if diff:
        return 0.5 * (-np.sin(val / 2) * mi - 1j * np.cos(val / 2) * mp)
    return np.cos(val / 2) * mi - 1j * np.sin(val / 2) * mp


class BasicGate:
    """Base of all gates: name, object qubits, control qubits."""

    n_qubits_fixed = True

    def __init__(self, name: str, n_qubits: int, obj_qubits=None, ctrl_qubits=None):
        self.name = name
        self.n_qubits = n_qubits
        self.obj_qubits: List[int] = _qubit_list(obj_qubits)
        self.ctrl_qubits: List[int] = _qubit_list(ctrl_qubits)
        self.hermitianed = False

    # --------------------------------------------------------------- placement
    def on(self, obj_qubits, ctrl_qubits=None):
        """Return a copy acting on ``obj_qubits`` controlled by ``ctrl_qubits``."""
        objs = _qubit_list(obj_qubits)
        ctrls = _qubit_list(ctrl_qubits)
        if not objs:
            raise ValueError("obj_qubits cannot be empty.")
        if any(q < 0 for q in objs + ctrls):
            raise ValueError("Qubit index should not be negative.")
        if len(set(objs)) != len(objs):
            raise RuntimeError(f"obj_qubits of {self.name} cannot have same qubits.")
        if len(set(ctrls)) != len(ctrls):
            raise RuntimeError(f"ctrl_qubits of {self.name} cannot have same qubits.")
        if set(objs) & set(ctrls):
            raise RuntimeError("obj_qubits and ctrl_qubits cannot have same qubits.")
        if self.n_qubits_fixed and len(objs) != self.n_qubits:
            raise ValueError(f"{self.name} acts on {self.n_qubits} qubit(s), but get {len(objs)} object qubits.")
        new = copy.deepcopy(self)
        new.obj_qubits = objs
        new.ctrl_qubits = ctrls
        if not self.n_qubits_fixed:
            new.n_qubits = len(objs)
        return new

    @property
    def parameterized(self) -> bool:
        return False

    def get_parameters(self) -> List[ParameterResolver]:
        return []

    def __params_prop__(self):
        keys, ansatz, encoder = [], [], []
        for pr in self.get_parameters():
            keys.extend(pr.params_name)
            ansatz.extend(pr.ansatz_parameters)
            encoder.extend(pr.encoder_parameters)
        return keys, ansatz, encoder

    def hermitian(self):
        return copy.deepcopy(self)

    def matrix(self, pr=None, full=False):  # pylint: disable=unused-argument
        raise NotImplementedError

    def __str__(self):
        s = self.name + ('†' if self.hermitianed else '')
        qs = ' '.join(str(q) for q in self.obj_qubits)
        if self.ctrl_qubits:
            qs += ' <-: ' + ' '.join(str(q) for q in self.ctrl_qubits)
        return f"{s}({qs})"

    __repr__ = __str__


class FixedGate(BasicGate):
    """A gate with a constant matrix (Pauli, H, S, T, SX, SWAP, ISWAP, custom constant matrices)."""

    def __init__(self, name, matrix_value, obj_qubits=None, ctrl_qubits=None, self_hermitian=False):
        matrix_value = np.asarray(matrix_value, dtype=complex)
        super().__init__(name, int(np.log2(matrix_value.shape[0])), obj_qubits, ctrl_qubits)
        self._matrix = matrix_value
        self.self_hermitian = self_hermitian

    def matrix(self, pr=None, full=False):  # pylint: disable=unused-argument
        if self.hermitianed:
            return np.conj(self._matrix).T.copy()
        return self._matrix.copy()

    def hermitian(self):
        new = copy.deepcopy(self)
        if not self.self_hermitian:
            new.hermitianed = not new.hermitianed
        return new


class XGate(FixedGate):
    def __init__(self):
        super().__init__('X', MAT['X'], self_hermitian=True)


class YGate(FixedGate):
    def __init__(self):
        super().__init__('Y', MAT['Y'], self_hermitian=True)


class ZGate(FixedGate):
    def __init__(self):
        super().__init__('Z', MAT['Z'], self_hermitian=True)


class IGate(FixedGate):
    def __init__(self):
        super().__init__('I', MAT['I'], self_hermitian=True)


class HGate(FixedGate):
    def __init__(self):
        super().__init__('H', MAT['H'], self_hermitian=True)


class SGate(FixedGate):
    def __init__(self):
        super().__init__('S', MAT['S'])


class TGate(FixedGate):
    def __init__(self):
        super().__init__('T', MAT['T'])


class SXGate(FixedGate):
    def __init__(self):
        super().__init__('SX', MAT['SX'])


class SWAPGate(FixedGate):
    def __init__(self):
        super().__init__('SWAP', MAT['SWAP'], self_hermitian=True)


class ISWAPGate(FixedGate):
    def __init__(self):
        super().__init__('ISWAP', MAT['ISWAP'])


class CNOTGate(FixedGate):
    """CNOT.on(obj, ctrl) is an X gate on ``obj`` controlled by ``ctrl`` (basicgate.py:454-456)."""

    def __init__(self):
        super().__init__('CNOT', MAT['X'], self_hermitian=True)

    def on(self, obj_qubits, ctrl_qubits=None):
        objs = _qubit_list(obj_qubits)
        ctrls = _qubit_list(ctrl_qubits)
        if len(objs) == 2 and not ctrls:
            objs, ctrls = [objs[0]], [objs[1]]
        g = XGate().on(objs, ctrls)
        return g


class UnivMathGate(FixedGate):
    """A constant custom matrix gate (basicgate.py:54-93)."""

    def __init__(self, name, matrix_value):
        matrix_value = np.asarray(matrix_value)
        if matrix_value.ndim != 2 or matrix_value.shape[0] != matrix_value.shape[1]:
            raise ValueError(f"matrix_value need a square matrix, but get shape {matrix_value.shape}")
        n = matrix_value.shape[0]
        if n & (n - 1) or n < 2:
            raise ValueError(f"Dimension of matrix_value need should be power of 2, but get {n}")
        super().__init__(name, matrix_value)


class Power(FixedGate):
    """Fractional power of a constant gate (basicgate.py:1756-1800)."""

    def __init__(self, gate, exponent=0.5):
        super().__init__(f'{gate.name}^{exponent}', fractional_matrix_power(gate.matrix(), exponent))
        self.gate = gate
        self.t = exponent


class ParameterGate(BasicGate):
    """A gate whose parameters are ParameterResolvers."""

    gate_id = GID_MATRIX

    def __init__(self, name, n_qubits, prs, obj_qubits=None, ctrl_qubits=None):
        super().__init__(name, n_qubits, obj_qubits, ctrl_qubits)
        self.prs: List[ParameterResolver] = [ParameterResolver(p) for p in prs]

    @property
    def coeff(self) -> ParameterResolver:
        return self.prs[0]

    @coeff.setter
    def coeff(self, value):
        self.prs[0] = ParameterResolver(value)

    @property
    def parameterized(self) -> bool:
        return any(not p.is_const() for p in self.prs)

    def get_parameters(self):
        return self.prs

    def values(self, pr=None):
        """Evaluate every parameter of this gate against ``pr``."""
        out = []
        for p in self.prs:
            if p.is_const():
                out.append(float(np.real(p.const)))
            else:
                if pr is None:
                    raise ValueError("The parameter is not set completed.")
                out.append(float(np.real(p.combination(pr).const)))
        return out

    def hermitian(self):
        new = copy.deepcopy(self)
        new.prs = [-p for p in new.prs]
        return new

    def matrix_of(self, vals) -> np.ndarray:
        raise NotImplementedError

    def diff_matrix_of(self, vals, idx) -> np.ndarray:
        raise NotImplementedError

    def matrix(self, pr=None, full=False):  # pylint: disable=unused-argument
        return self.matrix_of(self.values(pr))

    def diff_matrix(self, pr=None, about_what=None):
        """d(matrix)/d(about_what) through every parameter that contains it."""
        vals = self.values(pr)
        if about_what is None:
            names = [k for p in self.prs for k in p.params_name]
            if len(set(names)) != 1:
                raise ValueError("Should specific which parameter are going to do derivation.")
            about_what = names[0]
        out = 0
        for i, p in enumerate(self.prs):
            if about_what in p:
                out = out + p[about_what] * self.diff_matrix_of(vals, i)
        if isinstance(out, int):
            return np.zeros((1 << self.n_qubits, 1 << self.n_qubits), dtype=complex)
        return out

    def __str__(self):
        s = ', '.join(str(p) for p in self.prs)
        qs = ' '.join(str(q) for q in self.obj_qubits)
        if self.ctrl_qubits:
            qs += ' <-: ' + ' '.join(str(q) for q in self.ctrl_qubits)
        return f"{self.name}({s}|{qs})"

    __repr__ = __str__


class RX(ParameterGate):
    """exp(-i t/2 X); ApplyRX, cpu_vector_core_rot_pauli.cpp:432-446."""

    gate_id = GID_RX

    def __init__(self, pr):
        super().__init__('RX', 1, [pr])

    def matrix_of(self, v):
        c, s = np.cos(v[0] / 2), np.sin(v[0] / 2)
        return np.array([[c, -1j * s], [-1j * s, c]])

    def diff_matrix_of(self, v, idx):
        c, s = np.cos(v[0] / 2), np.sin(v[0] / 2)
        return 0.5 * np.array([[-s, -1j * c], [-1j * c, -s]])


class RY(ParameterGate):
    """exp(-i t/2 Y); ApplyRY, cpu_vector_core_rot_pauli.cpp:449-463."""

    gate_id = GID_RY

    def __init__(self, pr):
        super().__init__('RY', 1, [pr])

    def matrix_of(self, v):
        c, s = np.cos(v[0] / 2), np.sin(v[0] / 2)
        return np.array([[c, -s], [s, c]], dtype=complex)

    def diff_matrix_of(self, v, idx):
        c, s = np.cos(v[0] / 2), np.sin(v[0] / 2)
        return 0.5 * np.array([[-s, -c], [c, -s]], dtype=complex)


class RZ(ParameterGate):
    """exp(-i t/2 Z); ApplyRZ, cpu_vector_core_rot_pauli.cpp:526-541."""

    gate_id = GID_RZ

    def __init__(self, pr):
        super().__init__('RZ', 1, [pr])

    def matrix_of(self, v):
        return np.diag([np.exp(-0.5j * v[0]), np.exp(0.5j * v[0])])

    def diff_matrix_of(self, v, idx):
        return np.diag([-0.5j * np.exp(-0.5j * v[0]), 0.5j * np.exp(0.5j * v[0])])


class PhaseShift(ParameterGate):
    """diag(1, e^{i t}); ApplyPS, cpu_vector_core_z_like.cpp:95-130."""

    gate_id = GID_PS

    def __init__(self, pr):
        super().__init__('PS', 1, [pr])

    def matrix_of(self, v):
        return np.diag([1, np.exp(1j * v[0])])

    def diff_matrix_of(self, v, idx):
        return np.diag([0, 1j * np.exp(1j * v[0])])


class GlobalPhase(ParameterGate):
    """e^{-i t} I; ApplyGP, cpu_common/cpu_vector_core_other_gate.cpp:53-60."""

    gate_id = GID_GP

    def __init__(self, pr):
        super().__init__('GP', 1, [pr])

    def matrix_of(self, v):
        return np.exp(-1j * v[0]) * np.identity(2)

    def diff_matrix_of(self, v, idx):
        return -1j * np.exp(-1j * v[0]) * np.identity(2)


class _TwoQubitPauliRotation(ParameterGate):
    pauli = 'XX'

    def __init__(self, pr):
        super().__init__('R' + self.pauli.lower(), 2, [pr])
        self.name = 'R' + self.pauli[0].lower() + self.pauli[1].lower()

    def matrix_of(self, v):
        return two_qubit_rotation_matrix(self.pauli, v[0])

    def diff_matrix_of(self, v, idx):
        return two_qubit_rotation_matrix(self.pauli, v[0], diff=True)


class Rxx(_TwoQubitPauliRotation):
    """exp(-i t/2 X0 X1); ApplyRxx, cpu_vector_core_rot_pauli.cpp:31-86."""

    gate_id = GID_RXX
    pauli = 'XX'


class Ryy(_TwoQubitPauliRotation):
    """exp(-i t/2 Y0 Y1); ApplyRyy, cpu_vector_core_rot_pauli.cpp:322-377."""

    gate_id = GID_RYY
    pauli = 'YY'


class Rzz(_TwoQubitPauliRotation):
    """exp(-i t/2 Z0 Z1); ApplyRzz, cpu_vector_core_rot_pauli.cpp:380-428."""

    gate_id = GID_RZZ
    pauli = 'ZZ'


class Rxy(_TwoQubitPauliRotation):
    """exp(-i t/2 X_obj0 Y_obj1); ApplyRxy, cpu_vector_core_rot_pauli.cpp:89-144."""

    gate_id = GID_RXY
    pauli = 'XY'


class Rxz(_TwoQubitPauliRotation):
    """exp(-i t/2 X_obj0 Z_obj1); ApplyRxz, cpu_vector_core_rot_pauli.cpp:147-202."""

    gate_id = GID_RXZ
    pauli = 'XZ'


class Ryz(_TwoQubitPauliRotation):
    """exp(-i t/2 Y_obj0 Z_obj1); ApplyRyz, cpu_vector_core_rot_pauli.cpp:264-319."""

    gate_id = GID_RYZ
    pauli = 'YZ'


class Givens(ParameterGate):
    """Givens rotation on |01>,|10> (basicgate.py:617-704; ApplyGivens, cpu_vector_core_rot_pauli.cpp:205-261)."""

    gate_id = GID_GIVENS

    def __init__(self, pr):
        super().__init__('G', 2, [pr])

    def matrix_of(self, v):
        c, s = np.cos(v[0]), np.sin(v[0])
        return np.array([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]], dtype=complex)

    def diff_matrix_of(self, v, idx):
        c, s = np.cos(v[0]), np.sin(v[0])
        return np.array([[0, 0, 0, 0], [0, -s, -c, 0], [0, c, -s, 0], [0, 0, 0, 0]], dtype=complex)


class SWAPalpha(ParameterGate):
    """SWAP^alpha (basicgate.py:849-936; ApplySWAPalpha, cpu_vector_core_swap_like.cpp:107-150)."""

    gate_id = GID_SWAPALPHA

    def __init__(self, pr):
        super().__init__('SWAPalpha', 2, [pr])

    def matrix_of(self, v):
        e = np.exp(1j * np.pi * v[0])
        a, b = (1 + e) / 2, (1 - e) / 2
        return np.array([[1, 0, 0, 0], [0, a, b, 0], [0, b, a, 0], [0, 0, 0, 1]])

    def diff_matrix_of(self, v, idx):
        e = 0.5j * np.pi * np.exp(1j * np.pi * v[0])
        return np.array([[0, 0, 0, 0], [0, e, -e, 0], [0, -e, e, 0], [0, 0, 0, 0]])


class U3(ParameterGate):
    """U3(theta, phi, lambda) (gates.cpp:29-37; basicgate.py:2370-2505)."""

    gate_id = GID_U3

    def __init__(self, theta, phi, lam):
        super().__init__('U3', 1, [theta, phi, lam])

    @property
    def theta(self):
        return self.prs[0]

    @property
    def phi(self):
        return self.prs[1]

    @property
    def lamda(self):
        return self.prs[2]

    def hermitian(self):
        """U3(-theta, -lambda, -phi), basicgate.py:2445-2454."""
        new = copy.deepcopy(self)
        new.prs = [-self.prs[0], -self.prs[2], -self.prs[1]]
        return new

    def matrix_of(self, v):
        t, p, l = v
        c, s = np.cos(t / 2), np.sin(t / 2)
        return np.array([[c, -np.exp(1j * l) * s], [np.exp(1j * p) * s, np.exp(1j * (l + p)) * c]])

    def diff_matrix_of(self, v, idx):
        """U3DiffTheta/Phi/LambdaMatrix, gates.cpp:138-170."""
        t, p, l = v
        c, s = np.cos(t / 2), np.sin(t / 2)
        if idx == 0:
            return 0.5 * np.array([[-s, -np.exp(1j * l) * c], [np.exp(1j * p) * c, -np.exp(1j * (l + p)) * s]])
        if idx == 1:
            return np.array([[0, 0], [1j * np.exp(1j * p) * s, 1j * np.exp(1j * (l + p)) * c]])
        return np.array([[0, -1j * np.exp(1j * l) * s], [0, 1j * np.exp(1j * (l + p)) * c]])


class Rn(ParameterGate):
    """Rotation about (alpha, beta, gamma) (gates.cpp:48-72; basicgate.py:2232-2365)."""

    gate_id = GID_RN

    def __init__(self, alpha, beta, gamma):
        super().__init__('Rn', 1, [alpha, beta, gamma])

    def matrix_of(self, v):
        a, b, g = v
        f = np.sqrt(a * a + b * b + g * g)
        if f == 0:
            return np.identity(2, dtype=complex)
        h = (a * MAT['X'] + b * MAT['Y'] + g * MAT['Z']) / f
        return np.cos(f / 2) * np.identity(2) - 1j * np.sin(f / 2) * h

    def diff_matrix_of(self, v, idx):
        a, b, g = v
        f = np.sqrt(a * a + b * b + g * g)
        if f == 0:
            return np.zeros((2, 2), dtype=complex)
        comp = (a, b, g)[idx]
        sig = (MAT['X'], MAT['Y'], MAT['Z'])[idx]
        h = a * MAT['X'] + b * MAT['Y'] + g * MAT['Z']
        cc, sc = np.cos(f / 2), np.sin(f / 2)
        fa = comp / f
        return (-0.5 * fa * sc * np.identity(2) - 1j * h * fa * (cc / 2 / f - sc / f / f) - 1j * sig * sc / f)


class FSim(ParameterGate):
    """FSim(theta, phi) (gates.cpp:39-46; basicgate.py:2512-2640)."""

    gate_id = GID_FSIM

    def __init__(self, theta, phi):
        super().__init__('FSim', 2, [theta, phi])

    @property
    def theta(self):
        return self.prs[0]

    @property
    def phi(self):
        return self.prs[1]

    def matrix_of(self, v):
        t, p = v
        a, b = np.cos(t), -1j * np.sin(t)
        return np.array([[1, 0, 0, 0], [0, a, b, 0], [0, b, a, 0], [0, 0, 0, np.exp(-1j * p)]])

    def diff_matrix_of(self, v, idx):
        t, p = v
        if idx == 0:
            a, b = -np.sin(t), -1j * np.cos(t)
            return np.array([[0, 0, 0, 0], [0, a, b, 0], [0, b, a, 0], [0, 0, 0, 0]])
        out = np.zeros((4, 4), dtype=complex)
        out[3, 3] = -1j * np.exp(-1j * p)
        return out


class RotPauliString(ParameterGate):
    """exp(-i t/2 P) for a Pauli string P on the object qubits (basicgate.py:1567-1675; ApplyRPS)."""

    gate_id = GID_RPS
    n_qubits_fixed = True

    def __init__(self, pauli_string: str, pr):
        for p in pauli_string:
            if p not in 'ixyzIXYZ':
                raise ValueError(f"Unknown pauli operator {p}.")
        self.pauli_string = pauli_string.upper()
        super().__init__('RPS', len(pauli_string), [pr])

    def matrix_of(self, v):
        mp = pauli_string_matrix(self.pauli_string)
        return np.cos(v[0] / 2) * np.identity(len(mp)) - 1j * np.sin(v[0] / 2) * mp

    def diff_matrix_of(self, v, idx):
        mp = pauli_string_matrix(self.pauli_string)
        return 0.5 * (-np.sin(v[0] / 2) * np.identity(len(mp)) - 1j * np.cos(v[0] / 2) * mp)


class ParamNonHerm(ParameterGate):
    """A parameterized custom matrix gate built by :func:`gene_univ_parameterized_gate`."""

    gate_id = GID_CUSTOM
    n_qubits_fixed = True

    def __init__(self, name, n_qubits, matrix_generator, diff_matrix_generator, pr):
        super().__init__(name, n_qubits, [pr])
        self.matrix_generator = matrix_generator
        self.diff_matrix_generator = diff_matrix_generator

    def hermitian(self):
        """Same parameter, conjugate-transposed matrices (basicgate.py:1938-1947)."""
        new = copy.deepcopy(self)
        new.hermitianed = not self.hermitianed
        return new

    def matrix_of(self, v):
        m = np.asarray(self.matrix_generator(v[0]), dtype=complex)
        return np.conj(m).T.copy() if self.hermitianed else m

    def diff_matrix_of(self, v, idx):
        m = np.asarray(self.diff_matrix_generator(v[0]), dtype=complex)
        return np.conj(m).T.copy() if self.hermitianed else m


def gene_univ_parameterized_gate(name, matrix_generator, diff_matrix_generator):
    """Build a parameterized custom gate class (basicgate.py:1808-1960).

    ``matrix_generator(x)`` returns the 2^k x 2^k matrix and ``diff_matrix_generator(x)``
    its derivative with respect to ``x``.  The matrices are evaluated on the host for
    every parameter value and uploaded; everything else runs on the device.
    """
    m0 = np.asarray(matrix_generator(0.123))
    n_qubits = int(np.log2(m0.shape[0]))

    class _ParamNonHerm(ParamNonHerm):
        def __init__(self, pr):
            super().__init__(name, n_qubits, matrix_generator, diff_matrix_generator, pr)

    return _ParamNonHerm


class Measure(BasicGate):
    """Computational-basis measurement of one qubit (measurement.py; ApplyMeasure, vector_state.tpp:440-462)."""

    def __init__(self, key: str = None, reset_to=None):
        super().__init__('M', 1)
        self.key = key
        self.reset_to = reset_to

    def on(self, obj_qubits, ctrl_qubits=None):
        if ctrl_qubits:
            raise ValueError("Measure gate cannot have control qubits.")
        new = super().on(obj_qubits)
        if new.key is None:
            new.key = f"q{new.obj_qubits[0]}"
        return new

    def __str__(self):
        return f"M({self.key})"


class BarrierGate(BasicGate):
    """A no-op that only separates gates in drawings."""

    n_qubits_fixed = False

    def __init__(self, show=True):
        super().__init__('BARRIER', 0)
        self.show = show


class NoiseGate(BasicGate):
    """A quantum channel, simulated as a stochastic trajectory (VectorState::ApplyChannel,
    vector_state.tpp:465-709; classes of mindquantum/core/gates/channel.py)."""

    def hermitian(self):
        new = copy.deepcopy(self)
        new.hermitianed = not new.hermitianed
        return new


def _check_real(name, v):
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise TypeError(f"Unsupported type for {name}, get {type(v)}.")


class PauliChannel(NoiseGate):
    """X, Y, Z with probabilities px, py, pz, identity otherwise (channel.py:125-230)."""

    def __init__(self, px: float, py: float, pz: float, name: str = 'PC'):
        super().__init__(name, 1)
        for k, v in (('px', px), ('py', py), ('pz', pz)):
            _check_real(k, v)
        if min(px, py, pz) < 0.0:
            raise ValueError("Probability cannot be negative value.")
        if not 0 <= px + py + pz <= 1:
            raise ValueError("Required total probability P = px + py + pz ∈ [0,1].")
        self.px, self.py, self.pz = float(px), float(py), float(pz)

    def hermitian(self):
        return copy.deepcopy(self)

    def cumulative_probs(self):
        """[0, px, px + py, px + py + pz, 1] (PauliChannel, ccsrc/include/ops/basic_gate.h:341-352)."""
        probs = [self.px, self.py, self.pz, 1 - self.px - self.py - self.pz]
        out, acc = [0.0], 0.0
        for p in probs:
            acc += p
            out.append(acc)
        return out


class BitFlipChannel(PauliChannel):
    def __init__(self, p: float):
        super().__init__(p, 0, 0, 'BFC')


class PhaseFlipChannel(PauliChannel):
    def __init__(self, p: float):
        super().__init__(0, 0, p, 'PFC')


class BitPhaseFlipChannel(PauliChannel):
    def __init__(self, p: float):
        super().__init__(0, p, 0, 'BPFC')


class GroupedPauliChannel(NoiseGate):
    """One independent Pauli channel per object qubit, rows of ``probs`` = (px, py, pz) (channel.py:32-123)."""

    def __init__(self, probs):
        if not isinstance(probs, np.ndarray):
            raise TypeError(f"probs requires a numpy.ndarray, but get {type(probs)}")
        if not np.issubdtype(probs.dtype, np.floating):
            raise TypeError(f"probs requires a real number type, but get {probs.dtype}")
        if np.any(probs < 0.0):
            raise ValueError("probs cannot be negative value.")
        if probs.ndim != 2:
            raise ValueError(f"probs requires a two dimension array, but get dimension with {probs.shape}")
        if probs.shape[1] != 3:
            raise ValueError(f"The second dimension of probs should be two, but get {probs.shape[1]}")
        wrong = np.where(probs.sum(axis=1) > 1)[0]
        if wrong.shape[0]:
            raise ValueError(f"Wrong probs for {wrong[0]}-pauli channel: {probs[wrong[0]]}")
        super().__init__('GPC', probs.shape[0])
        self.probs = probs

    def hermitian(self):
        return copy.deepcopy(self)


class DepolarizingChannel(NoiseGate):
    """Depolarizing channel on n qubits with parameter p (channel.py:425-528)."""

    def __init__(self, p: float, n_qubits: int = 1):
        super().__init__('DC', n_qubits)
        _check_real('argument p', p)
        if not 0 <= p <= 4**n_qubits / (4**n_qubits - 1):
            raise ValueError(f"Required argument p ∈ [0, {4**n_qubits}/{4**n_qubits - 1}], but get p = {p}.")
        self.p = p

    def hermitian(self):
        return copy.deepcopy(self)


class AmplitudeDampingChannel(NoiseGate):
    """Amplitude damping with coefficient gamma (channel.py:530-606)."""

    def __init__(self, gamma: float):
        super().__init__('ADC', 1)
        _check_real('gamma', gamma)
        if not 0 <= gamma <= 1:
            raise ValueError("Required damping coefficient gamma ∈ [0,1].")
        self.gamma = gamma


class PhaseDampingChannel(NoiseGate):
    """Phase damping with coefficient gamma (channel.py:608-684)."""

    def __init__(self, gamma: float):
        super().__init__('PDC', 1)
        _check_real('gamma', gamma)
        if not 0 <= gamma <= 1:
            raise ValueError("Required damping coefficient gamma ∈ [0,1].")
        self.gamma = gamma


class KrausChannel(NoiseGate):
    """A single-qubit channel given by its Kraus operators (channel.py:686-766)."""

    def __init__(self, name: str, kraus_op):
        kraus_op = np.asarray(kraus_op)
        if not np.issubdtype(kraus_op.dtype, np.number):
            raise TypeError(f"{name} requires a numerical array, but get {kraus_op.dtype}")
        for mat in kraus_op:
            if mat.ndim != 2:
                raise ValueError(f"matrix_value require shape of 2, but get shape of {mat.shape}")
            if mat.shape[0] != mat.shape[1]:
                raise ValueError(f"matrix_value need a square matrix, but get shape {mat.shape}")
            if mat.shape[0] != 2:
                raise ValueError(f"Dimension of matrix_value need should be 2, but get {mat.shape[0]}")
        total = sum(np.conj(m).T @ m for m in kraus_op.astype(np.complex128))
        if not np.allclose(total, np.eye(2), atol=1e-6):
            raise ValueError(f"kraus_op need to satisfy the completeness condition, but get {total}")
        super().__init__(name, 1)
        self.kraus_op = kraus_op


class ThermalRelaxationChannel(NoiseGate):
    """Thermal relaxation with times T1, T2 and the gate time (channel.py:768-871)."""

    def __init__(self, t1: float, t2: float, gate_time: float):
        super().__init__('TRC', 1)
        for k, v in (('t1', t1), ('t2', t2), ('gate_time', gate_time)):
            _check_real(k, v)
        if t1 <= 0 or t2 <= 0:
            raise ValueError(f"T1 and T2 must be positive, but get T1={t1}, T2={t2}")
        if gate_time < 0:
            raise ValueError(f"gate time cannot be negative, but get {gate_time}")
        if t2 >= 2 * t1:
            raise ValueError("(T2 >= 2 * T1) is invalid case for thermal relaxation channel.")
        self.t1, self.t2, self.gate_time = t1, t2, gate_time


# Singletons with the reference's names
X = XGate()
Y = YGate()
Z = ZGate()
I = IGate()  # noqa: E741
H = HGate()
S = SGate()
T = TGate()
SX = SXGate()
SWAP = SWAPGate()
ISWAP = ISWAPGate()
CNOT = CNOTGate()
