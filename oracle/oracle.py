"""CPU oracle for the MindQuantum state-vector hot path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, and only as the checker / the timed reference CPU implementation.  The
product (``mindquantum_b200``) never imports it.

What it restates (reference file:line, paths inside mindquantum-ai/mindquantum):
  * ``VectorState::ApplyGate`` dispatch, ccsrc/include/simulator/vector/vector_state.tpp:166-437,
    with the per-gate kernels of the CPU policy (ccsrc/lib/simulator/vector/detail/cpu_common/*)
    restated in ``mqvector_oracle.c``;
  * ``ExpectDiffGate`` / ``ExpectDiffU3`` / ``ExpectDiffRn`` / ``ExpectDiffFSim``,
    vector_state.tpp:778-946, with the diff matrices of cpu_vector_core_gate_expect.cpp and
    ccsrc/lib/mq_base/gates/gates.cpp:29-170;
  * ``GradientHelper::HermitianAdjointGradient`` / ``LeftSizeGrad`` / ``GradRealDouble`` /
    ``GeneratePMap`` and the Jacobi of ``Parameterizable`` (ccsrc/include/simulator/vector/gradient.h:100-197,
    ccsrc/include/ops/basic_gate.h:208-241, ccsrc/lib/math/pr/parameter_resolver.cpp:560-573);
  * ``GetExpectation`` (vector_state.tpp:712-726), ``ApplyHamiltonian`` (vector_state.tpp:963-974),
    with ``Csr_Dot_Vec`` / ``ExpectationOfCsr`` (ccsrc/include/core/sparse/algo.h:160-200) for
    Hamiltonians given as sparse matrices;
  * ``GetExpectationWithGradParameterShiftOneMulti`` / ``MultiMulti`` (vector_state.tpp:1033-1305)
    in ``get_expectation_with_grad_parameter_shift``, with the shift table of ``shift_rule``;
  * ``ApplyChannel`` and the channel kernels (vector_state.tpp:465-709) in ``apply_channel``, and the
    parameter-shift loop with stochastic channels in ``get_expectation_with_grad_parameter_shift_noisy``;
  * ``SamplingMeasurementEndingWithoutNoise`` (vector_state.tpp:1326-1373) with the reference's
    random streams (std::mt19937 + std::uniform_real_distribution<double>), restated in
    ``_Mt19937`` / ``_uniform``.

The hermitian circuit is built exactly as the reference Python does (reversed daggers with
negated parameter coefficients; U3 -> U3(-t,-l,-p)), and the gradient is accumulated through
the Jacobi of the daggered gates, so the oracle follows the reference algorithm step for step.

Gates are read duck-typed from gate objects: ``name``, ``obj_qubits``, ``ctrl_qubits``,
``prs`` (parameter expressions with ``const`` and ``items()``), ``hermitianed``,
``pauli_string``, ``matrix_generator`` / ``diff_matrix_generator`` (custom parameterized
gates) and ``matrix()`` for constant custom matrices (user data).  The standard gates use the
oracle's own formulas below, never the gate object's matrices.
"""
from __future__ import annotations

import copy
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, 'liboracle.so')
_lib = None


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(['make', '-s', '-C', _HERE, 'liboracle.so'], check=True)


def lib():
    global _lib  # pylint: disable=global-statement
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, 'mqvector_oracle.c')
        ):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_I = ctypes.c_int
_U64 = ctypes.c_uint64
_D = ctypes.c_double


def _declare(L):
    for suf in ('d', 'f'):
        getattr(L, f'orc_apply_single_matrix_{suf}').argtypes = [_P, _I, _I, _U64, _P]
        getattr(L, f'orc_apply_two_matrix_{suf}').argtypes = [_P, _I, _I, _I, _U64, _P]
        getattr(L, f'orc_apply_n_matrix_{suf}').argtypes = [_P, _I, _P, _I, _U64, _P]
        getattr(L, f'orc_apply_xlike_{suf}').argtypes = [_P, _I, _I, _U64, _D, _D, _D, _D]
        getattr(L, f'orc_apply_zlike_{suf}').argtypes = [_P, _I, _I, _U64, _D, _D]
        getattr(L, f'orc_apply_rzz_{suf}').argtypes = [_P, _I, _I, _I, _U64, _D]
        getattr(L, f'orc_apply_rps_{suf}').argtypes = [_P, _I, _U64, _U64, _U64, _I, _U64, _D]
        getattr(L, f'orc_apply_pauli_string_{suf}').argtypes = [_P, _I, _U64, _U64, _U64, _I, _U64]
        getattr(L, f'orc_apply_terms_{suf}').argtypes = [_P, _P, _I, _I, _P, _P, _P, _P, _P]
        getattr(L, f'orc_expectation_of_terms_{suf}').argtypes = [_P, _P, _I, _I, _P, _P, _P, _P, _P, _P]
        getattr(L, f'orc_vdot_{suf}').argtypes = [_P, _P, _I, _P]
        getattr(L, f'orc_expect_diff_matrix_{suf}').argtypes = [_P, _P, _I, _P, _I, _U64, _P, _P]
        getattr(L, f'orc_expect_diff_rps_{suf}').argtypes = [_P, _P, _I, _U64, _U64, _U64, _I, _U64, _D, _P]
        getattr(L, f'orc_cumulative_probs_{suf}').argtypes = [_P, _I, _P]
        getattr(L, f'orc_lower_bound_{suf}').argtypes = [_P, _U64, _P, _U64, _P]
        getattr(L, f'orc_csr_dot_vec_{suf}').argtypes = [_P, _P, _P, _U64, _P, _P]
        getattr(L, f'orc_expectation_of_csr_{suf}').argtypes = [_P, _P, _P, _U64, _P, _P, _P]
    L.orc_num_threads.restype = _I
    L.orc_set_num_threads.argtypes = [_I]


def set_num_threads(t):
    lib().orc_set_num_threads(int(t))


def num_threads():
    return lib().orc_num_threads()


def _ptr(a):
    """Data pointer of a C-contiguous array (the C kernels index it densely)."""
    if not a.flags['C_CONTIGUOUS']:
        raise ValueError("the oracle's C kernels need C-contiguous arrays")
    return a.ctypes.data_as(ctypes.c_void_p)


def _suf(qs):
    return 'd' if qs.dtype == np.complex128 else 'f'


def _mask(qubits):
    m = 0
    for q in qubits:
        m |= 1 << int(q)
    return m


def _mat_arg(m):
    return np.ascontiguousarray(np.asarray(m, dtype=np.complex128)).view(np.float64)


# ----------------------------------------------------------------------------- state kernels
def zero_state(n, dtype=np.complex128):
    qs = np.zeros(1 << n, dtype=dtype)
    qs[0] = 1
    return qs


def apply_matrix(qs, n, objs, ctrls, m):
    """ApplyMatrixGate dispatch (single / two / N-qubit matrix kernels)."""
    L, s = lib(), _suf(qs)
    ma = _mat_arg(m)
    cm = _mask(ctrls)
    if len(objs) == 1:
        getattr(L, f'orc_apply_single_matrix_{s}')(_ptr(qs), n, int(objs[0]), cm, _ptr(ma))
    elif len(objs) == 2:
        getattr(L, f'orc_apply_two_matrix_{s}')(_ptr(qs), n, int(objs[0]), int(objs[1]), cm, _ptr(ma))
    else:
        oa = np.asarray(objs, dtype=np.int32)
        getattr(L, f'orc_apply_n_matrix_{s}')(_ptr(qs), n, _ptr(oa), len(objs), cm, _ptr(ma))


def expect_diff_matrix(bra, ket, n, objs, ctrls, m):
    """<bra| m |ket> over the gate's groups (ExpectDiffSingle/Two/NQubitsMatrix)."""
    L, s = lib(), _suf(bra)
    out = np.zeros(2)
    oa = np.asarray(objs, dtype=np.int32)
    getattr(L, f'orc_expect_diff_matrix_{s}')(_ptr(bra), _ptr(ket), n, _ptr(oa), len(objs), _mask(ctrls),
                                              _ptr(_mat_arg(m)), _ptr(out))
    return complex(out[0], out[1])


def pauli_mask_of(pauli_string, objs):
    """GenPauliMask (ccsrc/lib/simulator/utils.cpp:28-40) for letters on objs."""
    mx = my = mz = 0
    ny = 0
    for p, q in zip(pauli_string.upper(), objs):
        if p == 'X':
            mx |= 1 << q
        elif p == 'Y':
            my |= 1 << q
            ny += 1
        elif p == 'Z':
            mz |= 1 << q
    return mx, my, mz, ny


def ham_masks(ham):
    """Term masks of a Hamiltonian-like object with ``ham_termlist`` [((q, 'X'),...), coeff]."""
    terms = ham.ham_termlist
    nt = len(terms)
    mx = np.zeros(nt, np.uint64)
    my = np.zeros(nt, np.uint64)
    mz = np.zeros(nt, np.uint64)
    ny = np.zeros(nt, np.int32)
    cf = np.zeros(nt, np.float64)
    for t, (k, v) in enumerate(terms):
        a, b, c, d = pauli_mask_of(''.join(p for _, p in k), [q for q, _ in k])
        mx[t], my[t], mz[t], ny[t], cf[t] = a, b, c, d, float(np.real(v))
    return mx, my, mz, ny, cf


_FRONTEND = 2   # HowTo.FRONTEND: a user-given sparse matrix (mindquantum/core/operators/hamiltonian.py:26-32)


def _csr_arrays(ham, dtype):
    m = ham.sparse_matrix
    return (np.ascontiguousarray(m.indptr, dtype=np.int64), np.ascontiguousarray(m.indices, dtype=np.int64),
            np.ascontiguousarray(m.data, dtype=dtype))


def apply_terms(qs, n, ham):
    """ApplyTerms: returns H|qs> in a fresh buffer (cpu_vector_core_policy.cpp:133-161); a sparse
    matrix Hamiltonian goes through Csr_Dot_Vec instead (VectorState::ApplyHamiltonian,
    vector_state.tpp:963-974)."""
    L, s = lib(), _suf(qs)
    out = np.zeros_like(qs)
    if getattr(ham, 'how_to', 0) == _FRONTEND:
        ip, ix, dt = _csr_arrays(ham, qs.dtype)
        getattr(L, f'orc_csr_dot_vec_{s}')(_ptr(ip), _ptr(ix), _ptr(dt), 1 << n, _ptr(qs), _ptr(out))
        return out
    mx, my, mz, ny, cf = ham_masks(ham)
    getattr(L, f'orc_apply_terms_{s}')(_ptr(qs), _ptr(out), n, len(cf), _ptr(mx), _ptr(my), _ptr(mz), _ptr(ny),
                                       _ptr(cf))
    return out


def expectation_of_terms(bra, ket, n, ham):
    """ExpectationOfTerms (cpu_vector_core_policy.cpp:212-261), or ExpectationOfCsr for a sparse
    matrix Hamiltonian (vector_state.tpp:712-726)."""
    L, s = lib(), _suf(bra)
    out = np.zeros(2)
    if getattr(ham, 'how_to', 0) == _FRONTEND:
        ip, ix, dt = _csr_arrays(ham, bra.dtype)
        getattr(L, f'orc_expectation_of_csr_{s}')(_ptr(ip), _ptr(ix), _ptr(dt), 1 << n, _ptr(bra), _ptr(ket),
                                                  _ptr(out))
        return complex(out[0], out[1])
    mx, my, mz, ny, cf = ham_masks(ham)
    getattr(L, f'orc_expectation_of_terms_{s}')(_ptr(bra), _ptr(ket), n, len(cf), _ptr(mx), _ptr(my), _ptr(mz),
                                                _ptr(ny), _ptr(cf), _ptr(out))
    return complex(out[0], out[1])


def vdot(bra, ket, n):
    L, s = lib(), _suf(bra)
    out = np.zeros(2)
    getattr(L, f'orc_vdot_{s}')(_ptr(bra), _ptr(ket), n, _ptr(out))
    return complex(out[0], out[1])


# ----------------------------------------------------------------------------- gate semantics
def _pr_value(pr, prd):
    """ParameterResolver::Combination(pr).const_value, real part (vector_state.tpp:236 etc.)."""
    val = complex(pr.const)
    for k, c in pr.items():
        val += c * prd[k]
    return val.real


def _rot_xx_like(kind, c, s):
    """4x4 matrices of the two-qubit Pauli rotations with index b(obj0) + 2 b(obj1)
    (ApplyRxx/Rxy/Rxz/Ryz/Ryy/Rzz, cpu_vector_core_rot_pauli.cpp:31-428; c, s as in the kernels)."""
    z = 0
    if kind == 'Rxx':
        s = -1j * s
        return np.array([[c, z, z, s], [z, c, s, z], [z, s, c, z], [s, z, z, c]])
    if kind == 'Ryy':
        s = 1j * s
        return np.array([[c, z, z, s], [z, c, -s, z], [z, -s, c, z], [s, z, z, c]])
    if kind == 'Rxy':
        return np.array([[c, z, z, -s], [z, c, -s, z], [z, s, c, z], [s, z, z, c]])
    if kind == 'Rxz':
        s = -1j * s
        return np.array([[c, s, z, z], [s, c, z, z], [z, z, c, -s], [z, z, -s, c]])
    if kind == 'Ryz':
        return np.array([[c, -s, z, z], [s, c, z, z], [z, z, c, s], [z, z, -s, c]])
    if kind == 'Rzz':
        e, me = c + 1j * s, c - 1j * s
        return np.diag([me, e, e, me])
    raise KeyError(kind)


def _u3(t, p, l):
    """U3Matrix, gates.cpp:29-37."""
    c, s = math.cos(t / 2), math.sin(t / 2)
    el, ep = complex(math.cos(l), math.sin(l)), complex(math.cos(p), math.sin(p))
    return np.array([[c, -el * s], [ep * s, el * ep * c]])


def _rn(a, b, g, diff=None):
    """RnMatrix / RnDiff*Matrix, gates.cpp:48-136."""
    X = np.array([[0, 1], [1, 0]], complex)
    Y = np.array([[0, -1j], [1j, 0]], complex)
    Z = np.array([[1, 0], [0, -1]], complex)
    I2 = np.identity(2, dtype=complex)
    f = math.sqrt(a * a + b * b + g * g)
    if diff is None:
        if f == 0:
            return I2
        v2 = np.array([[g / f, a / f - 1j * b / f], [a / f + 1j * b / f, -g / f]])
        return np.cos(f / 2) * I2 - v2 * 1j * np.sin(f / 2)
    if f == 0:
        return np.zeros((2, 2), complex)
    comp, sig = [(a, X), (b, Y), (g, Z)][diff]
    h = X * a + Y * b + Z * g
    fa = comp / f
    cc, sc = math.cos(f / 2), math.sin(f / 2)
    return I2 * fa / -2 * sc - h * fa * 1j * (cc / 2 / f - sc / f / f) - sig * 1j * sc / f


def _fsim(t, p, diff=None):
    """FSimMatrix / FSimDiffTheta/PhiMatrix, gates.cpp:39-46, 144-163."""
    if diff is None:
        a, b = math.cos(t), -1j * math.sin(t)
        return np.array([[1, 0, 0, 0], [0, a, b, 0], [0, b, a, 0], [0, 0, 0, np.exp(-1j * p)]])
    if diff == 0:
        a, b = -math.sin(t), -1j * math.cos(t)
        return np.array([[0, 0, 0, 0], [0, a, b, 0], [0, b, a, 0], [0, 0, 0, 0]])
    out = np.zeros((4, 4), complex)
    out[3, 3] = np.exp(-1j * (p + math.pi / 2))
    return out


_TWO_ROT = ('Rxx', 'Ryy', 'Rzz', 'Rxy', 'Rxz', 'Ryz')
_SQ2 = math.sqrt(0.5)


def _gate_kind(g):
    return type(g).__name__ if type(g).__name__ not in ('_ParamNonHerm',) else 'ParamNonHerm'


def gate_matrix(g, prd):
    """The matrix that VectorState::ApplyGate applies for gate ``g`` (None for X/Y/Z-like/RPS paths)."""
    name = g.name
    if name in ('RX', 'RY', 'RZ', 'PS', 'GP') or name in _TWO_ROT or name in ('G', 'SWAPalpha'):
        v = _pr_value(g.prs[0], prd)
        c, s = math.cos(v / 2), math.sin(v / 2)
        if name == 'RX':   # ApplyRX: a = cos, b = -sin, m = [[a, ib], [ib, a]]
            return np.array([[c, -1j * s], [-1j * s, c]])
        if name == 'RY':   # ApplyRY
            return np.array([[c, -s], [s, c]], dtype=complex)
        if name == 'RZ':   # ApplyRZ: [[a - ib, 0], [0, a + ib]]
            return np.array([[c - 1j * s, 0], [0, c + 1j * s]])
        if name == 'PS':
            return np.array([[1, 0], [0, complex(math.cos(v), math.sin(v))]])
        if name == 'GP':   # ApplyGP: exp(-i v) on both diagonal entries
            e = complex(math.cos(-v), math.sin(-v))
            return np.array([[e, 0], [0, e]])
        if name in _TWO_ROT:
            return _rot_xx_like(name, c, s)
        if name == 'G':    # ApplyGivens uses cos(v), sin(v)
            cv, sv = math.cos(v), math.sin(v)
            return np.array([[1, 0, 0, 0], [0, cv, -sv, 0], [0, sv, cv, 0], [0, 0, 0, 1]])
        e = complex(math.cos(math.pi * v), math.sin(math.pi * v))  # SWAPalpha
        a, b = (1 + e) / 2, (1 - e) / 2
        return np.array([[1, 0, 0, 0], [0, a, b, 0], [0, b, a, 0], [0, 0, 0, 1]])
    if name == 'U3':
        return _u3(*[_pr_value(p, prd) for p in g.prs])
    if name == 'Rn':
        return _rn(*[_pr_value(p, prd) for p in g.prs])
    if name == 'FSim':
        return _fsim(*[_pr_value(p, prd) for p in g.prs])
    if hasattr(g, 'matrix_generator'):   # CustomGate with a parameter
        v = _pr_value(g.prs[0], prd)
        m = np.asarray(g.matrix_generator(v), dtype=complex)
        return np.conj(m).T if g.hermitianed else m
    if name == 'H':
        return np.array([[_SQ2, _SQ2], [_SQ2, -_SQ2]], dtype=complex)
    if name == 'SX':       # ApplySX / ApplySXdag, cpu_vector_core_other_gate.cpp:37-51
        a = complex(0.5, -0.5) if g.hermitianed else complex(0.5, 0.5)
        b = a.conjugate()
        return np.array([[a, b], [b, a]])
    if name == 'SWAP':
        return np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)
    if name == 'ISWAP':    # ApplyISWAP, frac = -1 when daggered
        f = -1j if g.hermitianed else 1j
        return np.array([[1, 0, 0, 0], [0, 0, f, 0], [0, f, 0, 0], [0, 0, 0, 1]])
    return np.asarray(g.matrix(), dtype=complex)   # CustomGate / Power with a constant matrix


def apply_gate(qs, n, g, prd):
    """VectorState::ApplyGate (vector_state.tpp:166-437) for one gate (no measurement)."""
    name = g.name
    L, s = lib(), _suf(qs)
    objs, ctrls = list(g.obj_qubits), list(g.ctrl_qubits)
    cm = _mask(ctrls)
    if name in ('I', 'BARRIER'):
        return
    if name == 'X':        # ApplyX -> ApplyXLike(1, 1)
        getattr(L, f'orc_apply_xlike_{s}')(_ptr(qs), n, objs[0], cm, 1, 0, 1, 0)
    elif name == 'Y':      # ApplyY -> ApplyXLike(-i, i)
        getattr(L, f'orc_apply_xlike_{s}')(_ptr(qs), n, objs[0], cm, 0, -1, 0, 1)
    elif name == 'Z':
        getattr(L, f'orc_apply_zlike_{s}')(_ptr(qs), n, objs[0], cm, -1, 0)
    elif name == 'S':
        getattr(L, f'orc_apply_zlike_{s}')(_ptr(qs), n, objs[0], cm, 0, -1 if g.hermitianed else 1)
    elif name == 'T':
        getattr(L, f'orc_apply_zlike_{s}')(_ptr(qs), n, objs[0], cm, _SQ2, -_SQ2 if g.hermitianed else _SQ2)
    elif name == 'Rzz':
        getattr(L, f'orc_apply_rzz_{s}')(_ptr(qs), n, objs[0], objs[1], cm, _pr_value(g.prs[0], prd))
    elif name == 'RPS':
        mx, my, mz, ny = pauli_mask_of(g.pauli_string, objs)
        getattr(L, f'orc_apply_rps_{s}')(_ptr(qs), n, mx, my, mz, ny, cm, _pr_value(g.prs[0], prd))
    elif name == 'M':
        raise ValueError("measurement is handled by apply_circuit")
    else:
        apply_matrix(qs, n, objs, ctrls, gate_matrix(g, prd))


def _diff_matrices(g, prd):
    """Per-parameter-slot derivative matrices of ExpectDiffGate (vector_state.tpp:778-946)."""
    name = g.name
    if name in ('RX', 'RY', 'RZ', 'PS', 'GP', 'G', 'SWAPalpha') or name in _TWO_ROT:
        v = _pr_value(g.prs[0], prd)
        c, s = -0.5 * math.sin(v / 2), 0.5 * math.cos(v / 2)
        if name == 'RX':   # ExpectDiffRX: [[c, -i s], [-i s, c]]
            return [np.array([[c, -1j * s], [-1j * s, c]])]
        if name == 'RY':
            return [np.array([[c, -s], [s, c]], dtype=complex)]
        if name == 'RZ':
            return [np.array([[c - 1j * s, 0], [0, c + 1j * s]])]
        if name == 'PS':   # ExpectDiffPS: (-sin v + i cos v) on the |1> half
            return [np.array([[0, 0], [0, -math.sin(v) + 1j * math.cos(v)]])]
        if name == 'GP':   # ExpectDiffGP: -i exp(-i v)
            e = -1j * complex(math.cos(-v), math.sin(-v))
            return [np.array([[e, 0], [0, e]])]
        if name in _TWO_ROT:   # the kernels with diff=true: c = -sin/2, s = cos/2
            return [_rot_xx_like(name, c, s)]
        if name == 'G':
            cv, sv = -math.sin(v), math.cos(v)
            return [np.array([[0, 0, 0, 0], [0, cv, -sv, 0], [0, sv, cv, 0], [0, 0, 0, 0]])]
        e = 0.5j * math.pi * complex(math.cos(math.pi * v), math.sin(math.pi * v))  # SWAPalpha
        return [np.array([[0, 0, 0, 0], [0, e, -e, 0], [0, -e, e, 0], [0, 0, 0, 0]])]
    if name == 'U3':       # U3Diff{Theta,Phi,Lambda}Matrix, gates.cpp:138-170
        t, p, l = [_pr_value(q, prd) for q in g.prs]
        md = 0.5 * _u3(t + math.pi, p, l)
        mp = _u3(t, p + math.pi / 2, l)
        mp[0, 0] = 0
        mp[0, 1] = 0
        ml = _u3(t, p, l + math.pi / 2)
        ml[0, 0] = 0
        ml[1, 0] = 0
        return [md, mp, ml]
    if name == 'Rn':
        a, b, c = [_pr_value(q, prd) for q in g.prs]
        return [_rn(a, b, c, 0), _rn(a, b, c, 1), _rn(a, b, c, 2)]
    if name == 'FSim':
        t, p = [_pr_value(q, prd) for q in g.prs]
        return [_fsim(t, p, 0), _fsim(t, p, 1)]
    if hasattr(g, 'diff_matrix_generator'):
        v = _pr_value(g.prs[0], prd)
        m = np.asarray(g.diff_matrix_generator(v), dtype=complex)
        return [np.conj(m).T if g.hermitianed else m]
    raise ValueError(f"Expectation of gate {name} not implement.")


def expect_diff_gate(bra, ket, n, g, prd):
    """ExpectDiffGate: one complex value per parameter slot of ``g``."""
    if g.name == 'RPS':
        mx, my, mz, ny = pauli_mask_of(g.pauli_string, g.obj_qubits)
        out = np.zeros(2)
        getattr(lib(), f'orc_expect_diff_rps_{_suf(bra)}')(_ptr(bra), _ptr(ket), n, mx, my, mz, ny,
                                                             _mask(g.ctrl_qubits), _pr_value(g.prs[0], prd), _ptr(out))
        return [complex(out[0], out[1])]
    mats = _diff_matrices(g, prd)
    res = []
    for slot, m in enumerate(mats):
        pr = g.prs[slot]
        if len(pr.params_name) == len(pr.no_grad_parameters):   # ExpectDiffU3: skip const slots
            res.append(0j)
        else:
            res.append(expect_diff_matrix(bra, ket, n, g.obj_qubits, g.ctrl_qubits, m))
    return res


def jacobi(g):
    """Parameterizable::GetJacobi: ({name: column}, matrix[n_pr][n_names]) of requires-grad params."""
    title = {}
    for pr in g.prs:
        for k in pr.requires_grad_parameters:
            title.setdefault(k, len(title))
    jac = np.zeros((len(g.prs), len(title)), dtype=complex)
    for i, pr in enumerate(g.prs):
        for k in pr.requires_grad_parameters:
            jac[i, title[k]] = pr[k]
    return title, jac


def gate_requires_grad(g):
    return hasattr(g, 'prs') and any(len(p.params_name) != len(p.no_grad_parameters) for p in g.prs)


def hermitian_gate(g):
    """The daggered gate the reference's Python builds (basic.py:510-515, basicgate.py:2445-2454)."""
    return g.hermitian()


# ----------------------------------------------------------------------------- drivers
def reduced_density_matrix(qs, n, kept_qubits):
    """GetReducedDensityMatrix, ccsrc/lib/simulator/vector/detail/cpu_common/cpu_vector_core_policy.cpp:335-383:
    for every pair (i, j) of basis states whose traced bits agree, rho[i_kept][j_kept] +=
    qs[i] conj(qs[j]), bit k of i_kept being bit sorted(kept)[k] of i.  Pure-Python loops: small n."""
    kept = sorted(kept_qubits)
    traced = [q for q in range(n) if q not in kept]
    rho = np.zeros((1 << len(kept), 1 << len(kept)), dtype=np.complex128)

    def sub(i, qubits):
        return sum(((i >> q) & 1) << k for k, q in enumerate(qubits))

    for i in range(1 << n):
        for j in range(1 << n):
            if sub(i, traced) == sub(j, traced):
                rho[sub(i, kept), sub(j, kept)] += qs[i] * np.conj(qs[j])
    return rho


class OracleSim:
    """A VectorState restatement: holds a numpy state and applies circuits with the C kernels."""

    def __init__(self, n, dtype=np.complex128, state=None):
        self.n = n
        self.dtype = dtype
        self.qs = zero_state(n, dtype) if state is None else np.array(state, dtype=dtype)

    def apply_circuit(self, circ, prd=None, draw=None):
        """Apply gates; channels draw from ``draw`` (the simulator's uniform stream)."""
        prd = prd or {}
        for g in circ:
            if g.name == 'M':
                raise ValueError("oracle apply_circuit does not sample measurements")
            if is_channel(g):
                if draw is None:
                    raise ValueError("a noise channel needs a random stream")
                apply_channel(self.qs, self.n, g, draw)
            else:
                apply_gate(self.qs, self.n, g, prd)
        return self

    def get_qs(self):
        return self.qs.copy()


def get_expectation(n, ham, circ, prd=None, dtype=np.complex128, init_state=None):
    """VectorState::GetExpectation (vector_state.tpp:712-726)."""
    sim = OracleSim(n, dtype, init_state).apply_circuit(circ, prd)
    return expectation_of_terms(sim.qs, sim.qs, n, ham)


def left_size_grad(n, psi_l, psi_r, herm_circ, hams, prd, p_map):
    """GradientHelper::LeftSizeGrad (gradient.h:160-197)."""
    n_hams = len(hams)
    f_and_g = np.zeros((n_hams, 1 + len(p_map)), dtype=complex)
    psi_rs = [psi_r if i == 0 else psi_r.copy() for i in range(n_hams)]
    for i in range(n_hams):
        psi_rs[i] = apply_terms(psi_rs[i], n, hams[i])
        f_and_g[i, 0] = vdot(psi_l, psi_rs[i], n)
    for g in herm_circ:
        apply_gate(psi_l, n, g, prd)
        if gate_requires_grad(g):
            title, jac = jacobi(g)
            if title:
                for j in range(n_hams):
                    intrin = np.array(expect_diff_gate(psi_l, psi_rs[j], n, g, prd))
                    p_grad = intrin @ jac
                    for name, idx in title.items():
                        f_and_g[j, 1 + p_map[name]] += p_grad[idx]
        for j in range(n_hams):
            apply_gate(psi_rs[j], n, g, prd)
    return f_and_g


def get_expectation_with_grad(n, hams, circ, enc_data, ans_data, enc_names, ans_names,
                              dtype=np.complex128, init_state=None):
    """GradientHelper::HermitianAdjointGradient (gradient.h:100-121) incl. GradRealDouble.

    Returns the reference layout ``[n_prs][n_hams][1 + n_enc + n_ans]`` complex.
    """
    herm = [hermitian_gate(g) for g in reversed(list(circ))]
    enc_data = np.atleast_2d(np.asarray(enc_data, dtype=np.float64)) if len(enc_names) else np.zeros((1, 0))
    ans_data = np.asarray(ans_data, dtype=np.float64).reshape(-1)
    p_map = {k: i for i, k in enumerate(enc_names)}
    p_map.update({k: i + len(enc_names) for i, k in enumerate(ans_names)})
    out = []
    for idx in range(enc_data.shape[0]):
        prd = dict(zip(enc_names, enc_data[idx].tolist()))
        prd.update(dict(zip(ans_names, ans_data.tolist())))
        sim = OracleSim(n, dtype, init_state).apply_circuit(circ, prd)
        psi_l = sim.qs
        psi_r = psi_l.copy()
        out.append(left_size_grad(n, psi_l, psi_r, herm, hams, prd, p_map))
    res = np.array(out)
    res[:, :, 1:] = res[:, :, 1:] + np.conj(res[:, :, 1:])   # GradRealDouble
    return res




# ----------------------------------------------------------------------------- noise channels
_CHANNELS = ('PC', 'BFC', 'PFC', 'BPFC', 'GPC', 'DC', 'ADC', 'PDC', 'TRC')


def is_channel(g):
    return g.name in _CHANNELS or hasattr(g, 'kraus_op')


def _qubit_prob(qs, q, bit):
    """OneStateVdot / ZeroStateVdot of a state with itself: sum of |amp|^2 where qubit q == bit."""
    sel = ((np.arange(qs.size) >> q) & 1) == bit
    return float(np.sum(np.abs(qs[sel].astype(np.complex128)) ** 2))


def _x_like(qs, n, q, ctrls, v1, v2):
    """ApplyXLike (cpu_vector_core_x_like.cpp:29-57): new[i] = old[j] v1, new[j] = old[i] v2."""
    v1, v2 = complex(v1), complex(v2)
    getattr(lib(), f'orc_apply_xlike_{_suf(qs)}')(_ptr(qs), n, q, _mask(ctrls), v1.real, v1.imag, v2.real, v2.imag)


def _i_like(qs, n, q, ctrls, a, b):
    """ApplyILike: diag(a, b) on qubit q (under the controls)."""
    apply_matrix(qs, n, [q], ctrls, np.array([[a, 0], [0, b]], dtype=np.complex128))


def _pauli(qs, n, which, q, ctrls):
    if which == 0:
        _x_like(qs, n, q, ctrls, 1, 1)
    elif which == 1:
        _x_like(qs, n, q, ctrls, -1j, 1j)
    elif which == 2:
        getattr(lib(), f'orc_apply_zlike_{_suf(qs)}')(_ptr(qs), n, q, _mask(ctrls), -1, 0)


def _pauli_index(cum, r):
    """lower_bound over [0, px, px+py, px+py+pz, 1]: 0 = X, 1 = Y, 2 = Z, 3 = I (vector_state.tpp:492-503)."""
    import bisect

    it = bisect.bisect_left(cum, r)
    return it - 1 if it > 0 else 0


def apply_channel(qs, n, g, draw):
    """VectorState::ApplyChannel and the channel kernels (vector_state.tpp:465-709), in place.

    ``draw()`` is the simulator's uniform(0, 1) stream; every branch draws exactly as the
    reference does, so a trajectory is reproduced draw for draw.
    """
    objs, ctrls = list(g.obj_qubits), list(g.ctrl_qubits)
    if g.name in ('PC', 'BFC', 'PFC', 'BPFC'):
        _pauli(qs, n, _pauli_index(g.cumulative_probs(), draw()), objs[0], ctrls)
    elif g.name == 'GPC':
        mx = my = mz = 0
        ny = 0
        for q, row in zip(objs, g.probs):
            px, py, pz = (float(v) for v in row)
            cum = [0.0, px, px + py, px + py + pz, px + py + pz + (1 - px - py - pz)]
            k = _pauli_index(cum, draw())
            if k == 0:
                mx |= 1 << q
            elif k == 1:
                my |= 1 << q
                ny += 1
            elif k == 2:
                mz |= 1 << q
        getattr(lib(), f'orc_apply_pauli_string_{_suf(qs)}')(_ptr(qs), n, mx, my, mz, ny, 0)
    elif g.name == 'DC':
        def uniform(idx):
            while idx < len(objs):
                p_i = draw()
                if p_i < 0.25:
                    _pauli(qs, n, 0, objs[idx], ctrls)
                elif p_i < 0.5:
                    _pauli(qs, n, 1, objs[idx], ctrls)
                elif p_i < 0.75:
                    _pauli(qs, n, 2, objs[idx], ctrls)
                idx += 1

        idx, p = 0, float(g.p)
        while idx < len(objs):
            if draw() < p * 3.0 / 4.0:
                p_i = draw()
                _pauli(qs, n, 0 if p_i < 1.0 / 3.0 else (1 if p_i < 2.0 / 3.0 else 2), objs[idx], ctrls)
                uniform(idx + 1)
                break
            if not 4 > 3 * p:
                break
            idx, p = idx + 1, p / (4 - 3 * p)
    elif hasattr(g, 'kraus_op'):
        total = 1.0
        for m in np.asarray(g.kraus_op, dtype=np.complex128):
            if abs(m[0, 1]) < 1e-6 and abs(m[1, 0]) < 1e-6 and abs(m[0, 0] - m[1, 1]) < 1e-6:
                prob = float((m[0, 0] * np.conj(m[0, 0])).real)
                rel = prob / total
                total -= prob
                if draw() < rel:
                    if m[0, 0].imag >= 1e-6:
                        qs *= m[0, 0] / math.sqrt(prob)
                    return
            else:
                tmp = qs.copy()
                apply_matrix(tmp, n, objs, ctrls, m)
                prob = float(np.vdot(tmp, tmp).real)
                rel = prob / total
                total -= prob
                if draw() < rel:
                    qs[:] = tmp * (1 / math.sqrt(prob))
                    return
    elif g.name in ('ADC', 'PDC'):
        renorm = _qubit_prob(qs, objs[0], 1)
        if renorm < 1e-6:
            return
        gamma = float(g.gamma)
        prob = gamma * renorm
        if draw() <= prob:
            if g.name == 'ADC':
                _x_like(qs, n, objs[0], ctrls, 1 / math.sqrt(renorm), 0)
            else:
                _i_like(qs, n, objs[0], ctrls, 0, 1 / math.sqrt(renorm))
        else:
            _i_like(qs, n, objs[0], ctrls, 1 / math.sqrt(1 - prob), math.sqrt(1 - gamma) / math.sqrt(1 - prob))
    elif g.name == 'TRC':
        t1, t2, tg = float(g.t1), float(g.t2), float(g.gate_time)
        e1, e2 = math.exp(-tg / t1), math.exp(-tg / t2)
        p_reset = 1 - e1
        q = objs[0]
        if t1 >= t2:
            pz = e1 * (1 - e2 / e1) / 2
            r = draw()
            if r < 1 - pz - p_reset:
                return
            if r < 1 - p_reset:
                _pauli(qs, n, 2, q, ctrls)
            else:
                zero = _qubit_prob(qs, q, 0)
                if draw() < zero:
                    _i_like(qs, n, q, ctrls, 1 / math.sqrt(zero), 0)
                else:
                    _x_like(qs, n, q, ctrls, 1 / math.sqrt(1 - zero), 0)
        elif 2 * t1 > t2:
            r = draw()
            root = math.sqrt(p_reset * p_reset + 4 * e2 * e2)
            ev0, ev1 = (2 - p_reset + root) / 2, (2 - p_reset - root) / 2
            vec0, vec1 = (ev0 - e1) / e2, (ev1 - e1) / e2
            zero = _qubit_prob(qs, q, 0)
            one = 1 - zero
            c0 = vec0 * vec0 * zero + one
            p0 = c0 * ev0 / (vec0 * vec0 + 1)
            if r < p0:
                _i_like(qs, n, q, ctrls, vec0 / math.sqrt(c0), 1 / math.sqrt(c0))
            elif r < 1 - p_reset * one:
                c1 = vec1 * vec1 * zero + one
                _i_like(qs, n, q, ctrls, vec1 / math.sqrt(c1), 1 / math.sqrt(c1))
            else:
                _x_like(qs, n, q, ctrls, 1 / math.sqrt(one), 0)
    else:
        raise ValueError(f"{g.name} is not a noise channel.")


class UniformStream:
    """std::uniform_real_distribution<double>(lo, hi) over std::mt19937(seed): the reference's rng_."""

    def __init__(self, seed, lo=0.0, hi=1.0):
        self.eng = _Mt19937(int(seed))
        self.lo, self.hi = lo, hi

    def __call__(self):
        return _uniform(self.eng, self.lo, self.hi)


def get_expectation_with_grad_parameter_shift_noisy(n, hams, circ, enc_data, ans_data, enc_names, ans_names,
                                                    draw, dtype=np.complex128, init_state=None, n_thread=None):
    """The parameter-shift loop of vector_state.tpp:1033-1230 with stochastic channels: every
    evaluation runs one trajectory of a copy re-seeded with int(draw() * 10000) from the
    simulator's stream ``draw``, and every Hamiltonian copy consumes one more draw, in the
    reference's order (Hamiltonians in groups of n_thread, the Hamiltonian loop inside the gate loop).
    """
    gates = [g for g in circ]
    enc_data = np.atleast_2d(np.asarray(enc_data, dtype=np.float64)) if len(enc_names) else np.zeros((1, 0))
    ans_data = np.asarray(ans_data, dtype=np.float64).reshape(-1)
    p_map = {k: i for i, k in enumerate(enc_names)}
    p_map.update({k: i + len(enc_names) for i, k in enumerate(ans_names)})
    n_h = len(hams)
    n_thread = min(15, n_h) if n_thread is None else max(1, min(n_thread, 15, n_h))
    out = np.zeros((enc_data.shape[0], n_h, 1 + len(p_map)), dtype=np.complex128)

    def trajectory(gate_list, prd):
        sim = OracleSim(n, dtype, init_state)
        sub = UniformStream(int(draw() * 10000))
        for g in gate_list:
            if is_channel(g):
                apply_channel(sim.qs, n, g, sub)
            else:
                apply_gate(sim.qs, n, g, prd)
        return sim.qs

    for s in range(enc_data.shape[0]):
        prd = dict(zip(enc_names, enc_data[s].tolist()))
        prd.update(dict(zip(ans_names, ans_data.tolist())))
        base = trajectory(gates, prd)
        for start in range(0, n_h, n_thread):
            group = range(start, min(start + n_thread, n_h))
            draw()                                   # the group's copy of the state
            for j in group:
                draw()                               # its Hamiltonian copy
                out[s, j, 0] = expectation_of_terms(base, base, n, hams[j])
            for gi, g in enumerate(gates):
                prs = getattr(g, 'prs', None)
                if is_channel(g) or not prs or not any(len(p.requires_grad_parameters) for p in prs):
                    continue
                shift, coeff, multi = shift_rule(g)
                for j in group:
                    for k, p in enumerate(prs):
                        if p.is_const():
                            continue
                        f = []
                        for sign in (-1.0, 1.0):
                            shifted, pr_s = g, prd
                            if multi:
                                key = min(p.keys())
                                pr_s = dict(prd)
                                pr_s[key] = prd[key] + sign * shift / float(np.real(p[key]))
                            else:
                                shifted = copy.copy(g)
                                shifted.prs = list(prs)
                                shifted.prs[k] = p + sign * shift
                            qs = trajectory(gates[:gi] + [shifted] + gates[gi + 1:], pr_s)
                            draw()                   # the Hamiltonian copy of this evaluation
                            f.append(expectation_of_terms(qs, qs, n, hams[j]))
                        intrin = coeff * float(np.real(f[1] - f[0]))
                        for name in p.requires_grad_parameters:
                            out[s, j, 1 + p_map[name]] += intrin * float(np.real(p[name]))
    return out

# ----------------------------------------------------------------------------- parameter shift
_PS_EXACT = ('RX', 'RY', 'RZ', 'Rxx', 'Ryy', 'Rzz', 'Rxy', 'Rxz', 'Ryz', 'GP', 'PS', 'U3')
_PS_MULTI = ('U3', 'FSim')


def shift_rule(g):
    """(shift, coefficient, shifts-the-parameter-value) of one gate, vector_state.tpp:1076-1174.

    Rotation-like gates: +-pi/2 and 1/2; SWAPalpha: +-1/2 and pi/2; every other supported gate and
    every controlled gate: central difference with step 1e-3.  U3 and FSim keep their angles
    outside the coefficient list the shift edits, so the reference shifts the value of the first
    (lexicographically smallest) parameter of the angle instead, which moves every gate using it.
    """
    custom = hasattr(g, 'matrix_generator')
    if not (custom or g.name in _PS_EXACT or g.name in _PS_MULTI or g.name in ('G', 'SWAPalpha')):
        raise RuntimeError(f"gate {g.name} not supported for parameter shift rule.")
    if custom:
        shift, coeff = 0.001, 0.5 / 0.001
    elif g.name in _PS_EXACT:
        shift, coeff = math.pi / 2, 0.5
    elif g.name == 'SWAPalpha':
        shift, coeff = 0.5, math.pi / 2
    else:
        shift, coeff = 0.001, 0.5 / 0.001
    if len(g.ctrl_qubits):
        shift, coeff = 0.001, 0.5 / 0.001
    return shift, coeff, (not custom and g.name in _PS_MULTI)


def get_expectation_with_grad_parameter_shift(n, hams, circ, enc_data, ans_data, enc_names, ans_names,
                                              dtype=np.complex128, init_state=None):
    """GetExpectationWithGradParameterShiftOneMulti / MultiMulti (vector_state.tpp:1033-1305).

    For every gate whose parameters require a gradient and every non-constant angle k of it, the
    circuit is evaluated with the angle shifted down and up; coeff * Re(f+ - f-) is the derivative
    with respect to the angle, and the gate's Jacobi row spreads it over the named parameters.
    Returns ``[n_prs][n_hams][1 + n_enc + n_ans]`` complex.
    """
    gates = [g for g in circ]
    enc_data = np.atleast_2d(np.asarray(enc_data, dtype=np.float64)) if len(enc_names) else np.zeros((1, 0))
    ans_data = np.asarray(ans_data, dtype=np.float64).reshape(-1)
    p_map = {k: i for i, k in enumerate(enc_names)}
    p_map.update({k: i + len(enc_names) for i, k in enumerate(ans_names)})
    out = np.zeros((enc_data.shape[0], len(hams), 1 + len(p_map)), dtype=np.complex128)

    def values(gate_list, prd):
        qs = OracleSim(n, dtype, init_state).apply_circuit(gate_list, prd).qs
        return np.array([expectation_of_terms(qs, qs, n, h) for h in hams])

    for s in range(enc_data.shape[0]):
        prd = dict(zip(enc_names, enc_data[s].tolist()))
        prd.update(dict(zip(ans_names, ans_data.tolist())))
        out[s, :, 0] = values(gates, prd)
        for gi, g in enumerate(gates):
            prs = getattr(g, 'prs', None)
            if not prs or not any(len(p.requires_grad_parameters) for p in prs):
                continue
            shift, coeff, multi = shift_rule(g)
            for k, p in enumerate(prs):
                if p.is_const():
                    continue
                f = []
                for sign in (-1.0, 1.0):
                    shifted, pr_s = g, prd
                    if multi:
                        key = min(p.keys())
                        pr_s = dict(prd)
                        pr_s[key] = prd[key] + sign * shift / float(np.real(p[key]))
                    else:
                        shifted = copy.copy(g)
                        shifted.prs = list(prs)
                        shifted.prs[k] = p + sign * shift
                    f.append(values(gates[:gi] + [shifted] + gates[gi + 1:], pr_s))
                intrin = coeff * np.real(f[1] - f[0])
                for name in p.requires_grad_parameters:
                    out[s, :, 1 + p_map[name]] += intrin * float(np.real(p[name]))
    return out

# ----------------------------------------------------------------------------- sampling
class _Mt19937:
    """std::mt19937 (the reference's RndEngine, vector_state.h:67): the published MT19937 algorithm."""

    def __init__(self, seed):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            self.mt[i] = (1812433253 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.index = 624

    def _twist(self):
        mt = self.mt
        for i in range(624):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
            v = mt[(i + 397) % 624] ^ (y >> 1)
            if y & 1:
                v ^= 0x9908B0DF
            mt[i] = v
        self.index = 0

    def __call__(self):
        if self.index >= 624:
            self._twist()
        y = self.mt[self.index]
        self.index += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def _uniform(eng, a, b):
    """std::uniform_real_distribution<double>(a, b) on a 32-bit engine (libstdc++ generate_canonical:
    two draws, (x0 + x1 * 2^32) / 2^64, clamped below 1)."""
    x0 = eng()
    x1 = eng()
    r = (x0 + x1 * 4294967296.0) / 18446744073709551616.0
    if r >= 1.0:
        r = math.nextafter(1.0, 0.0)
    return r * (b - a) + a


def apply_measure(qs, n, q, rng):
    """VectorState::ApplyMeasure (vector_state.tpp:440-462) without reset: collapse qubit q."""
    idx = np.arange(1 << n)
    one = ((idx >> q) & 1).astype(bool)
    one_amp = float(np.sum(np.abs(qs[one]) ** 2))   # OneStateVdot(...).real()
    collapse_to_one = rng() < one_amp
    if collapse_to_one:
        qs[~one] = 0
        qs[one] *= 1 / math.sqrt(one_amp)
    else:
        qs[one] = 0
        qs[~one] *= 1 / math.sqrt(1 - one_amp)
    return int(collapse_to_one)


def sampling_general(n, circ, prd, shots, seed, dtype=np.complex128, init_state=None):
    """VectorState::Sampling (vector_state.tpp:1308-1323): re-simulate the circuit once per shot;
    the shot's measurements and noise channels draw from one stream seeded from ``seed``'s.

    Returns (keys in circuit order, samples[shots][n_keys]).
    """
    rng = _Mt19937(seed)
    keys = [g.key for g in circ if g.name == 'M']
    out = np.zeros((shots, len(keys)), dtype=np.int64)
    for s in range(shots):
        sub = _Mt19937(int(_uniform(rng, 1.0, float(1 << 20))))
        draw = lambda: _uniform(sub, 0.0, 1.0)   # noqa: E731  pylint: disable=cell-var-from-loop
        qs = zero_state(n, dtype) if init_state is None else np.array(init_state, dtype=dtype)
        for g in circ:
            if g.name == 'M':
                out[s, keys.index(g.key)] = apply_measure(qs, n, g.obj_qubits[0], draw)
            elif is_channel(g):
                apply_channel(qs, n, g, draw)
            else:
                apply_gate(qs, n, g, prd or {})
    return keys, out


def sampling_measure_ending(n, circ, prd, shots, seed, dtype=np.complex128, init_state=None):
    """SamplingMeasurementEndingWithoutNoise (vector_state.tpp:1326-1373).

    Returns an array [shots][n_measures] in the order of the measurement keys' first appearance.
    """
    rng = _Mt19937(seed)
    sub_seed = int(_uniform(rng, 1.0, float(1 << 20)))
    sim_rng = _Mt19937(sub_seed)
    m_qids, keys = [], []
    other = []
    for g in circ:
        if g.name == 'M':
            m_qids.append(g.obj_qubits[0])
            keys.append(g.key)
        else:
            other.append(g)
    sim = OracleSim(n, dtype, init_state).apply_circuit(other, prd)
    real = np.float64 if dtype == np.complex128 else np.float32
    cum = np.zeros(1 << n, dtype=real)
    getattr(lib(), f'orc_cumulative_probs_{_suf(sim.qs)}')(_ptr(sim.qs), n, _ptr(cum))
    sampled = np.array([_uniform(sim_rng, 0.0, 1.0) for _ in range(shots)], dtype=real)
    sampled.sort()
    res = np.zeros(shots, dtype=np.uint32)
    getattr(lib(), f'orc_lower_bound_{_suf(sim.qs)}')(_ptr(cum), 1 << n, _ptr(sampled), shots, _ptr(res))
    out = np.zeros((shots, len(keys)), dtype=np.int64)
    for c, q in enumerate(m_qids):
        out[:, c] = (res >> q) & 1
    return keys, out


# ----------------------------------------------------------------------- density matrices (mqmatrix)
# Dense restatements of the reference's density-matrix simulator (DensityMatrixState,
# ccsrc/include/simulator/densitymatrix/densitymatrix_state.tpp) for small registers, the way the
# reference's own tests check it (tests/st/test_simulator/test_method_of_mqmatrix.py builds the
# same dense products).  rho[i][j] with index bit q <-> qubit q.

def dm_gate_matrix(n, g, prd):
    """The 2^n x 2^n matrix of a unitary gate (with its controls): the oracle's own gate kernels
    applied to every basis state."""
    dim = 1 << n
    U = np.zeros((dim, dim), dtype=np.complex128)
    for j in range(dim):
        e = np.zeros(dim, dtype=np.complex128)
        e[j] = 1
        apply_gate(e, n, g, prd)
        U[:, j] = e
    return U


def _embed1(n, q, m):
    """A single-qubit operator m on qubit q of n, as a 2^n x 2^n matrix."""
    out = np.array([[1.0 + 0j]])
    for k in reversed(range(n)):
        out = np.kron(out, m if k == q else np.eye(2))
    return out


def dm_kraus_1q(g):
    """Kraus operators of a single-qubit channel as the reference's density-matrix policy applies
    them (cpu_densitymatrix_core_channel.cpp: ApplyPauli, ApplyAmplitudeDamping with its daggered
    form, ApplyPhaseDamping, ApplyKraus)."""
    if g.name in ('PC', 'BFC', 'PFC', 'BPFC'):
        px, py, pz = g.px, g.py, g.pz
        out = []
        for p, m in ((px, [[0, 1], [1, 0]]), (py, [[0, -1j], [1j, 0]]), (pz, [[1, 0], [0, -1]]),
                     (1 - px - py - pz, [[1, 0], [0, 1]])):
            if p > 1e-8:
                out.append(np.sqrt(p) * np.array(m, dtype=np.complex128))
        return out
    if g.name == 'ADC':
        k0 = np.array([[1, 0], [0, np.sqrt(1 - g.gamma)]], dtype=np.complex128)
        if getattr(g, 'hermitianed', False):
            return [k0, np.array([[0, 0], [np.sqrt(g.gamma), 0]], dtype=np.complex128)]
        return [k0, np.array([[0, np.sqrt(g.gamma)], [0, 0]], dtype=np.complex128)]
    if g.name == 'PDC':
        return [np.array([[1, 0], [0, np.sqrt(1 - g.gamma)]], dtype=np.complex128),
                np.array([[0, 0], [0, np.sqrt(g.gamma)]], dtype=np.complex128)]
    return [np.asarray(k, dtype=np.complex128) for k in g.kraus_op]


def dm_apply_channel(rho, n, g):
    """DensityMatrixState::ApplyChannel (densitymatrix_state.tpp:465-505): the channel's exact map."""
    objs = list(g.obj_qubits)
    if g.name == 'GPC':
        for q, row in zip(objs, g.probs):
            px, py, pz = (float(v) for v in row)
            from types import SimpleNamespace

            rho = dm_apply_channel(rho, n, SimpleNamespace(name='PC', px=px, py=py, pz=pz, obj_qubits=[q]))
        return rho
    if g.name == 'DC':
        # (1 - p) rho + p (I / 2^k  (x)  Tr_objs rho)   (ApplyDepolarizing)
        k = len(objs)
        paulis = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]), np.array([[1, 0], [0, -1]])]
        tw = np.zeros_like(rho)
        import itertools

        for combo in itertools.product(range(4), repeat=k):
            P = np.eye(1 << n, dtype=np.complex128)
            for q, c in zip(objs, combo):
                P = P @ _embed1(n, q, paulis[c])
            tw += P @ rho @ P.conj().T
        return (1 - g.p) * rho + g.p / 4 ** k * tw
    if g.name == 'TRC':
        # ApplyThermalRelaxation: rho_00 += (1 - e1) rho_11, coherences x e2, rho_11 x e1
        e1 = np.exp(-g.gate_time / g.t1)
        e2 = np.exp(-g.gate_time / g.t2)
        q = objs[0]
        dim = 1 << n
        idx = np.arange(dim)
        b = (idx >> q) & 1
        out = rho.copy()
        r1c1 = (b[:, None] == 1) & (b[None, :] == 1)
        off = b[:, None] != b[None, :]
        out[off] *= e2
        out[r1c1] *= e1
        # rho_00 block gains (1 - e1) of rho_11 block (same other bits)
        lo = idx[b == 0]
        out[np.ix_(lo, lo)] += (1 - e1) * rho[np.ix_(lo | (1 << q), lo | (1 << q))]
        return out
    out = np.zeros_like(rho)
    for K in dm_kraus_1q(g):
        Kf = _embed1(n, objs[0], K)
        out += Kf @ rho @ Kf.conj().T
    return out


def dm_apply_circuit(n, circ, prd, rho):
    """DensityMatrixState::ApplyCircuit (densitymatrix_state.tpp:743) for gates and channels."""
    rho = np.array(rho, dtype=np.complex128)
    for g in circ:
        if is_channel(g):
            rho = dm_apply_channel(rho, n, g)
        elif g.name in ('BARRIER', 'I'):
            continue
        else:
            U = dm_gate_matrix(n, g, prd)
            rho = U @ rho @ U.conj().T
    return rho


def dm_expectation(n, ham, rho):
    """Tr(H rho) (GetStateExpectation of the density-matrix policy)."""
    return complex(np.trace(ham_matrix(n, ham) @ rho))


def ham_matrix(n, ham):
    """The 2^n x 2^n matrix of a Pauli Hamiltonian, columns by apply_terms on basis states."""
    dim = 1 << n
    Hm = np.zeros((dim, dim), dtype=np.complex128)
    for j in range(dim):
        e = np.zeros(dim, dtype=np.complex128)
        e[j] = 1
        Hm[:, j] = apply_terms(e, n, ham)
    return Hm


def dm_expectation_with_grad(n, hams, circ, params, names, rho0):
    """f = Tr(H E(rho0)) and its gradient for every parameter row: d/dtheta of the map's output
    (dU rho U^dag + U rho dU^dag at every gate holding the parameter, then the rest of the map),
    which is the quantity the reference's GetExpectationWithReversibleGrad / NoiseGrad return.
    Returns [rows][n_hams][1 + len(names)] complex."""
    params = np.atleast_2d(np.asarray(params, dtype=np.float64))
    gates = [g for g in circ if g.name not in ('BARRIER', 'I')]
    Hs = [ham_matrix(n, h) for h in hams]
    out = np.zeros((params.shape[0], len(hams), 1 + len(names)), dtype=complex)
    for s, row in enumerate(params):
        prd = dict(zip(names, row.tolist()))
        states = [np.array(rho0, dtype=np.complex128)]
        for g in gates:
            states.append(dm_apply_circuit(n, [g], prd, states[-1]))
        for h, Hm in enumerate(Hs):
            out[s, h, 0] = np.trace(Hm @ states[-1])
        for k, g in enumerate(gates):
            if is_channel(g) or not getattr(g, 'parameterized', False):
                continue
            U = dm_gate_matrix(n, g, prd)
            for name in names:
                if not any(name in p.params_name for p in g.prs):
                    continue
                dU = _gate_diff_full(n, g, prd, name)
                D = dU @ states[k] @ U.conj().T + U @ states[k] @ dU.conj().T
                D = dm_apply_circuit(n, gates[k + 1:], prd, D)
                for h, Hm in enumerate(Hs):
                    out[s, h, 1 + names.index(name)] += np.trace(Hm @ D)
    return out


def _gate_diff_full(n, g, prd, name, eps=1e-6):
    """d/d(name) of the gate's full matrix: sum over the gate's angles of d(angle)/d(name) times the
    angle's derivative matrix (_diff_matrices, the reference's ExpectDiff matrices) embedded with
    the controls (zero where the controls are not all set).  Pauli-string rotations use a central
    difference of the exact matrices instead."""
    dim = 1 << n
    if g.name == 'RPS':
        lo, hi = dict(prd), dict(prd)
        lo[name] -= eps
        hi[name] += eps
        return (dm_gate_matrix(n, g, hi) - dm_gate_matrix(n, g, lo)) / (2 * eps)
    objs, ctrls = list(g.obj_qubits), list(g.ctrl_qubits)
    out = np.zeros((dim, dim), dtype=np.complex128)
    for pr, dm in zip(g.prs, _diff_matrices(g, prd)):
        if name not in pr.params_name:
            continue
        coeff = float(np.real(pr[name]))
        dm = np.asarray(dm, dtype=np.complex128)
        for j in range(dim):
            e = np.zeros(dim, dtype=np.complex128)
            e[j] = 1
            e0 = e.copy()
            apply_matrix(e, n, objs, ctrls, dm)
            apply_matrix(e0, n, objs, ctrls, np.zeros_like(dm))
            out[:, j] += coeff * (e - e0)
    return out
