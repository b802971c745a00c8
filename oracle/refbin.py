"""The reference's own simulators, built from its sources by oracle/Makefile: the CPU simulator
(oracle/_ref/libmqref.so) and its thrust GPU simulator `mqvector_gpu` built for sm_100a
(oracle/_ref/libmqref_gpu.so).  TEST INFRASTRUCTURE ONLY: tests/ use them to pin the oracle (and
the CUDA path) to the reference itself, and bench.py's reference arm times them; the product never
does.

Supported gates (at most one control, at most two object qubits): X, Y, Z, H, S, T, SX (and their
daggers), SWAP, ISWAP (and its dagger), RX, RY, RZ, Rxx, Ryy, Rzz, Rxy, Rxz, Ryz, Givens, GlobalPhase,
PhaseShift and SWAPalpha whose angle is ``coeff * p + const`` of at most one parameter; U3, Rn and
FSim whose angles share at most one parameter; measurements; Pauli, depolarizing, amplitude- and
phase-damping and thermal-relaxation channels.  Hamiltonians: Pauli strings with real coefficients.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_ref', 'libmqref.so')
GPU_LIB_PATH = os.path.join(_HERE, '_ref', 'libmqref_gpu.so')
_KINDS = {'X': 0, 'H': 1, 'RX': 2, 'RY': 3, 'RZ': 4, 'Z': 5, 'Rzz': 6, 'Y': 7, 'PS': 8, 'M': 9, 'SWAP': 18,
          'Rxx': 20, 'Ryy': 21, 'Rxy': 22, 'Rxz': 23, 'Ryz': 24, 'G': 25, 'GP': 26, 'SWAPalpha': 27}
_FLAGGED = {'S': 15, 'T': 16, 'SX': 17, 'ISWAP': 19}
_MULTI = {'U3': 28, 'Rn': 29, 'FSim': 30}
_CHANNELS = {'PC': 10, 'BFC': 10, 'PFC': 10, 'BPFC': 10, 'DC': 11, 'ADC': 12, 'PDC': 13, 'TRC': 14}


def _channel_args(g):
    if g.name in ('PC', 'BFC', 'PFC', 'BPFC'):
        return [g.px, g.py, g.pz]
    if g.name in ('DC', 'PDC'):
        return [g.p if g.name == 'DC' else g.gamma, 0.0, 0.0]
    if g.name == 'ADC':
        return [g.gamma, 0.0, 1.0 if getattr(g, 'hermitianed', False) else 0.0]
    return [g.t1, g.t2, g.gate_time]
_libs = {}


def available(device='cpu'):
    return os.path.exists(GPU_LIB_PATH if device == 'gpu' else LIB_PATH)


def lib(device='cpu'):
    """The CPU (``device='cpu'``) or thrust GPU (``device='gpu'``) build; entry points are named
    mqref_* and mqref_gpu_* respectively and take the same arguments."""
    if device not in _libs:
        path, target = (GPU_LIB_PATH, 'refgpu') if device == 'gpu' else (LIB_PATH, 'ref')
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle {target}, with the reference checkout)")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        pre = 'mqref_gpu_' if device == 'gpu' else 'mqref_'
        getattr(L, pre + 'apply').argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 8 + [ctypes.c_int, P, ctypes.c_int,
                                                                                      P]
        if device == 'cpu':
            L.mqref_sample.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 8 + [ctypes.c_int, P, ctypes.c_int,
                                                                            ctypes.c_uint, ctypes.c_int, P]
        for fn in (getattr(L, pre + 'grad'), getattr(L, pre + 'grad_c64')):
            fn.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 8 + [ctypes.c_int, P, P, P, P, ctypes.c_int,
                                                                    ctypes.c_int, P, ctypes.c_int, P]
        _libs[device] = (L, pre)
    return _libs[device]


def _angle(pr, names):
    """(param index or -1, coefficient, constant) of an angle of at most one parameter."""
    keys = list(pr.params_name)
    if len(keys) > 1:
        raise ValueError("one parameter per angle")
    if not keys:
        return -1, 0.0, float(np.real(pr.const))
    return names.index(keys[0]), float(np.real(pr[keys[0]])), float(np.real(pr.const))


def _gate_table(circ, names, mkeys=None):
    """Columns of the harness's gate table; measurement gates take the index of their key in
    ``mkeys`` (appended to in circuit order) as their param column.  ``ch`` holds six values per
    gate: channel arguments, the daggered flag of S / T / SX / ISWAP, or the constants and
    coefficients of the angles of U3 / Rn / FSim (which share one parameter)."""
    cols = {k: [] for k in ('kind', 'o0', 'o1', 'ctrl', 'param', 'coeff', 'cst', 'ch')}

    def row(kind, g, param=-1, coeff=0.0, cst=0.0, ch=(0.0,) * 6):
        if len(g.obj_qubits) > 2 or len(g.ctrl_qubits) > 1:
            raise ValueError(f"gate {g.name} on {g.obj_qubits} / {g.ctrl_qubits} is not supported by the harness")
        for k, v in (('kind', kind), ('o0', int(g.obj_qubits[0]) if len(g.obj_qubits) else 0),
                     ('o1', int(g.obj_qubits[1]) if len(g.obj_qubits) > 1 else -1),
                     ('ctrl', int(g.ctrl_qubits[0]) if g.ctrl_qubits else -1), ('param', param), ('coeff', coeff),
                     ('cst', cst)):
            cols[k].append(v)
        cols['ch'].extend(list(ch) + [0.0] * (6 - len(ch)))

    for g in circ:
        if g.name in _CHANNELS:
            row(_CHANNELS[g.name], g, ch=_channel_args(g))
        elif g.name == 'M' and mkeys is not None:
            mkeys.append(g.key)
            row(_KINDS['M'], g, param=len(mkeys) - 1)
        elif g.name in _FLAGGED:
            row(_FLAGGED[g.name], g, ch=(1.0 if g.hermitianed else 0.0,))
        elif g.name in _MULTI:
            ang = [_angle(pr, names) for pr in g.prs]
            params = {a[0] for a in ang if a[0] >= 0}
            if len(params) > 1:
                raise ValueError(f"{g.name}: the angles must share one parameter")
            pi = params.pop() if params else -1
            ch = [a[2] for a in ang] + [0.0] * (3 - len(ang)) + [a[1] for a in ang]
            row(_MULTI[g.name], g, param=pi, ch=ch)
        else:
            name = 'PS' if g.name in ('PS', 'PhaseShift') else g.name
            if name not in _KINDS:
                raise ValueError(f"gate {g.name} is not supported by the reference harness")
            prs = getattr(g, 'prs', None)
            pi, coeff, cst = _angle(prs[0], names) if prs else (-1, 0.0, 0.0)
            row(_KINDS[name], g, param=pi, coeff=coeff, cst=cst)
    ints = {k: np.ascontiguousarray(cols[k], dtype=np.int32) for k in ('kind', 'o0', 'o1', 'ctrl', 'param')}
    dbls = {k: np.ascontiguousarray(cols[k] if cols[k] else [0.0], dtype=np.float64) for k in ('coeff', 'cst', 'ch')}
    return ints, dbls


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def apply(n, circ, params, threads=0, device='cpu'):
    """VectorState::ApplyCircuit from |0...0> with parameter values ``params`` (circ.params_name order),
    complex128, on the reference's CPU or thrust GPU policy."""
    names = list(circ.params_name)
    ints, dbls = _gate_table(circ, names)
    out = np.zeros(2 << n, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
    L, pre = lib(device)
    st = getattr(L, pre + 'apply')(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']),
                           _p(ints['param']), _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), len(names), _p(p),
                           threads, _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_apply failed ({st})")
    return out[0::2] + 1j * out[1::2]


def grad_pshift(n, circ, ham, params, threads=0):
    """The reference's parameter-shift gradient (GetExpectationWithGradParameterShiftMultiMulti,
    complex128, CPU), every parameter an encoder input: [samples][1 + n_params] complex."""
    return grad(n, circ, ham, params, threads=threads, _entry='grad_pshift')


def grad(n, circ, ham, params, threads=0, complex64=False, device='cpu', _entry=None):
    """VectorState::GetExpectationWithGradMultiMulti for one Hamiltonian, every parameter an encoder
    input: params [samples][n_params] -> [samples][1 + n_params] complex (f, then the gradient), on
    the reference's CPU (``device='cpu'``) or thrust GPU (``device='gpu'``) policy."""
    names = list(circ.params_name)
    ints, dbls = _gate_table(circ, names)
    tl, tq, tp, tc = [], [], [], []
    for term, c in ham.ham_termlist:
        tl.append(len(term))
        tc.append(float(c))
        for q, pch in term:
            tq.append(int(q))
            tp.append(pch)
    tl = np.ascontiguousarray(tl, dtype=np.int32)
    tq = np.ascontiguousarray(tq if tq else [0], dtype=np.int32)
    tc = np.ascontiguousarray(tc, dtype=np.float64)
    tpb = ctypes.create_string_buffer(''.join(tp).encode() or b'\0')
    params = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    S = params.shape[0]
    out = np.zeros(S * (1 + len(names)) * 2, dtype=np.float64)
    L, pre = lib(device)
    fn = getattr(L, pre + (_entry or ('grad_c64' if complex64 else 'grad')))
    if _entry:
        fn.argtypes = L.mqref_grad.argtypes
        fn.restype = ctypes.c_int
    st = fn(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']), _p(ints['param']),
            _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), len(tl), _p(tl), _p(tq), ctypes.cast(tpb, ctypes.c_void_p),
            _p(tc),
            len(names), S, _p(params), threads, _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_grad failed ({st})")
    out = out.reshape(S, 1 + len(names), 2)
    return out[..., 0] + 1j * out[..., 1]


def sample(n, circ, params, shots, seed, ending=True):
    """Shots of ``circ`` from |0...0> by the reference's own samplers (complex128):
    SamplingMeasurementEndingWithoutNoise when ``ending``, else Sampling (one re-simulation per
    shot, mid-circuit measurements).  Returns (keys in circuit order, samples[shots][n_keys])."""
    names = list(circ.params_name)
    keys = []
    ints, dbls = _gate_table(circ, names, keys)
    p = np.ascontiguousarray(params if len(names) else [0.0], dtype=np.float64).reshape(-1)
    out = np.zeros(max(1, shots * len(keys)), dtype=np.int32)
    L, _ = lib('cpu')
    st = L.mqref_sample(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']),
                        _p(ints['param']), _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), len(names), _p(p), shots,
                        seed,
                        1 if ending else 0, _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_sample failed ({st})")
    return keys, out[:shots * len(keys)].reshape(shots, len(keys)).astype(np.int64)


def _ham_arrays(ham):
    tl, tq, tp, tc = [], [], [], []
    for term, c in ham.ham_termlist:
        tl.append(len(term))
        tc.append(float(c))
        for q, pch in term:
            tq.append(int(q))
            tp.append(pch)
    return (np.ascontiguousarray(tl, dtype=np.int32), np.ascontiguousarray(tq if tq else [0], dtype=np.int32),
            ctypes.create_string_buffer(''.join(tp).encode() or b'\0'), np.ascontiguousarray(tc, dtype=np.float64))


def dm_apply(n, circ, params):
    """The reference's density-matrix simulator (complex128): rho after ``circ`` (gates and
    channels) from |0...0><0...0|, as a 2^n x 2^n array."""
    names = list(circ.params_name)
    ints, dbls = _gate_table(circ, names)
    p = np.ascontiguousarray(params if len(names) else [0.0], dtype=np.float64).reshape(-1)
    out = np.zeros(2 << (2 * n), dtype=np.float64)
    L, _ = lib('cpu')
    P = ctypes.c_void_p
    L.mqref_dm_apply.argtypes = [ctypes.c_int, ctypes.c_int] + [P] * 8 + [ctypes.c_int, P, P]
    st = L.mqref_dm_apply(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']),
                          _p(ints['param']), _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), len(names), _p(p),
                          _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_dm_apply failed ({st})")
    d = 1 << n
    return (out[0::2] + 1j * out[1::2]).reshape(d, d)


def dm_grad(n, circ, ham, params):
    """The reference's density-matrix expectation gradient (GetExpectationWithNoiseGradMultiMulti
    with channels in ``circ``, else GetExpectationWithReversibleGradMultiMulti), every parameter an
    encoder input: params [samples][n_params] -> [samples][1 + n_params] complex."""
    names = list(circ.params_name)
    ints, dbls = _gate_table(circ, names)
    tl, tq, tpb, tc = _ham_arrays(ham)
    params = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    S = params.shape[0]
    out = np.zeros(S * (1 + len(names)) * 2, dtype=np.float64)
    L, _ = lib('cpu')
    P = ctypes.c_void_p
    L.mqref_dm_grad.argtypes = ([ctypes.c_int, ctypes.c_int] + [P] * 8 + [ctypes.c_int, P, P, P, P, ctypes.c_int,
                                                                         ctypes.c_int, P, P])
    st = L.mqref_dm_grad(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']),
                         _p(ints['param']), _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), len(tl), _p(tl),
                         _p(tq), ctypes.cast(tpb, ctypes.c_void_p), _p(tc), len(names), S, _p(params), _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_dm_grad failed ({st})")
    out = out.reshape(S, 1 + len(names), 2)
    return out[..., 0] + 1j * out[..., 1]


def grad_nonherm(n, circ, circ_left, ham, params, psi, phi):
    """The reference's non-Hermitian gradient <phi| U_l^dag H U_r(p) |psi>
    (GetExpectationNonHermitianWithGradMultiMulti, complex128, CPU) with ``circ_left`` fixed and the
    right circuit's parameters as encoder inputs: params [samples][n_params] ->
    [samples][1 + n_params] complex (f, then the gradient)."""
    names = list(circ.params_name)
    ri, rd = _gate_table(circ, names)
    li, ld = _gate_table(circ_left, [])
    tl, tq, tpb, tc = _ham_arrays(ham)
    params = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    S = params.shape[0]
    cplx = lambda v: np.ascontiguousarray(np.stack([np.real(v), np.imag(v)], axis=-1).reshape(-1))  # noqa: E731
    psi_a, phi_a = cplx(np.asarray(psi, dtype=np.complex128)), cplx(np.asarray(phi, dtype=np.complex128))
    out = np.zeros(S * (1 + len(names)) * 2, dtype=np.float64)
    L, _ = lib('cpu')
    P, I = ctypes.c_void_p, ctypes.c_int
    L.mqref_grad_nonherm.argtypes = ([I, I] + [P] * 8 + [I] + [P] * 8 + [P, P, I, P, P, P, P, I, I, P, P])
    tab = lambda i, d: [_p(i['kind']), _p(i['o0']), _p(i['o1']), _p(i['ctrl']), _p(i['param']),  # noqa: E731
                        _p(d['coeff']), _p(d['cst']), _p(d['ch'])]
    st = L.mqref_grad_nonherm(n, len(ri['kind']), *tab(ri, rd), len(li['kind']), *tab(li, ld), _p(psi_a), _p(phi_a),
                              len(tl), _p(tl), _p(tq), ctypes.cast(tpb, ctypes.c_void_p), _p(tc), len(names), S,
                              _p(params), _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_grad_nonherm failed ({st})")
    out = out.reshape(S, 1 + len(names), 2)
    return out[..., 0] + 1j * out[..., 1]


def grad_qram(n, circ, ham, ans, init_states):
    """The reference's QRAM gradient (QramExpectationWithGrad, complex128, CPU): the ansatz with
    values ``ans`` applied to every row of ``init_states`` [samples][2^n]; returns
    [samples][1 + n_params] complex (f, then the ansatz gradient)."""
    names = list(circ.params_name)
    ints, dbls = _gate_table(circ, names)
    tl, tq, tpb, tc = _ham_arrays(ham)
    init = np.asarray(init_states, dtype=np.complex128)
    S = init.shape[0]
    init_a = np.ascontiguousarray(np.stack([init.real, init.imag], axis=-1).reshape(-1))
    p = np.ascontiguousarray(ans if len(names) else [0.0], dtype=np.float64).reshape(-1)
    out = np.zeros(S * (1 + len(names)) * 2, dtype=np.float64)
    L, _ = lib('cpu')
    P, I = ctypes.c_void_p, ctypes.c_int
    L.mqref_grad_qram.argtypes = [I, I] + [P] * 8 + [I, P, P, P, P, I, I, P, P, P]
    st = L.mqref_grad_qram(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']),
                           _p(ints['param']), _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), len(tl), _p(tl),
                           _p(tq), ctypes.cast(tpb, ctypes.c_void_p), _p(tc), len(names), S, _p(p), _p(init_a),
                           _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_grad_qram failed ({st})")
    out = out.reshape(S, 1 + len(names), 2)
    return out[..., 0] + 1j * out[..., 1]


def grad_csr(n, circ, matrix, params):
    """The reference's gradient with a Hamiltonian given as a sparse matrix (CsrHdMatrix from the
    scipy CSR arrays, complex128, CPU), every parameter an encoder input: [samples][1 + n_params]."""
    names = list(circ.params_name)
    ints, dbls = _gate_table(circ, names)
    m = matrix.tocsr()
    indptr = np.ascontiguousarray(m.indptr, dtype=np.int64)
    indices = np.ascontiguousarray(m.indices if m.nnz else [0], dtype=np.int64)
    data = np.asarray(m.data if m.nnz else [0], dtype=np.complex128)
    data = np.ascontiguousarray(np.stack([data.real, data.imag], axis=-1).reshape(-1))
    params = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    S = params.shape[0]
    out = np.zeros(S * (1 + len(names)) * 2, dtype=np.float64)
    L, _ = lib('cpu')
    P, I = ctypes.c_void_p, ctypes.c_int
    L.mqref_grad_csr.argtypes = [I, I] + [P] * 8 + [ctypes.c_int64, P, P, P, I, I, P, P]
    st = L.mqref_grad_csr(n, len(ints['kind']), _p(ints['kind']), _p(ints['o0']), _p(ints['o1']), _p(ints['ctrl']),
                          _p(ints['param']), _p(dbls['coeff']), _p(dbls['cst']), _p(dbls['ch']), m.nnz, _p(indptr),
                          _p(indices), _p(data), len(names), S, _p(params), _p(out))
    if st != 0:
        raise RuntimeError(f"mqref_grad_csr failed ({st})")
    out = out.reshape(S, 1 + len(names), 2)
    return out[..., 0] + 1j * out[..., 1]
