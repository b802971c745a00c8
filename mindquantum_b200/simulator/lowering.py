"""Lower a Circuit into the C gate table of libmqb200 and own the resulting native program.

This replaces the reference's ``Circuit.get_cpp_obj`` lowering to ``mqbackend.gate.*`` objects
(mindquantum/core/circuit/circuit.py:1108-1130) and the per-call ``ParameterResolver::Combination``
of every gate (vector_state.tpp:236-343): each gate becomes a fixed record whose angles are
linear expressions over one parameter vector, evaluated on the device for every sample.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _native as N
from ..core import gates as G
from ..core.operators import HowTo


def _real(v):
    return float(np.real(v))


def lower_circuit(circuit, param_names, grad_names=None):
    """Gate records, parameter terms, constant matrices and custom-gate specs of a circuit."""
    index = {k: i for i, k in enumerate(param_names)}
    grad_set = set(param_names if grad_names is None else grad_names)
    descs, terms, pool, customs = [], [], [], []
    custom_cursor = 0
    for g in circuit:
        if isinstance(g, G.BarrierGate) or g.name == 'I':
            continue
        if isinstance(g, G.Measure):
            raise ValueError("measurement gates must be split off before lowering")
        d = N.GateDesc()
        objs = list(g.obj_qubits)
        ctrl = 0
        for q in g.ctrl_qubits:
            ctrl |= 1 << int(q)
        d.ctrl_mask = ctrl
        if isinstance(g, G.ParameterGate):
            d.gate_id = g.gate_id
            if isinstance(g, G.RotPauliString):
                d.n_obj = 0
                mx = my = mz = ny = 0
                for p, q in zip(g.pauli_string, objs):
                    if p == 'X':
                        mx |= 1 << q
                    elif p == 'Y':
                        my |= 1 << q
                        ny += 1
                    elif p == 'Z':
                        mz |= 1 << q
                d.pauli_x, d.pauli_y, d.pauli_z, d.pauli_ny = mx, my, mz, ny
            else:
                if len(objs) > N.MQB_MAX_OBJ:
                    raise ValueError(f"{g.name} acts on {len(objs)} qubits; at most {N.MQB_MAX_OBJ} are supported")
                d.n_obj = len(objs)
                for i, q in enumerate(objs):
                    d.obj[i] = q
            d.n_angles = len(g.prs)
            grad_bits = 0
            for a, pr in enumerate(g.prs):
                d.angle_const[a] = _real(pr.const)
                d.term_begin[a] = len(terms)
                cnt = 0
                for name, coeff in pr.items():
                    if name not in index:
                        raise ValueError(f"parameter {name} of {g} is not in the parameter list")
                    t = N.ParamTerm()
                    t.param = index[name]
                    wants = name in grad_set and name not in pr.no_grad_parameters
                    t.flags = 1 if wants else 0
                    t.coeff = _real(coeff)
                    terms.append(t)
                    cnt += 1
                    if wants:
                        grad_bits |= 1 << a
                d.term_count[a] = cnt
            d.grad_angles = grad_bits
            if g.gate_id == G.GID_CUSTOM:
                size = 1 << (2 * len(objs))
                d.matrix_offset = custom_cursor
                customs.append(CustomSpec(g, custom_cursor, size, 0))
                custom_cursor += 2 * size
        else:
            m = np.asarray(g.matrix(), dtype=np.complex128)
            if len(objs) > N.MQB_MAX_OBJ:
                raise ValueError(f"{g.name} acts on {len(objs)} qubits; at most {N.MQB_MAX_OBJ} are supported")
            d.gate_id = G.GID_MATRIX
            d.n_obj = len(objs)
            for i, q in enumerate(objs):
                d.obj[i] = q
            # a channel's superoperator on a vectorized density matrix: never fused
            d.flags = N.MQB_GATE_NONUNITARY if getattr(g, 'nonunitary', False) else 0
            d.matrix_offset = sum(x.size for x in pool)
            pool.append(m.reshape(-1))
        descs.append(d)
    return descs, terms, pool, customs, custom_cursor


class CustomSpec:
    """A parameterized custom gate whose matrices the host evaluates per sample."""

    def __init__(self, gate, offset, size, angle_index):
        self.gate = gate
        self.offset = offset      # complex entries into the per-sample custom block
        self.size = size          # entries of one matrix
        self.angle_index = angle_index


class Program:
    """A lowered circuit bound to a parameter-name order, owning an ``mqb_program``.

    Args:
        circuit: gates to lower (measurements and barriers must already be removed).
        n_qubits: register size.
        precision: ``N.MQB_PREC_C64`` or ``N.MQB_PREC_C128``.
        param_names: order of the parameter vector the program reads.
        grad_names: names whose gradients are wanted (others get no gradient slot).
        fuse: fused tile passes (default) or one kernel per gate (the reference's schedule).
        tile_bits: tile width of the fused passes (0: automatic).
        jit: generated pass kernels (None automatic, True always, False never).
    """

    def __init__(self, circuit, n_qubits, precision, param_names, grad_names=None, fuse=True, tile_bits=0, jit=None):
        self.n_qubits = n_qubits
        self.precision = precision
        self.param_names = list(param_names)
        descs, terms, pool, customs, custom_cursor = lower_circuit(circuit, self.param_names, grad_names)
        self.customs = customs
        self.custom_entries = custom_cursor
        self.n_gates = len(descs)
        gate_arr = (N.GateDesc * max(1, len(descs)))(*descs)
        term_arr = (N.ParamTerm * max(1, len(terms)))(*terms)
        pool_arr = np.concatenate(pool) if pool else np.zeros(1, dtype=np.complex128)
        self._pool = np.ascontiguousarray(pool_arr.astype(np.complex128)).view(np.float64)
        opts = N.ProgramOptions()
        opts.fuse = 1 if fuse else 0
        opts.tile_bits = tile_bits
        opts.jit = 0 if jit is None else (1 if jit else -1)
        handle = ctypes.c_void_p()
        N.call('mqb_program_create', n_qubits, precision, gate_arr, len(descs), term_arr, len(terms),
               len(self.param_names), self._pool.ctypes.data_as(ctypes.c_void_p), pool_arr.size,
               ctypes.byref(opts), ctypes.byref(handle))
        self.handle = handle
        info = N.ProgramInfo()
        N.call('mqb_program_get_info', self.handle, ctypes.byref(info))
        self.info = info

    def __del__(self):
        h = getattr(self, 'handle', None)
        if h is not None and h.value:
            try:
                N.lib().mqb_program_destroy(h)
            except Exception:  # pylint: disable=broad-except
                pass
            self.handle = None

    def grad_passes(self, n_hams):
        n_p, k = ctypes.c_int(), ctypes.c_int()
        N.call('mqb_program_grad_passes', self.handle, n_hams, ctypes.byref(n_p), ctypes.byref(k))
        return n_p.value, k.value

    def custom_block(self, params_2d):
        """Per-sample matrices of the custom parameterized gates: [batch][custom_entries] complex128."""
        if not self.customs:
            return None
        batch = params_2d.shape[0]
        out = np.zeros((batch, max(1, self.custom_entries)), dtype=np.complex128)
        for spec in self.customs:
            g = spec.gate
            pr = g.prs[0]
            for b in range(batch):
                val = _real(pr.const) + sum(_real(c) * params_2d[b, self.param_names.index(k)] for k, c in pr.items())
                out[b, spec.offset:spec.offset + spec.size] = g.matrix_of([val]).reshape(-1)
                out[b, spec.offset + spec.size:spec.offset + 2 * spec.size] = g.diff_matrix_of([val], 0).reshape(-1)
        return out


def plan_schedule(circuit, n_qubits, precision, tile_bits=0, fuse=True):
    """The pass schedule libmqb200 builds for ``circuit`` (host only, no GPU needed).

    Returns (order, pass_of, qmask, fused): gate indices (into the lowered gate list) in execution
    order, the pass of each executed gate, and per pass the tile qubit mask and kind.
    """
    descs, _, pool, _, _ = lower_circuit(circuit, circuit.params_name)
    n = len(descs)
    gate_arr = (N.GateDesc * max(1, n))(*descs)
    pool_arr = np.concatenate(pool) if pool else np.zeros(1, dtype=np.complex128)
    pool_f = np.ascontiguousarray(pool_arr.astype(np.complex128)).view(np.float64)
    order = np.zeros(max(1, n), np.int32)
    pass_of = np.zeros(max(1, n), np.int32)
    qmask = np.zeros(max(1, n), np.uint64)
    fused = np.zeros(max(1, n), np.int32)
    stages = np.zeros(max(1, n), np.int32)
    n_passes = ctypes.c_int()
    N.call('mqb_plan_schedule', n_qubits, precision, gate_arr, n, pool_f.ctypes.data_as(ctypes.c_void_p),
           pool_arr.size, tile_bits, 1 if fuse else 0, ctypes.byref(n_passes), order.ctypes.data_as(ctypes.c_void_p),
           pass_of.ctypes.data_as(ctypes.c_void_p), qmask.ctypes.data_as(ctypes.c_void_p),
           fused.ctypes.data_as(ctypes.c_void_p), stages.ctypes.data_as(ctypes.c_void_p))
    k = n_passes.value
    plan_schedule.last_stages = stages[:k]
    return order[:n], pass_of[:n], qmask[:k], fused[:k]


def jit_check(circuit, n_qubits, precision, tile_bits=0, n_hams=0):
    """Generate and compile (NVRTC, no GPU needed) the pass kernels of ``circuit``.

    Forward kernels, plus the backward kernels for ``n_hams`` Hamiltonians when n_hams > 0.
    Returns the number of distinct kernels; raises with the compiler log on failure.
    """
    descs, _, pool, _, _ = lower_circuit(circuit, circuit.params_name)
    n = len(descs)
    gate_arr = (N.GateDesc * max(1, n))(*descs)
    pool_arr = np.concatenate(pool) if pool else np.zeros(1, dtype=np.complex128)
    pool_f = np.ascontiguousarray(pool_arr.astype(np.complex128)).view(np.float64)
    count = ctypes.c_int()
    N.call('mqb_jit_check', n_qubits, precision, gate_arr, n, pool_f.ctypes.data_as(ctypes.c_void_p), pool_arr.size,
           tile_bits, n_hams, ctypes.byref(count))
    return count.value


def lowered(circuit, n_qubits, precision, param_names, grad_names=None, fuse=True, tile_bits=0, jit=None):
    """Program for ``circuit`` cached on the circuit object (invalidated when the circuit changes)."""
    key = (n_qubits, precision, tuple(param_names), None if grad_names is None else tuple(grad_names), fuse,
           tile_bits, jit, len(circuit))
    cache = getattr(circuit, '_mqb_cache', None)
    if cache is None:
        cache = {}
        try:
            circuit._mqb_cache = cache  # pylint: disable=protected-access
        except AttributeError:
            pass
    prog = cache.get(key)
    if prog is None:
        prog = Program(circuit, n_qubits, precision, param_names, grad_names, fuse, tile_bits, jit)
        cache[key] = prog
    return prog


class NativeHamiltonian:
    """An ``mqb_hamiltonian``: a Hamiltonian's Pauli masks, or its CSR matrix (``HowTo.FRONTEND``;
    ``hermitian`` takes the conjugate transpose, like ``get_cpp_obj(hermitian=True)``,
    mindquantum/core/operators/hamiltonian.py:216-245)."""

    def __init__(self, ham, n_qubits, precision, hermitian=False):
        handle = ctypes.c_void_p()
        if ham.how_to == HowTo.FRONTEND:
            m = ham.sparse_matrix
            if m.shape[0] != (1 << n_qubits):
                raise RuntimeError("Sparse hamiltonian size not match with quantum state size.")
            if hermitian:
                m = m.conjugate().T.tocsr()
            cdt = np.complex64 if precision == N.MQB_PREC_C64 else np.complex128
            self._arrays = (np.ascontiguousarray(m.indptr, dtype=np.int64),
                            np.ascontiguousarray(m.indices, dtype=np.int64), np.ascontiguousarray(m.data, dtype=cdt))
            ptr = [a.ctypes.data_as(ctypes.c_void_p) for a in self._arrays]
            N.call('mqb_ham_create_csr', n_qubits, precision, int(m.nnz), *ptr, ctypes.byref(handle))
        else:
            mx, my, mz, ny, cf = ham.pauli_masks()
            self._arrays = (np.ascontiguousarray(mx), np.ascontiguousarray(my), np.ascontiguousarray(mz),
                            np.ascontiguousarray(ny), np.ascontiguousarray(cf))
            ptr = [a.ctypes.data_as(ctypes.c_void_p) for a in self._arrays]
            N.call('mqb_ham_create', n_qubits, precision, *ptr, len(cf), ctypes.byref(handle))
        self.handle = handle
        self.n_qubits = n_qubits
        self.precision = precision

    def __del__(self):
        h = getattr(self, 'handle', None)
        if h is not None and h.value:
            try:
                N.lib().mqb_ham_destroy(h)
            except Exception:  # pylint: disable=broad-except
                pass
            self.handle = None


def native_ham(ham, n_qubits, precision, hermitian=False):
    """The native Hamiltonian of ``ham`` (cached on it; a sparse matrix's conjugate transpose when
    ``hermitian``; Pauli Hamiltonians have real coefficients and are their own)."""
    hermitian = bool(hermitian) and ham.how_to == HowTo.FRONTEND
    cache = getattr(ham, '_mqb_cache', None)
    if cache is None:
        cache = {}
        ham._mqb_cache = cache  # pylint: disable=protected-access
    key = (n_qubits, precision, hermitian, ham.how_to)
    if key not in cache:
        cache[key] = NativeHamiltonian(ham, n_qubits, precision, hermitian)
    return cache[key]
