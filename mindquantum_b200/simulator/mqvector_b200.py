"""MQVectorB200: the B200 state-vector backend behind ``Simulator('mqvector_b200', n)``.

It keeps the reference ``MQSim`` interface (mindquantum/simulator/mqsim.py:51-560): argument
checks, the encoder/ansatz split of ``get_expectation_with_grad`` and the result layout
``(f, g_enc, g_ans)`` with shapes ``[n_prs][n_hams]`` / ``[n_prs][n_hams][n_params]``.  The state
is a torch tensor on the current CUDA device; all arithmetic runs in libmqb200 through its C ABI.
"""
from __future__ import annotations

import ctypes
import math
import warnings

import numpy as np
import torch

from .. import _native as N
from ..core import gates as G
from ..core.circuit import Circuit
from ..core.operators import Hamiltonian, HowTo
from ..core.parameterresolver import ParameterResolver, to_pr
from ..dtype import complex64, complex128
from .backend_base import BackendBase
from .lowering import lowered, native_ham
from .measure_result import MeasureResult
from .parameter_shift import ShiftPlan
from .rng import Mt19937Uniform, UniformBlocks, UniformStreams
from .utils import GradOpsWrapper, _thread_balance, check_kept_qubits, qs_of_qubits, reduced_density_matrix


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _split_inputs(version, enc_names, ans_names, inputs_):
    """Encoder rows ``[n_prs][n_enc]`` and the ansatz vector of a grad operator call (mqsim.py:341-380)."""
    inputs = [np.array(x) if isinstance(x, list) else x for x in inputs_]
    if version == "both" and len(inputs) != 2:
        raise ValueError("Need two inputs!")
    if version in ("encoder", "ansatz") and len(inputs) != 1:
        raise ValueError("Need one input!")
    if version in ("both", "encoder"):
        enc = np.asarray(inputs[0], dtype=np.float64)
        enc = enc[None, :] if enc.ndim == 1 else enc
        if enc.ndim != 2 or enc.shape[1] != len(enc_names):
            raise ValueError(f"encoder data requires a two dimension array with {len(enc_names)} columns, "
                             f"but get shape {enc.shape}")
        ans = np.asarray(inputs[1], dtype=np.float64).reshape(-1) if version == "both" else np.zeros(0)
    else:
        enc = np.zeros((1, 0))
        ans = np.asarray(inputs[0], dtype=np.float64).reshape(-1)
    if ans.size != len(ans_names):
        raise ValueError(f"ansatz data requires {len(ans_names)} values, but get {ans.size}")
    return enc, ans


# |<psi|psi> - 1| above which a complex64 gradient whose backward sweep rebuilt states by reverse
# application warns (its gradients then carry errors of the same order)
NORM_DRIFT_WARN = 1e-4


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("the mqvector_b200 backend needs a CUDA device (B200, sm_100a); none is visible")


class MQVectorB200(BackendBase):
    """State-vector simulator on one B200.

    Args:
        name: backend name.
        n_qubits: number of qubits.
        seed: seed of the measurement random stream (std::mt19937 as in the reference).
        dtype: ``complex128`` (default) or ``complex64``.
        fuse: fused tile passes (default) or one kernel per gate.
        jit: generated pass kernels: None automatic (registers of 18 qubits and more), True always,
            False never (the precompiled tile kernels).
        device: CUDA device (default: the current one).
    """

    def __init__(self, name, n_qubits, seed=None, dtype=None, fuse=True, device=None, jit=None):
        _require_cuda()
        super().__init__(name, n_qubits, seed, dtype)
        if not isinstance(n_qubits, int) or n_qubits < 1:
            raise ValueError(f"n_qubits should be a positive integer, but get {n_qubits}")
        if seed is None:
            seed = int(np.random.randint(1, 2**23))
        self.seed = int(seed)
        self.fuse = fuse
        self.jit = jit
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        self._state = None          # None means |0...0>, like the reference's null state
        self._rng = Mt19937Uniform(self.seed)
        N.lib()

    # ------------------------------------------------------------------ basics
    @property
    def precision(self):
        return N.MQB_PREC_C64 if self.arithmetic_type == complex64 else N.MQB_PREC_C128

    @property
    def torch_dtype(self):
        return torch.complex64 if self.arithmetic_type == complex64 else torch.complex128

    @property
    def dtype(self):
        return self.arithmetic_type

    def device_name(self):
        return f"{self.n_qubits} qubits {self.name} simulator."

    def _zero_state(self, batch=None):
        shape = (1 << self.n_qubits,) if batch is None else (batch, 1 << self.n_qubits)
        s = torch.zeros(shape, dtype=self.torch_dtype, device=self.device)
        s[..., 0] = 1
        return s

    @property
    def state(self):
        """The state as a device tensor (allocated on first use)."""
        if self._state is None:
            self._state = self._zero_state()
        return self._state

    def reset(self):
        self._state = None

    def copy(self):
        sim = MQVectorB200(self.name, self.n_qubits, self.seed, self.arithmetic_type, self.fuse, self.device, self.jit)
        if self._state is not None:
            sim._state = self._state.clone()
        return sim

    def astype(self, dtype, seed=None):
        sim = MQVectorB200(self.name, self.n_qubits, self.seed if seed is None else seed, dtype, self.fuse, self.device,
                           self.jit)
        if self._state is not None:
            sim._state = self._state.to(sim.torch_dtype)
        return sim

    def get_qs(self, ket=False):
        qs = self.state.detach().to(torch.complex128).cpu().numpy()
        if ket:
            return '\n'.join(f"{v}¦{format(i, f'0{self.n_qubits}b')}⟩" for i, v in enumerate(qs) if abs(v) > 1e-12)
        return qs

    # pure-state answers of MQSim's density-matrix methods for a state vector (mqsim.py:546-597)
    def entropy(self):
        return 0.0

    def purity(self):
        return 1.0

    def get_pure_state_vector(self):
        return self.get_qs()

    def get_partial_trace(self, obj_qubits):
        raise ValueError(f"{self.name} simulator not support partial trace method.")

    def get_circuit_matrix(self, circuit, pr):
        """Matrix of ``circuit`` with parameters ``pr`` (mqsim.py:199-201): column j is the circuit
        applied to |j>, evaluated column by column on a scratch simulator of this size and dtype;
        measurement gates are dropped."""
        if not isinstance(circuit, Circuit):
            raise TypeError(f"circuit requires a Circuit, but get {type(circuit)}")
        body = circuit.remove_measure()
        dim = 1 << self.n_qubits
        sim = MQVectorB200(self.name, self.n_qubits, self.seed, self.arithmetic_type, self.fuse, self.device, self.jit)
        cols = []
        for j in range(dim):
            e = np.zeros(dim, dtype=np.complex128)
            e[j] = 1
            sim.set_qs(e)
            sim.apply_circuit(body, pr)
            cols.append(sim.get_qs())
        return np.array(cols).T

    def get_reduced_density_matrix(self, kept_qubits):
        """Density matrix of ``kept_qubits`` with the other qubits traced out (mqsim.py:559-570,
        VectorState::GetReducedDensityMatrix): computed on the device from the state."""
        kept = check_kept_qubits(kept_qubits, self.n_qubits)
        return reduced_density_matrix(self.state.detach(), self.n_qubits, kept)

    def get_qs_of_qubits(self, qubits, ket=False):
        """Reduced state of ``qubits``: a vector when it is pure, else its density matrix
        (mqsim.py:598-626)."""
        return qs_of_qubits(self, qubits, ket)

    def set_qs(self, quantum_state):
        """Set the state; the vector is normalised first (mqsim.py:538-544)."""
        v = np.asarray(quantum_state)
        if v.ndim != 1:
            raise ValueError(f"vec requires a 1-dimensional array, but get {v.shape}")
        n = np.log2(v.shape[0])
        if n % 1 != 0:
            raise ValueError(f"vec size {v.shape[0]} is not power of 2")
        if int(n) != self.n_qubits:
            raise ValueError(f"{int(n)} qubits vec does not match with simulation qubits ({self.n_qubits})")
        norm = np.sqrt(np.sum(np.abs(v) ** 2))
        if norm == 0.0:
            raise ValueError("Wrong quantum state.")
        self._state = torch.as_tensor(v / norm, dtype=self.torch_dtype).to(self.device)

    def set_state_tensor(self, t):
        """Set the state from a device tensor without normalising (zero-copy when dtype/device match)."""
        if t.shape != (1 << self.n_qubits,):
            raise ValueError(f"state must have shape ({1 << self.n_qubits},)")
        self._state = t.to(device=self.device, dtype=self.torch_dtype).contiguous()

    # ------------------------------------------------------------------ gate application
    def _params_tensor(self, prog, pr):
        names = prog.param_names
        if not names:
            return torch.zeros((1, 1), dtype=torch.float64, device=self.device), np.zeros((1, 0))
        vals = np.array([[float(np.real(pr[k])) for k in names]], dtype=np.float64)
        return torch.as_tensor(vals, device=self.device), vals

    def _custom_tensor(self, prog, params_np):
        blk = prog.custom_block(params_np)
        if blk is None:
            return None
        return torch.as_tensor(np.ascontiguousarray(blk).view(np.float64), device=self.device)

    def _apply_segment(self, states, circuit, pr, batch=1):
        """Apply a measurement-free circuit in place to ``states`` ([batch][2^n]); ``pr`` is one
        ParameterResolver for every state, or ``(names, rows)`` with one row of values per state."""
        names = circuit.params_name
        prog = lowered(circuit, self.n_qubits, self.precision, names, None, self.fuse, jit=self.jit)
        if prog.n_gates == 0:
            return
        if isinstance(pr, tuple):
            all_names, rows = pr
            cols = [all_names.index(k) for k in prog.param_names]
            params_np = np.ascontiguousarray(rows[:, cols] if cols else np.zeros((batch, 1)), dtype=np.float64)
            params = torch.as_tensor(params_np, device=self.device)
            stride = params_np.shape[1]
        else:
            params, params_np = self._params_tensor(prog, pr)
            stride = 0
        custom = self._custom_tensor(prog, params_np)
        if custom is not None and custom.shape[0] != batch:   # the custom block has one row per state
            custom = custom.expand(batch, -1).contiguous()
        ws_bytes = ctypes.c_size_t()
        N.call('mqb_apply_workspace_size', prog.handle, batch, ctypes.byref(ws_bytes))
        ws = torch.empty(ws_bytes.value, dtype=torch.uint8, device=self.device)
        N.call('mqb_apply', prog.handle, _ptr(states), batch, _ptr(params), stride, _ptr(custom), _ptr(ws),
               ws_bytes.value, _stream())

    def _measure(self, state, gate, rng):
        """ApplyMeasure (vector_state.tpp:440-462) on one state: draw, collapse, optional reset."""
        return int(self._measure_rows(state.view(1, -1), gate, UniformStreams([rng]))[0])

    def _measure_rows(self, states, gate, streams):
        """ApplyMeasure on every trajectory of ``states`` at once: P(q = 1) of all of them in one
        reduction, one draw each from its own stream, the collapse (the projector over the square
        root of the outcome's probability) in one launch, then X where a reset asks for it."""
        q = gate.obj_qubits[0]
        rows = np.arange(states.shape[0])
        one = self._rows_norm(states, rows, self._P1, q)
        to_one = streams.take(rows) < one
        prob = np.where(to_one, one, 1.0 - one)
        with np.errstate(divide='ignore'):
            scale = np.where(prob > 0, 1.0 / np.sqrt(np.where(prob > 0, prob, 1.0)), 0.0)
        mats = np.zeros((len(rows), 2, 2), dtype=np.complex128)
        mats[to_one, 1, 1] = scale[to_one]
        mats[~to_one, 0, 0] = scale[~to_one]
        self._rows_apply(states, rows, mats, q)
        if gate.reset_to is not None:
            self._rows_apply(states, rows[to_one.astype(int) != int(gate.reset_to)], self._PAULI[0], q)
        return to_one.astype(np.int64)

    @staticmethod
    def _split(circuit):
        """The circuit as unitary segments, measurements and channels (cached on the circuit)."""
        key = len(circuit)
        cached = getattr(circuit, '_mqb_split', None)
        if cached is not None and cached[0] == key:
            return cached[1]
        parts, segment = [], Circuit()
        for g in circuit:
            if isinstance(g, (G.Measure, G.NoiseGate)):
                if len(segment):
                    parts.append(segment)
                    segment = Circuit()
                parts.append(g)
            elif not isinstance(g, G.BarrierGate):
                segment.append(g)
        if len(segment):
            parts.append(segment)
        try:
            circuit._mqb_split = (key, parts)  # pylint: disable=protected-access
        except AttributeError:
            pass
        return parts

    def _run(self, state, circuit, pr, rng):
        """Apply ``circuit`` in place; measurements and channels draw from ``rng``
        (VectorState::ApplyCircuit, vector_state.tpp:949-960)."""
        res = self._run_batch(state.view(1, -1), circuit, pr, UniformStreams([rng]))
        return {k: int(v[0]) for k, v in res.items()}

    def _run_batch(self, states, circuit, pr, streams):
        """Run one trajectory of ``circuit`` per row of ``states`` ([B][2^n]) in place, trajectory b
        drawing from stream b of ``streams``: the unitary segments as one batched launch, every
        measurement and channel with each trajectory's draws in the reference's order and the
        state-dependent probabilities of all trajectories in one reduction and one copy to the
        host.  Returns {measurement key: outcomes [B]}."""
        B = states.shape[0]
        results = {}
        if not circuit.has_measure_gate and not circuit.is_noise_circuit:
            if len(circuit):
                self._apply_segment(states, circuit, pr, B)
            return results
        for part in self._split(circuit):
            if isinstance(part, G.Measure):
                results[part.key] = self._measure_rows(states, part, streams)
            elif isinstance(part, G.NoiseGate):
                self._channel_rows(states, part, streams)
            else:
                self._apply_segment(states, part, pr, B)
        return results

    # ------------------------------------------------------------------ noise channels
    _PAULI = np.array([[[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]]], dtype=np.complex128)
    _P0 = np.array([[1, 0], [0, 0]], dtype=np.complex128)
    _P1 = np.array([[0, 0], [0, 1]], dtype=np.complex128)

    def _rows_args(self, states, rows, mats, q, mask):
        k = len(rows)
        self._rows_keep = (np.ascontiguousarray(rows, dtype=np.int64), np.full(k, int(q), dtype=np.int32),
                           np.full(k, int(mask), dtype=np.uint64),
                           np.ascontiguousarray(np.broadcast_to(mats, (k, 2, 2)), dtype=np.complex128)
                           .reshape(k, 4).view(np.float64))
        vp = ctypes.c_void_p
        return [self.n_qubits, self.precision, _ptr(states), states.shape[0], k] + \
            [a.ctypes.data_as(vp) for a in self._rows_keep]

    def _rows_apply(self, states, rows, mats, q, mask=0):
        """mats[i] (or one 2x2 matrix for all) on qubit q of states[rows[i]] where every bit of
        ``mask`` is set, in place, one launch (mqb_rows_apply_matrix1)."""
        if len(rows):
            N.call('mqb_rows_apply_matrix1', *self._rows_args(states, rows, mats, q, mask), _stream())

    def _rows_norm(self, states, rows, mats, q, mask=0):
        """||M_i states[rows[i]]||^2 for every row in one reduction, copied to the host
        (mqb_rows_matrix1_norm); with M = [[1, 0], [0, 0]] or [[0, 0], [0, 1]] and no mask, the
        reference's ZeroStateVdot / OneStateVdot."""
        if not len(rows):
            return np.zeros(0)
        out = torch.empty(len(rows), dtype=torch.float64, device=self.device)
        N.call('mqb_rows_matrix1_norm', *self._rows_args(states, rows, mats, q, mask), _ptr(out), _stream())
        return out.cpu().numpy()

    @staticmethod
    def _pauli_index(cum, r):
        """lower_bound over [0, px, px+py, px+py+pz, 1] for every draw in ``r``: 0 = X, 1 = Y,
        2 = Z, 3 = identity."""
        it = np.searchsorted(np.asarray(cum, dtype=np.float64), r, side='left')
        return np.where(it > 0, it - 1, 0)

    def _channel_rows(self, states, g, streams):
        """One step of a channel on every trajectory of ``states`` at once
        (VectorState::ApplyChannel, vector_state.tpp:465-709).  Trajectory b draws from stream b
        in the reference's order; the probabilities that depend on the state (damping, Kraus,
        thermal relaxation) are FP64 reductions on the device, one per step for all trajectories;
        each trajectory's operator (the chosen Kraus operator over the square root of its
        probability, or a Pauli) is applied to all trajectories in one launch."""
        rows = np.arange(states.shape[0])
        objs = [int(q) for q in g.obj_qubits]
        mask = sum(1 << int(c) for c in g.ctrl_qubits)
        P = self._PAULI
        if isinstance(g, G.PauliChannel):
            k = self._pauli_index(g.cumulative_probs(), streams.take(rows))
            self._rows_apply(states, rows[k < 3], P[k[k < 3]], objs[0], mask)
        elif isinstance(g, G.GroupedPauliChannel):
            picks = []
            for q, prow in zip(objs, g.probs):
                px, py, pz = (float(v) for v in prow)
                cum = [0.0, px, px + py, px + py + pz, px + py + pz + (1 - px - py - pz)]
                picks.append((q, self._pauli_index(cum, streams.take(rows))))
            for q, k in picks:    # ApplyPauliString: no controls
                self._rows_apply(states, rows[k < 3], P[k[k < 3]], q)
        elif isinstance(g, G.DepolarizingChannel):
            active, idx, p = rows, 0, float(g.p)
            while idx < len(objs) and len(active):
                hit = streams.take(active) < p * 3.0 / 4.0
                chosen = active[hit]
                if len(chosen):
                    p_i = streams.take(chosen)
                    self._rows_apply(states, chosen, P[np.where(p_i < 1.0 / 3.0, 0, np.where(p_i < 2.0 / 3.0, 1, 2))],
                                     objs[idx], mask)
                    for q in objs[idx + 1:]:
                        p_i = streams.take(chosen)
                        sel = p_i < 0.75
                        k = np.where(p_i < 0.25, 0, np.where(p_i < 0.5, 1, 2))
                        self._rows_apply(states, chosen[sel], P[k[sel]], q, mask)
                active = active[~hit]
                if not 4 > 3 * p:
                    break
                idx, p = idx + 1, p / (4 - 3 * p)
        elif isinstance(g, G.KrausChannel):
            active = rows
            total = np.ones(len(rows))
            for m in np.asarray(g.kraus_op, dtype=np.complex128):
                if not len(active):
                    break
                if abs(m[0, 1]) < 1e-6 and abs(m[1, 0]) < 1e-6 and abs(m[0, 0] - m[1, 1]) < 1e-6:
                    prob = float((m[0, 0] * np.conj(m[0, 0])).real)
                    with np.errstate(divide='ignore', invalid='ignore'):
                        rel = prob / total[active]
                    total[active] -= prob
                    chosen = streams.take(active) < rel
                    if m[0, 0].imag >= 1e-6:   # identity with a phase
                        v = m[0, 0] / math.sqrt(prob)
                        self._rows_apply(states, active[chosen], np.array([[v, 0], [0, v]]), 0)
                else:
                    prob = self._rows_norm(states, active, m, objs[0], mask)
                    with np.errstate(divide='ignore', invalid='ignore'):
                        rel = prob / total[active]
                    total[active] -= prob
                    chosen = streams.take(active) < rel
                    self._rows_apply(states, active[chosen], m[None] / np.sqrt(prob[chosen])[:, None, None], objs[0],
                                     mask)
                active = active[~chosen]
        elif isinstance(g, (G.AmplitudeDampingChannel, G.PhaseDampingChannel)):
            renorm = self._rows_norm(states, rows, self._P1, objs[0])   # OneStateVdot: controls ignored
            live = renorm >= 1e-6
            act, rn = rows[live], renorm[live]
            if len(act):
                gamma = float(g.gamma)
                prob = gamma * rn
                jump = streams.take(act) <= prob
                stay = ~jump
                mats = np.zeros((len(act), 2, 2), dtype=np.complex128)
                if isinstance(g, G.AmplitudeDampingChannel):
                    mats[jump, 0, 1] = 1 / np.sqrt(rn[jump])
                else:
                    mats[jump, 1, 1] = 1 / np.sqrt(rn[jump])
                mats[stay, 0, 0] = 1 / np.sqrt(1 - prob[stay])
                mats[stay, 1, 1] = math.sqrt(1 - gamma) / np.sqrt(1 - prob[stay])
                self._rows_apply(states, act, mats, objs[0], mask)
        elif isinstance(g, G.ThermalRelaxationChannel):
            t1, t2, tg = float(g.t1), float(g.t2), float(g.gate_time)
            e1, e2 = math.exp(-tg / t1), math.exp(-tg / t2)
            p_reset = 1 - e1
            q = objs[0]
            if t1 >= t2:
                pz = e1 * (1 - e2 / e1) / 2
                r = streams.take(rows)
                self._rows_apply(states, rows[(r >= 1 - pz - p_reset) & (r < 1 - p_reset)], P[2], q, mask)
                reset = rows[r >= 1 - p_reset]
                if len(reset):
                    zero = self._rows_norm(states, reset, self._P0, q)   # ZeroStateVdot
                    to_zero = streams.take(reset) < zero
                    mats = np.zeros((len(reset), 2, 2), dtype=np.complex128)
                    mats[to_zero, 0, 0] = 1 / np.sqrt(zero[to_zero])
                    mats[~to_zero, 0, 1] = 1 / np.sqrt(1 - zero[~to_zero])
                    self._rows_apply(states, reset, mats, q, mask)
            elif 2 * t1 > t2:
                r = streams.take(rows)
                root = math.sqrt(p_reset * p_reset + 4 * e2 * e2)
                ev0, ev1 = (2 - p_reset + root) / 2, (2 - p_reset - root) / 2
                vec0, vec1 = (ev0 - e1) / e2, (ev1 - e1) / e2
                zero = self._rows_norm(states, rows, self._P0, q)   # ZeroStateVdot
                one = 1 - zero
                c0 = vec0 * vec0 * zero + one
                c1 = vec1 * vec1 * zero + one
                b0 = r < c0 * ev0 / (vec0 * vec0 + 1)
                b1 = ~b0 & (r < 1 - p_reset * one)
                b2 = ~b0 & ~b1
                mats = np.zeros((len(rows), 2, 2), dtype=np.complex128)
                mats[b0, 0, 0] = vec0 / np.sqrt(c0[b0])
                mats[b0, 1, 1] = 1 / np.sqrt(c0[b0])
                mats[b1, 0, 0] = vec1 / np.sqrt(c1[b1])
                mats[b1, 1, 1] = 1 / np.sqrt(c1[b1])
                mats[b2, 0, 1] = 1 / np.sqrt(one[b2])
                self._rows_apply(states, rows, mats, q, mask)
        else:
            raise ValueError(f"{g.name} is not a noise channel.")

    def _check_pr(self, circuit, pr):
        if circuit.params_name:
            if pr is None:
                raise ValueError("Applying a parameterized circuit needs a parameter_resolver.")
            pr = to_pr(pr, circuit.params_name)
            for k in circuit.params_name:
                if k not in pr:
                    raise ValueError(f"Parameter {k} is missing in the parameter resolver.")
            if pr.is_complex:
                warnings.warn("Simulator does not support complex number, the imaginary part will be ignored",
                              UserWarning, stacklevel=3)
            return pr
        return ParameterResolver()

    def apply_circuit(self, circuit, pr=None):
        """Apply a circuit; measurements collapse the state and are returned as a MeasureResult."""
        if not isinstance(circuit, Circuit):
            raise TypeError(f"circuit requires a Circuit, but get {type(circuit)}")
        if self.n_qubits < circuit.n_qubits:
            raise ValueError(f"Circuit has {circuit.n_qubits} qubits, which is more than simulator qubits.")
        pr = self._check_pr(circuit, pr)
        res = self._run(self.state, circuit, pr, self._rng)
        if res:
            out = MeasureResult()
            keys = circuit.all_measures.keys()
            out.add_measure(keys)
            out.collect_data([[res[k] for k in out.keys]])
            return out
        return None

    def apply_gate(self, gate, pr=None, diff=False):
        """Apply one gate; ``diff=True`` applies the gate's derivative matrix (vector_state.tpp:166-437)."""
        if not isinstance(gate, G.BasicGate):
            raise TypeError(f"gate requires a quantum gate, but get {type(gate)}")
        if isinstance(gate, G.BarrierGate):
            return None
        if max(gate.obj_qubits + gate.ctrl_qubits) >= self.n_qubits:
            raise ValueError(f"qubits of gate {gate} is higher than simulator qubits.")
        if isinstance(gate, G.Measure):
            return self._measure(self.state, gate, self._rng)
        circ = Circuit([gate])
        pr = self._check_pr(circ, pr)
        if diff and gate.parameterized:
            # derivative matrix on the controlled subspace, zero elsewhere (SetToZeroExcept)
            names = [k for p in gate.get_parameters() for k in p.params_name]
            dm = gate.diff_matrix(pr, names[0] if len(set(names)) == 1 else None)
            qubits = gate.obj_qubits + gate.ctrl_qubits
            k, c = len(gate.obj_qubits), len(gate.ctrl_qubits)
            full = np.zeros((1 << (k + c), 1 << (k + c)), dtype=complex)
            base = ((1 << c) - 1) << k
            full[base:base + (1 << k), base:base + (1 << k)] = dm
            circ = Circuit([G.UnivMathGate('diff', full).on(qubits)])
            pr = ParameterResolver()
        self._apply_segment(self.state, circ, pr)
        return None

    def apply_hamiltonian(self, hamiltonian):
        if not isinstance(hamiltonian, Hamiltonian):
            raise TypeError(f"hamiltonian requires a Hamiltonian, but get {type(hamiltonian)}")
        self._check_ham(hamiltonian)
        h = native_ham(hamiltonian, self.n_qubits, self.precision)
        out = torch.empty_like(self.state)
        N.call('mqb_apply_hamiltonian', h.handle, _ptr(self.state), _ptr(out), 1, _stream())
        self._state = out

    def _check_ham(self, ham):
        """_check_hamiltonian_qubits_number (mindquantum/utils/type_value_check.py:51-63)."""
        if ham.how_to != HowTo.ORIGIN:
            if ham.n_qubits != self.n_qubits:
                raise ValueError(f"Hamiltonian qubits is {ham.n_qubits}, not match with simulator qubits number "
                                 f"{self.n_qubits}")
        elif ham.n_qubits > self.n_qubits:
            raise ValueError(f"Hamiltonian qubits is {ham.n_qubits}, which is bigger than simulator qubits.")

    # ------------------------------------------------------------------ expectations
    def _sub_seed(self, sim):
        """static_cast<unsigned>(static_cast<calc_type>(rng_()) * (1 << 20)) on ``sim``'s stream."""
        d = sim._rng.draw()  # pylint: disable=protected-access
        if self.precision == N.MQB_PREC_C64:
            return int(np.float32(np.float32(d) * np.float32(1 << 20)))
        return int(d * (1 << 20))

    def get_expectation(self, hamiltonian, circ_right=None, circ_left=None, simulator_left=None, pr=None):
        """<psi| circ_left^dag H circ_right |psi> (GetExpectation, vector_state.tpp:712-768)."""
        if not isinstance(hamiltonian, Hamiltonian):
            raise TypeError(f"hamiltonian requires a Hamiltonian, but get {type(hamiltonian)}")
        self._check_ham(hamiltonian)
        circ_right = Circuit() if circ_right is None else circ_right
        pr = ParameterResolver() if pr is None else to_pr(pr, circ_right.params_name)
        # sub-streams as the reference seeds its copies: int(float(draw) * 2^20), the bra's first
        # (from simulator_left's stream when there is one), vector_state.tpp:712-768
        if circ_left is None and simulator_left is None:
            ket = self.state.clone()
            self._run(ket, circ_right, pr, Mt19937Uniform(self._sub_seed(self)))
            bra = ket
        else:
            src = self if simulator_left is None else getattr(simulator_left, 'backend', simulator_left)
            if isinstance(src, BackendBase) and not isinstance(src, MQVectorB200):
                raise TypeError("simulator_left should be a mqvector_b200 simulator")
            if src.n_qubits != self.n_qubits or src.dtype != self.dtype:
                raise ValueError("simulator_left should have the same qubits and dtype")
            bra_seed = self._sub_seed(src)
            ket_seed = self._sub_seed(self)
            ket = self.state.clone()
            self._run(ket, circ_right, pr, Mt19937Uniform(ket_seed))
            bra = src.state.clone()
            self._run(bra, circ_right if circ_left is None else circ_left, pr, Mt19937Uniform(bra_seed))
        h = native_ham(hamiltonian, self.n_qubits, self.precision)
        out = torch.zeros(2, dtype=torch.float64, device=self.device)
        N.call('mqb_expectation', h.handle, _ptr(bra), _ptr(ket), 1, _ptr(out), _stream())
        o = out.cpu().numpy()
        return complex(o[0], o[1])

    def expectation_with_grad_tensor(self, hams, circuit, params, param_names, grad_names=None, init_state=None,
                                     ckpt_stride=None):
        """Batched forward + adjoint gradient on device tensors.

        Args:
            hams: list of Hamiltonian.
            circuit: parameterized circuit (no measurement).
            params: float64 CUDA tensor [batch][len(param_names)].
            param_names: parameter order of ``params``.
            grad_names: names that need gradients (default: all).
            init_state: None (|0...0>), [2^n] or [batch][2^n] tensor.
            ckpt_stride: passes between stored states (None: choose from free memory).
        Returns:
            f: float64 [batch][n_hams][2] (re, im); grad: float64 [batch][n_hams][n_params].
        """
        prog = lowered(circuit, self.n_qubits, self.precision, param_names, grad_names, self.fuse, jit=self.jit)
        nh = [native_ham(h, self.n_qubits, self.precision) for h in hams]
        params = params.to(device=self.device, dtype=torch.float64).contiguous()
        batch = params.shape[0]
        custom = None
        if prog.customs:
            custom = self._custom_tensor(prog, params.detach().cpu().numpy())
        init_batched = 0
        init = None
        if init_state is not None:
            init = init_state.to(device=self.device, dtype=self.torch_dtype).contiguous()
            init_batched = 1 if init.dim() == 2 else 0
        ham_arr = (ctypes.c_void_p * len(nh))(*[h.handle.value for h in nh])
        # the previous call's workspace (kept for its norm checks) goes back to the allocator first,
        # so this call can take the same memory
        self._last_grad = None
        stride = self._choose_stride(prog, batch, len(nh)) if ckpt_stride is None else int(ckpt_stride)
        ws_bytes = ctypes.c_size_t()
        N.call('mqb_grad_workspace_size', prog.handle, batch, len(nh), stride, ctypes.byref(ws_bytes))
        ws = torch.empty(ws_bytes.value, dtype=torch.uint8, device=self.device)
        f = torch.empty((batch, len(nh), 2), dtype=torch.float64, device=self.device)
        g = torch.empty((batch, len(nh), max(1, len(param_names))), dtype=torch.float64, device=self.device)
        N.call('mqb_expectation_with_grad', prog.handle, ham_arr, len(nh), _ptr(init), init_batched, batch,
               _ptr(params), params.shape[1] if params.dim() == 2 else 0, _ptr(custom), _ptr(f), _ptr(g), stride,
               _ptr(ws), ws_bytes.value, _stream())
        # the workspace keeps this call's FP64 norm checks until the next call (norm_checks())
        self._last_grad = (prog, ws, ws_bytes.value, batch, len(nh), stride)
        return f, g[:, :, :len(param_names)]

    def norm_checks(self):
        """<psi|psi> in FP64 at the norm checks of the last complex64 gradient call: [checks][batch].

        The checks follow every ceil(sqrt(P))-th of the P forward passes and the last one, then every
        ceil(sqrt(P))-th state the backward sweep rebuilds by applying passes in reverse (checkpoint
        stride 0 or > 1).  Empty for complex128.  Synchronizes the stream."""
        if getattr(self, '_last_grad', None) is None:
            return np.zeros((0, 0))
        prog, ws, ws_bytes, batch, n_hams, stride = self._last_grad
        n = ctypes.c_int()
        N.call('mqb_grad_norm_checks', prog.handle, _ptr(ws), ws_bytes, batch, n_hams, stride, None, 0,
               ctypes.byref(n), _stream())
        out = np.zeros((max(1, n.value), batch), dtype=np.float64)
        if n.value:
            N.call('mqb_grad_norm_checks', prog.handle, _ptr(ws), ws_bytes, batch, n_hams, stride,
                   out.ctypes.data_as(ctypes.c_void_p), n.value, ctypes.byref(n), _stream())
        return out[:n.value]

    def norm_drift(self):
        """max |<psi|psi> - 1| over the norm checks of the last gradient call (0.0 without checks)."""
        c = self.norm_checks()
        return float(np.max(np.abs(c - 1.0))) if c.size else 0.0

    def _choose_stride(self, prog, batch, n_hams):
        """Store the state after every pass when it fits in 85% of free memory, else every sqrt(P) passes.

        Free memory counts what torch's caching allocator holds unused (the previous call's
        workspace), which the driver reports as taken."""
        free, _ = torch.cuda.mem_get_info(self.device)
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        for stride in (1, max(2, int(math.ceil(math.sqrt(max(1, prog.grad_passes(n_hams)[0]))))), 0):
            ws = ctypes.c_size_t()
            N.call('mqb_grad_workspace_size', prog.handle, batch, n_hams, stride, ctypes.byref(ws))
            if ws.value <= 0.85 * free:
                return stride
        return 0

    def get_expectation_with_grad(self, hams, circ_right, circ_left=None, simulator_left=None, parallel_worker=None,
                                  pr_shift=False):
        """Build the grad operator of ``hams`` on ``circ_right`` (mqsim.py:255-439)."""
        if isinstance(hams, Hamiltonian):
            hams = [hams]
        elif not isinstance(hams, list):
            raise TypeError(f"hams requires a Hamiltonian or a list of Hamiltonian, but get {type(hams)}")
        for h in hams:
            if not isinstance(h, Hamiltonian):
                raise TypeError(f"hams's element requires a Hamiltonian, but get {type(h)}")
            self._check_ham(h)
        if not isinstance(circ_right, Circuit):
            raise TypeError(f"circ_right requires a Circuit, but get {type(circ_right)}")
        if circ_right.is_noise_circuit:
            if circ_left is not None or simulator_left is not None:
                raise ValueError("noise circuit use parameter shift rule to get grad, which not support circ_left "
                                 "and simulator_left.")
            pr_shift = True    # mqsim.py:281-287
        if circ_left is not None or simulator_left is not None:
            if circ_left is not None and circ_left.is_noise_circuit:
                raise ValueError("noise left circuit not support yet.")
            # the reference takes the non-Hermitian branch before looking at pr_shift (mqsim.py:384-401)
            return self._non_hermitian_grad_ops(hams, circ_right, circ_left, simulator_left, parallel_worker)
        if pr_shift:
            return self._parameter_shift_grad_ops(hams, circ_right, parallel_worker)
        if circ_right.has_measure_gate:
            raise ValueError("circuit for variational algorithm cannot have measure gate")
        if self.n_qubits < circ_right.n_qubits:
            raise ValueError(f"Simulator has {self.n_qubits} qubits, but circuit has {circ_right.n_qubits} qubits.")
        ans_names = circ_right.ansatz_params_name
        enc_names = circ_right.encoder_params_name
        if set(ans_names) & set(enc_names):
            raise RuntimeError("Parameter cannot be both encoder and ansatz parameter.")
        version = "both"
        if not ans_names:
            version = "encoder"
        if not enc_names:
            version = "ansatz"
        names = enc_names + ans_names
        sim = self

        def grad_ops(*inputs_):
            enc, ans = _split_inputs(version, enc_names, ans_names, inputs_)
            params = np.concatenate([enc, np.broadcast_to(ans, (enc.shape[0], ans.size))], axis=1)
            init = sim._state
            f, g = sim.expectation_with_grad_tensor(hams, circ_right, torch.as_tensor(params), names, init_state=init)
            f = f.cpu().numpy()
            g = g.cpu().numpy()
            if sim.precision == N.MQB_PREC_C64 and sim._last_grad[5] != 1:
                # states rebuilt by reverse application: report a norm that moved
                drift = sim.norm_drift() if init is None else 0.0
                if drift > NORM_DRIFT_WARN:
                    warnings.warn(f"complex64 gradient: the state's norm drifted by {drift:.2e} while the backward "
                                  f"sweep rebuilt it (checkpoint stride {sim._last_grad[5]}); use complex128 or "
                                  f"more memory for stored states", RuntimeWarning, stacklevel=2)
            fc = f[..., 0] + 1j * f[..., 1]
            gc = g.astype(np.complex128)
            if version == 'both':
                return fc, gc[:, :, :len(enc_names)], gc[:, :, len(enc_names):]
            return fc, gc

        wrapper = GradOpsWrapper(grad_ops, hams, circ_right, circ_left, enc_names, ans_names, parallel_worker, self)
        wrapper.set_str(f"{self.n_qubits} qubit{'' if self.n_qubits == 1 else 's'} {self.name} VQA Operator")
        # the same evaluation on device tensors, for the autograd operators (framework/operations.py)
        wrapper.device_grad = lambda params: sim.expectation_with_grad_tensor(
            hams, circ_right, params, names, init_state=sim._state)  # pylint: disable=protected-access
        return wrapper

    # ------------------------------------------------------------------ non-Hermitian gradient
    def _batched_states(self, circuit, names, init, params):
        """[batch][2^n]: ``circuit`` applied to ``init`` for every parameter row."""
        B = params.shape[0]
        st = init.reshape(1, -1).repeat(B, 1)   # always a copy: the circuit is applied in place
        prog = lowered(circuit, self.n_qubits, self.precision, names, None, self.fuse, jit=self.jit)
        if prog.n_gates == 0:
            return st
        custom = self._custom_tensor(prog, params.cpu().numpy()) if prog.customs else None
        ws_bytes = ctypes.c_size_t()
        N.call('mqb_apply_workspace_size', prog.handle, B, ctypes.byref(ws_bytes))
        ws = torch.empty(max(256, ws_bytes.value), dtype=torch.uint8, device=self.device)
        N.call('mqb_apply', prog.handle, _ptr(st), B, _ptr(params), params.shape[1], _ptr(custom), _ptr(ws),
               ws_bytes.value, _stream())
        return st

    def _adjoint_with_lambda(self, circuit, names, init, lam, params):
        """[batch][len(names)] complex: sum over gates of <lam_g| dU_g |psi_{g-1}>, psi from ``init``."""
        B = params.shape[0]
        prog = lowered(circuit, self.n_qubits, self.precision, names, None, self.fuse, jit=self.jit)
        custom = self._custom_tensor(prog, params.cpu().numpy()) if prog.customs else None
        stride = self._choose_stride(prog, B, 1)
        ws_bytes = ctypes.c_size_t()
        N.call('mqb_grad_workspace_size', prog.handle, B, 1, stride, ctypes.byref(ws_bytes))
        ws = torch.empty(max(256, ws_bytes.value), dtype=torch.uint8, device=self.device)
        out = []
        for lam_k in (lam, lam * 1j):   # Re <lam|..> and Re <i lam|..> = Im <lam|..>
            lam_k = lam_k.contiguous()
            g = torch.zeros((B, max(1, len(names))), dtype=torch.float64, device=self.device)
            N.call('mqb_adjoint_with_lambda', prog.handle, _ptr(lam_k), 1, _ptr(init), 0, B, _ptr(params),
                   params.shape[1], _ptr(custom), _ptr(g), stride, _ptr(ws), ws_bytes.value, _stream())
            out.append(g[:, :len(names)])
        return torch.complex(out[0], out[1])

    def _non_hermitian_grad_ops(self, hams, circ_right, circ_left, simulator_left, parallel_worker):
        """f = <phi| U_l^dag H U_r |psi> and its gradient over both circuits' parameters
        (GradientHelper::NonHermitianAdjointGradient, ccsrc/include/simulator/vector/gradient.h:83-98,
        199-268; mindquantum/simulator/mqsim.py:282-392).

        The right circuit's gradient is sum <lambda_g| dU_g |psi_{g-1}> with lambda = H U_l phi carried
        back through U_r; the left circuit's is the conjugate of the same sweep over U_l with
        lambda = H U_r psi.  Each sweep runs with lambda and with i lambda (real and imaginary parts).
        """
        if simulator_left is not None:
            simulator_left = getattr(simulator_left, 'backend', simulator_left)
            if not isinstance(simulator_left, MQVectorB200):
                raise TypeError("simulator_left should be a mqvector_b200 simulator")
            if simulator_left.n_qubits != self.n_qubits:
                raise ValueError(f"simulator_left should have the same n_qubits as this simulator, which is "
                                 f"{self.n_qubits}, but get {simulator_left.n_qubits}")
            if simulator_left.dtype != self.dtype:
                raise TypeError(f"simulator_left should have the same data type as this simulator (aka "
                                f"{self.dtype}), but get {simulator_left.dtype}.")
        sim_left = self if simulator_left is None else simulator_left
        circ_left = circ_right if circ_left is None else circ_left
        if not isinstance(circ_left, Circuit):
            raise TypeError(f"circ_left requires a Circuit, but get {type(circ_left)}")
        if circ_left.has_measure_gate or circ_right.has_measure_gate:
            raise ValueError("circuit for variational algorithm cannot have measure gate")
        ans_names = list(circ_right.ansatz_params_name)
        enc_names = list(circ_right.encoder_params_name)
        ans_names += [k for k in circ_left.ansatz_params_name if k not in ans_names]
        enc_names += [k for k in circ_left.encoder_params_name if k not in enc_names]
        if set(ans_names) & set(enc_names):
            raise RuntimeError("Parameter cannot be both encoder and ansatz parameter.")
        n_circ = max(circ_left.n_qubits, circ_right.n_qubits)
        if self.n_qubits < n_circ:
            raise ValueError(f"Simulator has {self.n_qubits} qubits, but circuit has {n_circ} qubits.")
        version = "both" if (ans_names and enc_names) else ("encoder" if enc_names else "ansatz")
        names = enc_names + ans_names
        sim = self

        def grad_ops(*inputs_):
            enc, ans = _split_inputs(version, enc_names, ans_names, inputs_)
            params = torch.as_tensor(np.concatenate([enc, np.broadcast_to(ans, (enc.shape[0], ans.size))], axis=1),
                                     device=sim.device).contiguous()
            B = params.shape[0]
            psi0, phi0 = sim.state, sim_left.state
            psi_r = sim._batched_states(circ_right, names, psi0, params)
            psi_l = sim._batched_states(circ_left, names, phi0, params)
            res = np.zeros((B, len(hams), 1 + len(names)), dtype=np.complex128)
            for h_i, ham in enumerate(hams):
                nh = native_ham(ham, sim.n_qubits, sim.precision)
                nh_herm = native_ham(ham, sim.n_qubits, sim.precision, hermitian=True)
                out = torch.zeros((B, 2), dtype=torch.float64, device=sim.device)
                N.call('mqb_expectation', nh.handle, _ptr(psi_l), _ptr(psi_r), B, _ptr(out), _stream())
                h_l = torch.empty_like(psi_l)   # H^dag psi_l (RightSizeGrad's herm_hams, gradient.h:199-217)
                N.call('mqb_apply_hamiltonian', nh_herm.handle, _ptr(psi_l), _ptr(h_l), B, _stream())
                h_r = torch.empty_like(psi_r)
                N.call('mqb_apply_hamiltonian', nh.handle, _ptr(psi_r), _ptr(h_r), B, _stream())
                g = sim._adjoint_with_lambda(circ_right, names, psi0, h_l, params)
                g = g + sim._adjoint_with_lambda(circ_left, names, phi0, h_r, params).conj()
                o = out.cpu().numpy()
                res[:, h_i, 0] = o[:, 0] + 1j * o[:, 1]
                res[:, h_i, 1:] = g.cpu().numpy()
            if version == 'both':
                return res[:, :, 0], res[:, :, 1:1 + len(enc_names)], res[:, :, 1 + len(enc_names):]
            return res[:, :, 0], res[:, :, 1:]

        wrapper = GradOpsWrapper(grad_ops, hams, circ_right, circ_left, enc_names, ans_names, parallel_worker, self)
        wrapper.set_str(f"{self.n_qubits} qubit{'' if self.n_qubits == 1 else 's'} {self.name} VQA Operator")
        return wrapper

    # ------------------------------------------------------------------ parameter shift
    def _row_expectations(self, circuit, names, init, rows, hams):
        """<psi_r|H_h|psi_r> for psi_r = circuit(rows[r]) applied to ``init``: ``[n_rows][n_hams]`` complex.

        Rows run through the batched forward kernels in chunks that take at most 40 % of the free
        device memory."""
        n_rows = rows.shape[0]
        if rows.shape[1] == 0:
            rows = np.zeros((n_rows, 1))
        S = (1 << self.n_qubits) * (8 if self.precision == N.MQB_PREC_C64 else 16)
        free, _ = torch.cuda.mem_get_info(self.device)
        chunk = int(max(1, min(n_rows, 2048, (0.4 * free) // S)))
        nhs = [native_ham(h, self.n_qubits, self.precision) for h in hams]
        out = torch.empty((len(hams), n_rows, 2), dtype=torch.float64, device=self.device)
        for a in range(0, n_rows, chunk):
            p = torch.as_tensor(rows[a:a + chunk], dtype=torch.float64, device=self.device).contiguous()
            st = self._batched_states(circuit, names, init, p)
            for h, nh in enumerate(nhs):
                N.call('mqb_expectation', nh.handle, _ptr(st), _ptr(st), p.shape[0], _ptr(out[h, a:a + p.shape[0]]),
                       _stream())
            del st
        o = out.cpu().numpy()
        return (o[..., 0] + 1j * o[..., 1]).T

    def _trajectory_chunk(self, count):
        """Trajectories run at once: at most 40 % of the free device memory, at most 4096."""
        S = (1 << self.n_qubits) * (8 if self.precision == N.MQB_PREC_C64 else 16)
        free, _ = torch.cuda.mem_get_info(self.device)
        return int(max(1, min(count, 4096, (0.4 * free) // S)))

    def _noisy_shift(self, plan, P, hams, n_thread):
        """Parameter shift over stochastic channels, one trajectory per evaluation, in the
        reference's order of random draws (vector_state.tpp:1033-1230): every evaluation runs on a
        copy of the state re-seeded with int(draw * 10000) from this simulator's stream, every
        Hamiltonian copy consumes one more draw, Hamiltonians go in groups of ``n_thread`` and the
        Hamiltonian loop sits inside the gate loop.

        The draws of this simulator's stream are taken first, in that order, which fixes every
        trajectory's seed; the trajectories then run as batches (those measured with the same
        Hamiltonian together) and f and g are summed in the reference's order."""
        rows = plan.rows(P)
        R, E = plan.rows_per_sample, plan.n_shifts
        nhs = [native_ham(h, self.n_qubits, self.precision) for h in hams]
        n_prs, n_h = P.shape[0], len(hams)
        by_gate = {}
        for e, gi in enumerate(plan.gate_of):
            by_gate.setdefault(gi, []).append(e)
        job_row, job_seed, job_ham = [], [], []

        def job(row, ham):
            job_row.append(row)
            job_seed.append(int(self._rng.draw() * 10000))
            job_ham.append(ham)
            return len(job_row) - 1

        terms = []   # (s, j, base job) and (s, j, e, minus job, plus job), the reference's order
        for s in range(n_prs):
            base = job(s * R, -1)
            for start in range(0, n_h, n_thread):
                group = range(start, min(start + n_thread, n_h))
                self._rng.draw()
                for j in group:
                    self._rng.draw()
                    terms.append((s, j, base))
                for gi in sorted(by_gate):
                    for j in group:
                        for e in by_gate[gi]:
                            km = job(s * R + 1 + e, j)
                            self._rng.draw()
                            kp = job(s * R + 1 + E + e, j)
                            self._rng.draw()
                            terms.append((s, j, e, km, kp))
        values = {}
        for ham in range(-1, n_h):
            ids = [k for k, h in enumerate(job_ham) if h == ham]
            chunk = self._trajectory_chunk(max(1, len(ids)))
            for a in range(0, len(ids), chunk):
                part = ids[a:a + chunk]
                states = self.state.reshape(1, -1).repeat(len(part), 1)
                self._run_batch(states, plan.circuit, (list(plan.slot_names), rows[[job_row[k] for k in part]]),
                                UniformBlocks([job_seed[k] for k in part]))
                targets = range(n_h) if ham < 0 else (ham,)
                res = torch.zeros((len(targets), len(part), 2), dtype=torch.float64, device=self.device)
                for t, j in enumerate(targets):
                    N.call('mqb_expectation', nhs[j].handle, _ptr(states), _ptr(states), len(part), _ptr(res[t]),
                           _stream())
                res = res.cpu().numpy()
                for t, j in enumerate(targets):
                    for i, k in enumerate(part):
                        values[k, j] = complex(res[t, i, 0], res[t, i, 1])
                del states
        f = np.zeros((n_prs, n_h), dtype=np.complex128)
        g = np.zeros((n_prs, n_h, plan.J.shape[1]), dtype=np.complex128)
        for t in terms:
            if len(t) == 3:
                s, j, base = t
                f[s, j] = values[base, j]
            else:
                s, j, e, km, kp = t
                g[s, j] += plan.coeff[e] * (values[kp, j] - values[km, j]).real * plan.J[e]
        return f, g

    def _parameter_shift_grad_ops(self, hams, circ, parallel_worker):
        """Gradients by the parameter-shift rule (mqsim.py:401-411;
        ``GetExpectationWithGradParameterShiftMultiMulti``, vector_state.tpp:1033-1305), every
        shifted circuit of every sample evaluated as one batch (``parameter_shift.ShiftPlan``)."""
        if circ.has_measure_gate:
            raise ValueError("circuit for variational algorithm cannot have measure gate")
        if self.n_qubits < circ.n_qubits:
            raise ValueError(f"Simulator has {self.n_qubits} qubits, but circuit has {circ.n_qubits} qubits.")
        ans_names = list(circ.ansatz_params_name)
        enc_names = list(circ.encoder_params_name)
        if set(ans_names) & set(enc_names):
            raise RuntimeError("Parameter cannot be both encoder and ansatz parameter.")
        version = "both" if (ans_names and enc_names) else ("encoder" if enc_names else "ansatz")
        plan = ShiftPlan(circ, enc_names + ans_names)
        sim = self

        noisy = circ.is_noise_circuit

        def grad_ops(*inputs_):
            enc, ans = _split_inputs(version, enc_names, ans_names, inputs_)
            P = np.concatenate([enc, np.broadcast_to(ans, (enc.shape[0], ans.size))], axis=1)
            n_thread = max(1, min(_thread_balance(P.shape[0], len(hams), parallel_worker)[1], 15, len(hams)))
            if noisy:
                f, g = sim._noisy_shift(plan, P, hams, n_thread)
            else:
                F = sim._row_expectations(plan.circuit, plan.slot_names, sim.state, plan.rows(P), hams)
                f, g = plan.combine(F)
                # the reference seeds every evaluation from the simulator's stream: advance it alike
                n_groups = -(-len(hams) // n_thread)
                sim._rng.draw(P.shape[0] * (1 + n_groups + len(hams) * (1 + 4 * plan.n_shifts)))
            if version == 'both':
                return f, g[:, :, :len(enc_names)], g[:, :, len(enc_names):]
            return f, g

        wrapper = GradOpsWrapper(grad_ops, hams, circ, None, enc_names, ans_names, parallel_worker, self)
        wrapper.set_str(f"{self.n_qubits} qubit{'' if self.n_qubits == 1 else 's'} {self.name} VQA Operator")
        return wrapper

    # ------------------------------------------------------------------ sampling
    def sampling(self, circuit, pr=None, shots=1, seed=None):
        """Sample measurement outcomes (mqsim.py:456-491; vector_state.tpp:1308-1373)."""
        if not isinstance(circuit, Circuit):
            raise TypeError(f"circuit requires a Circuit, but get {type(circuit)}")
        if not circuit.has_measure_gate:
            raise ValueError("circuit must have at least one measurement gate.")
        if self.n_qubits < circuit.n_qubits:
            raise ValueError(f"Circuit has {circuit.n_qubits} qubits, which is more than simulator qubits.")
        if not isinstance(shots, (int, np.integer)) or shots < 1:
            raise ValueError(f"sampling shots should be a positive integer, but get {shots}")
        pr = self._check_pr(circuit, pr)
        if seed is None:
            seed = int(np.random.randint(1, 2 << 20))
        res = MeasureResult()
        res.add_measure(circuit.all_measures.keys())
        key_map = res.keys_map
        rng = Mt19937Uniform(seed)
        samples = np.zeros((shots, len(key_map)), dtype=np.int64)
        if circuit.is_measure_end and not circuit.is_noise_circuit:
            sub = int(rng.draw(low=1.0, high=float(1 << 20)))
            sim_rng = Mt19937Uniform(sub)
            m_gates = [g for g in circuit if isinstance(g, G.Measure)]
            other = Circuit([g for g in circuit if not isinstance(g, (G.Measure, G.BarrierGate))])
            st = self.state.clone()
            if len(other):
                self._apply_segment(st, other, pr)
            u = sim_rng.draw(shots)
            if self.arithmetic_type == complex64:
                u = u.astype(np.float32).astype(np.float64)
            u.sort()
            u_t = torch.as_tensor(u, device=self.device)
            idx = torch.empty(shots, dtype=torch.int64, device=self.device)
            scratch_bytes = ctypes.c_size_t()
            N.call('mqb_sample_scratch_size', self.n_qubits, ctypes.byref(scratch_bytes))
            scratch = torch.empty(scratch_bytes.value, dtype=torch.uint8, device=self.device)
            N.call('mqb_sample_indices', self.n_qubits, self.precision, _ptr(st), _ptr(u_t), shots, _ptr(idx),
                   _ptr(scratch), scratch_bytes.value, _stream())
            r = idx.cpu().numpy()
            for g in m_gates:
                samples[:, key_map[g.key]] = (r >> g.obj_qubits[0]) & 1
        else:
            # every shot is a trajectory on its own stream, seeded from ``rng`` in shot order; the
            # shots run as batches of trajectories
            seeds = [int(rng.draw(low=1.0, high=float(1 << 20))) for _ in range(shots)]
            chunk = self._trajectory_chunk(shots)
            for a in range(0, shots, chunk):
                part = seeds[a:a + chunk]
                states = self.state.reshape(1, -1).repeat(len(part), 1)
                outs = self._run_batch(states, circuit, pr, UniformBlocks(part))
                for k, v in outs.items():
                    samples[a:a + len(part), key_map[k]] = v
                del states
        res.collect_data(samples)
        return res
