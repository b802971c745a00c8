"""The density-matrix backend ``mqmatrix_b200``: MindQuantum's ``mqmatrix`` on the B200 kernels.

The reference keeps rho as a 2^n x 2^n matrix with its own kernels (DensityMatrixState,
ccsrc/include/simulator/densitymatrix/densitymatrix_state.tpp).  Here rho is vectorized,
vec(rho)[i 2^n + j] = rho_ij, and lives as the state of a 2n-qubit register of the state-vector
engine: column index j on qubits 0..n-1, row index i on qubits n..2n-1.  Then

* a gate U on qubits Q acts as U on the row qubits Q + n and conj(U) on the column qubits Q
  (rho -> U rho U^dag), so a circuit becomes a doubled circuit of the same parameters and runs on
  the fused pass kernels unchanged;
* a channel becomes its superoperator, sum_k K_k (x) conj(K_k) on (q + n, q), or the reference's
  direct map for depolarizing and thermal relaxation (cpu_densitymatrix_core_channel.cpp); these
  are non-unitary constant matrices that run in passes of their own;
* Tr(H rho) = <vec(H)|vec(rho)>, with vec(H) = (H (x) I) vec(I) made by the Hamiltonian kernels;
* the gradient of Tr(H E(rho_0)) is linear in vec(rho): it is the adjoint sweep with the given
  lambda = vec(H) (mqb_adjoint_with_lambda, Re sum <lambda|dS|rho>), where the row and column
  copies of a gate share its parameters; that sum equals the reference's 2 Re Tr(H dU rho U^dag)
  (GetExpectationWithReversibleGrad / GetExpectationWithNoiseGrad, densitymatrix_state.tpp:791-983).
  With channels the sweep stores every pass's state, so no non-unitary op is ever undone.
"""
from __future__ import annotations

import copy
import ctypes
import itertools

import numpy as np
import torch

from .. import _native as N
from ..core import gates as G
from ..core.circuit import Circuit
from ..core.operators import Hamiltonian, HowTo, QubitOperator
from ..dtype import complex128
from .backend_base import BackendBase
from .lowering import lowered, native_ham
from .measure_result import MeasureResult
from .mqvector_b200 import MQVectorB200, _ptr, _split_inputs, _stream
from .rng import Mt19937Uniform
from .utils import GradOpsWrapper, check_kept_qubits, qs_of_qubits

_CHANNEL_NAMES = ('PC', 'BFC', 'PFC', 'BPFC', 'GPC', 'DC', 'ADC', 'PDC', 'TRC')
# conj(exp(-i t/2 G)) = exp(-i (-t)/2 G) when the generator G is real, itself when G is imaginary
_NEGATE = {'RX', 'RZ', 'PS', 'GP', 'Rxx', 'Ryy', 'Rzz', 'Rxz', 'SWAPalpha'}
_SAME = {'RY', 'Rxy', 'Ryz', 'G'}


class SuperOperator(G.UnivMathGate):
    """A channel's superoperator on (column qubits, row qubits) of a vectorized density matrix."""

    nonunitary = True

    def __init__(self, name, matrix_value):
        super().__init__(name, matrix_value)


def is_channel(g):
    return isinstance(g, G.NoiseGate) or g.name in _CHANNEL_NAMES


def conj_gate(g):
    """A gate whose matrix is the complex conjugate of ``g``'s, on the same qubits (parameters
    kept symbolic, so the row and column copies share them)."""
    if isinstance(g, G.ParameterGate):
        new = copy.deepcopy(g)
        name = g.name
        if isinstance(g, G.ParamNonHerm):
            mg, dg = g.matrix_generator, g.diff_matrix_generator
            new.matrix_generator = lambda x, _m=mg: np.conj(np.asarray(_m(x), dtype=complex))
            new.diff_matrix_generator = lambda x, _d=dg: np.conj(np.asarray(_d(x), dtype=complex))
        elif name in _NEGATE:
            new.prs = [-p for p in g.prs]
        elif name in _SAME:
            pass
        elif name == 'U3':
            new.prs = [g.prs[0], -g.prs[1], -g.prs[2]]
        elif name == 'Rn':
            new.prs = [-g.prs[0], g.prs[1], -g.prs[2]]
        elif name == 'FSim':
            new.prs = [-g.prs[0], -g.prs[1]]
        elif isinstance(g, G.RotPauliString):
            if g.pauli_string.count('Y') % 2 == 0:
                new.prs = [-p for p in g.prs]
        else:
            raise NotImplementedError(f"density matrix: no conjugation rule for {name}")
        return new
    m = np.conj(np.asarray(g.matrix(), dtype=np.complex128))
    return G.UnivMathGate(g.name + '*', m).on(list(g.obj_qubits), list(g.ctrl_qubits) or None)


def _kraus_superop(kraus):
    return sum(np.kron(k, np.conj(k)) for k in kraus)


def _kraus_1q(g):
    """Kraus operators of a single-qubit channel, as the reference's density-matrix policy applies
    them (cpu_densitymatrix_core_channel.cpp: ApplyPauli, ApplyAmplitudeDamping incl. its daggered
    form, ApplyPhaseDamping, ApplyKraus)."""
    if g.name in ('PC', 'BFC', 'PFC', 'BPFC'):
        out = []
        for p, m in ((g.px, [[0, 1], [1, 0]]), (g.py, [[0, -1j], [1j, 0]]), (g.pz, [[1, 0], [0, -1]]),
                     (1 - g.px - g.py - g.pz, [[1, 0], [0, 1]])):
            if p > 1e-8:
                out.append(np.sqrt(p) * np.array(m, dtype=np.complex128))
        return out
    if g.name == 'ADC':
        k0 = np.array([[1, 0], [0, np.sqrt(1 - g.gamma)]], dtype=np.complex128)
        if g.hermitianed:
            return [k0, np.array([[0, 0], [np.sqrt(g.gamma), 0]], dtype=np.complex128)]
        return [k0, np.array([[0, np.sqrt(g.gamma)], [0, 0]], dtype=np.complex128)]
    if g.name == 'PDC':
        return [np.array([[1, 0], [0, np.sqrt(1 - g.gamma)]], dtype=np.complex128),
                np.array([[0, 0], [0, np.sqrt(g.gamma)]], dtype=np.complex128)]
    if hasattr(g, 'kraus_op'):
        return [np.asarray(k, dtype=np.complex128) for k in g.kraus_op]
    raise NotImplementedError(f"density matrix: channel {g.name}")


_PAULIS = [np.eye(2, dtype=np.complex128), np.array([[0, 1], [1, 0]], dtype=np.complex128),
           np.array([[0, -1j], [1j, 0]], dtype=np.complex128), np.array([[1, 0], [0, -1]], dtype=np.complex128)]


def _superops(g, n):
    objs = list(g.obj_qubits)
    if g.ctrl_qubits:
        raise NotImplementedError("density matrix: controlled channels")
    if g.name == 'GPC':
        out = []
        for q, row in zip(objs, g.probs):
            px, py, pz = (float(v) for v in row)
            ks = [np.sqrt(p) * m for p, m in ((px, _PAULIS[1]), (py, _PAULIS[2]), (pz, _PAULIS[3]),
                                              (1 - px - py - pz, _PAULIS[0])) if p > 1e-8]
            out.append((_kraus_superop(ks), [q, q + n]))
        return out
    if g.name == 'DC':
        # (1 - p) rho + p (I / 2^k (x) Tr_objs rho) = (1 - p) rho + p / 4^k sum_P P rho P
        k = len(objs)
        kraus = []
        for combo in itertools.product(range(4), repeat=k):
            P = np.array([[1.0 + 0j]])
            for c in reversed(combo):   # matrix index bit b <-> objs[b]
                P = np.kron(P, _PAULIS[c])
            w = (1 - g.p + g.p / 4 ** k) if not any(combo) else g.p / 4 ** k
            if w > 0:
                kraus.append(np.sqrt(w) * P)
        return [(_kraus_superop(kraus), objs + [q + n for q in objs])]
    if g.name == 'TRC':
        # ApplyThermalRelaxation: rho_00 += (1 - e1) rho_11, coherences x e2, rho_11 x e1
        e1 = np.exp(-g.gate_time / g.t1)
        e2 = np.exp(-g.gate_time / g.t2)
        S = np.diag([1.0, e2, e2, e1]).astype(np.complex128)
        S[0, 3] = 1 - e1
        return [(S, [objs[0], objs[0] + n])]
    return [(_kraus_superop(_kraus_1q(g)), [objs[0], objs[0] + n])]


def doubled_circuit(circ, n):
    """The circuit acting on vec(rho) (2n qubits), with the same parameters."""
    out = []
    for g in circ:
        if isinstance(g, G.BarrierGate) or g.name == 'I':
            continue
        if isinstance(g, G.Measure):
            raise ValueError("density matrix: measurement gates must be split off")
        if is_channel(g):
            for S, objs in _superops(g, n):
                out.append(SuperOperator(g.name + '_superop', S).on(objs))
            continue
        objs, ctrls = list(g.obj_qubits), list(g.ctrl_qubits)
        row = copy.deepcopy(g)
        row.obj_qubits = [q + n for q in objs]
        row.ctrl_qubits = [q + n for q in ctrls]
        out.append(row)
        out.append(conj_gate(g))
    c = Circuit(out)
    return c


def _shifted_operator(ham, n, conj=False):
    """The Hamiltonian's Pauli sum on the row qubits (q + n), or its complex conjugate on the column
    qubits (a Pauli string with an odd number of Y changes sign)."""
    op = QubitOperator()
    for term, coeff in ham.ham_termlist:
        if conj:
            sign = -1.0 if sum(1 for _, p in term if p == 'Y') % 2 else 1.0
            s = ' '.join(f"{p}{q}" for q, p in term)
            op += QubitOperator(s, sign * coeff) if s else QubitOperator('', sign * coeff)
        else:
            s = ' '.join(f"{p}{q + n}" for q, p in term)
            op += QubitOperator(s, coeff) if s else QubitOperator('', coeff)
    return op


class MQMatrixB200(BackendBase):
    """Density-matrix simulator (the reference's ``mqmatrix`` surface: mqsim.py, with the density
    matrix specifics at mqsim.py:245, :389-399, :497-600)."""

    def __init__(self, name, n_qubits, seed=None, dtype=None, fuse=True, device=None, jit=None):
        super().__init__(name, n_qubits, seed, dtype if dtype is not None else complex128)
        if seed is None:
            seed = int(np.random.randint(1, 2**23))
        self.seed = seed
        self.engine = MQVectorB200(name, 2 * n_qubits, seed, self.arithmetic_type, fuse, device, jit)
        self._ham_vec = {}
        self._rng = Mt19937Uniform(seed)   # the measurement stream of apply_circuit

    # ------------------------------------------------------------------ state
    @property
    def device(self):
        return self.engine.device

    @property
    def precision(self):
        return self.engine.precision

    def _rho_tensor(self):
        return self.engine.state

    def reset(self):
        self.engine.reset()

    def copy(self):
        sim = MQMatrixB200(self.name, self.n_qubits, self.seed, self.arithmetic_type, self.engine.fuse,
                           self.engine.device, self.engine.jit)
        sim.engine.set_state_tensor(self.engine.state.clone())
        return sim

    def astype(self, dtype, seed=None):
        sim = MQMatrixB200(self.name, self.n_qubits, self.seed if seed is None else seed, dtype, self.engine.fuse,
                           self.engine.device, self.engine.jit)
        sim.engine.set_state_tensor(self.engine.state.clone())
        return sim

    def get_qs(self, ket=False):
        if ket:
            raise ValueError("density matrix simulator cannot return a ket string.")
        d = 1 << self.n_qubits
        return self.engine.state.detach().to(torch.complex128).cpu().numpy().reshape(d, d)

    def set_qs(self, quantum_state):
        """A vector (normalised, rho = v v^dag) or a density matrix (checked, trace-normalised)
        (mqsim.py:497-544, _set_matrix_state)."""
        state = np.asarray(quantum_state)
        n = np.log2(state.shape[0])
        if n % 1 != 0:
            raise ValueError(f"vec size {state.shape[0]} is not power of 2")
        if int(n) != self.n_qubits:
            raise ValueError(f"{int(n)} qubits vec does not match with simulation qubits ({self.n_qubits})")
        if state.ndim == 1:
            norm = np.sqrt(np.sum(np.abs(state) ** 2))
            if norm == 0.0:
                raise ValueError("Wrong quantum state.")
            v = state / norm
            rho = np.outer(v, np.conj(v))
        elif state.ndim == 2:
            if not np.allclose(state, state.T.conj(), atol=1e-6):
                raise ValueError("density matrix must be hermitian.")
            if (np.real(state.diagonal()) < 0).any():
                raise ValueError("the diagonal terms in density matrix cannot be negative.")
            tr = np.real(np.trace(state))
            if tr == 0.0:
                raise ValueError("Wrong quantum state.")
            rho = state / tr
        else:
            raise ValueError("State must be 1D vector or 2D density matrix")
        self.engine.set_state_tensor(torch.as_tensor(np.ascontiguousarray(rho).reshape(-1),
                                                     dtype=self.engine.torch_dtype))

    # ------------------------------------------------------------------ evolution
    def apply_circuit(self, circuit, pr=None):
        if not isinstance(circuit, Circuit):
            raise TypeError(f"circuit requires a Circuit, but get {type(circuit)}")
        if self.n_qubits < circuit.n_qubits:
            raise ValueError(f"Circuit has {circuit.n_qubits} qubits, which is more than simulator qubits.")
        res = MeasureResult()
        res.add_measure(circuit.all_measures.keys())
        rng = self._rng
        key_map = res.keys_map
        samples = {}
        segment = []
        pr = self.engine._check_pr(circuit, pr)   # pylint: disable=protected-access
        for g in list(circuit) + [None]:
            if g is None or isinstance(g, G.Measure):
                if segment:
                    dc = doubled_circuit(Circuit(segment), self.n_qubits)
                    if len(dc):
                        self.engine._apply_segment(self.engine.state, dc, pr)   # pylint: disable=protected-access
                    segment = []
                if g is not None:
                    samples[g.key] = self._measure(g, rng)
            else:
                segment.append(g)
        if not samples:
            return None
        out = np.zeros((1, len(key_map)), dtype=np.int64)
        for k, v in samples.items():
            out[0, key_map[k]] = v
        res.collect_data(out)
        return res

    def apply_gate(self, gate, pr=None, diff=False):
        if diff:
            raise NotImplementedError("density matrix: apply_gate with diff")
        return self.apply_circuit(Circuit([gate]), pr)

    def _diag(self):
        d = 1 << self.n_qubits
        return torch.diagonal(self.engine.state.view(d, d)).real.to(torch.float64)

    def _measure(self, g, rng):
        """DensityMatrixState::ApplyMeasure (densitymatrix_state.tpp:523-535): draw, collapse, reset."""
        q = g.obj_qubits[0]
        d = 1 << self.n_qubits
        idx = torch.arange(d, device=self.device)
        diag = self._diag()
        one = float(diag[(idx >> q) & 1 == 1].sum().item())
        bit = 1 if rng.draw() < one else 0
        rho = self.engine.state.view(d, d)
        keep = ((idx >> q) & 1) == bit
        mask = (keep[:, None] & keep[None, :]).to(rho.dtype)
        rho = rho * mask / (one if bit else 1 - one)
        self.engine.set_state_tensor(rho.reshape(-1).contiguous())
        if g.reset_to is not None and bit != g.reset_to:
            self.apply_circuit(Circuit([G.X.on(q)]))
        return bit

    def apply_hamiltonian(self, hamiltonian):
        """rho -> H rho H (DensityMatrixState::ApplyHamiltonian with the policy's ApplyTerms): H on the
        row qubits, conj(H) on the column qubits."""
        if not isinstance(hamiltonian, Hamiltonian) or hamiltonian.how_to == HowTo.FRONTEND:
            raise NotImplementedError("density matrix: apply_hamiltonian takes a Pauli Hamiltonian")
        n2 = 2 * self.n_qubits
        for conj in (False, True):
            h = native_ham(Hamiltonian(_shifted_operator(hamiltonian, self.n_qubits, conj)), n2, self.precision)
            out = torch.empty_like(self.engine.state)
            N.call('mqb_apply_hamiltonian', h.handle, _ptr(self.engine.state), _ptr(out), 1, _stream())
            self.engine.set_state_tensor(out)

    # ------------------------------------------------------------------ expectations
    def _vec_h(self, ham):
        """vec(H) = (H (x) I) vec(I) on the doubled register (cached per Hamiltonian object)."""
        key = id(ham)
        hit = self._ham_vec.get(key)
        if hit is not None and hit[0] is ham:
            return hit[1]
        n, d = self.n_qubits, 1 << self.n_qubits
        if ham.how_to == HowTo.FRONTEND:
            m = ham.sparse_matrix.toarray()
            vec = torch.as_tensor(np.ascontiguousarray(m).reshape(-1), dtype=self.engine.torch_dtype,
                                  device=self.device)
        else:
            ident = torch.zeros(d * d, dtype=self.engine.torch_dtype, device=self.device)
            ident[torch.arange(d, device=self.device) * (d + 1)] = 1
            h = native_ham(Hamiltonian(_shifted_operator(ham, n)), 2 * n, self.precision)
            vec = torch.empty_like(ident)
            N.call('mqb_apply_hamiltonian', h.handle, _ptr(ident), _ptr(vec), 1, _stream())
        self._ham_vec[key] = (ham, vec)
        return vec

    def _expect(self, ham, states):
        """Tr(H rho_b) for states [batch][4^n]: FP64 <vec(H)|vec(rho_b)>."""
        vh = self._vec_h(ham)
        B = states.shape[0]
        out = torch.zeros((B, 2), dtype=torch.float64, device=self.device)
        lam = vh.reshape(1, -1).expand(B, -1).contiguous()
        N.call('mqb_vdot', 2 * self.n_qubits, self.precision, _ptr(lam), _ptr(states), B, _ptr(out), _stream())
        return out

    def get_expectation(self, hamiltonian, circ_right=None, circ_left=None, simulator_left=None, pr=None):
        if circ_left is not None or simulator_left is not None:
            raise NotImplementedError("Non hermitian case for get_expectation not implement for mqmatrix yet.")
        st = self.engine.state.clone()
        if circ_right is not None and len(circ_right):
            pr = self.engine._check_pr(circ_right, pr)   # pylint: disable=protected-access
            dc = doubled_circuit(circ_right, self.n_qubits)
            if len(dc):
                self.engine._apply_segment(st, dc, pr)   # pylint: disable=protected-access
        o = self._expect(hamiltonian, st.reshape(1, -1)).cpu().numpy()
        return complex(o[0, 0], o[0, 1])

    def expectation_with_grad_tensor(self, hams, circuit, params, param_names):
        """f [batch][n_hams] and grad [batch][n_hams][n_params] (float64 device tensors) of Tr(H E(rho))."""
        params = params.to(device=self.device, dtype=torch.float64).contiguous()
        B = params.shape[0]
        dc = doubled_circuit(circuit, self.n_qubits)
        names = list(param_names)
        prog = lowered(dc, 2 * self.n_qubits, self.precision, names, None, self.engine.fuse, jit=self.engine.jit)
        init = self.engine.state
        f = torch.zeros((B, len(hams)), dtype=torch.float64, device=self.device)
        g = torch.zeros((B, len(hams), max(1, len(names))), dtype=torch.float64, device=self.device)
        states = self.engine._batched_states(dc, names, init, params)   # pylint: disable=protected-access
        custom = self.engine._custom_tensor(prog, params.cpu().numpy()) if prog.customs else None  # pylint: disable=protected-access
        has_channel = any(getattr(x, 'nonunitary', False) for x in dc)
        stride = 1 if has_channel else self.engine._choose_stride(prog, B, 1)   # pylint: disable=protected-access
        ws_bytes = ctypes.c_size_t()
        N.call('mqb_grad_workspace_size', prog.handle, B, 1, stride, ctypes.byref(ws_bytes))
        ws = torch.empty(max(256, ws_bytes.value), dtype=torch.uint8, device=self.device)
        for h, ham in enumerate(hams):
            f[:, h] = self._expect(ham, states)[:, 0]
            lam = self._vec_h(ham)
            gh = torch.zeros((B, max(1, len(names))), dtype=torch.float64, device=self.device)
            N.call('mqb_adjoint_with_lambda', prog.handle, _ptr(lam), 0, _ptr(init), 0, B, _ptr(params),
                   params.shape[1], _ptr(custom), _ptr(gh), stride, _ptr(ws), ws_bytes.value, _stream())
            g[:, h] = gh
        return f, g[:, :, :len(names)]

    def get_expectation_with_grad(self, hams, circ_right, circ_left=None, simulator_left=None, parallel_worker=None,
                                  pr_shift=False):
        """The grad operator of ``hams`` on ``circ_right`` (mqsim.py:255-439, density-matrix branches)."""
        if isinstance(hams, Hamiltonian):
            hams = [hams]
        elif not isinstance(hams, list):
            raise TypeError(f"hams requires a Hamiltonian or a list of Hamiltonian, but get {type(hams)}")
        for h in hams:
            if not isinstance(h, Hamiltonian):
                raise TypeError(f"hams's element requires a Hamiltonian, but get {type(h)}")
        if not isinstance(circ_right, Circuit):
            raise TypeError(f"circ_right requires a Circuit, but get {type(circ_right)}")
        if circ_left is not None or simulator_left is not None:
            raise NotImplementedError("Non hermitian case for get_expectation not implement for mqmatrix yet.")
        if pr_shift:
            raise NotImplementedError("density matrix: parameter-shift gradients")
        if circ_right.has_measure_gate:
            raise ValueError("circuit for variational algorithm cannot have measure gate")
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
            f, g = sim.expectation_with_grad_tensor(hams, circ_right, torch.as_tensor(params), names)
            fc = f.cpu().numpy().astype(np.complex128)
            gc = g.cpu().numpy().astype(np.complex128)
            if version == 'both':
                return fc, gc[:, :, :len(enc_names)], gc[:, :, len(enc_names):]
            return fc, gc

        wrapper = GradOpsWrapper(grad_ops, hams, circ_right, circ_left, enc_names, ans_names, parallel_worker, self)
        wrapper.set_str(f"{self.n_qubits} qubit{'' if self.n_qubits == 1 else 's'} {self.name} VQA Operator")
        return wrapper

    # ------------------------------------------------------------------ other density-matrix methods
    def purity(self):
        """Tr(rho^2) = sum |rho_ij|^2 (rho Hermitian)."""
        v = self.engine.state.reshape(1, -1)
        out = torch.zeros((1, 2), dtype=torch.float64, device=self.device)
        N.call('mqb_vdot', 2 * self.n_qubits, self.precision, _ptr(v), _ptr(v), 1, _ptr(out), _stream())
        return float(out[0, 0].item())

    def get_partial_trace(self, obj_qubits):
        """Trace out ``obj_qubits`` (mqsim.py get_partial_trace)."""
        rho = self.get_qs()
        n = self.n_qubits
        t = rho.reshape([2] * (2 * n))
        # axis k of the reshaped row index is qubit n-1-k
        for q in sorted(obj_qubits, reverse=True):
            m = t.ndim // 2
            ax = m - 1 - q
            t = np.trace(t, axis1=ax, axis2=ax + m)
        d = 1 << (n - len(obj_qubits))
        return t.reshape(d, d)

    def get_reduced_density_matrix(self, kept_qubits):
        kept = check_kept_qubits(kept_qubits, self.n_qubits)
        drop = [q for q in range(self.n_qubits) if q not in kept]
        return self.get_partial_trace(drop)

    def get_qs_of_qubits(self, qubits, ket=False):
        """Reduced state of ``qubits`` (mqsim.py:598-626)."""
        return qs_of_qubits(self, qubits, ket)

    def get_circuit_matrix(self, circuit, pr):
        """Unitary of a channel-free ``circuit`` (mqsim.py:199-201), from the state-vector engine."""
        if circuit.is_noise_circuit:
            raise ValueError("a circuit with noise channels has no circuit matrix")
        return MQVectorB200('mqvector_b200', self.n_qubits, self.seed, self.arithmetic_type).get_circuit_matrix(
            circuit, pr)

    def entropy(self):
        ev = np.real(np.linalg.eigvals(self.get_qs()))
        return float(-sum(x * np.log(x) for x in ev if x > 0))

    def get_pure_state_vector(self):
        if 1 - self.purity() > 1e-6:
            raise ValueError("Cannot transform mixed density matrix to vector.")
        w, v = np.linalg.eigh(self.get_qs())
        vec = v[:, np.argmax(w)]
        k = int(np.argmax(np.abs(vec)))
        return vec * np.exp(-1j * np.angle(vec[k]))

    def sampling(self, circuit, pr=None, shots=1, seed=None):
        """DensityMatrixState::SamplingMeasurementEndingWithoutNoise / Sampling
        (densitymatrix_state.tpp:1115-1160): the measurements of every shot are drawn from a
        copy of the state with the shot's own seed."""
        if not isinstance(circuit, Circuit):
            raise TypeError(f"circuit requires a Circuit, but get {type(circuit)}")
        if not circuit.has_measure_gate:
            raise ValueError("circuit must have at least one measurement gate.")
        if not isinstance(shots, (int, np.integer)) or shots < 1:
            raise ValueError(f"sampling shots should be a positive integer, but get {shots}")
        if seed is None:
            seed = int(np.random.randint(1, 2 << 20))
        res = MeasureResult()
        res.add_measure(circuit.all_measures.keys())
        key_map = res.keys_map
        rng = Mt19937Uniform(seed)
        samples = np.zeros((shots, len(key_map)), dtype=np.int64)
        base = self.copy()
        if circuit.is_measure_end and not circuit.is_noise_circuit:
            base.seed = int(rng.draw(low=1.0, high=float(1 << 20)))
            other = Circuit([g for g in circuit if not isinstance(g, (G.Measure, G.BarrierGate))])
            if len(other):
                base.apply_circuit(other, pr)
            rng = Mt19937Uniform(int(rng.draw(low=1.0, high=float(1 << 20))))
            circuit = Circuit([g for g in circuit if isinstance(g, G.Measure)])
        for s in range(shots):
            sim = base.copy()
            sim._rng = Mt19937Uniform(int(rng.draw(low=1.0, high=float(1 << 20))))   # pylint: disable=protected-access
            out = sim.apply_circuit(circuit, pr)
            samples[s] = out.samples[0]
        res.collect_data(samples)
        return res
