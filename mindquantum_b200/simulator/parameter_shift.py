"""Parameter-shift gradients as one batched forward evaluation.

The reference (``GetExpectationWithGradParameterShiftOneMulti`` / ``MultiMulti``,
ccsrc/include/simulator/vector/vector_state.tpp:1033-1305) re-runs the whole circuit twice for
every non-constant angle of every gate that needs a gradient, one evaluation after the other.
Here every non-constant angle becomes a parameter of its own (a slot) in a copy of the circuit,
so a sample's angles are one slot vector V = C p + c, and every shifted evaluation is a row
V - D_e or V + D_e.  All rows of all samples run through the batched forward kernels and the
expectation kernel in chunks that fit the device; the host combines them:

    g[h][name] = sum_e coeff_e * Re(f_h(V + D_e) - f_h(V - D_e)) * J_e[name]

where J_e is the gate's Jacobi row of that angle (requires-grad parameters only,
parameter_resolver.cpp:560-573).
"""
from __future__ import annotations

import copy
import math

import numpy as np

from ..core import gates as G
from ..core.circuit import Circuit
from ..core.parameterresolver import ParameterResolver

_EXACT = (G.RX, G.RY, G.RZ, G.Rxx, G.Ryy, G.Rzz, G.Rxy, G.Rxz, G.Ryz, G.GlobalPhase, G.PhaseShift, G.U3)
_VALUE_SHIFTED = (G.U3, G.FSim)
_SUPPORTED = _EXACT + _VALUE_SHIFTED + (G.Givens, G.SWAPalpha, G.ParamNonHerm)


def shift_rule(gate):
    """(shift, coefficient, shifts-the-parameter-value) of a gate (vector_state.tpp:1076-1174).

    Rotation-like gates, PS, GP and U3: +-pi/2 with coefficient 1/2 (exact for generators with
    eigenvalue gap 1); SWAPalpha: +-1/2 with pi/2; Givens, FSim and custom gates, and every
    controlled gate: a central difference with step 1e-3.  U3 and FSim read their angles from
    members the reference's shift does not edit, so it moves the value of the angle's first
    parameter (in name order) instead, which shifts every gate that uses that parameter.
    """
    if not isinstance(gate, _SUPPORTED):
        raise RuntimeError(f"gate {gate.name} not supported for parameter shift rule.")
    if isinstance(gate, _EXACT):
        shift, coeff = math.pi / 2, 0.5
    elif isinstance(gate, G.SWAPalpha):
        shift, coeff = 0.5, math.pi / 2
    else:
        shift, coeff = 0.001, 0.5 / 0.001
    if gate.ctrl_qubits:
        shift, coeff = 0.001, 0.5 / 0.001
    return shift, coeff, isinstance(gate, _VALUE_SHIFTED)


class ShiftPlan:
    """The slot circuit and the shift rows of one circuit over the parameter names ``names``."""

    def __init__(self, circuit, names):
        names = list(names)
        index = {k: i for i, k in enumerate(names)}
        gates, C, c0 = [], [], []
        shifts = []   # (kind, position, amount, coeff, jacobi row, gate index)
        for gi, g in enumerate(circuit):
            if not isinstance(g, G.ParameterGate) or not g.parameterized:
                gates.append(g)    # constant gates, measurements and channels stay as they are
                continue
            new = copy.copy(g)
            new.prs = list(g.prs)
            slot_of = {}
            for k, p in enumerate(g.prs):
                if p.is_const():
                    continue
                row = np.zeros(len(names))
                for key, v in p.items():
                    row[index[key]] = float(np.real(v))
                slot_of[k] = len(C)
                C.append(row)
                c0.append(float(np.real(p.const)))
                new.prs[k] = ParameterResolver({f'_slot{slot_of[k]}': 1.0})
            gates.append(new)
            if not any(p.requires_grad_parameters for p in g.prs):
                continue
            shift, coeff, by_value = shift_rule(g)
            for k, j in slot_of.items():
                p = g.prs[k]
                jac = np.zeros(len(names))
                for name in p.requires_grad_parameters:
                    jac[index[name]] = float(np.real(p[name]))
                if by_value:
                    key = min(p.keys())
                    shifts.append(('value', index[key], shift / float(np.real(p[key])), coeff, jac, gi))
                else:
                    shifts.append(('slot', j, shift, coeff, jac, gi))
        self.names = names
        self.circuit = Circuit(gates)
        self.slot_names = [f'_slot{j}' for j in range(len(C))]
        self.C = np.array(C, dtype=np.float64).reshape(len(C), len(names))
        self.c0 = np.array(c0, dtype=np.float64)
        self.n_shifts = len(shifts)
        self.D = np.zeros((len(shifts), len(C)))
        self.gate_of = [sh[5] for sh in shifts]   # circuit position of every shifted angle
        for e, (kind, pos, amount, _, _, _) in enumerate(shifts):
            if kind == 'slot':
                self.D[e, pos] = amount
            else:
                self.D[e] = amount * self.C[:, pos]
        self.coeff = np.array([s[3] for s in shifts], dtype=np.float64)
        self.J = np.array([s[4] for s in shifts], dtype=np.float64).reshape(len(shifts), len(names))

    @property
    def rows_per_sample(self):
        return 1 + 2 * self.n_shifts

    def rows(self, P):
        """Slot vectors ``[n_prs * (1 + 2E)][n_slots]``: per sample the unshifted row, then the E
        rows shifted down, then the E rows shifted up."""
        P = np.atleast_2d(np.asarray(P, dtype=np.float64))
        V = P @ self.C.T + self.c0
        R = np.concatenate([V[:, None, :], V[:, None, :] - self.D[None], V[:, None, :] + self.D[None]], axis=1)
        return np.ascontiguousarray(R.reshape(-1, len(self.slot_names)))

    def combine(self, F):
        """Expectations of the rows ``[n_prs * (1 + 2E)][n_hams]`` (complex) -> f ``[n_prs][n_hams]``
        and the gradient ``[n_prs][n_hams][n_names]`` (complex, zero imaginary part)."""
        E = self.n_shifts
        F = np.asarray(F).reshape(-1, 1 + 2 * E, F.shape[-1])
        intrin = self.coeff[None, :, None] * np.real(F[:, 1 + E:] - F[:, 1:1 + E])
        g = np.einsum('seh,en->shn', intrin, self.J)
        return F[:, 0], g.astype(np.complex128)
