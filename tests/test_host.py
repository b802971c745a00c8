"""Host-side tests (no GPU): the C ABI library, the pass scheduler, lowering and the Python API."""
import ctypes
import os
import re

import numpy as np
import pytest

from mindquantum_b200 import _native as N
from mindquantum_b200.core import gates as G
from mindquantum_b200.core.circuit import UN, Circuit, qft
from mindquantum_b200.core.operators import Hamiltonian, QubitOperator
from mindquantum_b200.core.parameterresolver import ParameterResolver
from mindquantum_b200.simulator.lowering import lower_circuit, plan_schedule
from mindquantum_b200.simulator.rng import Mt19937Uniform
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_loads_and_exports_every_declared_symbol():
    L = N.lib()
    header = open(os.path.join(ROOT, 'include', 'mqb200.h'), encoding='utf8').read()
    declared = set(re.findall(r'MQB_API\s+(?:int|const char \*)\s*(mqb_\w+)\(', header))
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert set(N.SIGNATURES) | {'mqb_last_error'} == declared
    assert L.mqb_version() >= 100


def test_gate_ids_match_header():
    text = open(os.path.join(ROOT, 'mindquantum_b200', 'csrc', 'mqb_gate_ids.h'), encoding='utf8').read()
    ids = {k: int(v) for k, v in re.findall(r'#define (GID_\w+) (\d+)', text)}
    for k, v in ids.items():
        if k == 'GID_COUNT':
            continue
        assert getattr(G, k) == v, k


def _random_circuit(rng, n, n_gates, kinds=None):
    kinds = kinds or ['h', 'x', 'cx', 'rx', 'ry', 'rz', 'rzz', 'u3', 'swap', 'cz', 'ccx', 'rxy', 'fsim', 'ps',
                      'ry1', 'crx', 'crz', 'ccz', 'crzz', 'y', 'cu3']
    c = Circuit()
    for i in range(n_gates):
        k = kinds[rng.integers(len(kinds))]
        qs = [int(q) for q in rng.permutation(n)[:3]]
        if k == 'h':
            c += G.H.on(qs[0])
        elif k == 'x':
            c += G.X.on(qs[0])
        elif k == 'cx':
            c += G.X.on(qs[0], qs[1])
        elif k == 'ccx':
            c += G.X.on(qs[0], qs[1:3])
        elif k == 'cz':
            c += G.Z.on(qs[0], qs[1])
        elif k == 'rx':
            c += G.RX(f'p{i}').on(qs[0])
        elif k == 'ry':
            c += G.RY(f'p{i}').on(qs[0], qs[1])
        elif k == 'rz':
            c += G.RZ(f'p{i}').on(qs[0])
        elif k == 'ps':
            c += G.PhaseShift(f'p{i}').on(qs[0], qs[2])
        elif k == 'rzz':
            c += G.Rzz(f'p{i}').on(qs[:2])
        elif k == 'rxy':
            c += G.Rxy(f'p{i}').on(qs[:2], qs[2])
        elif k == 'u3':
            c += G.U3(f'a{i}', f'b{i}', f'c{i}').on(qs[0])
        elif k == 'swap':
            c += G.SWAP.on(qs[:2])
        elif k == 'fsim':
            c += G.FSim(f'a{i}', f'b{i}').on(qs[:2])
        elif k == 'ry1':
            c += G.RY(f'p{i}').on(qs[0])
        elif k == 'crx':
            c += G.RX(f'p{i}').on(qs[0], qs[1])
        elif k == 'crz':
            c += G.RZ(f'p{i}').on(qs[0], qs[1])
        elif k == 'ccz':
            c += G.Z.on(qs[0], qs[1:3])
        elif k == 'crzz':
            c += G.Rzz(f'p{i}').on(qs[:2], qs[2])
        elif k == 'y':
            c += G.Y.on(qs[0])
        elif k == 'cu3':
            c += G.U3(f'a{i}', f'b{i}', f'c{i}').on(qs[0], qs[1])
    return c


def _targets_and_touched(g):
    dense = set()
    if not (g.name in ('RZ', 'PS', 'GP', 'Rzz', 'Z', 'S', 'T') and not g.hermitianed and True):
        dense = set(g.obj_qubits)
    if g.name in ('Z', 'S', 'T', 'RZ', 'PS', 'GP', 'Rzz'):
        dense = set()
    return dense, set(g.obj_qubits) | set(g.ctrl_qubits)


@pytest.mark.parametrize("n,K,prec", [(6, 4, 1), (9, 6, 0), (12, 8, 1), (14, 10, 0), (5, 13, 0)])
def test_schedule_is_a_valid_reordering(n, K, prec):
    rng = np.random.default_rng(n * 100 + K)
    c = _random_circuit(rng, n, 120)
    order, pass_of, qmask, fused = plan_schedule(c, n, prec, tile_bits=K)
    gates = [g for g in c]
    assert sorted(order.tolist()) == list(range(len(gates)))
    # every pair of gates sharing a qubit keeps its relative order
    pos = {int(g): i for i, g in enumerate(order)}
    for i in range(len(gates)):
        ti = set(gates[i].obj_qubits) | set(gates[i].ctrl_qubits)
        for j in range(i + 1, len(gates)):
            tj = set(gates[j].obj_qubits) | set(gates[j].ctrl_qubits)
            if ti & tj:
                assert pos[i] < pos[j], (i, j)
    # fused passes: K tile qubits containing the low contiguity qubits and every non-diagonal target
    c_bits = 4 if prec == 0 else 3
    for e, gi in enumerate(order):
        p = pass_of[e]
        if not fused[p]:
            continue
        qm = int(qmask[p])
        rb = 5 if prec == 0 else 4           # register bits of the forward tile kernel
        kk = min(n, max(K, rb + 5))
        assert bin(qm).count('1') == kk
        ce = kk if n <= kk else min(c_bits, max(1, kk - 2))
        assert qm & ((1 << ce) - 1) == (1 << ce) - 1
        dense, _ = _targets_and_touched(gates[gi])
        for q in dense:
            assert qm >> q & 1, (gates[gi], bin(qm))
    # executing in the planned order gives the same state
    prd = {k: float(v) for k, v in zip(c.params_name, rng.uniform(0, 2 * np.pi, len(c.params_name)))}
    ref = O.OracleSim(n).apply_circuit(c, prd).qs
    re_ordered = Circuit([gates[i] for i in order])
    got = O.OracleSim(n).apply_circuit(re_ordered, prd).qs
    assert np.allclose(ref, got, atol=1e-12)


def test_hea_pass_counts():
    from reference_circuits import hea_circuit

    c = hea_circuit(26, 12)
    _, _, qmask, fused = plan_schedule(c, 26, 0, tile_bits=13)
    assert all(fused)
    # 924 gates in far fewer state sweeps than the 924 of the per-gate schedule
    assert len(qmask) <= 32


def test_lowering_records():
    c = Circuit().rx({'a': 2.0, 'b': -1.0}, 3, 1).u3('a', 0.5, 'c', 2)
    c += G.UnivMathGate('m', G.H.matrix()).on(0)
    c += G.RotPauliString('XZY', 'b').on([0, 2, 4])
    descs, terms, pool, customs, _ = lower_circuit(c, ['a', 'b', 'c'])
    assert descs[0].gate_id == G.GID_RX and descs[0].n_obj == 1 and descs[0].obj[0] == 3
    assert descs[0].ctrl_mask == 2 and descs[0].n_angles == 1 and descs[0].term_count[0] == 2
    assert [(t.param, t.coeff) for t in terms[:2]] == [(0, 2.0), (1, -1.0)]
    assert descs[1].gate_id == G.GID_U3 and descs[1].n_angles == 3 and descs[1].grad_angles == 0b101
    assert descs[1].angle_const[1] == 0.5
    assert descs[2].gate_id == G.GID_MATRIX and len(pool) == 1
    assert descs[3].gate_id == G.GID_RPS and descs[3].pauli_x == 1 and descs[3].pauli_z == 4 and descs[3].pauli_y == 16
    assert descs[3].pauli_ny == 1


def test_invalid_gate_tables_are_rejected_on_the_host():
    d = N.GateDesc()
    d.gate_id = G.GID_RX
    d.n_obj = 1
    d.obj[0] = 7
    arr = (N.GateDesc * 1)(d)
    out = [np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.uint64), np.zeros(1, np.int32)]
    n_p = ctypes.c_int()
    st = N.lib().mqb_plan_schedule(4, 0, arr, 1, None, 0, 0, 1, ctypes.byref(n_p),
                                   *[o.ctypes.data_as(ctypes.c_void_p) for o in out], None)
    assert st == -1 and b'out of range' in N.lib().mqb_last_error()
    d.obj[0] = 1
    d.ctrl_mask = 2
    arr = (N.GateDesc * 1)(d)
    st = N.lib().mqb_plan_schedule(4, 0, arr, 1, None, 0, 0, 1, ctypes.byref(n_p),
                                   *[o.ctypes.data_as(ctypes.c_void_p) for o in out], None)
    assert st == -1 and b'overlap' in N.lib().mqb_last_error()


def test_rng_matches_reference_streams():
    u = Mt19937Uniform(1234)
    eng = O._Mt19937(1234)  # pylint: disable=protected-access
    for _ in range(50):
        assert u.draw() == O._uniform(eng, 0.0, 1.0)  # pylint: disable=protected-access
    v = Mt19937Uniform(42).draw(5, 1.0, float(1 << 20))
    eng = O._Mt19937(42)  # pylint: disable=protected-access
    assert np.allclose(v, [O._uniform(eng, 1.0, float(1 << 20)) for _ in range(5)], rtol=0, atol=0)


def test_parameter_resolver_and_circuit_bookkeeping():
    pr = ParameterResolver({'a': 1, 'b': 2}, const=0.5)
    assert (2 * pr - pr).expression() == pr.expression()
    assert pr.combination({'a': 3, 'b': 4}).const == 0.5 + 3 + 8
    c = Circuit().rx('a', 0).ry('b', 1).as_encoder()
    c += Circuit().rz('c', 0).rzz({'d': 2, 'a': 0.0}, [0, 1]).as_ansatz() if False else Circuit().rz('c', 0)
    assert c.encoder_params_name == ['a', 'b'] and c.ansatz_params_name == ['c']
    h = c.hermitian()
    assert h[0].name == 'RZ' and h[0].coeff['c'] == -1.0
    u3h = G.U3('t', 'p', 'l').on(0).hermitian()
    assert u3h.prs[1].params_name == ['l'] and u3h.prs[2].params_name == ['p']
    q = qft(range(3))
    assert sum(1 for g in q if g.name == 'SWAP') == 1
    assert Circuit(UN(G.H, 3)).n_qubits == 3


def test_qubit_operator_and_masks():
    op = QubitOperator('X0 Y1', 2.0) + QubitOperator('Z2', -1.0) + QubitOperator('', 0.5)
    h = Hamiltonian(op)
    mx, my, mz, ny, cf = h.pauli_masks()
    assert list(mx) == [1, 0, 0] and list(my) == [2, 0, 0] and list(mz) == [0, 4, 0]
    assert list(ny) == [1, 0, 0] and list(cf) == [2.0, -1.0, 0.5]
    prod = QubitOperator('X0') * QubitOperator('Y0')
    assert prod.terms == {((0, 'Z'),): 1j}
    assert np.allclose(h.matrix(3), h.matrix(3).conj().T)
