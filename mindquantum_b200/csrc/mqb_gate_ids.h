// Gate ids of the lowered gate table (mqb_gate_desc.gate_id).  The Python lowering in
// mindquantum_b200/core/gates.py uses the same numbers (checked by tests/test_host.py).
#ifndef MQB_GATE_IDS_H_
#define MQB_GATE_IDS_H_

#define GID_MATRIX 0     // constant matrix from the const pool (X, H, SWAP, custom matrices, ...)
#define GID_RX 1
#define GID_RY 2
#define GID_RZ 3
#define GID_PS 4         // phase shift diag(1, e^{i t})
#define GID_GP 5         // global phase e^{-i t}
#define GID_RXX 6
#define GID_RYY 7
#define GID_RZZ 8
#define GID_RXY 9
#define GID_RXZ 10
#define GID_RYZ 11
#define GID_GIVENS 12
#define GID_SWAPALPHA 13
#define GID_U3 14
#define GID_RN 15
#define GID_FSIM 16
#define GID_RPS 17       // exp(-i t/2 P), P a Pauli string (masks in the gate descriptor)
#define GID_CUSTOM 18    // parameterized custom matrix; matrices uploaded per sample by the caller
#define GID_COUNT 19

#endif
