"""Circuit, gate, operator and parameter classes of the state-vector path."""
from . import gates
from .circuit import UN, Circuit, SwapParts, qft
from .gates import (CNOT, H, I, ISWAP, S, SWAP, SX, T, X, Y, Z, BarrierGate, BasicGate, FSim, GlobalPhase,
                    Givens, Measure, ParameterGate, PhaseShift, Power, RotPauliString, Rn, RX, Rxx, Rxy, Rxz, RY,
                    Ryy, Ryz, RZ, Rzz, SWAPalpha, U3, UnivMathGate, gene_univ_parameterized_gate)
from .operators import Hamiltonian, HowTo, QubitOperator
from .parameterresolver import PR, ParameterResolver
