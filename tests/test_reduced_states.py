"""Reduced states of the simulators: get_reduced_density_matrix and get_qs_of_qubits.

The reduction (``simulator.utils.reduced_density_matrix``, M M^H of the state viewed as
[kept bits][traced bits]) is checked against the oracle's restatement of the reference's
GetReducedDensityMatrix (ccsrc/lib/simulator/vector/detail/cpu_common/cpu_vector_core_policy.cpp:335-383)
on host tensors, and the pure/mixed logic of get_qs_of_qubits (mindquantum/simulator/mqsim.py:598-626)
on a stand-in backend; on a B200 both backends are checked through the Simulator facade, with
the reference's argument errors.  Tolerance 1e-12 (complex128).
"""
import numpy as np
import pytest
import torch

from mindquantum_b200.simulator.utils import check_kept_qubits, qs_of_qubits, reduced_density_matrix
from oracle import oracle as O


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("kept", [[0], [3], [4, 1], [0, 2, 3], [1, 2, 3, 4]])
def test_reduction_matches_the_reference_algorithm(kept):
    n = 5
    qs = _random_state(n, 7 + len(kept))
    rho = reduced_density_matrix(torch.from_numpy(qs), n, check_kept_qubits(kept, n))
    assert np.max(np.abs(rho - O.reduced_density_matrix(qs, n, kept))) <= 1e-12


def test_kept_qubit_checks():
    with pytest.raises(ValueError, match="repeated"):
        check_kept_qubits([1, 1], 4)
    with pytest.raises(ValueError, match="less than total"):
        check_kept_qubits([0, 1, 2, 3], 4)
    with pytest.raises(ValueError, match="out of range"):
        check_kept_qubits([5], 4)
    assert check_kept_qubits(2, 4) == [2]


class _Backend:
    """A state-vector backend stand-in: the state is a host array."""

    def __init__(self, qs):
        self.qs = qs
        self.n_qubits = int(np.log2(qs.size))

    def get_qs(self, ket=False):
        return self.qs

    def get_reduced_density_matrix(self, kept):
        return reduced_density_matrix(torch.from_numpy(self.qs), self.n_qubits, check_kept_qubits(kept, self.n_qubits))


def test_qs_of_qubits_pure_and_mixed():
    # |psi> = (|00> + |11>)/sqrt(2) on qubits 0, 1, times |+> on qubit 2: qubit 2 alone is pure,
    # qubit 0 alone is mixed (I/2)
    bell = np.zeros(4, dtype=np.complex128)
    bell[0] = bell[3] = 1 / np.sqrt(2)
    plus = np.array([1, 1], dtype=np.complex128) / np.sqrt(2)
    qs = np.kron(plus, bell)   # qubit 2 is the most significant bit
    be = _Backend(qs)
    vec = qs_of_qubits(be, 2)
    assert vec.shape == (2,) and np.max(np.abs(vec - plus)) <= 1e-12
    rho = qs_of_qubits(be, [0])
    assert np.max(np.abs(rho - np.eye(2) / 2)) <= 1e-12
    assert 'mixed state' in qs_of_qubits(be, [0], ket=True)
    assert qs_of_qubits(be, [0, 1, 2]) is qs
    with pytest.raises(TypeError):
        qs_of_qubits(be, 'q0')
    with pytest.raises(ValueError):
        qs_of_qubits(be, [3])


@pytest.mark.gpu
def test_reduced_states_on_both_backends():
    from mindquantum_b200 import complex128, workloads as W
    from mindquantum_b200.simulator import Simulator

    n = 6
    circ, _, params = W.hea(n, 2, 1, seed=4, encoder=False)
    pr = dict(zip(circ.params_name, params[0].tolist()))
    qs = O.OracleSim(n).apply_circuit(circ, pr).qs
    sv = Simulator('mqvector_b200', n, dtype=complex128)
    sv.apply_circuit(circ, pr)
    dm = Simulator('mqmatrix_b200', n, dtype=complex128)
    dm.apply_circuit(circ, pr)
    for kept in ([0], [5, 2], [1, 3, 4]):
        ref = O.reduced_density_matrix(qs, n, kept)
        assert np.max(np.abs(sv.get_reduced_density_matrix(kept) - ref)) <= 1e-12
        assert np.max(np.abs(dm.get_reduced_density_matrix(kept) - ref)) <= 1e-12
        a, b = sv.get_qs_of_qubits(kept), dm.get_qs_of_qubits(kept)
        assert a.shape == b.shape and np.max(np.abs(a - b)) <= 1e-10
    with pytest.raises(ValueError):
        sv.get_reduced_density_matrix([0, 1, 2, 3, 4, 5])
    with pytest.raises(NotImplementedError):
        sv.set_threads_number(4)
    # the pure-state answers of the density-matrix methods on a state vector (mqsim.py:546-597)
    be = sv.backend
    assert be.entropy() == 0 and be.purity() == 1.0
    assert np.max(np.abs(be.get_pure_state_vector() - qs)) <= 1e-12
    with pytest.raises(ValueError, match="partial trace"):
        be.get_partial_trace([0])


@pytest.mark.gpu
def test_circuit_matrix_on_both_backends():
    """get_circuit_matrix (mqsim.py:199-201): column j is the circuit applied to |j>, against the
    oracle's columns (1e-12), on the state-vector and the density-matrix backend."""
    from mindquantum_b200 import complex128, workloads as W
    from mindquantum_b200.simulator import Simulator

    n = 4
    circ, _, params = W.hea(n, 2, 1, seed=6, encoder=False)
    pr = dict(zip(circ.params_name, params[0].tolist()))
    ref = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    for j in range(1 << n):
        e = np.zeros(1 << n, dtype=np.complex128)
        e[j] = 1
        ref[:, j] = O.OracleSim(n, state=e).apply_circuit(circ, pr).qs
    for backend in ('mqvector_b200', 'mqmatrix_b200'):
        m = Simulator(backend, n, dtype=complex128).backend.get_circuit_matrix(circ, pr)
        assert m.shape == ref.shape and np.max(np.abs(m - ref)) <= 1e-12
