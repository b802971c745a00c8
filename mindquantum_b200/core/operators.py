"""Pauli operators and Hamiltonians.

``QubitOperator`` mirrors the reference qubit operator for Pauli-string sums (term keys are
tuples of ``(qubit, 'X'|'Y'|'Z')`` sorted by qubit).  ``Hamiltonian`` mirrors
mindquantum/core/operators/hamiltonian.py:26-245: the term-list mode (real coefficients,
imaginary parts discarded with a warning, as the reference does; each term lowered to the
reference ``PauliMask`` (mask_x, mask_y, mask_z, num_y; ccsrc/lib/simulator/utils.cpp:28-40)),
``.sparse(n)``, and Hamiltonians given as a ``scipy.sparse.csr_matrix``.
"""
from __future__ import annotations

import numbers
import re
import warnings
from typing import Dict, Tuple

import numpy as np

from ..dtype import complex128, to_mq_type

Term = Tuple[Tuple[int, str], ...]

# single-qubit Pauli products: (a, b) -> (phase, result)
_PAULI_PROD = {
    ('X', 'X'): (1, 'I'), ('Y', 'Y'): (1, 'I'), ('Z', 'Z'): (1, 'I'),
    ('X', 'Y'): (1j, 'Z'), ('Y', 'X'): (-1j, 'Z'),
    ('Y', 'Z'): (1j, 'X'), ('Z', 'Y'): (-1j, 'X'),
    ('Z', 'X'): (1j, 'Y'), ('X', 'Z'): (-1j, 'Y'),
}


def _parse_term(term) -> Term:
    if isinstance(term, str):
        out = {}
        for tok in term.split():
            m = re.fullmatch(r'([XYZxyz])(\d+)', tok)
            if not m:
                raise ValueError(f"Invalid Pauli token {tok!r}.")
            q = int(m.group(2))
            if q in out:
                raise ValueError(f"Duplicated qubit {q} in {term!r}.")
            out[q] = m.group(1).upper()
        return tuple(sorted(out.items()))
    if isinstance(term, (tuple, list)):
        return tuple(sorted((int(q), p.upper()) for q, p in term))
    raise TypeError(f"Cannot parse Pauli term {term!r}.")


class QubitOperator:
    """Sum of Pauli strings with complex coefficients."""

    def __init__(self, term=None, coefficient=1.0):
        self.terms: Dict[Term, complex] = {}
        if term is not None:
            self.terms[_parse_term(term)] = coefficient

    @classmethod
    def _from_terms(cls, terms):
        out = cls()
        out.terms = {k: v for k, v in terms.items() if v != 0}
        return out

    def __add__(self, other):
        if isinstance(other, numbers.Number):
            other = QubitOperator('', other)
        terms = dict(self.terms)
        for k, v in other.terms.items():
            terms[k] = terms.get(k, 0) + v
        return QubitOperator._from_terms(terms)

    __radd__ = __add__

    def __neg__(self):
        return QubitOperator._from_terms({k: -v for k, v in self.terms.items()})

    def __sub__(self, other):
        return self + (-other)

    def __rsub__(self, other):
        return (-self) + other

    def __mul__(self, other):
        if isinstance(other, numbers.Number):
            return QubitOperator._from_terms({k: v * other for k, v in self.terms.items()})
        if isinstance(other, QubitOperator):
            terms = {}
            for ka, va in self.terms.items():
                for kb, vb in other.terms.items():
                    d = dict(ka)
                    phase = 1
                    for q, p in kb:
                        if q in d:
                            ph, r = _PAULI_PROD[(d[q], p)]
                            phase *= ph
                            if r == 'I':
                                del d[q]
                            else:
                                d[q] = r
                        else:
                            d[q] = p
                    key = tuple(sorted(d.items()))
                    terms[key] = terms.get(key, 0) + va * vb * phase
            return QubitOperator._from_terms(terms)
        raise TypeError(f"Cannot multiply QubitOperator by {type(other)}.")

    def __rmul__(self, other):
        if isinstance(other, numbers.Number):
            return self * other
        raise TypeError(f"Cannot multiply {type(other)} by QubitOperator.")

    def __truediv__(self, other):
        return self * (1.0 / other)

    def astype(self, dtype):  # pylint: disable=unused-argument
        return self

    def compress(self, abs_tol=1e-12):
        return QubitOperator._from_terms({k: v for k, v in self.terms.items() if abs(v) > abs_tol})

    @property
    def n_qubits(self):
        qs = [q for k in self.terms for q, _ in k]
        return max(qs) + 1 if qs else 0

    def matrix(self, n_qubits=None):
        """Dense little-endian matrix of this operator."""
        n = self.n_qubits if n_qubits is None else n_qubits
        mats = {'X': np.array([[0, 1], [1, 0]]), 'Y': np.array([[0, -1j], [1j, 0]]), 'Z': np.diag([1, -1])}
        out = np.zeros((1 << n, 1 << n), dtype=complex)
        for k, v in self.terms.items():
            d = dict(k)
            m = np.array([[1]], dtype=complex)
            for q in range(n):
                m = np.kron(mats[d[q]] if q in d else np.identity(2), m)
            out += v * m
        return out

    def __str__(self):
        if not self.terms:
            return "0"
        return " +\n".join(f"{v} [{' '.join(f'{p}{q}' for q, p in k)}]" for k, v in self.terms.items())

    __repr__ = __str__


class HowTo:
    """How a Hamiltonian is applied (mindquantum/core/operators/hamiltonian.py:26-32)."""

    ORIGIN = 0     # Pauli term list
    BACKEND = 1    # Pauli terms, treated as a sparse matrix of a fixed register size
    FRONTEND = 2   # a user-given sparse matrix


class Hamiltonian:
    """A Hamiltonian: a real-coefficient Pauli sum or a sparse matrix (hamiltonian.py:35-245).

    ``Hamiltonian(QubitOperator)`` keeps the term list (``HowTo.ORIGIN``; imaginary parts of the
    coefficients discarded with a warning, as the reference does); ``.sparse(n)`` marks it as a
    sparse Hamiltonian of exactly ``n`` qubits (``HowTo.BACKEND``: the reference converts the
    terms to a CSR matrix on the CPU; here the same operator keeps running through the Pauli
    kernels).  ``Hamiltonian(scipy.sparse.csr_matrix)`` (``HowTo.FRONTEND``) applies the matrix
    itself with the device CSR kernel.
    """

    def __init__(self, hamiltonian, dtype=None):
        import scipy.sparse as sp

        if isinstance(hamiltonian, sp.csr_matrix):
            if len(hamiltonian.shape) != 2 or hamiltonian.shape[0] != hamiltonian.shape[1]:
                raise ValueError(
                    f"Hamiltonian requires a two dimension square csr_matrix, but get shape {hamiltonian.shape}")
            if np.log2(hamiltonian.shape[0]) % 1 != 0:
                raise ValueError(f"size of hamiltonian sparse matrix should be power of 2, but get {hamiltonian.shape}")
            self.ham_dtype = to_mq_type(dtype) if dtype is not None else to_mq_type(hamiltonian.dtype)
            self._hamiltonian = None
            self._ham_termlist = None
            self._sparse_matrix = hamiltonian
            self.how_to = HowTo.FRONTEND
            self.n_qubits = int(np.log2(hamiltonian.shape[0]))
            return
        if not isinstance(hamiltonian, QubitOperator):
            raise TypeError(f"Require a QubitOperator or a csr_matrix, but get {type(hamiltonian)}!")
        self.ham_dtype = to_mq_type(dtype) if dtype is not None else complex128
        self._hamiltonian = hamiltonian
        self._sparse_matrix = None
        self.how_to = HowTo.ORIGIN
        self.n_qubits = hamiltonian.n_qubits
        self._ham_termlist = []
        warned = False
        for k, v in hamiltonian.terms.items():
            v = complex(v)
            if abs(v.imag) > 1e-8 and not warned:
                warnings.warn(
                    "Hamiltonian coefficients must be real numbers. Imaginary part will be discarded.",
                    UserWarning,
                    stacklevel=2,
                )
                warned = True
            self._ham_termlist.append((k, v.real))

    @property
    def dtype(self):
        return self.ham_dtype

    @property
    def hamiltonian(self):
        if self.how_to == HowTo.FRONTEND:
            raise ValueError("Cannot get QubitOperator: this Hamiltonian was constructed from a sparse matrix.")
        return self._hamiltonian

    @property
    def ham_termlist(self):
        if self.how_to == HowTo.FRONTEND:
            raise ValueError("Cannot get Pauli term list: this Hamiltonian was constructed from a sparse matrix.")
        return self._ham_termlist

    @property
    def sparse_matrix(self):
        """The matrix as ``scipy.sparse.csr_matrix``."""
        if self.how_to != HowTo.FRONTEND:
            import scipy.sparse as sp

            return sp.csr_matrix(self._hamiltonian.matrix(self.n_qubits))
        return self._sparse_matrix

    def sparse(self, n_qubits=1):
        """Mark the Hamiltonian as sparse on exactly ``n_qubits`` qubits (hamiltonian.py:122-136)."""
        if self.how_to != HowTo.ORIGIN:
            raise ValueError('Already a sparse hamiltonian.')
        if n_qubits < self.n_qubits:
            raise ValueError(f"Can not sparse a {self.n_qubits} qubits hamiltonian to {n_qubits} hamiltonian.")
        self.n_qubits = n_qubits
        self.how_to = HowTo.BACKEND
        return self

    def astype(self, dtype):
        if self.how_to == HowTo.FRONTEND:
            return Hamiltonian(self._sparse_matrix, dtype)
        return Hamiltonian(self._hamiltonian, dtype)

    def pauli_masks(self):
        """(mask_x, mask_y, mask_z, num_y, coeff) arrays; GenPauliMask, ccsrc/lib/simulator/utils.cpp:28-40."""
        terms = self.ham_termlist
        nt = len(terms)
        mx = np.zeros(nt, dtype=np.uint64)
        my = np.zeros(nt, dtype=np.uint64)
        mz = np.zeros(nt, dtype=np.uint64)
        ny = np.zeros(nt, dtype=np.int32)
        cf = np.zeros(nt, dtype=np.float64)
        for t, (k, v) in enumerate(terms):
            for q, p in k:
                bit = np.uint64(1) << np.uint64(q)
                if p == 'X':
                    mx[t] |= bit
                elif p == 'Y':
                    my[t] |= bit
                    ny[t] += 1
                else:
                    mz[t] |= bit
            cf[t] = v
        return mx, my, mz, ny, cf

    def matrix(self, n_qubits=None):
        if self.how_to == HowTo.FRONTEND:
            return self._sparse_matrix
        return self._hamiltonian.matrix(n_qubits)

    def __str__(self):
        if self.how_to == HowTo.FRONTEND:
            return str(self._sparse_matrix)
        return str(self._hamiltonian)

    __repr__ = __str__
