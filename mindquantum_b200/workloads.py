"""Synthetic variational workloads of the state-vector path (seeded, reproducible).

Each builder returns circuits, Hamiltonians and parameter arrays drawn from
``numpy.random.default_rng(seed)`` in a fixed order (angles, then Hamiltonian coefficients, then
encoder data), so a workload is fully named by its sizes and its seed:

* ``hea``: hardware-efficient ansatz, per layer RY then RZ on every qubit and a CNOT ladder
  q_i -> q_{i+1}; H = sum a_i Z_i Z_{i+1} + sum b_i X_i, a, b ~ N(0, 1).
* ``qnn``: RX(x_j) encoder with x ~ U[0, pi], per layer RY and RZ on every qubit and a CZ ring
  (i, i+1 mod n); Hamiltonians Z_0 .. Z_{m-1} evaluated separately.
* ``uneven_u3``: circuits of different qubit counts, per layer U3 on every qubit and brick CNOTs
  (even layers (0,1),(2,3)..., odd layers (1,2),(3,4)...), each with its own random Pauli
  Hamiltonian (strings of weight 1..4 on distinct qubits, coefficients N(0, 1)).
* ``qaoa_maxcut``: QAOA on a random 3-regular graph: H on every qubit, then per layer
  Rzz(gamma_l) on every edge and RX(beta_l) on every qubit, gamma, beta ~ U[0, pi];
  H = sum over edges Z_i Z_j.
"""
import numpy as np

from .core import gates as G
from .core.circuit import Circuit
from .core.operators import Hamiltonian, QubitOperator


def hea(n, layers, batch, seed=0, encoder=True):
    """(circuit, Hamiltonian, params[batch][2 n layers]); the angles are the encoder part when ``encoder``."""
    circ = Circuit()
    k = 0
    for _ in range(layers):
        for q in range(n):
            circ += G.RY(f'p{k}').on(q)
            k += 1
        for q in range(n):
            circ += G.RZ(f'p{k}').on(q)
            k += 1
        for q in range(n - 1):
            circ += G.X.on(q + 1, q)
    if encoder:
        circ.as_encoder()
    rng = np.random.default_rng(seed)
    params = rng.uniform(0, 2 * np.pi, size=(batch, k))
    a = rng.normal(size=n - 1)
    b = rng.normal(size=n)
    op = QubitOperator()
    for i in range(n - 1):
        op += QubitOperator(f'Z{i} Z{i + 1}', float(a[i]))
    for i in range(n):
        op += QubitOperator(f'X{i}', float(b[i]))
    return circ, Hamiltonian(op), params


def qnn(n, layers, samples, n_obs=4, seed=0):
    """(circuit, [Hamiltonian Z_0..Z_{n_obs-1}], enc[samples][n], ans[2 n layers])."""
    enc = Circuit([G.RX(f'x{j}').on(j) for j in range(n)]).as_encoder()
    ans = Circuit()
    k = 0
    for _ in range(layers):
        for q in range(n):
            ans += G.RY(f'w{k}').on(q)
            k += 1
        for q in range(n):
            ans += G.RZ(f'w{k}').on(q)
            k += 1
        for q in range(n):
            ans += G.Z.on((q + 1) % n, q)
    circ = enc + ans
    rng = np.random.default_rng(seed)
    ans_data = rng.uniform(0, 2 * np.pi, size=k)
    enc_data = rng.uniform(0, np.pi, size=(samples, n))
    hams = [Hamiltonian(QubitOperator(f'Z{i}')) for i in range(n_obs)]
    return circ, hams, enc_data, ans_data


def _u3_brick(n, layers, prefix):
    c = Circuit()
    for layer in range(layers):
        for q in range(n):
            c += G.U3(f'{prefix}t{layer}_{q}', f'{prefix}p{layer}_{q}', f'{prefix}l{layer}_{q}').on(q)
        for q in range(layer % 2, n - 1, 2):
            c += G.X.on(q + 1, q)
    return c


def random_pauli_hamiltonian(n, n_terms, rng, max_weight=4):
    op = QubitOperator()
    for _ in range(n_terms):
        w = int(rng.integers(1, max_weight + 1))
        qs = rng.permutation(n)[:w]
        ps = rng.integers(0, 3, size=w)
        s = ' '.join(f"{'XYZ'[p]}{q}" for p, q in zip(ps, qs))
        op += QubitOperator(s, float(rng.normal()))
    return Hamiltonian(op)


def uneven_u3(count, n_min, n_max, layers, n_terms=10, seed=0):
    """[(n, circuit, Hamiltonian, params[3 n layers])] with n ~ U{n_min..n_max} per circuit."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, size=count)
    out = []
    for i, n in enumerate(ns):
        n = int(n)
        c = _u3_brick(n, layers, f'c{i}')
        params = rng.uniform(0, 2 * np.pi, size=len(c.params_name))
        out.append([n, c, None, params])
    for item in out:   # Hamiltonian coefficients after every angle
        item[2] = random_pauli_hamiltonian(item[0], n_terms, rng)
    return [tuple(x) for x in out]


def regular_graph_edges(n, degree=3, seed=0):
    import networkx as nx  # pylint: disable=import-outside-toplevel

    g = nx.random_regular_graph(degree, n, seed=seed)
    return sorted((min(u, v), max(u, v)) for u, v in g.edges())


def qaoa_maxcut(n, p, seed=0):
    """(circuit, Hamiltonian, params[2 p], edges): ansatz parameters g0..g{p-1}, b0..b{p-1}."""
    edges = regular_graph_edges(n, 3, seed)
    circ = Circuit([G.H.on(q) for q in range(n)])
    for layer in range(p):
        for (i, j) in edges:
            circ += G.Rzz(f'g{layer}').on([i, j])
        for q in range(n):
            circ += G.RX(f'b{layer}').on(q)
    rng = np.random.default_rng(seed)
    params = rng.uniform(0, np.pi, size=len(circ.params_name))
    op = QubitOperator()
    for (i, j) in edges:
        op += QubitOperator(f'Z{i} Z{j}')
    return circ, Hamiltonian(op), params, edges


def pauli_csr(ham, n, dtype=np.complex128):
    """The 2^n x 2^n matrix of a Pauli Hamiltonian as ``scipy.sparse.csr_matrix``, built per flip
    mask without a dense matrix: P|i> = i^{n_y} (-1)^{popcount(i & (m_y | m_z))} |i ^ m_flip>, so
    row r has one entry per distinct flip mask f, at column r ^ f."""
    import scipy.sparse as sp

    mx, my, mz, ny, cf = ham.pauli_masks()
    dim = 1 << n
    cols_of, vals_of = [], []
    rows = np.arange(dim, dtype=np.int64)
    flips = sorted({int(a) | int(b) for a, b in zip(mx, my)})
    for f in flips:
        col = rows ^ f
        val = np.zeros(dim, dtype=np.complex128)
        for t in range(len(cf)):
            if (int(mx[t]) | int(my[t])) != f:
                continue
            sign = 1 - 2 * (np.bitwise_count(col & np.int64(int(my[t]) | int(mz[t]))) & 1).astype(np.int64)
            val += cf[t] * (1j ** int(ny[t])) * sign
        cols_of.append(col)
        vals_of.append(val)
    cols = np.stack(cols_of)            # [flips][dim]
    vals = np.stack(vals_of)
    order = np.argsort(cols, axis=0)
    cols = np.take_along_axis(cols, order, axis=0).T.reshape(-1)
    vals = np.take_along_axis(vals, order, axis=0).T.reshape(-1).astype(dtype)
    indptr = np.arange(0, dim * len(flips) + 1, len(flips), dtype=np.int64)
    return sp.csr_matrix((vals, cols, indptr), shape=(dim, dim))
