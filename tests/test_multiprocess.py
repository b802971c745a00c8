"""Replica sharding across ranks (world size 2, gloo on CPU; no GPU needed).

Each rank evaluates its own slice of the encoder samples with the CPU oracle and the ansatz
gradients are summed with an all-reduce; the result must equal the single-process sum over the
whole batch, and the shards must tile the batch exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mindquantum_b200.parallel import ansatz_gradient, shard, shard_bounds


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _problem():
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit
    from mindquantum_b200.core.operators import Hamiltonian, QubitOperator

    n = 4
    enc = Circuit([G.RX(f'x{i}').on(i) for i in range(n)]).as_encoder()
    ans = Circuit()
    for i in range(n):
        ans += G.RY(f'w{i}').on(i)
    for i in range(n - 1):
        ans += G.X.on(i + 1, i)
    circ = enc + ans
    hams = [Hamiltonian(QubitOperator('Z0')), Hamiltonian(QubitOperator('X1 Z2', 0.5))]
    rng = np.random.default_rng(3)
    x = rng.uniform(0, np.pi, (7, n))
    w = rng.uniform(0, 2 * np.pi, n)
    dout = rng.normal(size=(7, 2))
    return circ, hams, x, w, dout


def _grads(circ, hams, x, w):
    from oracle import oracle as O

    res = O.get_expectation_with_grad(4, hams, circ, x, w, circ.encoder_params_name, circ.ansatz_params_name)
    return res[:, :, 1 + len(circ.encoder_params_name):]


def _worker(rank, world, port, out_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist

    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        circ, hams, x, w, dout = _problem()
        g = _grads(circ, hams, shard(x, rank, world), w)
        total = ansatz_gradient(g, shard(dout, rank, world))
        if rank == 0:
            np.save(out_path, total.numpy())
    finally:
        dist.destroy_process_group()


def test_shard_bounds_tile_the_batch():
    for n in (0, 1, 7, 8, 13):
        for world in (1, 2, 3, 5):
            spans = [shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_two_rank_replicas_match_single_process(tmp_path):
    out = str(tmp_path / 'g.npy')
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method='spawn')
    circ, hams, x, w, dout = _problem()
    ref = ansatz_gradient(_grads(circ, hams, x, w), dout).numpy()
    got = np.load(out)
    assert np.allclose(got, ref, atol=1e-12)


@pytest.mark.parametrize("world", [2])
def test_shard_is_a_view_of_the_batch(world):
    t = torch.arange(10)
    assert torch.equal(torch.cat([shard(t, r, world) for r in range(world)]), t)
