"""The multi-process path of bench.py on the CPU: two gloo ranks.

Every rank runs an independent replica of the step; the job's time is the slowest
rank's, reduced with an all-reduce MAX.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from datetime import timedelta

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=30))
    try:
        got = bench.max_over_ranks(10.0 * (rank + 1), dist, torch.device("cpu"))
        results[rank] = got
    finally:
        dist.destroy_process_group()


def test_time_is_the_slowest_ranks():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank, args=(world, port, results), nprocs=world, join=True,
                       start_method="spawn")
    assert dict(results) == {0: 20.0, 1: 20.0}


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(3.5, None, torch.device("cpu")) == 3.5


def test_shares_tile_the_items_and_balance_the_work():
    from tree_d_3d_b200 import _shards

    rng = torch.Generator().manual_seed(3)
    for world in (1, 2, 3, 5):
        work = torch.rand(1000, generator=rng, dtype=torch.float64) ** 4
        b = _shards.bounds(work, world)
        assert b[0] == 0 and b[-1] == 1000 and b == sorted(b) and len(b) == world + 1
        total, biggest = float(work.sum()), float(work.max())
        for r in range(world):
            mine = float(work[b[r]: b[r + 1]].sum())
            assert abs(mine - total / world) <= biggest + 1e-9
    assert _shards.bounds(torch.zeros(0), 3) == [0, 0, 0, 0]


def _fmm_rank(rank, world, port, results):
    """One rank of the reference's MPI decomposition of the log FMM
    (src/tree_d_3d/flat_tree.py:1505-1539, :1600-1631) on the oracle's kernels: this
    rank's M2L pairs, the locals summed over the ranks (the product's allsum), L2L,
    this rank's leaves (L2P) and P2P pairs, the fields summed over the ranks."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from datetime import timedelta

    import numpy as np

    from oracle import flat_tree_oracle as oracle
    from tree_d_3d_b200 import _shards

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        oracle.set_threads(1)
        rng = np.random.default_rng(7)
        pos = rng.normal(0, 0.3, (2, 6000)).clip(-0.99, 0.99)
        q = rng.normal(size=6000)
        tree = oracle.OracleTree(pos, q, (0, 0, 1), kernel="log", order=10)
        L, p = oracle.lib(), oracle._p
        m2l, p2p = tree.lists(0.5)
        count, order = tree.node_count, tree.order
        pairs = _shards.share(torch.ones(len(m2l)), rank, world)
        local = np.zeros((2, count, order + 1))
        mine = np.ascontiguousarray(m2l[pairs])
        if len(mine):
            rows, partners = tree.m2l_rows(mine)
            coeff = oracle.m2l_coefficients(order, False)
            L.fmm_m2l_host(p(rows), count, p(partners), p(tree.node_center),
                           p(tree.node_center), p(tree.moment_re), p(tree.moment_im), p(coeff),
                           p(local[0]), p(local[1]), order)
        local = _shards.allsum(torch.from_numpy(local), None).numpy()
        local_re, local_im = np.ascontiguousarray(local[0]), np.ascontiguousarray(local[1])
        tree._downward(local_re, local_im, oracle.binomial_table(2 * order + 1))
        counts = tree.node_end - tree.node_start
        leaves = _shards.share(torch.from_numpy(np.where(tree.node_child < 0, counts, 0)),
                               rank, world)
        a, b = counts[p2p[:, 0]], counts[p2p[:, 1]]
        near = _shards.share(torch.from_numpy(np.where(p2p[:, 0] == p2p[:, 1], 0.5 * a * a,
                                                       a * b)), rank, world)
        spos, scharge = tree.sorted_sources()
        n = pos.shape[1]
        out = np.zeros((3, n))
        status = np.zeros(1, dtype=np.int64)
        lo = leaves.start
        for nodes, run in (((lo, leaves.stop), (0, 0)), ((0, 0), (near.start, near.stop))):
            k, m = nodes[1] - nodes[0], run[1] - run[0]
            if not k and not m:
                continue
            sub = np.ascontiguousarray(p2p[run[0]:run[1]] if m else p2p[:1])
            f = np.zeros((2, n))
            ph = np.zeros(n)
            L.fmm_evaluate_host(p(spos), n, p(scharge), k,
                                p(np.ascontiguousarray(tree.node_center[nodes[0]:])),
                                p(np.ascontiguousarray(tree.node_start[nodes[0]:])),
                                p(np.ascontiguousarray(tree.node_end[nodes[0]:])),
                                p(np.ascontiguousarray(tree.node_child[nodes[0]:])),
                                p(np.ascontiguousarray(local_re[nodes[0]:])),
                                p(np.ascontiguousarray(local_im[nodes[0]:])), order, p(sub), m,
                                0.0, 1, p(ph), p(f), n, p(status))
            out[0] += ph
            out[1:] += f
        out = _shards.allsum(torch.from_numpy(out), None).numpy()
        st = _shards.allmax(torch.from_numpy(status.copy()), None)
        phi0, field0 = tree.fmm(theta=0.5)
        phi = np.empty(n)
        field = np.empty((2, n))
        phi[tree.perm] = out[0]
        field[:, tree.perm] = out[1:]
        err = max(np.abs(phi - phi0).max() / np.abs(phi0).max(),
                  np.abs(field - field0).max() / np.abs(field0).max())
        results[rank] = (float(err), int(st.item()), pairs.start, pairs.stop)
    finally:
        dist.destroy_process_group()


def test_fmm_decomposed_over_two_gloo_ranks_equals_one_process():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_fmm_rank, args=(world, port, results), nprocs=world, join=True,
                       start_method="spawn")
    got = dict(results)
    assert set(got) == {0, 1}
    for rank in (0, 1):
        err, status, _, _ = got[rank]
        assert status == 0 and err < 1e-12
    assert got[0][3] == got[1][2]  # the two runs of pairs meet
