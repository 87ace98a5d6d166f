"""The FMM's work shares over ranks, emulated on one GPU.

Every rank of a replicated-source FMM (``FlatQuadtree(comm=...)``) takes a run of the
M2L pairs and a run of the leaves; the sum of the ranks' partial locals, after the
L2L, and the sum of their partial near fields must give the single-process FMM.  The
ranks run here one after another on one GPU (no rank waits for another); the sums
that ``all_reduce`` makes between GPUs are made by hand.  FP64 within 1e-12, mixed
within 1e-6 of the single-process mixed FMM (other partial-sum orders).
"""

from __future__ import annotations

import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel,precision", [("log", "fp64"), ("log", "mixed"),
                                              ("coulomb", "fp64"), ("coulomb", "mixed")])
@pytest.mark.parametrize("world", [2, 3])
def test_rank_shares_sum_to_the_single_process_fmm(kernel, precision, world):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic
    from tree_d_3d_b200._utils import status_word

    pos, q = synthetic.mixture8(150_000, seed=60 + world)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    eps = 1e-3 if kernel == "coulomb" else 0.0
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel=kernel, order=12, precision=precision)
    phi0, field0 = tree.fmm(theta=0.5, softening=eps)
    parts = [tree._shard(0.5, r, world) for r in range(world)]
    # the shares tile the pairs and the nodes
    n_pairs = tree._lists(0.5)["m2l"].shape[0]
    assert parts[0]["pairs"].start == 0 and parts[-1]["pairs"].stop == n_pairs
    assert parts[0]["leaves"].start == 0 and parts[-1]["leaves"].stop == tree.node_count
    for a, b in zip(parts, parts[1:]):
        assert a["pairs"].stop == b["pairs"].start and a["leaves"].stop == b["leaves"].start
    partial = [tree._shard_locals(p, eps) for p in parts]
    local_a = sum(p[0] for p in partial)
    local_b = local_a if kernel == "coulomb" else sum(p[1] for p in partial)
    tree._full_downward(local_a, local_b)
    phi = torch.zeros_like(phi0)
    field = torch.zeros_like(field0)
    for p in parts:
        ph, fl, status = torch.zeros_like(phi0), torch.zeros_like(field0), status_word(P.device)
        tree._shard_near(p, local_a, local_b, eps, True, ph, fl, status)
        assert int(status.item()) == 0
        phi += ph
        field += fl
    tree._check_tensor_cores()
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert relative(phi.cpu().numpy(), phi0.cpu().numpy()) < tol
    assert relative(field.cpu().numpy(), field0.cpu().numpy()) < tol
