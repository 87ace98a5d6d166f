"""Work shares and collectives of the FMM over ranks with replicated sources.

The reference's MPI design (src/tree_d_3d/flat_tree.py:627-637 ``_share``, :830-851
``_fmm_shares``, the allsums of :1536-1539 and :1629-1631): every rank holds every
particle and builds the same tree and interaction lists; each takes a contiguous run
of the M2L pairs and of the leaves with about an even share of their work; the partial
local expansions and the partial fields are completed by a sum over the ranks
(``all_reduce``), the coincidence status by a maximum.  Here the ranks are the
processes of a ``torch.distributed`` group (NCCL between GPUs; gloo on the CPU for the
host-side tests), one GPU each.
"""

from __future__ import annotations

import torch


def bounds(work: torch.Tensor, world: int) -> list:
    """Cut points 0 = b_0 <= ... <= b_world = n of [0, n) into ``world`` contiguous runs
    of about equal total ``work`` (non-negative): b_k is the first index whose running
    sum reaches k / world of the total."""
    n = int(work.numel())
    if world <= 1 or n == 0:
        return [0] + [n] * max(world, 1)
    running = torch.cumsum(work.to(torch.float64).reshape(-1), 0)
    marks = running[-1] * torch.arange(1, world, dtype=torch.float64, device=work.device) / world
    cuts = torch.searchsorted(running, marks).clamp_(0, n).tolist()
    return [0] + [int(c) for c in cuts] + [n]


def share(work: torch.Tensor, rank: int, world: int) -> slice:
    """This rank's run of items (``bounds``)."""
    b = bounds(work, world)
    return slice(b[rank], b[rank + 1])


def leaf_work(tree, rows: torch.Tensor, partners: torch.Tensor) -> torch.Tensor:
    """Near-field work of every cell: for a non-empty leaf, its particles times (its
    partner leaves' particles + the order of its local expansion), the P2P and L2P of
    the leaf's row; zero otherwise."""
    counts = (tree.node_end - tree.node_start).to(torch.float64)
    n_entries = int(partners.numel())
    pc = counts[partners[:n_entries]] if n_entries else counts.new_zeros(0)
    running = torch.cat((counts.new_zeros(1), torch.cumsum(pc, 0)))
    row_sum = running[rows[1:]] - running[rows[:-1]]
    leaf = (tree.node_child < 0) & (counts > 0)
    return torch.where(leaf, counts * (row_sum + tree.order + 1), torch.zeros_like(counts))


def allsum(tensor: torch.Tensor, comm) -> torch.Tensor:
    """Sum ``tensor`` over the ranks of ``comm``, in place."""
    import torch.distributed as dist

    dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=comm)
    return tensor


def allmax(tensor: torch.Tensor, comm) -> torch.Tensor:
    """Maximum of ``tensor`` over the ranks of ``comm``, in place."""
    import torch.distributed as dist

    dist.all_reduce(tensor, op=dist.ReduceOp.MAX, group=comm)
    return tensor


def rank_and_world(comm) -> tuple:
    import torch.distributed as dist

    return dist.get_rank(comm), dist.get_world_size(comm)
