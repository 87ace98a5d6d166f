"""Parity at the workload configurations' full sizes, against the oracle on the host cores.

Config 2: 200k line charges from a 2D Gaussian (sigma 0.3), log kernel, order 12,
``fmm()`` at the sources.  Config 3: 1M points from the 8-Gaussian mixture (charges +-1,
net zero): the tree build, the interaction lists, the Barnes-Hut walk at theta 0.3 / 0.5
/ 0.7 (Coulomb, softening 1e-3), the log FMM at orders 8 / 12 / 16, the Coulomb FMM at
orders 8 and 12, and ``fmm_at`` on 1M uniform targets for both kernels.  The particle
sets are those of ``bench.py`` (``synthetic`` with its seeds).

Integer outputs (node arrays, permutation, levels, lists) must be identical; fields
within 1e-12 normwise (max|a - b| / max|b|), the FP64 parity bound of the reference's
own CPU/GPU comparisons.  The oracle runs with OpenMP on every host core (about half a
minute of CPU work in all on 16 cores).
"""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu
TOL = 1e-12
N = 1_000_000
SEED = 3  # the bench's particle set


def _np(t):
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


@pytest.fixture(scope="module")
def cpu(oracle):
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


@pytest.fixture(scope="module")
def mixture():
    from tree_d_3d_b200 import synthetic

    pos, q = synthetic.mixture8(N, seed=SEED)
    return pos, q, torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")


@pytest.fixture(scope="module")
def targets():
    t = np.random.default_rng(SEED + 2).uniform(-1, 1, (2, N))
    return t, torch.tensor(t, device="cuda")


def test_config2_log_fmm_200k(cpu):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.gaussian(200_000, 0.3, seed=2)
    ref = cpu.OracleTree(pos, q, (0, 0, 1), kernel="log", order=12)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel="log", order=12)
    a = ref.fmm(theta=0.5)
    b = tree.fmm(theta=0.5)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL
    m2l, p2p = ref.lists(0.5)
    lists = tree._lists(0.5)
    np.testing.assert_array_equal(_np(lists["m2l"]), m2l)
    np.testing.assert_array_equal(_np(lists["p2p"]), p2p)


def test_config3_build_and_lists_identical(cpu, mixture):
    """Every node array, the permutation, the levels and the sorted positions of the 1M
    tree, and the mutual M2L / P2P lists in the reference's order."""
    from tree_d_3d_b200 import FlatQuadtree, Quad

    pos, q, pos_d, q_d = mixture
    ref = cpu.OracleTree(pos, q, (0, 0, 1), kernel="log", order=12)
    tree = FlatQuadtree(pos_d, q_d, Quad(0, 0, 1), kernel="log", order=12)
    assert tree.node_count == ref.node_count
    for name in ("perm", "node_center", "node_half", "node_start", "node_end", "node_child",
                 "node_depth"):
        np.testing.assert_array_equal(_np(getattr(tree, name)), getattr(ref, name), err_msg=name)
    np.testing.assert_array_equal(tree.levels, ref.levels)
    np.testing.assert_array_equal(_np(tree._sorted_pos), ref.sorted_pos)
    m2l, p2p = ref.lists(0.5)
    lists = tree._lists(0.5)
    np.testing.assert_array_equal(_np(lists["m2l"]), m2l)
    np.testing.assert_array_equal(_np(lists["p2p"]), p2p)


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_config3_walk(cpu, mixture, theta):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    pos, q, pos_d, q_d = mixture
    idx = np.arange(N)
    ref = cpu.OracleTree(pos, q, (0, 0, 1), kernel="coulomb")
    tree = FlatQuadtree(pos_d, q_d, Quad(0, 0, 1), kernel="coulomb")
    a = ref.evaluate(pos, exclude=idx, theta=theta, softening=1e-3)
    b = tree.evaluate(pos_d, exclude=torch.arange(N, device="cuda"), theta=theta, softening=1e-3)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL


@pytest.mark.parametrize("order", [8, 12, 16])
def test_config3_log_fmm(cpu, mixture, order):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    pos, q, pos_d, q_d = mixture
    ref = cpu.OracleTree(pos, q, (0, 0, 1), kernel="log", order=order)
    tree = FlatQuadtree(pos_d, q_d, Quad(0, 0, 1), kernel="log", order=order)
    a = ref.fmm(theta=0.5)
    b = tree.fmm(theta=0.5)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL


@pytest.mark.parametrize("order", [8, 12])
def test_config3_coulomb_fmm(cpu, mixture, order):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    pos, q, pos_d, q_d = mixture
    ref = cpu.OracleTree(pos, q, (0, 0, 1), kernel="coulomb", order=order)
    tree = FlatQuadtree(pos_d, q_d, Quad(0, 0, 1), kernel="coulomb", order=order)
    a = ref.fmm(theta=0.5, softening=1e-3)
    b = tree.fmm(theta=0.5, softening=1e-3)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL


@pytest.mark.parametrize("kernel,eps", [("log", 0.0), ("coulomb", 1e-3)])
def test_config3_fmm_at_1m_targets(cpu, mixture, targets, kernel, eps):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    pos, q, pos_d, q_d = mixture
    t, t_d = targets
    ref = cpu.OracleTree(pos, q, (0, 0, 1), kernel=kernel, order=12)
    tree = FlatQuadtree(pos_d, q_d, Quad(0, 0, 1), kernel=kernel, order=12)
    a = ref.fmm_at(t, theta=0.5, softening=eps)
    b = tree.fmm_at(t_d, theta=0.5, softening=eps)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL
