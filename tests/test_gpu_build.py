"""The GPU tree build and moments against the reference's golden vectors.

Trees are integer work plus exactly replicated floating-point centres: every node
array, the permutation, the levels and the sorted positions must be identical.  The
moments sum in the reference's order without FMA contraction, so they are compared
for equality as well.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

TREE_ARRAYS = ("perm", "node_center", "node_half", "node_start", "node_end", "node_child",
               "node_depth")


def _np(t):
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def assert_tree(tree, data, prefix):
    assert tree.node_count == int(data[f"{prefix}/node_count"])
    for name in TREE_ARRAYS:
        np.testing.assert_array_equal(_np(getattr(tree, name)), data[f"{prefix}/{name}"],
                                      err_msg=name)
    np.testing.assert_array_equal(tree.levels, data[f"{prefix}/levels"])


@pytest.mark.parametrize("cloud", ["uniform", "circle", "clustered", "lattice", "coincident"])
def test_build_is_identical(cloud):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("build")
    pos = data[f"{cloud}/pos"]
    tree = FlatQuadtree(pos, np.ones(pos.shape[1]), Quad(0, 0, 1), leaf_capacity=6)
    assert_tree(tree, data, cloud)
    perm = _np(tree.perm)
    assert np.array_equal(np.sort(perm), np.arange(pos.shape[1]))
    np.testing.assert_array_equal(_np(tree._sorted_pos), pos[:, perm])


def test_build_deep_chain_depths_and_offset_root():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("build")
    tree = FlatQuadtree(data["chain/pos"], [1, 1, -1], Quad(0, 0, 1), leaf_capacity=1)
    assert_tree(tree, data, "chain")
    assert tree.node_count == 1 + 4 * 48 and int(tree.node_depth.max()) == 48
    assert tree.root.count == 3
    for leaf, depth in ((1, 10), (8, 48)):
        key = f"cloud300_l{leaf}_d{depth}"
        tree = FlatQuadtree(data[f"{key}/pos"], np.ones(300), Quad(0, 0, 1),
                            leaf_capacity=leaf, max_depth=depth)
        assert_tree(tree, data, key)
    root = data["offroot/root"]
    pos = data["offroot/pos"]
    tree = FlatQuadtree(pos, np.zeros(pos.shape[1]), Quad(*root), leaf_capacity=16)
    assert_tree(tree, data, "offroot")


def test_too_small_node_buffer_restarts_the_build():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("build")
    pos = data["clustered/pos"]
    tree = FlatQuadtree.__new__(FlatQuadtree)
    # the constructor with a capacity of 8 nodes: must restart and give the same tree
    original = FlatQuadtree._build
    FlatQuadtree._build = lambda self, capacity=None: original(self, 8)
    try:
        tree = FlatQuadtree(pos, np.ones(pos.shape[1]), Quad(0, 0, 1), leaf_capacity=6)
    finally:
        FlatQuadtree._build = original
    assert tree.build_restarts > 0
    assert_tree(tree, data, "clustered")


def test_moments_are_identical():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("moments")
    pos, charge = data["pos"], data["charge"]
    tree = FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=8)
    assert_tree(tree, data, "coulomb")
    for name in ("node_q", "node_qabs", "node_p", "node_s"):
        np.testing.assert_array_equal(_np(getattr(tree, name)), data[f"coulomb/{name}"],
                                      err_msg=name)
    tree = FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=8, kernel="log", order=12)
    for name in ("node_qabs", "moment_re", "moment_im", "node_q", "node_p"):
        np.testing.assert_array_equal(_np(getattr(tree, name)), data[f"log/{name}"],
                                      err_msg=name)
    for order in (4, 12):
        tree = FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=8, order=order)
        np.testing.assert_array_equal(_np(tree._cartesian_moments()), data[f"cart{order}/moments"])


@pytest.mark.parametrize("order,capacity", [(1, 40), (7, 70), (12, 8), (12, 100), (15, 33)])
@pytest.mark.parametrize("adjoint", [False, True])
def test_log_moments_of_low_orders_equal_the_coefficient_per_thread_form(order, capacity,
                                                                         adjoint):
    """Orders below 16 (leaf moments a thread per leaf, M2M 16 lanes per node) against
    the first coefficients of order 20 (a thread per node and coefficient): a_n does not
    depend on the order, so the bits agree.  Leaves of several dozen particles; plain
    and dipole (adjoint) terms."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, _lib

    rng = np.random.default_rng(order + capacity)
    pos = np.concatenate([rng.uniform(-1, 1, (2, 6000)), rng.normal(0.3, 0.01, (2, 3000))], 1)
    charge = rng.normal(size=pos.shape[1])
    dipole = None
    results = []
    for p in (order, 20):
        tree = FlatQuadtree(pos, charge, Quad(0, 0, 1), kernel="log", order=p,
                            leaf_capacity=capacity)
        if not adjoint:
            results.append((tree.node_qabs, tree.moment_re[:, : order + 1],
                            tree.moment_im[:, : order + 1]))
            continue
        dev, count = tree.device, tree.node_count
        if dipole is None:
            dipole = torch.tensor(rng.normal(size=(2, pos.shape[1])), device=dev)
        levels = np.ascontiguousarray(tree.levels, dtype=np.int64)
        binom = tree._binomial()
        wabs = torch.empty(count, dtype=torch.float64, device=dev)
        mre = torch.empty((count, p + 1), dtype=torch.float64, device=dev)
        mim = torch.empty_like(mre)
        _lib.call("td3_log_moments_adjoint", levels.ctypes.data, len(levels) - 1, p,
                  tree._sorted_pos.data_ptr(), tree._sorted_charge.data_ptr(),
                  dipole.data_ptr(), pos.shape[1], tree.node_center.data_ptr(),
                  tree.node_start.data_ptr(), tree.node_end.data_ptr(),
                  tree.node_child.data_ptr(), binom.data_ptr(), binom.shape[0],
                  wabs.data_ptr(), mre.data_ptr(), mim.data_ptr(), _lib.stream(dev))
        results.append((wabs, mre[:, : order + 1], mim[:, : order + 1]))
    for low, high in zip(*results):
        assert torch.equal(low, high)


@pytest.mark.parametrize("kernel", ["log", "coulomb"])
def test_set_charges_equals_a_new_tree(kernel):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(8)
    pos = rng.uniform(-1, 1, (2, 3000))
    first, second = rng.normal(size=3000), rng.normal(size=3000)
    tree = FlatQuadtree(pos, first, Quad(0, 0, 1), kernel=kernel, leaf_capacity=16)
    tree.set_charges(second)
    fresh = FlatQuadtree(pos, second, Quad(0, 0, 1), kernel=kernel, leaf_capacity=16)
    names = ("moment_re", "moment_im") if kernel == "log" else ("node_q", "node_p", "node_s")
    for name in names + ("node_qabs",):
        assert torch.equal(getattr(tree, name), getattr(fresh, name)), name
    with pytest.raises(ValueError, match="one entry per particle"):
        tree.set_charges(second[:10])


def test_validation_and_empty_tree():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    with pytest.raises(ValueError, match=r"\(2, N\)"):
        FlatQuadtree(np.zeros((3, 2)), np.zeros(3), Quad(0, 0, 1))
    with pytest.raises(ValueError, match="outside tree bounds"):
        FlatQuadtree([[2.0], [0.0]], [1.0], Quad(0, 0, 1))
    with pytest.raises(ValueError, match="finite"):
        FlatQuadtree([[np.nan], [0.0]], [1.0], Quad(0, 0, 1))
    with pytest.raises(ValueError, match="kernel"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), kernel="yukawa")
    with pytest.raises(ValueError, match="order"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), order=65)
    with pytest.raises(ValueError, match="same length"):
        FlatQuadtree([[0.0], [0.0]], [1.0, 2.0], Quad(0, 0, 1))
    tree = FlatQuadtree(np.zeros((2, 0)), np.zeros(0), Quad(0, 0, 1))
    tree.set_charges(np.zeros(0))
    assert tree.node_count == 1


def test_large_build_is_a_valid_tree():
    """1M clustered points: the permutation is a permutation, every split node's
    children tile its range, leaves respect the capacity, digits follow the centres."""
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(3)
    n = 1_000_000
    pos = rng.normal(0, 0.2, (2, n)).clip(-0.999, 0.999)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.ones(n, device="cuda",
                        dtype=torch.float64), Quad(0, 0, 1), leaf_capacity=8)
    perm = tree.perm
    assert torch.equal(torch.sort(perm).values, torch.arange(n, device="cuda"))
    child, start, end = tree.node_child, tree.node_start, tree.node_end
    split = child >= 0
    first = child[split]
    assert torch.equal(start[first], start[split])
    assert torch.equal(end[first + 3], end[split])
    for c in range(3):
        assert torch.equal(end[first + c], start[first + c + 1])
    leaves = ~split
    assert int(((end - start)[leaves] > 8).sum()) == 0
    assert torch.equal(tree._sorted_pos, tree.pos[:, perm])


@pytest.mark.parametrize("scale,depth", [(1e-5, 48), (1e-8, 48), (1e-8, 20), (1e-12, 48)])
def test_build_of_fine_clusters_matches_the_oracle(oracle, scale, depth):
    """Clusters 2^-17 to 2^-40 of the root: trees whose splits go past the first 16
    levels of the quadrant paths, past 32 levels, or stop at max_depth."""
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(int(-np.log10(scale)) + depth)
    pos = np.concatenate([rng.uniform(-1, 1, (2, 3000)),
                          0.3 + scale * rng.normal(size=(2, 2000)),
                          -0.51 + scale * rng.uniform(-1, 1, (2, 500))], axis=1)
    ref = oracle.OracleTree(pos, np.ones(pos.shape[1]), (0.0, 0.0, 1.0), leaf_capacity=5,
                            max_depth=depth)
    tree = FlatQuadtree(pos, np.ones(pos.shape[1]), Quad(0, 0, 1), leaf_capacity=5,
                        max_depth=depth)
    assert tree.node_count == ref.node_count
    for name in TREE_ARRAYS:
        np.testing.assert_array_equal(_np(getattr(tree, name)), getattr(ref, name)[: ref.node_count]
                                      if name != "perm" else ref.perm, err_msg=name)
    np.testing.assert_array_equal(tree.levels, ref.levels)


@pytest.mark.parametrize("order", [4, 8, 12])
def test_moments_in_one_launch_are_the_bits_of_the_level_pass(order, monkeypatch):
    """The one-launch upward pass (the last child forms its parent) against the
    level-by-level pass, for the forward moments and the adjoint ones (monopoles and
    point dipoles): identical arrays."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, flat_tree, synthetic

    pos, q = synthetic.mixture8(200_000, seed=70 + order)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel="log", order=order)
    rng = np.random.default_rng(order)
    w = torch.tensor(rng.normal(size=pos.shape[1]), device="cuda")
    d = torch.tensor(rng.normal(size=pos.shape), device="cuda")
    binom = tree._binomial()
    runs = {}
    for one in (True, False):
        monkeypatch.setattr(flat_tree, "MOMENTS_ONE_LAUNCH", one)
        tree._moments()
        out = [_np(tree.moment_re).copy(), _np(tree.moment_im).copy(), _np(tree.node_qabs).copy()]
        mre, mim = torch.empty_like(tree.moment_re), torch.empty_like(tree.moment_im)
        wabs = torch.empty_like(tree.node_qabs)
        tree._log_moments_into(w, d, binom, wabs, mre, mim)
        runs[one] = out + [_np(mre), _np(mim), _np(wabs)]
    for a, b in zip(runs[True], runs[False]):
        np.testing.assert_array_equal(a, b)
