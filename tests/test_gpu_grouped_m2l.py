"""The grouped tensor-core M2L of the mixed form (td3_m2l_groups, td3_fmm_m2l_grouped).

The grouping is integer work, checked on the host: every directed translation of the
M2L list appears exactly once; a run holds one operator key and distinct rows of its
tile; a translation is on the operator table exactly when its depth difference is at
most one and its lattice offset within the table's span; off-table translations form
one run per destination row, after the table's runs of their tile.  The products
(3xTF32 on the tensor cores, FP32 accumulation over up to four runs) give the locals of the FP64 M2L to FP32 accuracy --
1e-6 normwise, the mixed form's bound -- through the off-table formula as well, and the
same bits on every run (a fixed summation order).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _bits_for(v: int) -> int:
    b = 1
    while b < 32 and (1 << b) <= v:
        b += 1
    return b


def _node_at(levels: np.ndarray, qp: np.ndarray) -> np.ndarray:
    """Node of quadrant-order position qp (within each depth: all first children of the
    parents in order, then all second children, ...)."""
    lv = np.searchsorted(levels, qp, side="right") - 1
    start, size = levels[lv], levels[lv + 1] - levels[lv]
    off = qp - start
    quarter = np.maximum(size // 4, 1)
    node = start + 4 * (off % quarter) + off // quarter
    return np.where(size % 4 == 0, node, qp)


@pytest.fixture(autouse=True)
def _grouped_form(monkeypatch):
    """The mixed fmm takes the grouped products in this module."""
    from tree_d_3d_b200 import flat_tree

    monkeypatch.setattr(flat_tree, "M2L_GROUPED", True)


def _trees(n, order, seed, symmetric=False):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.mixture8(n, seed=seed)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    ref = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=order, symmetric=symmetric)
    mixed = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=order, symmetric=symmetric,
                         precision="mixed")
    return ref, mixed


def test_groups_hold_every_translation_once_in_runs_of_one_key():
    ref, tree = _trees(150_000, 12, seed=11)
    lists = tree._lists(0.5)
    g = lists["groups"]
    m2l = lists["m2l"].cpu().numpy()
    e = 2 * m2l.shape[0]
    keys = g["keys"].cpu().numpy().view(np.uint32)[:e].astype(np.int64)
    vals = g["vals"].cpu().numpy().view(np.uint32)[:e].astype(np.int64)
    tile_run = g["tile_run"].cpu().numpy().astype(np.int64)
    run_start = g["run_start"].cpu().numpy().astype(np.int64)
    span = g["span"]
    side = 2 * span + 1
    n_keys = 3 * side * side
    kb = _bits_for(n_keys + 127)
    tile, key = keys >> kb, keys & ((1 << kb) - 1)
    src, row = vals >> 7, vals & 127
    dst = _node_at(tree.levels, tile * 128 + row)
    # the directed translations, each once
    got = np.sort(dst * tree.node_count + src)
    want = np.sort(np.concatenate([m2l[:, 0] * tree.node_count + m2l[:, 1],
                                   m2l[:, 1] * tree.node_count + m2l[:, 0]]))
    np.testing.assert_array_equal(got, want)
    # keys: on the table exactly for |dl| <= 1 and offsets within the span
    depth = tree.node_depth.cpu().numpy()
    center, half = tree.node_center.cpu().numpy(), tree.node_half.cpu().numpy()
    dl = depth[src] - depth[dst]
    hmin = np.minimum(half[src], half[dst])
    u = np.rint((center[dst] - center[src]) / hmin[:, None]).astype(np.int64)
    on = (np.abs(dl) <= 1) & (np.abs(u) <= span).all(axis=1)
    want_key = np.where(on, ((dl + 1) * side + u[:, 0] + span) * side + u[:, 1] + span,
                        n_keys + row)
    np.testing.assert_array_equal(key, want_key)
    assert on.mean() > 0.99
    # runs: one key, distinct rows, inside one tile; the off-table runs (one row each)
    # after the table's runs
    n_tiles = (tree.node_count + 127) // 128
    assert tile_run.shape[0] == n_tiles + 1 and tile_run[-1] > 0
    n_runs = tile_run[-1]
    assert run_start[n_runs] == e and np.all(np.diff(run_start[: n_runs + 1]) > 0)
    for t in range(0, n_tiles, 7):
        for r in range(tile_run[t], tile_run[t + 1]):
            a, b = run_start[r], run_start[r + 1]
            assert np.all(tile[a:b] == t) and np.all(key[a:b] == key[a])
            if key[a] < n_keys:
                assert b - a <= 128 and len(np.unique(row[a:b])) == b - a
                assert r == tile_run[t] or key[run_start[r - 1]] < key[a]
            else:
                assert np.all(row[a:b] == key[a] - n_keys)


@pytest.mark.parametrize("order", [4, 8, 12, 14])
def test_grouped_locals_match_fp64(order):
    ref, tree = _trees(150_000, order, seed=20 + order)
    fp64 = [t.cpu().numpy() for t in ref._log_locals(ref._lists(0.5))]
    lists = tree._lists(0.5)
    assert "groups" in lists and "m2l_rows" not in dict.keys(lists)
    got = [t.cpu().numpy() for t in tree._log_locals(lists)]
    tree._check_tensor_cores()
    again = [t.cpu().numpy() for t in tree._log_locals(lists)]
    for part in (0, 1):
        assert relative(got[part], fp64[part]) < TOL
        assert np.array_equal(again[part], got[part])


def test_grouped_matches_the_per_translation_fp32_form(monkeypatch):
    from tree_d_3d_b200 import flat_tree

    ref, tree = _trees(150_000, 12, seed=31, symmetric=True)
    grouped = [t.cpu().numpy() for t in tree._log_locals(tree._lists(0.45))]
    tree._check_tensor_cores()
    monkeypatch.setattr(flat_tree, "M2L_GROUPED", False)
    tree._traversals.clear()
    lanes = [t.cpu().numpy() for t in tree._log_locals(tree._lists(0.45))]
    fp64 = [t.cpu().numpy() for t in ref._log_locals(ref._lists(0.45))]
    for part in (0, 1):
        assert relative(grouped[part], lanes[part]) < TOL
        assert relative(grouped[part], fp64[part]) < TOL


def test_off_table_translations_take_the_per_translation_formula(monkeypatch):
    """A span of 3 puts every same-depth translation (offsets of 6 half-widths and more)
    off the table: the CTAs' CUDA-core path must give the same locals."""
    from tree_d_3d_b200 import flat_tree

    monkeypatch.setattr(flat_tree, "_group_span", lambda theta: 3)
    ref, tree = _trees(60_000, 12, seed=5)
    lists = tree._lists(0.5)
    assert lists["groups"]["span"] == 3
    got = [t.cpu().numpy() for t in tree._log_locals(lists)]
    tree._check_tensor_cores()
    fp64 = [t.cpu().numpy() for t in ref._log_locals(ref._lists(0.5))]
    for part in (0, 1):
        assert relative(got[part], fp64[part]) < TOL


@pytest.mark.parametrize("theta", [0.3, 0.7])
def test_grouped_fmm_field_at_other_openings(theta):
    ref, tree = _trees(300_000, 12, seed=9)
    _, f64 = ref.fmm(theta=theta)
    _, fmx = tree.fmm(theta=theta)
    assert "groups" in tree._lists(theta)
    assert relative(fmx.cpu().numpy(), f64.cpu().numpy()) < TOL
