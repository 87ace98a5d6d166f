"""The GPU FMM against the reference's golden vectors and the oracle.

Interaction lists are integer work: identical pairs, in the reference's order, and
identical CSR rows.  Fields use FMA and another summation order: 1e-12 normwise.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, relative

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _np(t):
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def test_log_fmm_lists_and_fields_match_golden():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("fmm")
    pos, q = data["log/pos"], data["log/charge"]
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=12)
    phi, field = tree.fmm(theta=0.5)
    lists = tree._lists(0.5)
    np.testing.assert_array_equal(_np(lists["m2l"]), data["log/m2l"])
    np.testing.assert_array_equal(_np(lists["p2p"]), data["log/p2p"])
    np.testing.assert_array_equal(_np(lists["m2l_rows"]), data["log/m2l_rows"])
    np.testing.assert_array_equal(_np(lists["m2l_partners"]), data["log/m2l_partners"])
    assert tree.fmm_pairs == tuple(int(v) for v in data["log/sizes"])
    assert relative(phi, data["log/phi"]) < TOL
    assert relative(field, data["log/field"]) < TOL
    phi, field = tree.fmm(theta=0.5, softening=0.005, potential=False)
    assert not np.any(phi)
    assert relative(field, data["log/eps/field"]) < TOL
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=12, symmetric=True)
    phi, field = tree.fmm(theta=0.4)
    assert relative(phi, data["log/sym/phi"]) < TOL
    assert relative(field, data["log/sym/field"]) < TOL
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=8, leaf_capacity=1)
    phi, field = tree.fmm(theta=0.6)
    assert relative(phi, data["log/leaf1/phi"]) < TOL
    assert relative(field, data["log/leaf1/field"]) < TOL


@pytest.mark.parametrize("order,leaf", [(12, 8), (20, 32), (40, 16), (64, 4)])
def test_log_fmm_matches_oracle(oracle, order, leaf):
    rng = np.random.default_rng(order)
    n = 60_000
    pos = rng.normal(0, 0.3, (2, n))
    pos = pos[:, np.all(np.abs(pos) < 1, axis=0)]
    q = rng.normal(size=pos.shape[1])
    from tree_d_3d_b200 import FlatQuadtree, Quad

    ref = oracle.OracleTree(pos, q, (0, 0, 1), kernel="log", order=order, leaf_capacity=leaf)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel="log", order=order, leaf_capacity=leaf)
    a = ref.fmm(theta=0.55, softening=1e-4)
    b = tree.fmm(theta=0.55, softening=1e-4)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL
    m2l, p2p = ref.lists(0.55)
    lists = tree._lists(0.55)
    np.testing.assert_array_equal(_np(lists["m2l"]), m2l)
    np.testing.assert_array_equal(_np(lists["p2p"]), p2p)


def test_fmm_validation_and_coincidence():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(2)
    pos = rng.normal(0, 0.2, (2, 400)).clip(-0.99, 0.99)
    q = rng.normal(0.3, 1, 400)
    q[::7] = 0.0
    pos[:, 2] = pos[:, 1]
    _, field = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log").fmm(softening=0.01)
    assert np.all(np.isfinite(field))
    with pytest.raises(ValueError, match="Coincident"):
        FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log").fmm()
    with pytest.raises(ValueError, match="theta"):
        FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log").fmm(theta=1.0)


def test_fmm_lists_survive_set_charges():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(8)
    pos = rng.uniform(-1, 1, (2, 3000))
    first, second = rng.normal(size=3000), rng.normal(size=3000)
    tree = FlatQuadtree(pos, first, Quad(0, 0, 1), kernel="log", leaf_capacity=16)
    tree.fmm()
    lists = tree._lists(0.5)
    tree.set_charges(second)
    assert tree._lists(0.5) is lists
    fresh = FlatQuadtree(pos, second, Quad(0, 0, 1), kernel="log", leaf_capacity=16)
    np.testing.assert_allclose(tree.fmm()[1], fresh.fmm()[1], rtol=0, atol=1e-10)


@pytest.mark.parametrize("order", [12, 40])
def test_downward_in_one_launch_equals_the_level_by_level_pass(order, monkeypatch):
    """Each leaf's local from its ancestors' own locals (one launch) against the
    reference's level-by-level L2L: the same leaf locals up to rounding."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, flat_tree, synthetic

    pos, q = synthetic.mixture8(100_000, seed=4)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel="log", order=order)
    lists = tree._lists(0.5)
    leaves = ((tree.node_child < 0) & (tree.node_end > tree.node_start)).cpu().numpy()
    monkeypatch.setattr(flat_tree, "DOWNWARD_LEAVES", True)
    one = [_np(t)[leaves] for t in tree._log_locals(lists)]
    monkeypatch.setattr(flat_tree, "DOWNWARD_LEAVES", False)
    levels = [_np(t)[leaves] for t in tree._log_locals(lists)]
    for a, b in zip(one, levels):
        assert relative(a, b) < 1e-13


@pytest.mark.parametrize("mutual", [True, False])
def test_pair_csr_rows_equal_the_oracle_at_full_lists(oracle, mutual):
    """td3_pair_csr (counting placement, rows ordered by input position) against the
    reference's pair_csr on the lists of a 300k-particle tree: the same rows, partners
    in the same order, every entry's row."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic
    from oracle.flat_tree_oracle import lib, _p

    pos, q = synthetic.mixture8(300_000, seed=17)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel="log", order=4)
    lists = tree._lists(0.5)
    for name in ("m2l", "p2p"):
        pairs = lists[name]
        rows, partners, entry = tree._rows(pairs, mutual, entry_rows=True)
        n = tree.node_count
        pn = np.ascontiguousarray(_np(pairs), dtype=np.int64)
        want_rows = np.zeros(n + 1, dtype=np.int64)
        want_partners = np.empty(max((2 if mutual else 1) * len(pn), 1), dtype=np.int64)
        cursor = np.empty(n, dtype=np.int64)
        lib().pair_csr(_p(pn), len(pn), 1 if mutual else 0, _p(want_rows), n, _p(want_partners),
                       _p(cursor))
        got_rows = _np(rows)
        np.testing.assert_array_equal(got_rows, want_rows)
        total = int(got_rows[-1])
        np.testing.assert_array_equal(_np(partners)[:total], want_partners[:total])
        row_of = np.repeat(np.arange(n), np.diff(want_rows))
        np.testing.assert_array_equal(_np(entry)[:total], row_of)
        assert np.all(_np(entry)[total:] == n)
