"""The Coulomb (Cartesian) FMM and fmm_at on the GPU against the reference.

Fields: 1e-12 normwise against the golden vectors and the oracle.  The one-way dual
lists of fmm_at come out breadth first (the reference walks depth first), so they are
compared row by row as sets; the target tree is identical.
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


@pytest.mark.parametrize("order", [4, 8, 12])
def test_coulomb_fmm_matches_golden(order):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("fmm")
    pos, q = data["coulomb/pos"], data["coulomb/charge"]
    eps = float(data[f"coulomb/p{order}/eps"])
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), order=order, leaf_capacity=16)
    phi, field = tree.fmm(theta=0.5, softening=eps)
    assert relative(phi, data[f"coulomb/p{order}/phi"]) < TOL
    assert relative(field, data[f"coulomb/p{order}/field"]) < TOL


@pytest.mark.parametrize("order,leaf", [(4, 8), (12, 32), (16, 16), (18, 16)])
def test_coulomb_fmm_matches_oracle(oracle, order, leaf):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.mixture8(40_000, seed=order)
    ref = oracle.OracleTree(pos, q, (0, 0, 1), order=order, leaf_capacity=leaf)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), order=order, leaf_capacity=leaf)
    a = ref.fmm(theta=0.5, softening=1e-3)
    b = tree.fmm(theta=0.5, softening=1e-3)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL


@pytest.mark.parametrize("softening", [0.0, 0.02])
def test_coulomb_fmm_converges_and_conserves_momentum(softening):
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    rng = np.random.default_rng(11)
    pos = np.concatenate(
        (rng.uniform(-0.9, 0.9, (2, 1500)), rng.normal(0.3, 0.05, (2, 1500))), axis=1
    ).clip(-0.99, 0.99)
    q = rng.normal(size=pos.shape[1])
    everyone = np.arange(pos.shape[1])
    phi_exact, exact = direct_field(pos, pos, q, exclude=everyone, softening=softening)
    errors = []
    for order in (2, 4, 6, 8):
        tree = FlatQuadtree(pos, q, Quad(0, 0, 1), order=order, leaf_capacity=16)
        phi, field = tree.fmm(theta=0.5, softening=softening)
        errors.append(relative(field, exact))
        assert np.max(np.abs(phi - phi_exact)) < 0.05 * np.max(np.abs(phi_exact))
        net = np.abs((q * field).sum(axis=1)).max()
        assert net < 1e-12 * np.abs(q * field).sum()
    assert errors[-1] < 1e-2 * errors[0] and all(np.diff(errors) < 0)


@pytest.mark.parametrize("order,tolerance", [(6, 1e-3), (10, 1e-5), (18, 1e-8)])
def test_log_fmm_converges_with_order(order, tolerance):
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    rng = np.random.default_rng(0)
    n = 3000
    pos = np.concatenate((rng.normal([[-0.3], [0.1]], 0.1, (2, n // 2)),
                          rng.normal([[0.4], [-0.2]], 0.25, (2, n - n // 2))), axis=1).clip(-0.99, 0.99)
    q = rng.normal(0.3, 1, n)
    ref_phi, ref_field = direct_field(pos, pos, q, exclude=np.arange(n), kernel="log")
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=order)
    phi, field = tree.fmm(theta=0.5)
    assert relative(phi, ref_phi) < tolerance
    assert relative(field, ref_field) < 10 * tolerance


def _rows_as_sets(rows, partners):
    rows, partners = _np(rows), _np(partners)
    return [tuple(sorted(partners[rows[i]:rows[i + 1]])) for i in range(len(rows) - 1)]


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
def test_fmm_at_matches_golden(kernel):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("fmm_at")
    order = 8 if kernel == "coulomb" else 16
    eps = 0.01 if kernel == "coulomb" else 0.0
    tree = FlatQuadtree(data["pos"], data["charge"], Quad(0, 0, 1), kernel=kernel, order=order,
                        leaf_capacity=16)
    phi, field = tree.fmm_at(data["targets"], exclude=data["exclude"], theta=0.5, softening=eps)
    assert relative(phi, data[f"{kernel}/phi"]) < TOL
    assert relative(field, data[f"{kernel}/field"]) < TOL
    targets = torch.tensor(data["targets"], device="cuda")
    ttree, lists = tree._target_plan(targets, 0.5, 16)
    prefix = f"{kernel}/target_tree"
    assert ttree.node_count == int(data[f"{prefix}/node_count"])
    for name in ("perm", "node_center", "node_half", "node_start", "node_end", "node_child"):
        np.testing.assert_array_equal(_np(getattr(ttree, name)), data[f"{prefix}/{name}"])
    assert _rows_as_sets(lists["m2l_rows"], lists["m2l_partners"]) == _rows_as_sets(
        data[f"{kernel}/m2l_rows"], data[f"{kernel}/m2l_partners"])
    assert _rows_as_sets(lists["p2p_rows"], lists["p2p_partners"]) == _rows_as_sets(
        data[f"{kernel}/p2p_rows"], data[f"{kernel}/p2p_partners"])
    no_phi, same = tree.fmm_at(data["targets"], exclude=data["exclude"], theta=0.5,
                               softening=eps, potential=False)
    assert not np.any(no_phi)
    np.testing.assert_allclose(same, field, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
def test_fmm_at_matches_oracle_on_large_targets(oracle, kernel):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.mixture8(60_000, seed=5)
    targets = np.random.default_rng(6).uniform(-1, 1, (2, 50_000))
    order = 12
    ref = oracle.OracleTree(pos, q, (0, 0, 1), kernel=kernel, order=order)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel=kernel, order=order)
    a = ref.fmm_at(targets, theta=0.5, softening=1e-3)
    b = tree.fmm_at(torch.tensor(targets, device="cuda"), theta=0.5, softening=1e-3)
    assert relative(_np(b[0]), a[0]) < TOL
    assert relative(_np(b[1]), a[1]) < TOL


def test_fmm_at_keeps_its_plan_across_new_charges():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(14)
    pos = rng.uniform(-0.9, 0.9, (2, 800))
    targets = rng.uniform(-0.9, 0.9, (2, 300))
    q, other = rng.normal(size=800), rng.normal(size=800)
    other[:400] = 0.0
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", leaf_capacity=8)
    tree.fmm_at(targets)
    plan = tree._plans[("targets", 0.5, 8)]
    tree.set_charges(other)
    got = tree.fmm_at(targets)
    assert tree._plans[("targets", 0.5, 8)] is plan
    fresh = FlatQuadtree(pos, other, Quad(0, 0, 1), kernel="log", leaf_capacity=8)
    np.testing.assert_allclose(got[1], fresh.fmm_at(targets)[1], rtol=1e-12, atol=1e-12)


def test_fmm_at_validation():
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    pos = np.array([[0.1, 0.5], [0.2, -0.3]])
    tree = FlatQuadtree(pos, np.ones(2), Quad(0, 0, 1))
    with pytest.raises(ValueError, match="Coincident"):
        tree.fmm_at(pos[:, :1])
    phi, field = tree.fmm_at(pos[:, :1], exclude=[0])
    _, ref = direct_field(pos[:, :1], pos, np.ones(2), exclude=[0])
    np.testing.assert_allclose(field, ref, rtol=1e-12)
    with pytest.raises(ValueError, match="theta"):
        tree.fmm_at(pos, theta=1.0)
    assert tree.fmm_at(np.zeros((2, 0)))[1].shape == (2, 0)
