"""The electrode solver's repeated multipole products (tree_d_3d_b200.electrodes) on
panel-like points, against the oracle's fmm_at / walk of the same tree.

Sources are quadrature nodes along curves (three circles and a segment), targets the
midpoints between neighbouring nodes plus some nodes themselves (those exclude their
own source).  Three products with new charges each must reuse the first product's
tree and target plan (no rebuild) and match the oracle within 1e-12 normwise.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu


def _panels(n_per_curve=12_000):
    t = np.linspace(0.0, 2 * np.pi, n_per_curve, endpoint=False)
    curves = [np.stack((0.3 * np.cos(t) - 0.4, 0.3 * np.sin(t) + 0.1)),
              np.stack((0.2 * np.cos(t) + 0.45, 0.25 * np.sin(t) - 0.2)),
              np.stack((0.1 * np.cos(t) + 0.1, 0.1 * np.sin(t) + 0.6)),
              np.stack((np.linspace(-0.9, 0.9, n_per_curve), np.full(n_per_curve, -0.7)))]
    nodes = np.concatenate(curves, axis=1)
    mids = 0.5 * (nodes[:, :-1] + nodes[:, 1:])[:, ::2]
    on_node = np.arange(0, nodes.shape[1], 5)
    targets = np.concatenate((mids, nodes[:, on_node]), axis=1)
    exclude = np.concatenate((np.full(mids.shape[1], -1), on_node)).astype(np.int64)
    return np.ascontiguousarray(nodes), np.ascontiguousarray(targets), exclude


def test_repeated_products_reuse_the_tree_and_plan_and_match_the_oracle(oracle):
    from tree_d_3d_b200.electrodes import FMM_AT_THETA, FMM_LEAF, FMM_ORDER, PanelSums

    nodes, targets, exclude = _panels()
    sums = PanelSums(torch.tensor(nodes, device="cuda"), torch.tensor(targets, device="cuda"),
                     exclude=torch.tensor(exclude, device="cuda"))
    rng = np.random.default_rng(4)
    ref_tree, plan = None, None
    for step in range(3):
        charges = rng.normal(size=nodes.shape[1])
        phi, field = sums(torch.tensor(charges, device="cuda"))
        tree = sums.tree
        if plan is None:
            first_tree = tree
            plan = dict(tree._plans)
            q = tree.root_quad
            ref_tree = oracle.OracleTree(nodes, charges, (q.xmid, q.ymid, q.half), kernel="log",
                                         order=FMM_ORDER, leaf_capacity=FMM_LEAF)
        else:
            assert tree is first_tree  # same source tree, new charges
            assert len(tree._plans) == 1
            for key, value in tree._plans.items():
                assert value[1] is plan[key][1]  # the same target tree and lists
            ref_tree.set_charges(charges)
        a = ref_tree.fmm_at(targets, exclude=exclude, theta=FMM_AT_THETA)
        assert relative(phi.cpu().numpy(), a[0]) < 1e-12
        assert relative(field.cpu().numpy(), a[1]) < 1e-12
    assert sums.products == 3


def test_few_targets_take_the_walk(oracle):
    from tree_d_3d_b200.electrodes import FMM_LEAF, FMM_ORDER, WALK_THETA, PanelSums

    nodes, targets, exclude = _panels(4000)
    few = np.ascontiguousarray(targets[:, exclude < 0][:, ::40])  # midpoints only
    sums = PanelSums(nodes, few)
    charges = np.random.default_rng(5).normal(size=nodes.shape[1])
    phi, field = sums(charges)
    assert isinstance(phi, np.ndarray) and sums.tree._plans == {}
    q = sums.tree.root_quad
    ref = oracle.OracleTree(nodes, charges, (q.xmid, q.ymid, q.half), kernel="log",
                            order=FMM_ORDER, leaf_capacity=FMM_LEAF)
    a = ref.evaluate(few, theta=WALK_THETA)
    assert relative(phi, a[0]) < 1e-12
    assert relative(field, a[1]) < 1e-12
    op = sums.as_operator()
    assert op.shape == (few.shape[1], nodes.shape[1])
    assert relative(op.matvec(charges), a[0]) < 1e-12
