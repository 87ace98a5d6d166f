"""The mixed-precision near field at the sources in two parts (td3_fmm_near_mixed /
td3_fmm_far_mixed and the adjoint pair: FP32 hi + lo pair arithmetic and the partial sums
of multi-segment leaves, then the FP64 far field per particle), the near part on a second
stream or on the caller's, against the one-launch mixed form and FP64, for the field, the
potential and the backward, both kernels, softened or not."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu


def _run(pos, q, kernel, eps, precision, split, w, e, overlap=True):
    from tree_d_3d_b200 import Quad, flat_tree
    from tree_d_3d_b200.autograd import fmm_field

    flat_tree.NEAR_SPLIT = split
    flat_tree.NEAR_OVERLAP = overlap
    P = torch.tensor(pos, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", requires_grad=True)
    phi, field = fmm_field(P, Q, Quad(0, 0, 1), kernel=kernel, order=12, softening=eps,
                           precision=precision)
    ((w * phi).sum() + (e * field).sum()).backward()
    return [t.detach().cpu().numpy() for t in (phi, field, Q.grad, P.grad)]


@pytest.mark.parametrize("segment", [256, 8])
@pytest.mark.parametrize("kernel,eps", [("log", 0.0), ("log", 1e-3), ("coulomb", 1e-3)])
def test_split_near_field_matches_one_launch_form_and_fp64(kernel, eps, segment, monkeypatch):
    from tree_d_3d_b200 import flat_tree, synthetic

    # segment 8: most leaves take several segments (the partial-sum path)
    monkeypatch.setattr(flat_tree, "NEAR_SEGMENT", segment)
    monkeypatch.setattr(flat_tree, "NEAR_SPLIT", True)
    monkeypatch.setattr(flat_tree, "NEAR_OVERLAP", True)
    pos, q = synthetic.mixture8(60_000, seed=70)
    rng = np.random.default_rng(71)
    w = torch.tensor(rng.normal(size=pos.shape[1]), device="cuda")
    e = torch.tensor(rng.normal(size=pos.shape), device="cuda")
    split = _run(pos, q, kernel, eps, "mixed", True, w, e)
    again = _run(pos, q, kernel, eps, "mixed", True, w, e)
    serial = _run(pos, q, kernel, eps, "mixed", True, w, e, overlap=False)
    one = _run(pos, q, kernel, eps, "mixed", False, w, e)
    fp64 = _run(pos, q, kernel, eps, "fp64", True, w, e)
    for a, b, s1, c, d in zip(split, again, serial, one, fp64):
        assert np.array_equal(a, b)  # fixed summation order
        # the near part on its own stream gives the bits of the one-stream call
        assert np.array_equal(a, s1)
        assert relative(a, c) < 1e-6
        assert relative(a, d) < 1e-6


def test_split_near_field_reports_coincident_charges(monkeypatch):
    from tree_d_3d_b200 import FlatQuadtree, Quad, flat_tree

    monkeypatch.setattr(flat_tree, "NEAR_SPLIT", True)
    rng = np.random.default_rng(5)
    pos = rng.uniform(-0.9, 0.9, (2, 3000))
    pos[:, 1] = pos[:, 0]
    P, Q = torch.tensor(pos, device="cuda"), torch.ones(3000, device="cuda", dtype=torch.float64)
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=8, precision="mixed")
    with pytest.raises(ValueError, match="Coincident"):
        tree.fmm(theta=0.5)
    # softened: no report, the pair counts
    phi, field = tree.fmm(theta=0.5, softening=1e-3)
    assert torch.isfinite(phi).all() and torch.isfinite(field).all()


def test_slot_leaves_and_rejections():
    from tree_d_3d_b200 import FlatQuadtree, Quad, _lib, synthetic

    pos, q = synthetic.uniform(20_000, seed=4)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=8, precision="mixed")
    leaf = tree._slot_leaves().cpu().numpy()
    start, end = tree.node_start.cpu().numpy(), tree.node_end.cpu().numpy()
    child = tree.node_child.cpu().numpy()
    assert (child[leaf] < 0).all()
    slots = np.arange(pos.shape[1])
    assert ((start[leaf] <= slots) & (slots < end[leaf])).all()
    # slot_leaf is required, the unit must be positive
    rc = _lib.lib().td3_fmm_evaluate_mixed(_lib.KERNEL_LOG, 0, 0, 0, 1, 0, 0, 0, 8, 0, 0, 0, 0,
                                           0, 0, 0, 0, 0, 0.0, 1, 1.0, 0, 0, 0, 0)
    assert rc == _lib.EINVAL
    rc = _lib.lib().td3_fmm_adjoint_mixed(_lib.KERNEL_LOG, 0, 0, 0, 1, 0, 0, 0, 8, 0, 0, 0, 0,
                                          1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0.0, -1.0, 0, 0, 0)
    assert rc == _lib.EINVAL
