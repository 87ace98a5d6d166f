"""The mixed-precision FMM (FP32 near field with compensated sums, FP32 M2L on
size-scaled expansions, FP64 M2M / L2L / L2P) against FP64 references.

The contract: field error at most 1e-6 normwise against the FP64 direct sum, on 4096
seeded sample targets, at p = 12 (config 2: 200k Gaussian line charges; config 3: 1M
8-Gaussian mixture).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _sample_error(tree, pos, q, kernel, eps, field, n_sample=4096, seed=0):
    from tree_d_3d_b200 import direct_field

    n = pos.shape[1]
    idx = torch.tensor(np.random.default_rng(seed).choice(n, n_sample, replace=False),
                       device=pos.device)
    _, ref = direct_field(pos[:, idx], pos, q, softening=eps, exclude=idx, kernel=kernel)
    return relative(field[:, idx].cpu().numpy(), ref.cpu().numpy())


@pytest.mark.parametrize("config", ["gaussian_200k", "mixture_1M"])
def test_mixed_log_fmm_error_against_direct(config):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    if config == "gaussian_200k":
        pos, q = synthetic.gaussian(200_000, 0.3, seed=2)
    else:
        pos, q = synthetic.mixture8(1_000_000, seed=3)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    errors = {}
    fields = {}
    for precision in ("fp64", "mixed"):
        tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=12, precision=precision)
        _, field = tree.fmm(theta=0.5)
        fields[precision] = field
        errors[precision] = _sample_error(tree, P, Q, "log", 0.0, field)
    assert errors["fp64"] < 1e-7
    assert errors["mixed"] < TOL
    assert relative(fields["mixed"].cpu().numpy(), fields["fp64"].cpu().numpy()) < TOL


@pytest.mark.parametrize("kernel,eps", [("log", 1e-3), ("coulomb", 1e-3)])
def test_mixed_fmm_and_fmm_at_match_fp64(kernel, eps):
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.mixture8(200_000, seed=7)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    targets = torch.tensor(np.random.default_rng(8).uniform(-1, 1, (2, 50_000)), device="cuda")
    out = {}
    for precision in ("fp64", "mixed"):
        tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel=kernel, order=12, precision=precision)
        out[precision] = (tree.fmm(theta=0.5, softening=eps),
                          tree.fmm_at(targets, theta=0.5, softening=eps))
    for which in (0, 1):
        for comp in (0, 1):
            a = out["mixed"][which][comp].cpu().numpy()
            b = out["fp64"][which][comp].cpu().numpy()
            assert relative(a, b) < TOL


@pytest.mark.parametrize("kernel", ["log", "coulomb"])
def test_mixed_backward_matches_fp64(kernel):
    from tree_d_3d_b200 import Quad, synthetic
    from tree_d_3d_b200.autograd import fmm_field

    pos, q = synthetic.uniform(100_000, seed=11)
    rng = np.random.default_rng(12)
    w = torch.tensor(rng.normal(size=pos.shape[1]), device="cuda")
    e = torch.tensor(rng.normal(size=pos.shape), device="cuda")
    eps = 1e-3 if kernel == "coulomb" else 0.0
    grads = {}
    for precision in ("fp64", "mixed"):
        P = torch.tensor(pos, device="cuda", requires_grad=True)
        Q = torch.tensor(q, device="cuda", requires_grad=True)
        phi, field = fmm_field(P, Q, Quad(0, 0, 1), kernel=kernel, order=12, softening=eps,
                               precision=precision)
        ((w * phi).sum() + (e * field).sum()).backward()
        grads[precision] = (Q.grad.cpu().numpy(), P.grad.cpu().numpy())
    assert relative(grads["mixed"][0], grads["fp64"][0]) < TOL
    assert relative(grads["mixed"][1], grads["fp64"][1]) < TOL


@pytest.mark.parametrize("kernel,eps,scale", [("log", 0.0, 1.0), ("log", 1e-3, 1.0),
                                              ("coulomb", 0.0, 1.0), ("coulomb", 1e-3, 1.0),
                                              ("log", 0.0, 1e-12), ("coulomb", 0.0, 1e12)])
def test_mixed_walk_matches_fp64_walk(kernel, eps, scale):
    """The mixed Barnes-Hut walk takes the FP64 walk's cells (exact decisions) and its
    field and potential agree with FP64 to 1e-6, also at length scales far from 1 (the
    FP32 far-field terms are formed in units of the distance and the cell size)."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.mixture8(200_000, seed=21)
    P = torch.tensor(pos * scale, device="cuda")
    Q = torch.tensor(q, device="cuda")
    idx = torch.arange(200_000, device="cuda")
    out = {}
    for precision in ("fp64", "mixed"):
        tree = FlatQuadtree(P, Q, Quad(0, 0, scale), kernel=kernel, order=12,
                            precision=precision)
        out[precision] = tree.evaluate(P, exclude=idx, theta=0.5, softening=eps * scale)
    for comp in (0, 1):
        assert relative(out["mixed"][comp].cpu().numpy(), out["fp64"][comp].cpu().numpy()) < TOL


@pytest.mark.parametrize("kernel,scale", [("log", 1e-12), ("log", 1e9), ("coulomb", 1e-12)])
def test_mixed_fmm_and_backward_at_extreme_length_scales(kernel, scale):
    """The mixed FMM works in units of the root half-width: at length scales far from 1
    its fields, potentials and gradients stay within 1e-6 of FP64."""
    from tree_d_3d_b200 import Quad, synthetic
    from tree_d_3d_b200.autograd import fmm_field

    pos, q = synthetic.mixture8(100_000, seed=31)
    rng = np.random.default_rng(32)
    w = torch.tensor(rng.normal(size=pos.shape[1]), device="cuda")
    e = torch.tensor(rng.normal(size=pos.shape), device="cuda")
    eps = 1e-3 * scale if kernel == "coulomb" else 0.0
    out = {}
    for precision in ("fp64", "mixed"):
        P = torch.tensor(pos * scale, device="cuda", requires_grad=True)
        Q = torch.tensor(q, device="cuda", requires_grad=True)
        phi, field = fmm_field(P, Q, Quad(0, 0, scale), kernel=kernel, order=12,
                               softening=eps, precision=precision)
        ((w * phi).sum() + (e * field).sum()).backward()
        out[precision] = [t.detach().cpu().numpy() for t in (phi, field, Q.grad, P.grad)]
    for a, b in zip(out["mixed"], out["fp64"]):
        assert relative(a, b) < TOL


@pytest.mark.parametrize("order", [4, 8, 12, 15])
def test_tensor_core_m2l_matches_cuda_core_m2l_and_fp64(order, monkeypatch):
    """The M2L matrix products on the tensor cores (3xTF32, tcgen05) give the locals of
    the FP32 CUDA-core form and of FP64 to FP32 accuracy, and the same bits every run
    (fixed summation order per destination)."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, flat_tree, synthetic

    monkeypatch.setattr(flat_tree, "M2L_GROUPED", False)  # the per-translation forms
    pos, q = synthetic.mixture8(150_000, seed=40 + order)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    ref = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=order)
    lists = ref._lists(0.5)
    fp64 = [t.cpu().numpy() for t in ref._log_locals(lists)]
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=order, precision="mixed")
    lists = tree._lists(0.5)
    runs = {}
    for tensor in (True, False):
        monkeypatch.setattr(flat_tree, "M2L_TENSOR_CORES", tensor)
        runs[tensor] = [t.cpu().numpy() for t in tree._log_locals(lists)]
        tree._check_tensor_cores()
    monkeypatch.setattr(flat_tree, "M2L_TENSOR_CORES", True)
    again = [t.cpu().numpy() for t in tree._log_locals(lists)]
    for part in (0, 1):
        assert relative(runs[True][part], fp64[part]) < 1e-6
        assert relative(runs[True][part], runs[False][part]) < 1e-6
        assert np.array_equal(again[part], runs[True][part])


@pytest.mark.parametrize("order", [4, 8, 12, 16])
def test_mixed_cartesian_m2l_matches_fp64(order):
    """The FP32 Cartesian M2L on size-scaled expansions (td3_cart_m2l_mixed) against the
    FP64 one on the same lists and moments: the locals to FP32 accuracy."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, synthetic

    pos, q = synthetic.mixture8(120_000, seed=50 + order)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    out = {}
    for precision in ("fp64", "mixed"):
        tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="coulomb", order=order,
                            precision=precision)
        lists = tree._lists(0.5)
        out[precision] = tree._cart_locals(lists["m2l_rows"], lists["m2l_partners"],
                                           lists["m2l"].shape[0], tree, 1e-3).cpu().numpy()
    assert relative(out["mixed"], out["fp64"]) < TOL
