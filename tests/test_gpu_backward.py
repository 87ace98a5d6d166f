"""The hand-written backward of the FMM field against exact gradients.

* U = 1/2 sum q phi: dU/dq = phi and dU/dx = -q E exactly; compared with the FP64
  direct sum;
* a general loss L = sum w phi + sum e . E: compared with torch autograd through a plain
  PyTorch FP64 direct-sum reference of the same kernel;
* central finite differences (h = 1e-6) on 64 seeded coordinates of N = 100k, with the
  tree topology frozen (positions moved within their cells).
The backward is the FMM approximation of the exact gradient, so it agrees with each to
the FMM's truncation error (about 1e-8 at p = 12): 1e-6 normwise, 1e-5 per coordinate
against finite differences.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("kernel,eps", [("log", 0.0), ("coulomb", 1e-3)])
def test_energy_gradient_matches_the_direct_sum(kernel, eps):
    from tree_d_3d_b200 import Quad, direct_field
    from tree_d_3d_b200.autograd import fmm_energy

    rng = np.random.default_rng(4)
    n = 20_000
    pos = torch.tensor(rng.uniform(-1, 1, (2, n)), device="cuda", requires_grad=True)
    q = torch.tensor(rng.normal(size=n), device="cuda", requires_grad=True)
    u = fmm_energy(pos, q, Quad(0, 0, 1), kernel=kernel, order=12, softening=eps)
    u.backward()
    phi, field = direct_field(pos.detach(), pos.detach(), q.detach(), softening=eps,
                              exclude=torch.arange(n, device="cuda"), kernel=kernel)
    assert relative(_np(q.grad), _np(phi)) < 1e-6
    assert relative(_np(pos.grad), _np(-q.detach() * field)) < 1e-6
    u = float(u.detach())
    assert abs(u - 0.5 * float((q.detach() * phi).sum())) < 1e-6 * abs(u)


def _torch_direct(pos, q, kernel, eps):
    """phi, E at every particle (own charge excluded) by plain PyTorch FP64 ops."""
    d = pos[:, :, None] - pos[:, None, :]
    r2 = d[0] ** 2 + d[1] ** 2 + eps * eps
    eye = torch.eye(pos.shape[1], dtype=torch.bool, device=pos.device)
    r2 = torch.where(eye, torch.ones_like(r2), r2)
    qj = torch.where(eye, torch.zeros_like(r2), q[None, :].expand_as(r2))
    if kernel == "log":
        phi = -(qj * torch.log(r2)).sum(1)
        e = (2 * qj / r2)[None] * d
    else:
        inv = r2.rsqrt()
        phi = (qj * inv).sum(1)
        e = (qj * inv ** 3)[None] * d
    return phi, e.sum(2)


@pytest.mark.parametrize("kernel,eps", [("log", 0.0), ("coulomb", 0.01)])
def test_vector_jacobian_product_matches_torch_autograd_of_the_direct_sum(kernel, eps):
    """The position gradient carries Hessians, one derivative more than the field, so
    its truncation error is larger: it must fall with the order and end below 1e-6."""
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.autograd import fmm_field

    rng = np.random.default_rng(9)
    n = 3000
    pos0 = np.concatenate((rng.normal(0.2, 0.1, (2, n // 2)), rng.uniform(-0.9, 0.9, (2, n - n // 2))),
                          axis=1).clip(-0.99, 0.99)
    q0 = rng.normal(size=n)
    w = torch.tensor(rng.normal(size=n), device="cuda")
    e = torch.tensor(rng.normal(size=(2, n)), device="cuda")

    def grads(order):
        pos = torch.tensor(pos0, device="cuda", requires_grad=True)
        q = torch.tensor(q0, device="cuda", requires_grad=True)
        if order is None:
            phi, field = _torch_direct(pos, q, kernel, eps)
        else:
            phi, field = fmm_field(pos, q, Quad(0, 0, 1), kernel=kernel, order=order, theta=0.5,
                                   softening=eps)
        ((w * phi).sum() + (e * field).sum()).backward()
        return _np(q.grad), _np(pos.grad)

    exact = grads(None)
    errors = []
    for order in (10, 14, 20):
        got = grads(order)
        errors.append((relative(got[0], exact[0]), relative(got[1], exact[1])))
    assert errors[-1][0] < 1e-6 and errors[-1][1] < 1e-6
    assert errors[0][1] > errors[1][1] > errors[2][1]


@pytest.mark.parametrize("kernel", ["log", "coulomb"])
def test_backward_matches_central_finite_differences(kernel):
    """Config-4 style: N = 100k uniform, q ~ N(0, 1), p = 12, 64 seeded coordinates."""
    from tree_d_3d_b200 import FlatQuadtree, Quad
    from tree_d_3d_b200.autograd import fmm_field

    rng = np.random.default_rng(12)
    n = 100_000
    eps = 1e-3 if kernel == "coulomb" else 0.0
    pos0 = torch.tensor(rng.uniform(-1, 1, (2, n)), device="cuda")
    q0 = torch.tensor(rng.normal(size=n), device="cuda")
    w = torch.tensor(rng.normal(size=n), device="cuda")
    e = torch.tensor(rng.normal(size=(2, n)), device="cuda")
    opts = dict(kernel=kernel, order=12, theta=0.5, softening=eps)
    pos = pos0.clone().requires_grad_(True)
    q = q0.clone().requires_grad_(True)
    phi, field = fmm_field(pos, q, Quad(0, 0, 1), **opts)
    ((w * phi).sum() + (e * field).sum()).backward()
    tree = FlatQuadtree(pos0, q0, Quad(0, 0, 1), kernel=kernel, order=12)

    def loss(p, c):
        tree._move_within_cells(p)
        tree.set_charges(c)
        a, b = tree.fmm(theta=0.5, softening=eps)
        return float((w * a).sum() + (e * b).sum())

    h = 1e-6
    picks = rng.choice(n, 64, replace=False)
    fd_x, bw_x, fd_q, bw_q = [], [], [], []
    for k, i in enumerate(picks):
        axis = k % 2
        p_plus, p_minus = pos0.clone(), pos0.clone()
        p_plus[axis, i] += h
        p_minus[axis, i] -= h
        try:
            fd_x.append((loss(p_plus, q0) - loss(p_minus, q0)) / (2 * h))
        except ValueError:  # moved across a cell boundary: topology not frozen
            continue
        bw_x.append(float(pos.grad[axis, i]))
    for i in picks[:16]:
        c_plus, c_minus = q0.clone(), q0.clone()
        c_plus[i] += h
        c_minus[i] -= h
        fd_q.append((loss(pos0, c_plus) - loss(pos0, c_minus)) / (2 * h))
        bw_q.append(float(q.grad[i]))
    assert len(fd_x) >= 48
    fd_x, bw_x = np.array(fd_x), np.array(bw_x)
    assert np.max(np.abs(fd_x - bw_x)) < 1e-5 * np.max(np.abs(bw_x))
    fd_q, bw_q = np.array(fd_q), np.array(bw_q)
    assert np.max(np.abs(fd_q - bw_q)) < 1e-5 * np.max(np.abs(bw_q))


def test_coincident_charges_are_reported_at_forward_or_after_backward():
    """Without gradients fmm_field raises at the forward like FlatQuadtree.fmm; with
    gradients the same ValueError comes at the end of the backward (the forward does
    not wait for the GPU)."""
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.autograd import fmm_field

    rng = np.random.default_rng(5)
    pos = rng.uniform(-0.9, 0.9, (2, 3000))
    pos[:, 1] = pos[:, 0]  # two charged particles on one point, unsoftened
    q = np.ones(3000)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    with pytest.raises(ValueError, match="Coincident"):
        fmm_field(P, Q, Quad(0, 0, 1), kernel="log", order=8)
    Qg = Q.clone().requires_grad_(True)
    phi, _ = fmm_field(P, Qg, Quad(0, 0, 1), kernel="log", order=8)
    with pytest.raises(ValueError, match="Coincident"):
        phi.sum().backward()
