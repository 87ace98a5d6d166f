"""Differentiable FMM fields: a hand-written backward behind torch.autograd.Function.

``fmm_field(positions, charges, root_quad, ...)`` returns the potential (N,) and field
(2, N) at the sources (``FlatQuadtree.fmm``) as tensors that carry gradients to the
positions (2, N) and the charges (N,).  ``fmm_energy`` is U = 1/2 sum q phi.

The backward of a loss L(phi, E) with w = dL/dphi and e = dL/dE is
    dL/dq_k = Psi(x_k),   dL/dx_k = -w_k E_k + q_k grad Psi(x_k) - (sum_j q_j Hess G) e_k,
Psi the potential of monopoles w and dipoles e at the sources: one transposed FMM pass
(the kernel is symmetric) with dipole terms in P2M, value and gradient in L2P, plus
the Hessian of the forward expansions and kernel Hessian-vector products in P2P
(``FlatQuadtree._fmm_adjoint``).  The tree and its interaction lists are built in the
forward and kept for the backward; the tree topology is not differentiated.

When the positions or charges require gradients, the check for coincident charges of
the forward (the ValueError of ``FlatQuadtree.fmm``) is read at the end of the backward,
so that the host queues the loss and the backward without waiting for the GPU; call
without gradients for the check at the forward.
"""

from __future__ import annotations

import torch

from tree_d_3d_b200._utils import _check, status_word
from tree_d_3d_b200.flat_tree import FlatQuadtree
from tree_d_3d_b200.quad import Quad


class _FMMField(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, charges, root, options):
        tree = FlatQuadtree(positions.detach(), charges.detach(), root,
                            kernel=options["kernel"], order=options["order"],
                            leaf_capacity=options["leaf_capacity"],
                            max_depth=options["max_depth"], symmetric=options["symmetric"],
                            precision=options["precision"])
        # with gradients on, the forward's coincident-charge report is read after the
        # backward has been queued, so the host does not wait for the GPU here
        deferred = any(ctx.needs_input_grad[:2])
        status = status_word(tree.device) if deferred else None
        phi, field = tree.fmm(theta=options["theta"], softening=options["softening"],
                              _status=status)
        ctx.tree = tree
        ctx.status = status
        ctx.options = options
        ctx.save_for_backward(field)
        return phi, field

    @staticmethod
    def backward(ctx, grad_phi, grad_field):
        (field,) = ctx.saved_tensors
        tree = ctx.tree
        ctx.tree = None  # the tree's buffers go as soon as the backward is done
        n = field.shape[1]
        if grad_phi is None:
            grad_phi = torch.zeros(n, dtype=torch.float64, device=field.device)
        if grad_field is None:
            grad_field = torch.zeros_like(field)
        qbar, xbar = tree._fmm_adjoint(ctx.options["theta"], ctx.options["softening"],
                                       grad_phi.contiguous(), grad_field.contiguous(), field)
        if ctx.status is not None:
            _check(ctx.status)
            tree._check_tensor_cores()
        return xbar, qbar, None, None


def fmm_field(positions: torch.Tensor, charges: torch.Tensor, root_quad: Quad, *,
              kernel: str = "log", order: int | None = None, theta: float = 0.5,
              softening: float = 0.0, leaf_capacity: int = 8, max_depth: int = 48,
              symmetric: bool = False, precision: str = "fp64"):
    """Differentiable (phi, field) at the sources by the FMM (see the module doc)."""
    options = {"kernel": kernel, "order": order, "theta": float(theta),
               "softening": float(softening), "leaf_capacity": leaf_capacity,
               "max_depth": max_depth, "symmetric": symmetric, "precision": precision}
    return _FMMField.apply(positions, charges, root_quad, options)


def fmm_energy(positions: torch.Tensor, charges: torch.Tensor, root_quad: Quad, **options):
    """U = 1/2 sum_i q_i phi_i (each particle's own charge excluded), differentiable."""
    phi, _ = fmm_field(positions, charges, root_quad, **options)
    return 0.5 * torch.sum(charges * phi)
