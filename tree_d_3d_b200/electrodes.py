"""The multipole products of the boundary-integral electrode solver, on the GPU.

The reference's ``BoundaryIntegralElectrodes`` (src/tree_d_3d/electrodes.py:514-1536)
solves for panel charges with GMRES whose every product is a free-space log sum from
charges on fixed source points (panel quadrature nodes) to fixed target points (panel
midpoints): ``_tree_sum`` (:1140-1160) keeps one tree per geometry and only sets new
charges on it (``set_charges``), and ``_sum_at`` (:267-271) sums by the FMM at the
targets (``fmm_at``, whose target tree and interaction lists are kept while the
targets stay the same) or, at few targets, by the Barnes-Hut walk.  The panel geometry
itself comes from simgeometry, which is not part of this package: ``PanelSums`` takes
the points as arrays.  Constants and rules are the reference's (:70-80).
"""

from __future__ import annotations

import numpy as np
import torch

from tree_d_3d_b200._utils import _device, _points, out, wants_numpy
from tree_d_3d_b200.flat_tree import FlatQuadtree
from tree_d_3d_b200.quad import Quad

#: Opening angle and leaf size of the panels' multipole sums (electrodes.py:70-76).
FMM_AT_THETA: float = 0.5
FMM_LEAF: int = 16
#: A sum at fewer targets than the sources over this ratio walks the tree instead, at
#: WALK_THETA (electrodes.py:77-79).
FMM_AT_RATIO: int = 8
WALK_THETA: float = 0.7
#: Expansion order of the panel solver's trees (its ``fmm_order`` default).
FMM_ORDER: int = 32


def _sum_at(tree: FlatQuadtree, points: torch.Tensor, exclude: torch.Tensor):
    """The raw sum of ``tree`` at ``points``: the FMM at many points, the walk at a few
    (electrodes.py:267-271)."""
    if points.shape[1] * FMM_AT_RATIO >= tree.pos.shape[1]:
        return tree.fmm_at(points, exclude=exclude, theta=FMM_AT_THETA)
    return tree.evaluate(points, exclude=exclude, theta=WALK_THETA)


def bounding_quad(points: torch.Tensor) -> Quad:
    """The root cell of a panel tree: the points' bounding square, widened by a relative
    1e-9 (electrodes.py:1143-1146)."""
    low = points.amin(dim=1).tolist()
    high = points.amax(dim=1).tolist()
    half = 0.5 * max(high[0] - low[0], high[1] - low[1]) * (1.0 + 1e-9) + 1e-300
    return Quad(0.5 * (low[0] + high[0]), 0.5 * (low[1] + high[1]), half)


class PanelSums:
    """Repeated log-kernel sums from charges on fixed ``sources`` (2, N) to fixed
    ``targets`` (2, M), the products of the electrode solver's iterations.

    The first product builds the tree of the sources (root: their bounding square;
    ``order`` and ``leaf_capacity`` the solver's) and, through ``fmm_at``, the target
    tree and the dual lists; later products only set the new charges and sum again.
    ``exclude[i]`` is a source index left out of target ``i`` (a target on a source
    node); -1 for none.  Returns the raw potential and field, without k_e, as
    ``direct_field(targets, sources, charges, kernel="log", exclude=exclude)`` would.
    """

    def __init__(self, sources, targets, *, exclude=None, order: int = FMM_ORDER,
                 leaf_capacity: int = FMM_LEAF, precision: str = "fp64") -> None:
        self.sources = _points(sources, "sources")
        self.targets = _points(targets, "targets")
        m = self.targets.shape[1]
        if exclude is None:
            exclude = torch.full((m,), -1, dtype=torch.int64, device=self.targets.device)
        self.exclude = _device(exclude, torch.int64).reshape(-1)
        if self.exclude.shape[0] != m:
            raise ValueError("exclude must have one entry per target")
        self.order = int(order)
        self.leaf_capacity = int(leaf_capacity)
        self.precision = precision
        self.tree: FlatQuadtree | None = None
        self.products = 0

    def __call__(self, charges):
        as_numpy = wants_numpy(charges)
        charges = _device(charges).reshape(-1)
        if charges.shape[0] != self.sources.shape[1]:
            raise ValueError("charges must have one entry per source")
        if self.tree is None:
            self.tree = FlatQuadtree(self.sources, charges, bounding_quad(self.sources),
                                     kernel="log", order=self.order,
                                     leaf_capacity=self.leaf_capacity,
                                     precision=self.precision)
        else:
            self.tree.set_charges(charges)
        self.products += 1
        return out(_sum_at(self.tree, self.targets, self.exclude), as_numpy)

    def matvec(self, charges) -> np.ndarray:
        """The potential at the targets (NumPy), for an iterative solver."""
        phi, _ = self(np.asarray(charges, dtype=float))
        return np.asarray(phi)

    def as_operator(self):
        """A SciPy LinearOperator (targets x sources) applying ``matvec``."""
        from scipy.sparse.linalg import LinearOperator

        shape = (self.targets.shape[1], self.sources.shape[1])
        return LinearOperator(shape, matvec=lambda x: self.matvec(np.ravel(x)), dtype=float)
