r"""Line charges between two grounded plates, by conformal mapping and the FMM.

Mirrors ``GroundedStripField`` of the reference (src/tree_d_3d/strip.py:115-327): line
charges in the strip ``0 < x < L`` between grounded plates at ``x = 0`` and ``x = L``.
The map ``zeta = exp(i pi z / L)`` sends the strip onto the upper half-plane, where each
charge has one image (``-q`` at ``conj(zeta)``), so the strip's potential is one
free-space log sum over 2N sources, evaluated by the FMM (or the Barnes-Hut walk at
probes, or the direct sum).  The map, the way back (with each charge's own regular
term: the image force of the plates) and the physical-plane softening of close pairs
run in libtreed3d.so (``td3_strip_map``, ``td3_strip_assemble``, ``td3_soften``); the
close pairs are found on the device on a hashed grid of the cutoff radius instead of the
reference's host k-d tree.  Tensor inputs give CUDA tensor results, NumPy inputs NumPy
results.
"""

from __future__ import annotations

import numpy as np
import torch

from tree_d_3d_b200 import _lib
from tree_d_3d_b200._utils import _device, out, status_word, wants_numpy
from tree_d_3d_b200.constants import K_E
from tree_d_3d_b200.flat_tree import FlatQuadtree, direct_field
from tree_d_3d_b200.quad import Quad


class GroundedStripField:
    """Field and potential of line charges between plates at x = 0 and x = L
    (strip.py:115-145: the same arguments, defaults and messages)."""

    def __init__(self, width: float, *, order: int = 14, theta: float = 0.5,
                 leaf_capacity: int = 32, k_e: float = K_E, method: str = "fmm",
                 softening: float = 0.0, cutoff: float = 6.0) -> None:
        if not np.isfinite(width) or width <= 0:
            raise ValueError("width must be finite and positive")
        if method not in ("fmm", "direct"):
            raise ValueError("method must be 'fmm' or 'direct'")
        self.width = float(width)
        self.order = int(order)
        self.theta = float(theta)
        self.leaf_capacity = int(leaf_capacity)
        self.k_e = float(k_e)
        self.method = method
        if not np.isfinite(softening) or softening < 0:
            raise ValueError("softening must be finite and nonnegative")
        if not cutoff > 1:
            raise ValueError("cutoff must exceed 1")
        self.softening = float(softening)
        self.cutoff = float(cutoff)

    # ------------------------------------------------------------------ the map
    def _map(self, points: torch.Tensor, charges: torch.Tensor | None):
        """td3_strip_map: the mapped points (2, n), or with ``charges`` the (2, 2n)
        charges-then-images and their charges; raises for a point off the strip."""
        n = points.shape[1]
        dev = points.device
        cols = 2 * n if charges is not None else n
        mapped = torch.empty((2, cols), dtype=torch.float64, device=dev)
        q = torch.empty(cols, dtype=torch.float64, device=dev) if charges is not None else None
        status = status_word(dev)
        _lib.call("td3_strip_map", points.data_ptr(), n, self.width,
                  charges.data_ptr() if charges is not None else 0, mapped.data_ptr(),
                  q.data_ptr() if q is not None else 0, status.data_ptr(), _lib.stream(dev))
        if int(status[0].item()):
            raise ValueError("Charges must lie strictly between the plates")
        return mapped, q

    def to_plane(self, positions):
        """zeta = exp(i pi z / L) as a complex array; ``positions`` is ``(2, N)``
        (strip.py:147-152)."""
        as_numpy = wants_numpy(positions)
        points = _device(positions).reshape(2, -1)
        mapped, _ = self._map(points, None)
        zeta = torch.complex(mapped[0], mapped[1])
        return zeta.cpu().numpy() if as_numpy else zeta

    @staticmethod
    def _root(xy: torch.Tensor) -> Quad:
        """strip.py:165-170: the square around the mapped points."""
        lo, hi = xy.amin(dim=1).tolist(), xy.amax(dim=1).tolist()
        centre = ((lo[0] + hi[0]) / 2, (lo[1] + hi[1]) / 2)
        half = float(max(hi[0] - lo[0], hi[1] - lo[1]) / 2) * (1 + 1e-9) + 1e-300
        return Quad(float(centre[0]), float(centre[1]), half)

    def _soften(self, targets, sources, charge, same, potential, phi, field, message):
        """td3_soften: close pairs softened (when softening > 0), then the k_e scale."""
        dev = targets.device
        status = status_word(dev)
        n = sources.shape[1]
        ws = _lib.workspace(_lib.query("td3_soften_workspace_size", n), dev)
        _lib.call("td3_soften", targets.data_ptr(), targets.shape[1], sources.data_ptr(),
                  charge.data_ptr(), n, 1 if same else 0, self.cutoff * self.softening,
                  self.softening, 1 if potential else 0, self.k_e, phi.data_ptr(),
                  field.data_ptr(), status.data_ptr(), ws.data_ptr(), ws.numel(),
                  _lib.stream(dev))
        if self.softening > 0 and int(status[0].item()):
            raise ValueError(message)

    # ------------------------------------------------------------------ at the charges
    def field_at_charges(self, positions, charges, *, potential: bool = True):
        """Potential (V) and field (V/m, shape (2, N)) acting on every charge
        (strip.py:203-250): all other charges and every image, including the charge's
        own (the image force of the plates)."""
        as_numpy = wants_numpy(positions)
        pos = _device(positions).reshape(2, -1)
        q = _device(charges).reshape(-1)
        n = pos.shape[1]
        dev = pos.device
        if q.shape[0] != n:
            # the reference maps first (a point off the strip is reported before this)
            self._map(pos, None)
            raise ValueError("positions and charges must have the same length")
        if not n:
            return out((torch.zeros(0, dtype=torch.float64, device=dev),
                        torch.zeros((2, 0), dtype=torch.float64, device=dev)), as_numpy)
        xy, sq = self._map(pos, q)
        if self.method == "fmm":
            tree = FlatQuadtree(xy, sq, self._root(xy), kernel="log", order=self.order,
                                leaf_capacity=self.leaf_capacity)
            phi_raw, raw = tree.fmm(theta=self.theta, potential=potential)
        else:
            exclude = torch.arange(2 * n, dtype=torch.int64, device=dev)
            phi_raw, raw = direct_field(xy, xy, sq, exclude=exclude, kernel="log")
        phi = torch.empty(n, dtype=torch.float64, device=dev)
        field = torch.empty((2, n), dtype=torch.float64, device=dev)
        _lib.call("td3_strip_assemble", xy.data_ptr(), 2 * n, n, self.width, q.data_ptr(),
                  phi_raw.data_ptr(), raw.data_ptr(), 2 * n, 1 if potential else 0,
                  phi.data_ptr(), field.data_ptr(), _lib.stream(dev))
        self._soften(pos, pos, q, True, potential, phi, field, "Coincident charges")
        return out((phi, field), as_numpy)

    # ------------------------------------------------------------------ at probes
    def potential(self, positions, charges, points):
        """Potential (V) at arbitrary ``points`` strictly between the plates."""
        return self.probe(positions, charges, points)[0]

    def probe(self, positions, charges, points):
        """Potential (V) and field (V/m, shape (2, M)) at ``points`` ``(2, M)``
        (strip.py:256-327); probes are not charges, so no self term applies."""
        as_numpy = wants_numpy(points)
        pos = _device(positions).reshape(2, -1)
        q = _device(charges).reshape(-1)
        targets = _device(points).reshape(2, -1)
        dev = targets.device
        if q.shape[0] != pos.shape[1]:
            self._map(pos, None)
            raise ValueError("positions and charges must have the same length")
        xy, sq = self._map(pos, q) if pos.shape[1] else (None, None)
        probes, _ = self._map(targets, None)
        m = probes.shape[1]
        if xy is None:
            return out((torch.zeros(m, dtype=torch.float64, device=dev),
                        torch.zeros((2, m), dtype=torch.float64, device=dev)), as_numpy)
        if self.method == "fmm":
            everything = torch.cat((xy, probes), dim=1)
            tree = FlatQuadtree(xy, sq, self._root(everything), kernel="log", order=self.order,
                                leaf_capacity=self.leaf_capacity)
            phi_raw, raw = tree.evaluate(probes, theta=self.theta)
        else:
            phi_raw, raw = direct_field(probes, xy, sq, kernel="log")
        phi = torch.empty(m, dtype=torch.float64, device=dev)
        field = torch.empty((2, m), dtype=torch.float64, device=dev)
        _lib.call("td3_strip_assemble", probes.data_ptr(), m, m, self.width, 0,
                  phi_raw.data_ptr(), raw.data_ptr(), m, 1, phi.data_ptr(), field.data_ptr(),
                  _lib.stream(dev))
        self._soften(targets, pos, q, False, True, phi, field,
                     "A probe coincides with a charge")
        return out((phi, field), as_numpy)


__all__ = ["GroundedStripField"]
