"""The square cells of the quadtrees (src/tree_d_3d/quad.py:6-63)."""

from __future__ import annotations


class Quad:
    """A square cell: centre (xmid, ymid) and half-width half."""

    xmid: float
    ymid: float
    half: float

    def __init__(self, x_mid: float, y_mid: float, half_size: float) -> None:
        self.xmid = x_mid
        self.ymid = y_mid
        self.half = half_size

    def contains(self, x: float, y: float) -> bool:
        """Closed-box membership, as the walks' inside test."""
        return (
            x >= self.xmid - self.half
            and x <= self.xmid + self.half
            and y >= self.ymid - self.half
            and y <= self.ymid + self.half
        )

    def northwest(self) -> Quad:
        return Quad(self.xmid - self.half / 2.0, self.ymid + self.half / 2.0, self.half / 2.0)

    def northeast(self) -> Quad:
        return Quad(self.xmid + self.half / 2.0, self.ymid + self.half / 2.0, self.half / 2.0)

    def southwest(self) -> Quad:
        return Quad(self.xmid - self.half / 2.0, self.ymid - self.half / 2.0, self.half / 2.0)

    def southeast(self) -> Quad:
        return Quad(self.xmid + self.half / 2.0, self.ymid - self.half / 2.0, self.half / 2.0)

    def __repr__(self) -> str:
        return f"Quad({self.xmid!r}, {self.ymid!r}, {self.half!r})"
