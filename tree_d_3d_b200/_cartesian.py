"""Index tables of the Cartesian expansions of the Coulomb FMM.

The same format as the reference's tables (src/tree_d_3d/_cartesian.py:29-107), which
the kernels read as flat lists of terms: a coefficient of multi-index (a, b), the
powers of x and y, sits at n (n + 1) / 2 + b with n = a + b <= p.

* moments of a cell about its centre c: m_a = sum_j q_j (r_j - c)^a;
* local expansion: phi(c + u) = sum_b T_b u^b;
* Taylor coefficients A_g(t) = D^g f(t) / g! of f = (x^2 + y^2 + eps^2)^(-1/2), by
  n R^2 A_g = -(2n - 1)(t_x A_{g-e_x} + t_y A_{g-e_y}) - (n - 1)(A_{g-2e_x} + A_{g-2e_y});
* M2L: T_b += sum_a (-1)^|a| C(a + b, a) m_a A_{a+b}, |a| + |b| <= p;
* M2M / L2L: shifts by s with the binomial C(g, b) s^(g - b).
"""

from __future__ import annotations

from math import comb

import numpy as np

_CACHE: dict = {}


def size(order: int) -> int:
    """Coefficients of total degree at most ``order``."""
    return (order + 1) * (order + 2) // 2


def index(a: int, b: int) -> int:
    """Position of coefficient (a, b)."""
    n = a + b
    return n * (n + 1) // 2 + b


def _pos(a: int, b: int) -> int:
    return index(a, b) if a >= 0 and b >= 0 else -1


def tables(order: int) -> dict:
    """The tables of ``order`` (cached): ex, ey, mono_parent, mono_dir, rec, grad,
    m2l rows (b, a, a+b) sorted by b with m2l_coef, shift rows (g, b, g-b) sorted by g
    with shift_coef; plus the row offsets m2l_start / shift_start per b / g."""
    if order in _CACHE:
        return _CACHE[order]
    n_coef = size(order)
    powers = [(n - b, b) for n in range(order + 1) for b in range(n + 1)]
    ex = np.array([a for a, _ in powers], dtype=np.int64)
    ey = np.array([b for _, b in powers], dtype=np.int64)
    mono_parent = np.zeros(n_coef, dtype=np.int64)
    mono_dir = np.zeros(n_coef, dtype=np.int64)
    rec = np.full((n_coef, 4), -1, dtype=np.int64)
    grad = np.full((n_coef, 2), -1, dtype=np.int64)
    for i, (a, b) in enumerate(powers):
        if a:
            mono_parent[i], mono_dir[i] = _pos(a - 1, b), 0
        elif b:
            mono_parent[i], mono_dir[i] = _pos(a, b - 1), 1
        rec[i] = (_pos(a - 1, b), _pos(a, b - 1), _pos(a - 2, b), _pos(a, b - 2))
        grad[i] = (_pos(a - 1, b), _pos(a, b - 1))
    m2l_rows, m2l_coef, m2l_start = [], [], [0]
    for ib, (bx, by) in enumerate(powers):
        for ia in range(size(order - bx - by)):
            ax, ay = powers[ia]
            m2l_rows.append((ib, ia, index(ax + bx, ay + by)))
            m2l_coef.append(float((-1) ** (ax + ay) * comb(ax + bx, ax) * comb(ay + by, ay)))
        m2l_start.append(len(m2l_rows))
    shift_rows, shift_coef, shift_start = [], [], [0]
    for ig, (gx, gy) in enumerate(powers):
        for bx in range(gx + 1):
            for by in range(gy + 1):
                shift_rows.append((ig, index(bx, by), index(gx - bx, gy - by)))
                shift_coef.append(float(comb(gx, bx) * comb(gy, by)))
        shift_start.append(len(shift_rows))
    # L2L by output coefficient: the shift rows of each b, in g order
    by_b = sorted(range(len(shift_rows)), key=lambda r: shift_rows[r][1])
    l2l_start = np.zeros(n_coef + 1, dtype=np.int32)
    for r in by_b:
        l2l_start[shift_rows[r][1] + 1] += 1
    l2l_start = np.cumsum(l2l_start).astype(np.int32)
    m2l_arr = np.array(m2l_rows, dtype=np.int64)
    out = {
        "m2l_a": m2l_arr[:, 1].astype(np.int32),
        "m2l_g": m2l_arr[:, 2].astype(np.int32),
        "m2l_start32": np.array(m2l_start, dtype=np.int32),
        "l2l_start": l2l_start,
        "l2l_g": np.array([shift_rows[r][0] for r in by_b], dtype=np.int32),
        "l2l_d": np.array([shift_rows[r][2] for r in by_b], dtype=np.int32),
        "l2l_coef": np.array([shift_coef[r] for r in by_b]),
        "ex": ex,
        "ey": ey,
        "mono_parent": mono_parent,
        "mono_dir": mono_dir,
        "rec": rec,
        "grad": grad,
        "m2l": np.array(m2l_rows, dtype=np.int64),
        "m2l_coef": np.array(m2l_coef),
        "m2l_start": np.array(m2l_start, dtype=np.int64),
        "shift": np.array(shift_rows, dtype=np.int64),
        "shift_coef": np.array(shift_coef),
        "shift_start": np.array(shift_start, dtype=np.int64),
    }
    _CACHE[order] = out
    return out
