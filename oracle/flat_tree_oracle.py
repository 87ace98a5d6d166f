"""CPU oracle of the field solver: the reference's CPU orchestration on NumPy arrays.

TEST INFRASTRUCTURE ONLY.  This module restates, step by step, the CPU code path of
the reference's ``FlatQuadtree`` (max-models/tree-d-3d,
``src/tree_d_3d/flat_tree.py``) and calls the C restatement of its kernels
(``oracle/oracle.c``).  It is imported by the tests (as the checker), by
``__graft_entry__.smoke`` and by ``bench.py``'s CPU baseline; the product never
imports it.

Every function cites the reference lines it follows; ``ft`` is
``src/tree_d_3d/flat_tree.py``.
"""

from __future__ import annotations

import ctypes
import os
import re
from math import comb

import numpy as np

from oracle.build import build as _build_library

_LIB = None
_P = ctypes.c_void_p
_I = ctypes.c_int64
_D = ctypes.c_double
_C = ctypes.c_int

#: C parameter types -> ctypes codes (pointer P, int64 I, double D, int C)
_TYPES = {"P": _P, "I": _I, "D": _D, "C": _C}


def _signatures(source: str) -> dict:
    """The ctypes argument codes of every ``void name(...)`` in ``oracle.c``."""
    out = {}
    for match in re.finditer(r"^void (\w+)\(([^)]*)\)", source, re.M):
        codes = []
        for param in match.group(2).split(","):
            param = " ".join(param.split())
            if "*" in param:
                codes.append("P")
            elif param.startswith("i64"):
                codes.append("I")
            elif param.startswith("double"):
                codes.append("D")
            elif param.startswith("int"):
                codes.append("C")
            else:
                raise ValueError(f"unknown parameter type: {param}")
        out[match.group(1)] = "".join(codes)
    return out



MAX_ORDER = 64
LOG_ORDER = 12
COULOMB_ORDER = 4
KERNELS = ("coulomb", "log")


def lib():
    """The C oracle, built on first use (``oracle/build.py``)."""
    global _LIB
    if _LIB is None:
        path = _build_library()
        _LIB = ctypes.CDLL(str(path))
        source = (path.parent / "oracle.c").read_text()
        for name, sig in _signatures(source).items():
            fn = getattr(_LIB, name)
            fn.argtypes = [_TYPES[c] for c in sig]
            fn.restype = None
    return _LIB


def set_threads(n: int) -> None:
    """The OpenMP thread count of the oracle's parallel loops."""
    os.environ["OMP_NUM_THREADS"] = str(int(n))
    try:
        gomp = ctypes.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(ctypes.c_int(int(n)))
    except OSError:
        pass


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(_P)


class CoincidentError(ValueError):
    pass


def _check(status) -> None:
    """ft: `_check` (src/tree_d_3d/_utils.py:26-35)."""
    code = int(status[0])
    if code > 0:
        raise ValueError("Coincident charges require positive softening")
    if code < 0:
        raise RuntimeError("traversal stack overflow")


# ----------------------------------------------------------------------------- tables
def binomial_table(size: int) -> np.ndarray:
    """ft:224-231 `_binomial_table`."""
    table = np.zeros((size, size))
    for row in range(size):
        table[row, 0] = 1.0
        for col in range(1, row + 1):
            table[row, col] = table[row - 1, col - 1] + table[row - 1, col]
    return table


def m2l_coefficients(order: int, symmetric: bool) -> np.ndarray:
    """ft:234-245 `_m2l_coefficients`."""
    binomial = binomial_table(2 * order + 1)
    coeff = np.zeros((order + 1, order + 1))
    for m in range(1, order + 1):
        coeff[0, m] = 1.0 / m
    for k in range(1, order + 1):
        coeff[k, 0] = 1.0 / k
        for m in range(1, order + 1):
            if k <= (order - m if symmetric else order):
                coeff[k, m] = binomial[k + m - 1, m] / k
    return coeff


def cart_size(order: int) -> int:
    """src/tree_d_3d/_cartesian.py:29-31."""
    return (order + 1) * (order + 2) // 2


def cart_index(a: int, b: int) -> int:
    """src/tree_d_3d/_cartesian.py:34-37."""
    n = a + b
    return n * (n + 1) // 2 + b


def cart_tables(order: int) -> dict:
    """src/tree_d_3d/_cartesian.py:40-107 `tables`."""
    n = cart_size(order)
    ex = np.empty(n, dtype=np.int64)
    ey = np.empty(n, dtype=np.int64)
    for deg in range(order + 1):
        for b in range(deg + 1):
            ex[cart_index(deg - b, b)] = deg - b
            ey[cart_index(deg - b, b)] = b

    def at(a, b):
        return cart_index(a, b) if a >= 0 and b >= 0 else -1

    mono_parent = np.zeros(n, dtype=np.int64)
    mono_dir = np.zeros(n, dtype=np.int64)
    rec = np.full((n, 4), -1, dtype=np.int64)
    grad = np.full((n, 2), -1, dtype=np.int64)
    for i in range(n):
        a, b = int(ex[i]), int(ey[i])
        if a > 0:
            mono_parent[i], mono_dir[i] = at(a - 1, b), 0
        elif b > 0:
            mono_parent[i], mono_dir[i] = at(a, b - 1), 1
        rec[i] = (at(a - 1, b), at(a, b - 1), at(a - 2, b), at(a, b - 2))
        grad[i] = (at(a - 1, b), at(a, b - 1))
    m2l, m2l_coef, shift, shift_coef = [], [], [], []
    for ib in range(n):
        bx, by = int(ex[ib]), int(ey[ib])
        for ia in range(cart_size(order - bx - by)):
            ax, ay = int(ex[ia]), int(ey[ia])
            m2l.append((ib, ia, cart_index(ax + bx, ay + by)))
            m2l_coef.append((-1) ** (ax + ay) * comb(ax + bx, ax) * comb(ay + by, ay))
    for ig in range(n):
        gx, gy = int(ex[ig]), int(ey[ig])
        for bx in range(gx + 1):
            for by in range(gy + 1):
                shift.append((ig, cart_index(bx, by), cart_index(gx - bx, gy - by)))
                shift_coef.append(comb(gx, bx) * comb(gy, by))
    return {
        "ex": ex,
        "ey": ey,
        "mono_parent": mono_parent,
        "mono_dir": mono_dir,
        "rec": rec,
        "grad": grad,
        "m2l": np.array(m2l, dtype=np.int64),
        "m2l_coef": np.array(m2l_coef, dtype=float),
        "shift": np.array(shift, dtype=np.int64),
        "shift_coef": np.array(shift_coef, dtype=float),
    }


# ----------------------------------------------------------------------------- direct
def direct_field(targets, pos, charge, *, softening=0.0, exclude=None, kernel="coulomb"):
    """ft:124-160 `direct_field` (CPU path)."""
    targets = np.ascontiguousarray(targets, dtype=float)
    pos = np.ascontiguousarray(pos, dtype=float)
    charge = np.ascontiguousarray(charge, dtype=float).reshape(-1)
    m, n = targets.shape[1], pos.shape[1]
    exclude = (
        np.full(m, -1, dtype=np.int64)
        if exclude is None
        else np.ascontiguousarray(exclude, dtype=np.int64).reshape(-1)
    )
    phi, field = np.zeros(m), np.zeros((2, m))
    if not m or not n:
        return phi, field
    status = np.zeros(1, dtype=np.int64)
    fn = lib().direct_log_sum if kernel == "log" else lib().direct_sum
    fn(_p(targets), m, m, _p(exclude), _p(pos), n, n, _p(charge), float(softening),
       _p(phi), _p(field), m, _p(status))
    _check(status)
    return phi, field


def pair_energy(pos, charge, softening):
    """The pair energy sum q_i q_j / sqrt(r^2 + eps^2) (K/pair_energy/pair_energy_pyccel.py)."""
    pos = np.ascontiguousarray(pos, dtype=float)
    charge = np.ascontiguousarray(charge, dtype=float)
    n = pos.shape[1]
    status, energy = np.zeros(1, dtype=np.int64), np.zeros(1)
    lib().pair_energy(_p(pos), n, n, _p(charge), float(softening), _p(status), _p(energy))
    _check(status)
    return float(energy[0])


# ----------------------------------------------------------------------------- tree
class OracleTree:
    """The reference's FlatQuadtree on the CPU (ft:437-1676), single process."""

    def __init__(self, positions, charges, root, *, leaf_capacity=8, max_depth=48,
                 kernel="coulomb", order=None, symmetric=False):
        # ft:760-800 validation (the subset the oracle needs)
        if kernel not in KERNELS:
            raise ValueError(f"kernel must be one of {KERNELS}")
        if order is None:
            order = LOG_ORDER if kernel == "log" else COULOMB_ORDER
        self.kernel, self.order, self.symmetric = kernel, int(order), bool(symmetric)
        self.root = tuple(float(v) for v in root)
        self.leaf_capacity, self.max_depth = int(leaf_capacity), int(max_depth)
        self.pos = np.ascontiguousarray(positions, dtype=float).copy()
        self.charge = np.ascontiguousarray(charges, dtype=float).reshape(-1).copy()
        n = self.pos.shape[1]
        self._traversals = {}
        self._cart = None
        if not n:
            self._empty()
            return
        count = self._build()
        self.node_count = int(count)
        for name in ("node_center", "node_half", "node_start", "node_end", "node_child",
                     "node_depth"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name)[:count]).copy())
        self._moments()

    def _empty(self):
        """ft:462-481 `_empty`."""
        x, y, h = self.root
        self.perm = np.empty(0, dtype=np.int64)
        self.node_count = 1
        self.node_center = np.array([[x, y]])
        self.node_half = np.array([h])
        self.node_start = np.zeros(1, dtype=np.int64)
        self.node_end = np.zeros(1, dtype=np.int64)
        self.node_child = np.full(1, -1, dtype=np.int64)
        self.node_depth = np.zeros(1, dtype=np.int64)
        self.levels = np.array([0, 1])
        self.node_q = np.zeros(1)
        self.node_qabs = np.zeros(1)
        self.node_p = np.zeros((1, 2))
        self.node_s = np.zeros((1, 3))
        self.moment_re = np.zeros((1, self.order + 1))
        self.moment_im = np.zeros((1, self.order + 1))
        self.sorted_pos = np.zeros((2, 1))

    def _build(self):
        """ft:483-530 `_build_host` with the capacity of ft:545."""
        n = self.pos.shape[1]
        capacity = 4 * (2 * n // self.leaf_capacity + 16)
        perm, slot_node, quadrant, new_perm, new_slot = (
            np.empty(n, dtype=np.int64) for _ in range(5)
        )
        new_sorted = np.empty((2, n + 1))
        sizes = np.zeros(3, dtype=np.int64)
        while True:
            sorted_pos = np.zeros((2, n + 1))
            sorted_pos[:, :n] = self.pos
            self.node_center = np.empty((capacity, 2))
            self.node_half = np.empty(capacity)
            self.node_start = np.empty(capacity, dtype=np.int64)
            self.node_end = np.empty(capacity, dtype=np.int64)
            self.node_child = np.empty(capacity, dtype=np.int64)
            self.node_depth = np.empty(capacity, dtype=np.int64)
            self.node_center[0] = self.root[:2]
            self.node_half[0] = self.root[2]
            levels = np.empty(capacity + 1, dtype=np.int64)
            cursor = np.empty(capacity, dtype=np.int64)
            lib().quadtree_build(
                _p(sorted_pos), n + 1, n, self.leaf_capacity, self.max_depth,
                _p(self.node_center), _p(self.node_half), _p(self.node_start),
                _p(self.node_end), _p(self.node_child), _p(self.node_depth), _p(perm),
                _p(levels), _p(slot_node), _p(quadrant), _p(cursor), capacity,
                _p(new_sorted), n + 1, _p(new_perm), _p(new_slot), _p(sizes))
            if not sizes[2]:
                break
            capacity *= 2
        self.perm = perm
        self.levels = levels[: sizes[1] + 1].copy()
        self.sorted_pos = np.ascontiguousarray(sorted_pos[:, :n])
        return int(sizes[0])

    def _moments(self):
        """ft:663-744 `_moments` (one process on the CPU: the upward kernels)."""
        count = self.node_count
        L = lib()
        n = self.pos.shape[1]
        self.node_q = np.empty(count)
        self.node_qabs = np.empty(count)
        self.node_p = np.empty((count, 2))
        self.node_s = np.empty((count, 3))
        self.stack_size = 3 * int(self.node_depth.max()) + 8
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        if self.kernel == "log":
            self.moment_re = np.empty((count, self.order + 1))
            self.moment_im = np.empty((count, self.order + 1))
            binom = binomial_table(2 * self.order + 1)
            L.log_moments_upward(
                _p(self.pos), n, _p(self.charge), _p(self.perm), _p(levels), len(levels),
                _p(self.node_center), _p(self.node_start), _p(self.node_end),
                _p(self.node_child), _p(binom), binom.shape[0], _p(self.node_qabs),
                _p(self.moment_re), _p(self.moment_im), self.order)
            self.node_q[:] = self.moment_re[:, 0]
            self.node_p[:, 0] = self.moment_re[:, 1]
            self.node_p[:, 1] = self.moment_im[:, 1]
            return
        self.moment_re = np.zeros((1, 1))
        self.moment_im = np.zeros((1, 1))
        L.quadtree_moments_upward(
            _p(self.pos), n, _p(self.charge), _p(self.perm), _p(levels), len(levels),
            _p(self.node_center), _p(self.node_start), _p(self.node_end),
            _p(self.node_child), _p(self.node_q), _p(self.node_qabs), _p(self.node_p),
            _p(self.node_s))

    def set_charges(self, charges):
        """ft:853-868 `set_charges`."""
        self.charge[...] = np.asarray(charges, dtype=float).reshape(-1)
        self._cart = None
        if self.pos.shape[1]:
            self._moments()

    def sorted_sources(self):
        """ft:879-889 `_sorted_sources`."""
        return (np.ascontiguousarray(self.sorted_pos),
                np.ascontiguousarray(self.charge[self.perm]))

    # ------------------------------------------------------------------ walk
    def evaluate(self, targets, *, exclude=None, theta=0.5, softening=0.0, potential=True):
        """ft:987-1061 `evaluate` (per-target walk; see oracle.c evaluate_quadtree)."""
        targets = np.ascontiguousarray(targets, dtype=float)
        m = targets.shape[1]
        exclude = (
            np.full(m, -1, dtype=np.int64)
            if exclude is None
            else np.ascontiguousarray(exclude, dtype=np.int64).reshape(-1)
        )
        phi, field = np.zeros(m), np.zeros((2, m))
        status = np.zeros(1, dtype=np.int64)
        n = self.pos.shape[1]
        if not n or not m:
            return phi, field
        L = lib()
        if self.kernel == "log":
            L.evaluate_log_quadtree(
                _p(targets), m, m, _p(exclude), _p(self.pos), n, _p(self.charge),
                _p(self.perm), _p(self.node_center), _p(self.node_half),
                _p(self.node_start), _p(self.node_end), _p(self.node_child),
                _p(self.node_qabs), _p(self.moment_re), _p(self.moment_im), self.order,
                float(theta), float(softening), self.stack_size, 1 if potential else 0,
                _p(phi), _p(field), m, _p(status))
        else:
            L.evaluate_quadtree(
                _p(targets), m, m, _p(exclude), _p(self.pos), n, _p(self.charge),
                _p(self.perm), _p(self.node_center), _p(self.node_half),
                _p(self.node_start), _p(self.node_end), _p(self.node_child),
                _p(self.node_q), _p(self.node_qabs), _p(self.node_p), _p(self.node_s),
                float(theta), float(softening), self.stack_size, 1 if potential else 0,
                _p(phi), _p(field), m, _p(status))
        _check(status)
        if not potential:
            phi[...] = 0.0
        return phi, field

    # ------------------------------------------------------------------ FMM
    def traverse(self, theta):
        """ft:1318-1358 `_traverse`: generations of fmm_traverse from (0, 0)."""
        L = lib()
        capacity = np.array([16, 16, 10]) * self.node_count + 64
        while True:
            m2l = np.empty((capacity[0], 2), dtype=np.int64)
            p2p = np.empty((capacity[1], 2), dtype=np.int64)
            frontier = np.zeros((capacity[2], 2), dtype=np.int64)
            nxt = np.empty((capacity[2], 2), dtype=np.int64)
            counts = np.zeros(4, dtype=np.int64)
            n_frontier = 1
            while n_frontier:
                counts[2] = 0
                L.fmm_traverse(
                    _p(self.node_center), _p(self.node_half), _p(self.node_start),
                    _p(self.node_end), _p(self.node_child), float(theta), _p(frontier),
                    n_frontier, _p(nxt), capacity[2], _p(m2l), capacity[0], _p(p2p),
                    capacity[1], _p(counts))
                if counts[3]:
                    break
                n_frontier = int(counts[2])
                frontier, nxt = nxt, frontier
            if not counts[3]:
                return m2l[: counts[0]].copy(), p2p[: counts[1]].copy()
            capacity = np.maximum(2 * capacity, counts[:3])

    def lists(self, theta):
        if theta not in self._traversals:
            self._traversals[theta] = self.traverse(theta)
        return self._traversals[theta]

    def m2l_rows(self, m2l):
        """ft:818-828 `_m2l_rows`: pair_csr, mutual."""
        rows = np.zeros(self.node_count + 1, dtype=np.int64)
        partners = np.empty(max(2 * len(m2l), 1), dtype=np.int64)
        cursor = np.empty(self.node_count, dtype=np.int64)
        pairs = np.ascontiguousarray(m2l, dtype=np.int64).reshape(-1, 2)
        lib().pair_csr(_p(pairs), len(m2l), 1, _p(rows), self.node_count, _p(partners),
                       _p(cursor))
        return rows, partners

    def fmm(self, *, theta=0.5, softening=0.0, potential=True):
        """ft:1460-1634 `fmm` (CPU, one process)."""
        if not 0 < theta < 1:
            raise ValueError("FMM theta must lie in (0, 1)")
        n = self.pos.shape[1]
        phi, field = np.zeros(n), np.zeros((2, n))
        if not n:
            return phi, field
        if self.kernel != "log":
            return self._coulomb_fmm(theta, softening)
        L = lib()
        m2l, p2p = self.lists(theta)
        order, count = self.order, self.node_count
        binom = binomial_table(2 * order + 1)
        local_re = np.zeros((count, order + 1))
        local_im = np.zeros((count, order + 1))
        if len(m2l):
            rows, partners = self.m2l_rows(m2l)
            coeff = m2l_coefficients(order, self.symmetric)
            L.fmm_m2l_host(_p(rows), count, _p(partners), _p(self.node_center),
                           _p(self.node_center), _p(self.moment_re), _p(self.moment_im),
                           _p(coeff), _p(local_re), _p(local_im), order)
        self._downward(local_re, local_im, binom)
        spos, scharge = self.sorted_sources()
        phi_sorted = np.zeros(n)
        field_sorted = np.zeros((2, n))
        status = np.zeros(1, dtype=np.int64)
        pairs = np.ascontiguousarray(p2p, dtype=np.int64).reshape(-1, 2)
        L.fmm_evaluate_host(_p(spos), n, _p(scharge), count, _p(self.node_center),
                            _p(self.node_start), _p(self.node_end), _p(self.node_child),
                            _p(local_re), _p(local_im), order, _p(pairs), len(p2p),
                            float(softening), 1 if potential else 0, _p(phi_sorted),
                            _p(field_sorted), n, _p(status))
        if int(status[0]):
            status[0] = self.perm[int(status[0]) - 1] + 1
        phi[self.perm] = phi_sorted
        field[:, self.perm] = field_sorted
        _check(status)
        self.fmm_pairs = (len(m2l), len(p2p))
        return phi, field

    def _downward(self, local_re, local_im, binom):
        """ft:1540-1552: fmm_downward level by level from the root."""
        for lo, hi in zip(self.levels[:-2], self.levels[1:-1]):
            lib().fmm_downward(int(lo), int(hi), _p(self.node_center), _p(self.node_child),
                               _p(binom), binom.shape[0], _p(local_re), _p(local_im),
                               self.order)

    def cartesian_moments(self):
        """ft:1063-1084 `_cartesian_moments`."""
        if self._cart is None:
            t = cart_tables(self.order)
            n = self.pos.shape[1]
            moments = np.empty((self.node_count, cart_size(self.order)))
            levels = np.ascontiguousarray(self.levels, dtype=np.int64)
            lib().cart_moments_upward(
                _p(self.pos), n, _p(self.charge), _p(self.perm), _p(levels), len(levels),
                _p(self.node_center), _p(self.node_start), _p(self.node_end),
                _p(self.node_child), _p(t["mono_parent"]), _p(t["mono_dir"]),
                _p(t["shift"]), _p(t["shift_coef"]), len(t["shift_coef"]), _p(moments),
                moments.shape[1])
            self._cart = moments
        return self._cart

    def _cart_downward(self, tree, local, t):
        levels = np.ascontiguousarray(tree.levels, dtype=np.int64)
        lib().cart_downward(_p(levels), len(levels), _p(tree.node_center),
                            _p(tree.node_child), _p(t["mono_parent"]), _p(t["mono_dir"]),
                            _p(t["shift"]), _p(t["shift_coef"]), len(t["shift_coef"]),
                            _p(local), local.shape[1])

    def _coulomb_fmm(self, theta, softening):
        """ft:1360-1428 `_coulomb_fmm`."""
        L = lib()
        n = self.pos.shape[1]
        m2l, p2p = self.lists(theta)
        t = cart_tables(self.order)
        nc = cart_size(self.order)
        local = np.zeros((self.node_count, nc))
        if len(m2l):
            rows, partners = self.m2l_rows(m2l)
            L.cart_m2l_host(_p(rows), self.node_count, _p(partners), _p(self.node_center),
                            _p(self.node_center), _p(self.cartesian_moments()), nc,
                            float(softening), _p(t["ex"]), _p(t["ey"]), _p(t["rec"]),
                            _p(t["m2l"]), _p(t["m2l_coef"]), len(t["m2l_coef"]), _p(local))
        self._cart_downward(self, local, t)
        spos, scharge = self.sorted_sources()
        phi_sorted, field_sorted = np.zeros(n), np.zeros((2, n))
        status = np.zeros(1, dtype=np.int64)
        pairs = np.ascontiguousarray(p2p, dtype=np.int64).reshape(-1, 2)
        L.cart_evaluate_host(_p(spos), n, _p(scharge), self.node_count,
                             _p(self.node_center), _p(self.node_start), _p(self.node_end),
                             _p(self.node_child), _p(local), nc, _p(t["mono_parent"]),
                             _p(t["mono_dir"]), _p(t["ex"]), _p(t["ey"]), _p(t["grad"]),
                             _p(pairs), len(p2p), float(softening), _p(phi_sorted),
                             _p(field_sorted), n, _p(status))
        if int(status[0]):
            status[0] = self.perm[int(status[0]) - 1] + 1
        _check(status)
        phi, field = np.zeros(n), np.zeros((2, n))
        phi[self.perm] = phi_sorted
        field[:, self.perm] = field_sorted
        self.fmm_pairs = (len(m2l), len(p2p))
        return phi, field

    # ------------------------------------------------------------------ fmm_at
    def dual_lists(self, tree, theta):
        """ft:1086-1122 `_dual_lists`: dual_traverse, then one-way pair_csr rows."""
        L = lib()
        depth = int(tree.node_depth.max()) + int(self.node_depth.max())
        stack = np.empty((3 * depth + 8, 2), dtype=np.int64)
        capacity = np.array([16, 8]) * (tree.node_count + self.node_count) + 64
        counts = np.zeros(3, dtype=np.int64)
        while True:
            m2l = np.empty((capacity[0], 2), dtype=np.int64)
            p2p = np.empty((capacity[1], 2), dtype=np.int64)
            L.dual_traverse(_p(tree.node_center), _p(tree.node_half), _p(tree.node_start),
                            _p(tree.node_end), _p(tree.node_child), _p(self.node_center),
                            _p(self.node_half), _p(self.node_start), _p(self.node_end),
                            _p(self.node_child), float(theta), _p(stack), len(stack),
                            _p(m2l), capacity[0], _p(p2p), capacity[1], _p(counts))
            if not counts[2]:
                break
            capacity = np.maximum(2 * capacity, counts[:2] + 64)
        rows = []
        for pairs, size in ((m2l, int(counts[0])), (p2p, int(counts[1]))):
            start = np.zeros(tree.node_count + 1, dtype=np.int64)
            partners = np.empty(max(size, 1), dtype=np.int64)
            cursor = np.empty(tree.node_count, dtype=np.int64)
            lib().pair_csr(_p(np.ascontiguousarray(pairs)), size, 0, _p(start),
                           tree.node_count, _p(partners), _p(cursor))
            rows.append((start, partners, size))
        return rows

    def target_tree(self, targets, leaf):
        """ft:1124-1149 `_target_plan`: the target tree's root and build."""
        m = targets.shape[1]
        lo, hi = targets.min(axis=1), targets.max(axis=1)
        centre = 0.5 * (lo + hi)
        half = 0.5 * float(np.max(hi - lo)) * (1 + 1e-12) + 1e-300
        return OracleTree(targets, np.zeros(m), (float(centre[0]), float(centre[1]), half),
                          leaf_capacity=leaf, max_depth=self.max_depth, kernel="coulomb")

    def fmm_at(self, targets, *, exclude=None, theta=0.5, softening=0.0, potential=True,
               leaf_capacity=None):
        """ft:1151-1316 `fmm_at`."""
        if not 0 < theta < 1:
            raise ValueError("FMM theta must lie in (0, 1)")
        targets = np.ascontiguousarray(targets, dtype=float)
        m, n = targets.shape[1], self.pos.shape[1]
        phi, field = np.zeros(m), np.zeros((2, m))
        if not m or not n:
            return phi, field
        exclude = (np.full(m, -1, dtype=np.int64) if exclude is None
                   else np.ascontiguousarray(exclude, dtype=np.int64).reshape(-1))
        leaf = self.leaf_capacity if leaf_capacity is None else int(leaf_capacity)
        tree = self.target_tree(targets, leaf)
        (m2l_rows, m2l_partners, n_m2l), (p2p_rows, p2p_partners, _) = self.dual_lists(tree, theta)
        L = lib()
        tpos, _ = tree.sorted_sources()
        texclude = np.ascontiguousarray(exclude[tree.perm])
        spos, scharge = self.sorted_sources()
        phi_sorted = np.empty(m)
        field_sorted = np.empty((2, m))
        if self.kernel == "log":
            order = self.order
            local_re = np.zeros((tree.node_count, order + 1))
            local_im = np.zeros((tree.node_count, order + 1))
            if n_m2l:
                coeff = m2l_coefficients(order, self.symmetric)
                L.fmm_m2l_host(_p(m2l_rows), tree.node_count, _p(m2l_partners),
                               _p(tree.node_center), _p(self.node_center), _p(self.moment_re),
                               _p(self.moment_im), _p(coeff), _p(local_re), _p(local_im), order)
            binom = binomial_table(2 * order + 1)
            for lo, hi in zip(tree.levels[:-2], tree.levels[1:-1]):
                L.fmm_downward(int(lo), int(hi), _p(tree.node_center), _p(tree.node_child),
                               _p(binom), binom.shape[0], _p(local_re), _p(local_im), order)
            L.log_targets_host(_p(tpos), m, _p(texclude), tree.node_count,
                               _p(tree.node_center), _p(tree.node_start), _p(tree.node_end),
                               _p(tree.node_child), _p(local_re), _p(local_im), order,
                               _p(p2p_rows), _p(p2p_partners), _p(spos), n, _p(scharge),
                               _p(self.perm), _p(self.node_start), _p(self.node_end),
                               float(softening), 1 if potential else 0, _p(phi_sorted),
                               _p(field_sorted), m)
        else:
            t = cart_tables(self.order)
            nc = cart_size(self.order)
            local = np.zeros((tree.node_count, nc))
            if n_m2l:
                L.cart_m2l_host(_p(m2l_rows), tree.node_count, _p(m2l_partners),
                                _p(tree.node_center), _p(self.node_center),
                                _p(self.cartesian_moments()), nc, float(softening),
                                _p(t["ex"]), _p(t["ey"]), _p(t["rec"]), _p(t["m2l"]),
                                _p(t["m2l_coef"]), len(t["m2l_coef"]), _p(local))
            self._cart_downward(tree, local, t)
            L.cart_targets_host(_p(tpos), m, _p(texclude), tree.node_count,
                                _p(tree.node_center), _p(tree.node_start), _p(tree.node_end),
                                _p(tree.node_child), _p(local), nc, _p(t["mono_parent"]),
                                _p(t["mono_dir"]), _p(t["ex"]), _p(t["ey"]), _p(t["grad"]),
                                _p(p2p_rows), _p(p2p_partners), _p(spos), n, _p(scharge),
                                _p(self.perm), _p(self.node_start), _p(self.node_end),
                                float(softening), _p(phi_sorted), _p(field_sorted), m)
        phi[tree.perm] = phi_sorted
        field[:, tree.perm] = field_sorted
        bad = np.flatnonzero(phi == 1.0e300)
        if bad.size:
            raise ValueError("Coincident charges require positive softening")
        if not potential:
            phi[:] = 0.0
        return phi, field
