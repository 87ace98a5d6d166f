"""The flat quadtree and direct sums on the GPU: a drop-in for tree-d-3d's field solver.

Mirrors src/tree_d_3d/flat_tree.py of the reference (``ft`` below): ``direct_field``,
``FlatNode`` and ``FlatQuadtree`` keep its signatures, defaults, validation messages
and semantics, with component-major (2, N) arrays.  The arrays live on the current
CUDA device as float64 / int64 tensors and every numeric step runs in libtreed3d.so
(hand-written sm_100a kernels behind the C ABI of include/treed3d.h).  Tensor inputs
give CUDA tensor results; NumPy or list inputs give NumPy results.
"""

from __future__ import annotations

import math
import weakref

import numpy as np
import torch

from tree_d_3d_b200 import _lib, _shards
from tree_d_3d_b200._trace import profile, region
from tree_d_3d_b200._utils import (
    _check,
    _device,
    _finite,
    _points,
    device,
    out,
    status_word,
    wants_numpy,
)
from tree_d_3d_b200.constants import K_E
from tree_d_3d_b200.quad import Quad

#: Highest expansion order (ft:46).
MAX_ORDER = 64

#: Default orders of the log kernel and of the Coulomb FMM (ft:50-51).
LOG_ORDER = 12
COULOMB_ORDER = 4

_KERNELS = ("coulomb", "log")

#: targets per group of the reference's CPU walk (ft:70); the GPU walk groups a warp
GROUP_SIZE = 32


def _kernel_code(kernel: str) -> int:
    return _lib.KERNEL_LOG if kernel == "log" else _lib.KERNEL_COULOMB


def _direct(targets, exclude, pos, charge, softening, kernel, potential=True):
    """Device tensors in, (phi, field) device tensors out; raises on coincidence."""
    dev = targets.device
    m, n = targets.shape[1], pos.shape[1]
    phi = torch.zeros(m, dtype=torch.float64, device=dev)
    field = torch.zeros((2, m), dtype=torch.float64, device=dev)
    if not m or not n:
        return phi, field
    status = status_word(dev)
    ws = _lib.workspace(_lib.query("td3_direct_sum_workspace_size", m, n), dev)
    _lib.call(
        "td3_direct_sum", _kernel_code(kernel), targets.data_ptr(), m, exclude.data_ptr(),
        pos.data_ptr(), charge.data_ptr(), n, float(softening), 1 if potential else 0,
        phi.data_ptr(), field.data_ptr(), status.data_ptr(), ws.data_ptr(), ws.numel(),
        _lib.stream(dev),
    )
    _check(status)
    return phi, field


@profile("flat_tree.direct_field")
def direct_field(targets, pos, charge, *, softening=0.0, exclude=None, compiled=True,
                 kernel="coulomb"):
    """Exact potential (M,) and field (2, M) at ``targets`` (2, M), without ``k_e``.

    ``pos`` (2, N) and ``charge`` (N,) are the sources; ``exclude[i]`` is the index of a
    source skipped for target ``i`` (-1 for none); ``kernel`` is ``"coulomb"`` or
    ``"log"``.  ft:124-160.  ``compiled`` is accepted for compatibility (the GPU path
    is always the compiled one).
    """
    if kernel not in _KERNELS:
        raise ValueError(f"kernel must be one of {_KERNELS}")
    as_numpy = wants_numpy(targets)
    targets = _points(targets, "targets")
    pos = _points(pos, "pos")
    charge = _device(charge).reshape(-1)
    m = targets.shape[1]
    if exclude is None:
        exclude = torch.full((m,), -1, dtype=torch.int64, device=targets.device)
    exclude = _device(exclude, torch.int64).reshape(-1)
    return out(_direct(targets, exclude, pos, charge, softening, kernel), as_numpy)


class FlatNode:
    """Read-only view of one node of a `FlatQuadtree` (ft:163-211)."""

    def __init__(self, tree: FlatQuadtree, index: int) -> None:
        self.tree = tree
        self.index = index

    @property
    def quad(self) -> Quad:
        x, y = self.tree.node_center[self.index].tolist()
        return Quad(float(x), float(y), float(self.tree.node_half[self.index]))

    @property
    def count(self) -> int:
        return int(self.tree.node_end[self.index] - self.tree.node_start[self.index])

    @property
    def total_charge(self) -> float:
        return float(self.tree.node_q[self.index])

    @property
    def total_abs_charge(self) -> float:
        return float(self.tree.node_qabs[self.index])

    @property
    def dipole(self) -> np.ndarray:
        return self.tree.node_p[self.index].cpu().numpy().copy()

    @property
    def second_moment(self) -> np.ndarray:
        sxx, sxy, syy = self.tree.node_s[self.index].tolist()
        return np.array([[sxx, sxy], [sxy, syy]])

    @property
    def particles(self) -> np.ndarray:
        """Indices of the particles inside this node."""
        tree = self.tree
        start, end = int(tree.node_start[self.index]), int(tree.node_end[self.index])
        return tree.perm[start:end].cpu().numpy()

    def is_external(self) -> bool:
        return int(self.tree.node_child[self.index]) < 0

    @property
    def children(self) -> tuple:
        first = int(self.tree.node_child[self.index])
        if first < 0:
            return (None, None, None, None)
        return tuple(FlatNode(self.tree, first + k) for k in range(4))


_NODE_ARRAYS = ("node_center", "node_half", "node_start", "node_end", "node_child", "node_depth")

#: small per-device tables shared by every tree (binomials, M2L matrices, Cartesian tables)
_TABLES: dict = {}


def _binomial_table(size: int) -> np.ndarray:
    """C(n, k) for 0 <= n, k < size as floats, by Pascal's rule in floating point
    (the values of the reference's table, ft:224-231)."""
    table = np.zeros((size, size))
    table[:, 0] = 1.0
    for row in range(1, size):
        table[row, 1 : row + 1] = table[row - 1, : row] + table[row - 1, 1 : row + 1]
    return table


def _m2l_coefficients(order: int, symmetric: bool) -> np.ndarray:
    """The real M2L matrix coeff[k, l] (ft:234-245): 1/l in row 0, 1/k in column 0,
    C(k + l - 1, l) / k elsewhere, zero beyond the triangle k <= p - l if symmetric."""
    binomial = _binomial_table(2 * order + 1)
    coeff = np.zeros((order + 1, order + 1))
    ls = np.arange(1, order + 1)
    coeff[0, 1:] = 1.0 / ls
    coeff[1:, 0] = 1.0 / ls
    for k in range(1, order + 1):
        for m in range(1, order + 1):
            if k <= (order - m if symmetric else order):
                coeff[k, m] = binomial[k + m - 1, m] / k
    return coeff


#: partners per near-field work segment (one warp each)
NEAR_SEGMENT = 256

#: the mixed-precision near field at the sources in three launches (td3_fmm_evaluate_mixed,
#: td3_fmm_adjoint_mixed: far field per particle, FP32 hi + lo pair arithmetic) instead of
#: the one-launch form of td3_fmm_evaluate / td3_fmm_adjoint with mixed = 1.
NEAR_SPLIT = True

#: with NEAR_SPLIT, the near part (pair sums) runs on a second stream while the M2L and the
#: downward pass run on the caller's stream; the far part follows both.
NEAR_OVERLAP = True

_SIDE_STREAMS: dict = {}


def _side_stream(device) -> "torch.cuda.Stream":
    """The second stream of ``device`` the near field's pair sums run on."""
    key = torch.device(device).index
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = torch.cuda.Stream(device=device)
    return _SIDE_STREAMS[key]

#: mixed-precision M2L matrix products on the tensor cores (tcgen05, 3xTF32; orders up
#: to 15) instead of FP32 CUDA-core arithmetic.  Off by default: the tensor-core form is
#: correct but, waiting on each 128-row tile, still slower than the CUDA-core form.
M2L_TENSOR_CORES = False

#: the log kernel's downward pass in one launch (each leaf's local from its ancestors'
#: own locals) instead of one L2L launch per level.  Off: at 1M particles the ancestor
#: walks take 1.5 ms per pass against 0.2 ms for the per-level launches.
DOWNWARD_LEAVES = False

#: the log kernel's upward pass in one launch (orders up to 12; the last child to finish
#: forms its parent) instead of one M2M launch per level; the same bits either way.
#: Off: its register use (244 per thread) leaves it at 0.55 ms per pass at 1M against
#: 0.22 ms for the per-level launches.
MOMENTS_ONE_LAUNCH = False

#: the mixed-precision M2L of ``fmm`` (mutual lists, log kernel, orders up to 14) as
#: tensor-core products grouped by translation (td3_m2l_groups, td3_fmm_m2l_grouped)
#: instead of the FP32 CUDA-core form (a lane per translation).  Off: 1.71 ms per launch
#: at 1M, p = 12, against 0.91 ms for the CUDA-core form.
M2L_GROUPED = False

#: the mixed-precision CUDA-core M2L with a group of 8 lanes per destination row
#: (td3_fmm_m2l_mixed_rows: partial sums in shared memory, packed 128-byte source records)
#: instead of a lane per entry across row boundaries (td3_fmm_m2l_mixed).
M2L_ROWS = True


def _group_span(theta: float) -> int:
    """Offsets (in units of the smaller half-width) covered by the grouped M2L's
    operator table: the lists of ``theta`` reach about 4.5 / theta; rarer, farther
    translations take the per-translation formula."""
    return int(min(max(math.ceil(5.5 / theta), 8), 24))


class _Lists(dict):
    """The interaction lists of one theta.  The CSR rows of the M2L list are made on
    first use: the grouped tensor-core M2L of the mixed form reads its own order."""

    def __init__(self, tree, **items):
        super().__init__(**items)
        self._tree = weakref.ref(tree)

    def __missing__(self, key):
        if key in ("m2l_rows", "m2l_partners", "m2l_entry_row") and "m2l" in self:
            rows, partners, entry = self._tree()._rows(self["m2l"], mutual=True, entry_rows=True)
            self.update(m2l_rows=rows, m2l_partners=partners, m2l_entry_row=entry)
            return dict.__getitem__(self, key)
        raise KeyError(key)


def _nearfield_plan(rows: torch.Tensor, tree, entries: int, end: torch.Tensor | None = None) -> dict:
    """The near-field work plan of one tree's leaf rows (td3_nearfield_plan): leaf rows
    cut into segments of at most NEAR_SEGMENT partners, and the partial-sum buffer of
    the rows that take several segments.  ``entries`` bounds the rows' partner count;
    ``end`` (default the tree's node_end) set to node_start leaves a leaf out."""
    dev = rows.device
    n_nodes = rows.shape[0] - 1
    capacity = n_nodes + entries // NEAR_SEGMENT + 1
    seg_leaf = torch.empty(capacity, dtype=torch.int32, device=dev)
    seg_range = torch.empty((capacity, 2), dtype=torch.int64, device=dev)
    seg_out = torch.empty(capacity, dtype=torch.int64, device=dev)
    sizes = np.zeros(2, dtype=np.int64)
    ws = _lib.workspace(_lib.query("td3_nearfield_plan_workspace_size", n_nodes), dev)
    end = tree.node_end if end is None else end
    _lib.call("td3_nearfield_plan", rows.data_ptr(), n_nodes, tree.node_child.data_ptr(),
              tree.node_start.data_ptr(), end.data_ptr(), NEAR_SEGMENT,
              seg_leaf.data_ptr(), seg_range.data_ptr(), seg_out.data_ptr(), capacity,
              sizes.ctypes.data, ws.data_ptr(), ws.numel(), _lib.stream(dev))
    n_seg = int(sizes[0])
    return {
        "seg_leaf": seg_leaf[:n_seg], "seg_range": seg_range[:n_seg], "seg_out": seg_out[:n_seg],
        "n_seg": n_seg, "partial_len": int(sizes[1]),
        "partial": torch.empty(3 * max(int(sizes[1]), 1), dtype=torch.float64, device=dev),
    }


def _device_table(key, make, dev, dtype=torch.float64):
    full = (key, dev)
    if full not in _TABLES:
        _TABLES[full] = torch.as_tensor(np.ascontiguousarray(make()), dtype=dtype, device=dev)
    return _TABLES[full]


class FlatQuadtree:
    """Array quadtree for point charges in a plane or for line charges, on the GPU.

    The tree and conventions of the reference (ft:437-1676): nodes holding more than
    ``leaf_capacity`` particles split into four until ``max_depth``; ``positions``
    (2, N) and ``charges`` (N,) are copied.  ``kernel="coulomb"`` keeps signed moments
    through the quadrupole, ``kernel="log"`` complex multipole expansions of ``order``
    terms.  ``comm`` (MPI sharing of the moments) is not supported: one GPU holds the
    whole tree.  ``precision="mixed"`` selects the mixed-precision forms of the FMM and
    of the Barnes-Hut walk: the same cells and pairs as FP64, near pairs and far-field
    terms in FP32 with compensated sums, M2M/L2L and the results in FP64.
    """

    def __init__(self, positions, charges, root_quad: Quad, *, leaf_capacity: int = 8,
                 max_depth: int = 48, compiled: bool = True, kernel: str = "coulomb",
                 order: int | None = None, symmetric: bool = False, comm=None,
                 precision: str = "fp64") -> None:
        # ft:760-800
        if kernel not in _KERNELS:
            raise ValueError(f"kernel must be one of {_KERNELS}")
        if order is None:
            order = LOG_ORDER if kernel == "log" else COULOMB_ORDER
        if isinstance(order, bool) or int(order) != order or order < 1:
            raise ValueError("order must be a positive integer")
        if order > MAX_ORDER:
            raise ValueError(f"order must be at most {MAX_ORDER}, got {order}")
        if comm is not None:
            import torch.distributed as dist

            if not (dist.is_available() and dist.is_initialized()):
                raise ValueError("comm must be a torch.distributed process group (the ranks "
                                 "that share the FMM), with the default group initialised")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.kernel = kernel
        self.order = int(order)
        #: the process group whose ranks share the FMM's work (None: one process)
        self.comm = comm if compiled else None
        self._rank, self._world = (0, 1) if self.comm is None else _shards.rank_and_world(comm)
        self.symmetric = bool(symmetric)
        self.precision = precision
        self._compiled = bool(compiled)
        _finite("half_size", root_quad.half, positive=True)
        _finite("xmid", root_quad.xmid)
        _finite("ymid", root_quad.ymid)
        for name, value in (("leaf_capacity", leaf_capacity), ("max_depth", max_depth)):
            if isinstance(value, bool) or int(value) != value or value < 1:
                raise ValueError(f"{name} must be a positive integer")
        self._numpy = wants_numpy(positions)
        self.pos = _points(positions, "positions").clone()
        self.charge = _device(charges).reshape(-1).clone()
        self.device = self.pos.device
        n = self.pos.shape[1]
        if self.charge.shape[0] != n:
            raise ValueError("positions and charges must have the same length")
        # finite positions inside the root (ft:788-794) are checked by the build itself
        self.leaf_capacity = int(leaf_capacity)
        self.max_depth = int(max_depth)
        self.root_quad = Quad(float(root_quad.xmid), float(root_quad.ymid), float(root_quad.half))
        self._traversals: dict = {}
        self._shard_cache: dict = {}
        self._cart_moments = None
        self._plans: dict = {}
        if not n:
            self._empty()
            return
        with region("flat_tree.build"):
            count = self._build()
        self.node_count = int(count)
        for name in _NODE_ARRAYS:  # views of the first `count` rows of the build's buffers
            setattr(self, name, getattr(self, name)[:count])
        with region("flat_tree.moments"):
            self._moments()

    # ------------------------------------------------------------------ build
    def _empty(self) -> None:
        """ft:462-481: the lone root of an empty tree."""
        dev, q = self.device, self.root_quad
        f64, i64 = torch.float64, torch.int64
        self.perm = torch.empty(0, dtype=i64, device=dev)
        self.node_count = 1
        self.node_center = torch.tensor([[q.xmid, q.ymid]], dtype=f64, device=dev)
        self.node_half = torch.tensor([q.half], dtype=f64, device=dev)
        self.node_start = torch.zeros(1, dtype=i64, device=dev)
        self.node_end = torch.zeros(1, dtype=i64, device=dev)
        self.node_child = torch.full((1,), -1, dtype=i64, device=dev)
        self.node_depth = torch.zeros(1, dtype=i64, device=dev)
        self.levels = np.array([0, 1])
        self.node_q = torch.zeros(1, dtype=f64, device=dev)
        self.node_qabs = torch.zeros(1, dtype=f64, device=dev)
        self.node_p = torch.zeros((1, 2), dtype=f64, device=dev)
        self.node_s = torch.zeros((1, 3), dtype=f64, device=dev)
        self.moment_re = torch.zeros((1, self.order + 1), dtype=f64, device=dev)
        self.moment_im = torch.zeros((1, self.order + 1), dtype=f64, device=dev)
        self._sorted_pos = torch.zeros((2, 0), dtype=f64, device=dev)
        self._sorted_charge = torch.zeros(0, dtype=f64, device=dev)

    def _build(self, capacity: int | None = None) -> int:
        """ft:483-625: the whole build in td3_quadtree_build, restarted with twice the
        node capacity while it reports the node arrays too small (ft:523-525)."""
        n = self.pos.shape[1]
        dev = self.device
        if capacity is None:
            capacity = 4 * (2 * n // self.leaf_capacity + 16)
        f64, i64 = torch.float64, torch.int64
        self.perm = torch.empty(n, dtype=i64, device=dev)
        self._sorted_pos = torch.empty((2, n), dtype=f64, device=dev)
        sizes = np.zeros(4, dtype=np.int64)
        while True:
            self.node_center = torch.empty((capacity, 2), dtype=f64, device=dev)
            self.node_half = torch.empty(capacity, dtype=f64, device=dev)
            self.node_start = torch.empty(capacity, dtype=i64, device=dev)
            self.node_end = torch.empty(capacity, dtype=i64, device=dev)
            self.node_child = torch.empty(capacity, dtype=i64, device=dev)
            self.node_depth = torch.empty(capacity, dtype=i64, device=dev)
            # the first node of each depth: at most max_depth + 2 entries
            levels = np.zeros(min(capacity, self.max_depth + 1) + 1, dtype=np.int64)
            ws = _lib.workspace(_lib.query("td3_quadtree_build_workspace_size", n, capacity), dev)
            q = self.root_quad
            rc = _lib.call_code(
                "td3_quadtree_build", self.pos.data_ptr(), n, q.xmid, q.ymid, q.half,
                self.leaf_capacity, self.max_depth, capacity, self.node_center.data_ptr(),
                self.node_half.data_ptr(), self.node_start.data_ptr(), self.node_end.data_ptr(),
                self.node_child.data_ptr(), self.node_depth.data_ptr(), self.perm.data_ptr(),
                self._sorted_pos.data_ptr(), levels.ctypes.data, sizes.ctypes.data,
                ws.data_ptr(), ws.numel(), _lib.stream(dev),
            )
            self.build_restarts = getattr(self, "build_restarts", 0)
            if rc == _lib.OK:
                break
            # the build checks the positions as ft:788-794 (one read for the whole build)
            if rc == _lib.EINVAL and sizes[3] == 1:
                raise ValueError("Particle position must be finite")
            if rc == _lib.EINVAL and sizes[3] == 2:
                raise ValueError("Particle lies outside tree bounds")
            if rc != _lib.ENEEDMORE:
                raise _lib.LibraryError(f"td3_quadtree_build failed with code {rc}")
            self.build_restarts += 1
            capacity = max(2 * capacity, int(sizes[0]))
        self.levels = levels[: sizes[1] + 1].copy()
        self._sorted_charge = self.charge[self.perm].contiguous()
        return int(sizes[0])

    # ------------------------------------------------------------------ moments
    def _binomial(self) -> torch.Tensor:
        size = 2 * self.order + 1
        return _device_table(("binomial", size), lambda: _binomial_table(size), self.device)

    def _moments(self) -> None:
        """ft:663-744: cell charges and multipole moments from the charges."""
        self._fwd_locals = None
        count, dev, f64 = self.node_count, self.device, torch.float64
        n = self.pos.shape[1]
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        stream = _lib.stream(dev)
        common = (self._sorted_pos.data_ptr(), self._sorted_charge.data_ptr(), n,
                  self.node_center.data_ptr(), self.node_start.data_ptr(),
                  self.node_end.data_ptr(), self.node_child.data_ptr())
        self.node_qabs = torch.empty(count, dtype=f64, device=dev)
        if self.kernel == "log":
            # the moments launch first (the GPU waits for them after the build's host
            # read); the derived node arrays follow
            self.moment_re = torch.empty((count, self.order + 1), dtype=f64, device=dev)
            self.moment_im = torch.empty((count, self.order + 1), dtype=f64, device=dev)
            binom = self._binomial()
            self._log_moments_into(self._sorted_charge, None, binom, self.node_qabs,
                                   self.moment_re, self.moment_im)
            self.node_q = self.moment_re[:, 0].clone()
            self.node_p = torch.stack((self.moment_re[:, 1], self.moment_im[:, 1]), dim=1)
            self.node_s = torch.zeros((count, 3), dtype=f64, device=dev)
            return
        self.node_q = torch.empty(count, dtype=f64, device=dev)
        self.node_p = torch.empty((count, 2), dtype=f64, device=dev)
        self.node_s = torch.zeros((count, 3), dtype=f64, device=dev)
        self.moment_re = torch.zeros((1, 1), dtype=f64, device=dev)
        self.moment_im = torch.zeros((1, 1), dtype=f64, device=dev)
        _lib.call("td3_quadtree_moments", levels.ctypes.data, len(levels) - 1, *common,
                  self.node_q.data_ptr(), self.node_qabs.data_ptr(), self.node_p.data_ptr(),
                  self.node_s.data_ptr(), stream)

    def _log_moments_into(self, weight, dipole, binom, qabs, mre, mim) -> None:
        """Complex moments of monopoles ``weight`` (tree order) and, when given, point
        dipoles ``dipole`` (2, N) into mre / mim: in one launch for orders up to 12
        (td3_log_moments_tree), else level by level (td3_log_moments[_adjoint]); the
        same bits either way."""
        n, stream = self.pos.shape[1], _lib.stream(self.device)
        if MOMENTS_ONE_LAUNCH and self.order <= 12:
            arrive = torch.empty(self.node_count, dtype=torch.int32, device=self.device)
            _lib.call("td3_log_moments_tree", self.node_count, self.order,
                      self._sorted_pos.data_ptr(), weight.data_ptr(),
                      0 if dipole is None else dipole.data_ptr(), n,
                      self.node_center.data_ptr(), self.node_start.data_ptr(),
                      self.node_end.data_ptr(), self.node_child.data_ptr(),
                      self._parents().data_ptr(), binom.data_ptr(), binom.shape[0],
                      qabs.data_ptr(), mre.data_ptr(), mim.data_ptr(), arrive.data_ptr(), stream)
            return
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        nodes = (self.node_center.data_ptr(), self.node_start.data_ptr(),
                 self.node_end.data_ptr(), self.node_child.data_ptr())
        if dipole is None:
            _lib.call("td3_log_moments", levels.ctypes.data, len(levels) - 1, self.order,
                      self._sorted_pos.data_ptr(), weight.data_ptr(), n, *nodes,
                      binom.data_ptr(), binom.shape[0], qabs.data_ptr(), mre.data_ptr(),
                      mim.data_ptr(), stream)
        else:
            _lib.call("td3_log_moments_adjoint", levels.ctypes.data, len(levels) - 1, self.order,
                      self._sorted_pos.data_ptr(), weight.data_ptr(), dipole.data_ptr(), n,
                      *nodes, binom.data_ptr(), binom.shape[0], qabs.data_ptr(),
                      mre.data_ptr(), mim.data_ptr(), stream)

    def _cartesian_tables(self):
        from tree_d_3d_b200 import _cartesian

        dev = self.device
        t = _cartesian.tables(self.order)
        out = {}
        for name, value in t.items():
            if value.dtype.kind == "f":
                dtype = torch.float64
            else:
                dtype = torch.int32 if value.dtype == np.int32 else torch.int64
            out[name] = _device_table(("cart", self.order, name), lambda v=value: v, dev, dtype)
        return out

    def _cartesian_moments(self) -> torch.Tensor:
        """ft:1063-1084: the Cartesian moments of every cell, kept until the charges change."""
        if self._cart_moments is None:
            from tree_d_3d_b200 import _cartesian

            t = self._cartesian_tables()
            n_coef = _cartesian.size(self.order)
            moments = torch.empty((self.node_count, n_coef), dtype=torch.float64,
                                  device=self.device)
            levels = np.ascontiguousarray(self.levels, dtype=np.int64)
            _lib.call("td3_cart_moments", levels.ctypes.data, len(levels) - 1,
                      self._sorted_pos.data_ptr(), self._sorted_charge.data_ptr(),
                      self.pos.shape[1], self.node_center.data_ptr(), self.node_start.data_ptr(),
                      self.node_end.data_ptr(), self.node_child.data_ptr(), t["ex"].data_ptr(),
                      t["ey"].data_ptr(), t["shift"].data_ptr(), t["shift_coef"].data_ptr(),
                      t["shift_start"].data_ptr(), n_coef, moments.data_ptr(),
                      _lib.stream(self.device))
            self._cart_moments = moments
        return self._cart_moments

    def set_charges(self, charges) -> None:
        """New charges (N,) for the same particles, without rebuilding (ft:853-868)."""
        charges = _device(charges).reshape(-1)
        if charges.shape[0] != self.pos.shape[1]:
            raise ValueError("charges must have one entry per particle")
        self.charge.copy_(charges)
        self._cart_moments = None
        if self.pos.shape[1]:
            self._sorted_charge = self.charge[self.perm].contiguous()
            self._moments()

    @property
    def root(self) -> FlatNode:
        return FlatNode(self, 0)

    def collect_nodes(self) -> list:
        """Views of every node that holds at least one particle (ft:870-877)."""
        occupied = torch.nonzero(self.node_end > self.node_start).flatten().tolist()
        return [FlatNode(self, int(i)) for i in occupied]

    # ------------------------------------------------------------------ walk
    @property
    def tree_depth(self) -> int:
        """The depth of the deepest node."""
        return len(self.levels) - 2

    def _target_order(self, targets: torch.Tensor) -> torch.Tensor:
        """ft:891-912: tree order for the sources themselves, else Morton order."""
        if targets.shape == self.pos.shape and torch.equal(targets, self.pos):
            return self.perm
        m = targets.shape[1]
        order = torch.empty(m, dtype=torch.int64, device=self.device)
        ws = _lib.workspace(_lib.query("td3_target_order_workspace_size", m), self.device)
        _lib.call("td3_target_order", targets.data_ptr(), m, order.data_ptr(), ws.data_ptr(),
                  ws.numel(), _lib.stream(self.device))
        return order

    def _walk(self, targets, exclude, theta, softening, potential, phi, field, status):
        m, n = targets.shape[1], self.pos.shape[1]
        order = self._target_order(targets)
        kernel = _kernel_code(self.kernel)
        ws = _lib.workspace(_lib.query("td3_walk_workspace_size", self.node_count, kernel),
                            self.device)
        hat = None
        if self._mixed and self.kernel == "log":
            hat = self._scaled_moments((self.moment_re, self.moment_im))
        _lib.call(
            "td3_evaluate_quadtree", kernel, targets.data_ptr(), m, exclude.data_ptr(),
            order.data_ptr(), self._sorted_pos.data_ptr(), self._sorted_charge.data_ptr(),
            self.perm.data_ptr(), n, self.node_count, self.node_center.data_ptr(),
            self.node_half.data_ptr(), self.node_start.data_ptr(), self.node_end.data_ptr(),
            self.node_child.data_ptr(), self.node_depth.data_ptr(), self.tree_depth,
            self.node_q.data_ptr(), self.node_qabs.data_ptr(), self.node_p.data_ptr(),
            self.node_s.data_ptr(), self.moment_re.data_ptr(), self.moment_im.data_ptr(),
            0 if hat is None else hat.data_ptr(), self.order, float(theta), float(softening),
            1 if potential else 0, self._mixed, phi.data_ptr(), field.data_ptr(),
            status.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream(self.device),
        )

    @profile("flat_tree.evaluate")
    def evaluate(self, targets, *, exclude=None, theta=0.5, softening=0.0, potential=True):
        """Potential (M,) and field (2, M) at ``targets`` (2, M) by the Barnes-Hut walk,
        without ``k_e`` (ft:987-1061).

        ``exclude[i]`` is a source index skipped for target ``i`` (-1: none);
        ``potential=False`` returns the potential as zeros (and skips the line-charge
        kernel's logarithms).
        """
        as_numpy = wants_numpy(targets)
        targets = _points(targets, "targets")
        m = targets.shape[1]
        if exclude is None:
            exclude = torch.full((m,), -1, dtype=torch.int64, device=self.device)
        exclude = _device(exclude, torch.int64).reshape(-1)
        phi = torch.zeros(m, dtype=torch.float64, device=self.device)
        field = torch.zeros((2, m), dtype=torch.float64, device=self.device)
        if self.pos.shape[1] and m:
            status = status_word(self.device)
            self._walk(targets, exclude, theta, softening, potential, phi, field, status)
            _check(status)
        if not potential:
            phi.zero_()
        return out((phi, field), as_numpy)

    def field_at(self, positions, *, theta: float = 0.5, k_e: float = K_E,
                 softening: float = 0.0, reference_radius: float = 1.0):
        """Potential (n,) and field (2, n) at probes (2, n), times ``k_e`` (ft:1648-1676).

        For line charges the potential is -2 k_e sum q ln(r / reference_radius).
        """
        theta = _finite("theta", theta, minimum=0)
        reference_radius = _finite("reference_radius", reference_radius, positive=True)
        k_e = _finite("k_e", k_e, minimum=0)
        softening = _finite("softening", softening, minimum=0)
        as_numpy = wants_numpy(positions)
        positions = _points(positions, "positions")
        if not bool(torch.isfinite(positions).all()):
            raise ValueError("positions must be finite")
        n = positions.shape[1]
        if k_e == 0:
            zeros = (torch.zeros(n, dtype=torch.float64, device=self.device),
                     torch.zeros((2, n), dtype=torch.float64, device=self.device))
            return out(zeros, as_numpy)
        phi, field = self.evaluate(positions, theta=theta, softening=softening)
        if self.kernel == "log":
            phi = phi + 2 * torch.sum(self.charge) * float(np.log(reference_radius))
        return out((k_e * phi, k_e * field), as_numpy)

    # ------------------------------------------------------------------ FMM lists
    def _traverse(self, theta: float):
        """ft:1318-1358: the mutual M2L and P2P pair lists, restarting with larger
        buffers while a generation overflows."""
        dev = self.device
        capacity = np.array([24, 16, 12]) * self.node_count + 64
        sizes = np.zeros(4, dtype=np.int64)
        while True:
            m2l = torch.empty((int(capacity[0]), 2), dtype=torch.int64, device=dev)
            p2p = torch.empty((int(capacity[1]), 2), dtype=torch.int64, device=dev)
            ws = _lib.workspace(_lib.query("td3_fmm_traverse_workspace_size", int(capacity[2]),
                                           self.node_count), dev)
            rc = _lib.call(
                "td3_fmm_traverse", self.node_center.data_ptr(), self.node_half.data_ptr(),
                self.node_start.data_ptr(), self.node_end.data_ptr(), self.node_child.data_ptr(),
                self.node_count, float(theta), m2l.data_ptr(), int(capacity[0]), p2p.data_ptr(),
                int(capacity[1]),
                int(capacity[2]), sizes.ctypes.data, ws.data_ptr(), ws.numel(), _lib.stream(dev))
            if rc == _lib.OK:
                return m2l[: sizes[0]], p2p[: sizes[1]]
            capacity = np.maximum(2 * capacity, sizes[:3] + 64)

    def _rows(self, pairs: torch.Tensor, mutual: bool, n_nodes: int | None = None,
              entry_rows: bool = False):
        """pair_csr (K/pair_csr/pair_csr_pyccel.py:12-45): rows by node of ``pairs``;
        with ``entry_rows`` also the row of every entry (int32)."""
        dev = self.device
        n_nodes = self.node_count if n_nodes is None else n_nodes
        count = pairs.shape[0]
        rows = torch.zeros(n_nodes + 1, dtype=torch.int64, device=dev)
        slots = max((2 if mutual else 1) * count, 1)
        partners = torch.empty(slots, dtype=torch.int64, device=dev)
        entry = torch.empty(slots, dtype=torch.int32, device=dev) if entry_rows else None
        ws = _lib.workspace(_lib.query("td3_pair_csr_workspace_size", count, int(mutual), n_nodes),
                            dev)
        _lib.call("td3_pair_csr", pairs.data_ptr(), count, int(mutual), n_nodes, rows.data_ptr(),
                  partners.data_ptr(), 0 if entry is None else entry.data_ptr(), ws.data_ptr(),
                  ws.numel(), _lib.stream(dev))
        return (rows, partners, entry) if entry_rows else (rows, partners)

    def _lists(self, theta: float) -> dict:
        """The interaction lists of ``theta``, their rows and the near-field plan, kept
        across set_charges (ft:1496-1498): they depend on the cells only."""
        if theta not in self._traversals:
            with region("flat_tree.traverse"):
                self._traversals[theta] = self._new_lists(theta)
        return self._traversals[theta]

    def _new_lists(self, theta: float) -> dict:
        """The mutual lists of ``theta`` (ft:1318-1358), the M2L translations in the
        order their M2L reads (CSR rows by destination, or the grouped order of the
        tensor-core form) and the near-field rows and plan."""
        m2l, p2p = self._traverse(theta)
        lists = _Lists(self, m2l=m2l, p2p=p2p)
        if self._grouped_m2l():
            lists["groups"] = self._m2l_groups(m2l, theta)
        else:
            lists["m2l_rows"]  # the CSR rows, made now
        p2p_rows, p2p_partners = self._rows(p2p, mutual=True)
        lists.update(p2p_rows=p2p_rows, p2p_partners=p2p_partners)
        lists["plan"] = _nearfield_plan(p2p_rows, self, 2 * p2p.shape[0])
        return lists

    def _grouped_m2l(self) -> bool:
        """Whether this tree's fmm takes the grouped tensor-core M2L."""
        return (M2L_GROUPED and self.kernel == "log" and self.precision == "mixed"
                and self.order <= 14 and self.node_count < (1 << 25)
                and 1 <= len(self.levels) - 1 <= 64)

    def _m2l_groups(self, m2l: torch.Tensor, theta: float) -> dict:
        """The directed translations of the mutual M2L list sorted by (tile of 128
        destinations, operator key), with the runs and tiles of that order
        (td3_m2l_groups)."""
        dev = self.device
        n_pairs = int(m2l.shape[0])
        e = 2 * n_pairs
        n_tiles = (self.node_count + 127) // 128
        span = _group_span(theta)
        keys = torch.empty(max(e, 1), dtype=torch.int32, device=dev)
        vals = torch.empty(max(e, 1), dtype=torch.int32, device=dev)
        tile_run = torch.empty(n_tiles + 1, dtype=torch.int32, device=dev)
        run_start = torch.empty(e + 1, dtype=torch.int32, device=dev)
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        ws = _lib.workspace(_lib.query("td3_m2l_groups_workspace_size", n_pairs), dev)
        _lib.call("td3_m2l_groups", m2l.data_ptr(), n_pairs, self.node_center.data_ptr(),
                  self.node_half.data_ptr(), self.node_depth.data_ptr(), levels.ctypes.data,
                  len(levels) - 1, self.node_count, span, keys.data_ptr(), vals.data_ptr(),
                  tile_run.data_ptr(), run_start.data_ptr(), ws.data_ptr(), ws.numel(),
                  _lib.stream(dev))
        return {"keys": keys, "vals": vals, "tile_run": tile_run, "run_start": run_start,
                "span": span}

    def _m2l_operators(self, span: int) -> torch.Tensor:
        """The grouped M2L's operator table for this order (td3_m2l_operators), made
        once per device."""
        key = (("m2l_ops", self.order, self.symmetric, span), self.device)
        if key not in _TABLES:
            nbytes = _lib.query("td3_m2l_operators_size", span)
            ops = torch.empty(nbytes // 4, dtype=torch.float32, device=self.device)
            _lib.call("td3_m2l_operators", self.order, self._m2l_matrix().data_ptr(), span,
                      ops.data_ptr(), _lib.stream(self.device))
            _TABLES[key] = ops
        return _TABLES[key]

    def _m2l_grouped(self, groups: dict, hat: torch.Tensor, local_re, local_im) -> None:
        """The grouped tensor-core M2L (td3_fmm_m2l_grouped) into the locals."""
        span = groups["span"]
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        coeff = np.ascontiguousarray(_m2l_coefficients(self.order, self.symmetric))
        _lib.call("td3_fmm_m2l_grouped", groups["tile_run"].data_ptr(),
                  groups["run_start"].data_ptr(), groups["keys"].data_ptr(),
                  groups["vals"].data_ptr(), self.node_count, levels.ctypes.data,
                  len(levels) - 1, self.node_center.data_ptr(), self.node_half.data_ptr(),
                  hat.data_ptr(), self.order, self._m2l_operators(span).data_ptr(), span,
                  coeff.ctypes.data, local_re.data_ptr(), local_im.data_ptr(),
                  self._tensor_status().data_ptr(), _lib.stream(self.device))

    def _m2l_matrix(self) -> torch.Tensor:
        key = ("m2l_coefficients", self.order, self.symmetric)
        return _device_table(key, lambda: _m2l_coefficients(self.order, self.symmetric),
                             self.device)

    # ------------------------------------------------------------------ FMM
    @profile("flat_tree.fmm")
    def fmm(self, *, theta: float = 0.5, softening: float = 0.0, potential: bool = True,
            _status: torch.Tensor | None = None):
        """Potential (N,) and field (2, N) at every source by the FMM, without ``k_e``
        (ft:1460-1634): complex expansions for ``kernel="log"``, Cartesian expansions of
        the softened kernel for ``kernel="coulomb"``; each particle's own charge
        excluded; ``potential=False`` returns zeros for the potential.

        ``_status`` (internal): a zeroed device status word that receives the
        coincident-charge report instead of a check here, for callers that read it later
        (the autograd function reads it after the backward) so the host does not wait
        for the GPU at the end of the call."""
        theta = _finite("theta", theta, minimum=0)
        if not 0 < theta < 1:
            raise ValueError("FMM theta must lie in (0, 1)")
        softening = _finite("softening", softening, minimum=0)
        n, dev = self.pos.shape[1], self.device
        phi = torch.zeros(n, dtype=torch.float64, device=dev)
        field = torch.zeros((2, n), dtype=torch.float64, device=dev)
        if not n:
            return out((phi, field), self._numpy)
        if self._world > 1:
            self._fmm_sharded(theta, softening, potential, phi, field)
            return out((phi, field), self._numpy)
        if self.kernel != "log":
            self._coulomb_fmm(theta, softening, phi, field, _status)
            return out((phi, field), self._numpy)
        lists = self._lists(theta)
        status = status_word(dev) if _status is None else _status
        if self._mixed and NEAR_SPLIT and NEAR_OVERLAP:
            # the M2L and L2L enqueued here first, then the pair sums on the second stream
            # (after the lists only): the M2L's blocks are dispatched first and the pair
            # sums fill the SMs the per-level L2L launches leave idle
            # (phi, field, status and the plan's buffer, which the second stream writes,
            # exist before the event it waits for)
            ready = torch.cuda.Event()
            ready.record(torch.cuda.current_stream(dev))
            local_re, local_im = self._log_locals(lists)
            self._fwd_locals = ((theta, softening), local_re, local_im)
            done = self._near_part(lists, _lib.KERNEL_LOG, softening, potential, phi, field,
                                   status, after=ready)
            torch.cuda.current_stream(dev).wait_event(done)
            _lib.call("td3_fmm_far_mixed", _lib.KERNEL_LOG, self._sorted_pos.data_ptr(),
                      self.perm.data_ptr(), n, self.node_center.data_ptr(), self.order,
                      local_re.data_ptr(), local_im.data_ptr(), self._slot_leaves().data_ptr(),
                      1 if potential else 0, phi.data_ptr(), field.data_ptr(),
                      _lib.stream(dev))
        else:
            local_re, local_im = self._log_locals(lists)
            self._fwd_locals = ((theta, softening), local_re, local_im)
            self._evaluate_near(lists, _lib.KERNEL_LOG, local_re, local_im, softening,
                                potential, phi, field, status)
        if _status is None:
            _check(status)
            self._check_tensor_cores()
        self.fmm_pairs = (int(lists["m2l"].shape[0]), int(lists["p2p"].shape[0]))
        return out((phi, field), self._numpy)

    def _log_locals(self, lists: dict, moments=None, downward: bool = True):
        """M2L into every cell's local expansion, then L2L down the tree (``moments``:
        (moment_re, moment_im), by default the tree's own; ``downward=False`` stops
        after the M2L)."""
        dev, count, w = self.device, self.node_count, self.order + 1
        mre, mim = moments if moments is not None else (self.moment_re, self.moment_im)
        local_re = torch.zeros((count, w), dtype=torch.float64, device=dev)
        local_im = torch.zeros((count, w), dtype=torch.float64, device=dev)
        stream = _lib.stream(dev)
        if lists["m2l"].shape[0]:
            self._m2l_log(lists, self, (mre, mim), local_re, local_im)
        if downward:
            self._downward(local_re, local_im, self.order, self._binomial())
        return local_re, local_im

    def _parents(self) -> torch.Tensor:
        """The parent of every node (int32, -1 for the root), kept with the tree."""
        if getattr(self, "_node_parent", None) is None:
            self._node_parent = torch.empty(self.node_count, dtype=torch.int32, device=self.device)
            _lib.call("td3_node_parents", self.node_count, self.node_child.data_ptr(),
                      self._node_parent.data_ptr(), _lib.stream(self.device))
        return self._node_parent

    def _downward(self, local_re, local_im, order, binom) -> None:
        """L2L of complex locals of ``order`` from the root down this tree (``binom`` the
        binomial table): in one launch, every leaf's local from its ancestors' own
        locals (td3_fmm_downward_leaves; internal cells keep their own M2L locals), or
        level by level as the reference (td3_fmm_downward) with DOWNWARD_LEAVES off."""
        if DOWNWARD_LEAVES:
            _lib.call("td3_fmm_downward_leaves", self.node_count, order,
                      self.node_center.data_ptr(), self._parents().data_ptr(),
                      self.node_start.data_ptr(), self.node_end.data_ptr(),
                      self.node_child.data_ptr(), binom.data_ptr(), binom.shape[0],
                      local_re.data_ptr(), local_im.data_ptr(), _lib.stream(self.device))
            return
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        _lib.call("td3_fmm_downward", levels.ctypes.data, len(levels) - 1,
                  self.node_center.data_ptr(), self._parents().data_ptr(),
                  self.node_start.data_ptr(), self.node_end.data_ptr(), order,
                  binom.data_ptr(), binom.shape[0], local_re.data_ptr(), local_im.data_ptr(),
                  _lib.stream(self.device))

    def _near_part(self, lists, kernel, softening, potential, phi, field, status, after):
        """td3_fmm_near_mixed on the second stream after the event ``after`` of the
        caller's stream; returns the event the far part waits for.  The tensors it reads
        and writes stay alive until the caller's stream has waited for the event."""
        dev = self.device
        side = _side_stream(dev)
        side.wait_event(after)
        plan = lists["plan"]
        _lib.call("td3_fmm_near_mixed", kernel, self._sorted_pos.data_ptr(),
                  self._sorted_charge.data_ptr(), self.perm.data_ptr(), self.pos.shape[1],
                  self.node_center.data_ptr(), self.node_start.data_ptr(),
                  self.node_end.data_ptr(), lists["p2p_partners"].data_ptr(),
                  plan["seg_leaf"].data_ptr(), plan["seg_range"].data_ptr(),
                  plan["seg_out"].data_ptr(), plan["n_seg"], plan["partial"].data_ptr(),
                  float(softening), 1 if potential else 0, self._unit, phi.data_ptr(),
                  field.data_ptr(), status.data_ptr(), side.cuda_stream)
        done = torch.cuda.Event()
        done.record(side)
        return done

    def _slot_leaves(self) -> torch.Tensor:
        """The leaf of every particle slot (td3_slot_leaves), kept with the tree."""
        if getattr(self, "_slot_leaf", None) is None:
            n = self.pos.shape[1]
            self._slot_leaf = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
            _lib.call("td3_slot_leaves", self.node_count, self.node_child.data_ptr(),
                      self.node_start.data_ptr(), self.node_end.data_ptr(),
                      self._slot_leaf.data_ptr(), _lib.stream(self.device))
        return self._slot_leaf

    def _evaluate_near(self, lists, kernel, local_a, local_b, softening, potential, phi, field,
                       status):
        """L2P + P2P at the sources (td3_fmm_evaluate) over the near-field plan; the
        mixed form as td3_fmm_evaluate_mixed (NEAR_SPLIT)."""
        plan = lists["plan"]
        n = self.pos.shape[1]
        if self._mixed and NEAR_SPLIT:
            _lib.call(
                "td3_fmm_evaluate_mixed", kernel, self._sorted_pos.data_ptr(),
                self._sorted_charge.data_ptr(), self.perm.data_ptr(), n,
                self.node_center.data_ptr(), self.node_start.data_ptr(),
                self.node_end.data_ptr(), self.order, local_a.data_ptr(), local_b.data_ptr(),
                lists.get("slot_leaf", self._slot_leaves()).data_ptr(),
                lists["p2p_partners"].data_ptr(),
                plan["seg_leaf"].data_ptr(), plan["seg_range"].data_ptr(),
                plan["seg_out"].data_ptr(), plan["n_seg"], plan["partial"].data_ptr(),
                float(softening), 1 if potential else 0, self._unit, phi.data_ptr(),
                field.data_ptr(), status.data_ptr(), _lib.stream(self.device))
            return
        _lib.call(
            "td3_fmm_evaluate", kernel, self._sorted_pos.data_ptr(),
            self._sorted_charge.data_ptr(), self.perm.data_ptr(), n, self.node_center.data_ptr(),
            self.node_start.data_ptr(), self.node_end.data_ptr(), self.order, local_a.data_ptr(),
            local_b.data_ptr(), lists["p2p_partners"].data_ptr(), plan["seg_leaf"].data_ptr(),
            plan["seg_range"].data_ptr(), plan["seg_out"].data_ptr(), plan["n_seg"],
            plan["partial"].data_ptr(), float(softening), 1 if potential else 0, self._mixed,
            self._unit,
            phi.data_ptr(), field.data_ptr(), status.data_ptr(), _lib.stream(self.device))

    @property
    def _mixed(self) -> int:
        return 1 if self.precision == "mixed" else 0

    @property
    def _unit(self) -> float:
        """The length unit of the mixed-precision kernels: the root half-width."""
        return self.root_quad.half

    def _scaled_moments(self, moments):
        """FP32 moments scaled by the cell size, hat_k = a_k / h^k (nodes, order + 1
        rounded up to even, 2; the pad pair is zero)."""
        mre, mim = moments
        width = (self.order + 2) & ~1
        hat = torch.empty((self.node_count, width, 2), dtype=torch.float32, device=self.device)
        _lib.call("td3_scale_moments", self.node_count, self.order, mre.data_ptr(),
                  mim.data_ptr(), self.node_half.data_ptr(), hat.data_ptr(),
                  _lib.stream(self.device))
        return hat

    def _source_records(self, moments):
        """Packed source cells of the row-group M2L (td3_pack_m2l_sources): centre (FP64),
        hat_k = a_k / h^k (FP32 pairs) and h / unit, td3_m2l_record_floats(order) floats
        per node."""
        mre, mim = moments
        width = _lib.lib().td3_m2l_record_floats(self.order)
        records = torch.empty((self.node_count, width), dtype=torch.float32,
                              device=self.device)
        _lib.call("td3_pack_m2l_sources", self.node_count, self.order, mre.data_ptr(),
                  mim.data_ptr(), self.node_center.data_ptr(), self.node_half.data_ptr(),
                  self._unit, records.data_ptr(), _lib.stream(self.device))
        return records

    def _tensor_status(self) -> torch.Tensor:
        """The device word the tensor-core M2L raises when a wait for the tensor cores
        runs out (checked by _check_tensor_cores)."""
        if getattr(self, "_tc_status", None) is None:
            self._tc_status = status_word(self.device)
        return self._tc_status

    def _check_tensor_cores(self) -> None:
        """Raise if a tensor-core M2L of this tree did not complete (reads the word)."""
        word = getattr(self, "_tc_status", None)
        if word is not None and int(word.item()) != 0:
            word.zero_()
            raise RuntimeError("the tensor cores did not complete an M2L (a bounded wait ran "
                               "out); the local expansions are incomplete")

    def _m2l_log(self, lists, dst, moments, local_re, local_im):
        """Log-kernel M2L from this tree's cells into ``dst``'s over the rows of
        ``lists``: FP64, or FP32 on moments scaled by the cell size for
        ``precision="mixed"`` (orders up to 20), the matrix products on the tensor cores
        for orders up to 15 (M2L_TENSOR_CORES)."""
        stream = _lib.stream(self.device)
        mre, mim = moments
        if self.precision == "mixed" and self.order <= 20:
            groups = lists.get("groups") if dst is self else None
            if groups is not None:
                self._m2l_grouped(groups, self._scaled_moments(moments), local_re, local_im)
                return
            rows, partners = lists["m2l_rows"], lists["m2l_partners"]
            coeff = np.ascontiguousarray(_m2l_coefficients(self.order, self.symmetric))
            tensor = 1 if M2L_TENSOR_CORES and self.order <= 15 else 0
            if M2L_ROWS and not tensor:
                records = self._source_records(moments)
                _lib.call("td3_fmm_m2l_mixed_rows", rows.data_ptr(), partners.data_ptr(),
                          dst.node_count, dst.node_center.data_ptr(), dst.node_half.data_ptr(),
                          records.data_ptr(), self.order, coeff.ctypes.data, self._unit,
                          local_re.data_ptr(), local_im.data_ptr(), stream)
                return
            hat = self._scaled_moments(moments)
            _lib.call("td3_fmm_m2l_mixed", rows.data_ptr(), lists["m2l_entry_row"].data_ptr(),
                      partners.data_ptr(), dst.node_count,
                      dst.node_center.data_ptr(), dst.node_half.data_ptr(),
                      self.node_center.data_ptr(), self.node_half.data_ptr(), hat.data_ptr(),
                      self.order, coeff.ctypes.data, self._unit, tensor, local_re.data_ptr(),
                      local_im.data_ptr(), self._tensor_status().data_ptr() if tensor else 0,
                      stream)
            return
        rows, partners = lists["m2l_rows"], lists["m2l_partners"]
        _lib.call("td3_fmm_m2l", rows.data_ptr(), partners.data_ptr(), dst.node_count,
                  dst.node_center.data_ptr(), self.node_center.data_ptr(), mre.data_ptr(),
                  mim.data_ptr(), self.order, self._m2l_matrix().data_ptr(), local_re.data_ptr(),
                  local_im.data_ptr(), stream)

    # ------------------------------------------------------------------ backward
    @profile("flat_tree.fmm_backward")
    def _fmm_adjoint(self, theta: float, softening: float, weight: torch.Tensor,
                     dipole: torch.Tensor, efield: torch.Tensor):
        """The backward of ``fmm`` at the sources: for upstream gradients ``weight`` =
        dL/dphi (N,) and ``dipole`` = dL/dE (2, N), and the forward field ``efield``,
        returns (dL/dq (N,), dL/dx (2, N)) by one adjoint FMM pass (monopole + dipole
        sources) plus the Hessian of the forward expansions."""
        from tree_d_3d_b200 import _cartesian

        lists = self._lists(theta)
        n, dev, count = self.pos.shape[1], self.device, self.node_count
        sw = weight.to(torch.float64)[self.perm].contiguous()
        sd = dipole.to(torch.float64)[:, self.perm].contiguous()
        efield = efield.to(torch.float64).contiguous()
        levels = np.ascontiguousarray(self.levels, dtype=np.int64)
        stream = _lib.stream(dev)
        kept = getattr(self, "_fwd_locals", None)
        if kept is not None and kept[0] != (theta, softening):
            kept = None
        overlap = self._mixed and NEAR_SPLIT and NEAR_OVERLAP
        if overlap:
            # what the second stream writes is allocated before the event it waits for,
            # so it cannot take memory that work enqueued after the event still uses
            plan = lists["plan"]
            partial = torch.empty(6 * max(plan["partial_len"], 1), dtype=torch.float64,
                                  device=dev)
            qbar = torch.empty(n, dtype=torch.float64, device=dev)
            xbar = torch.empty((2, n), dtype=torch.float64, device=dev)
            ready = torch.cuda.Event()
            ready.record(torch.cuda.current_stream(dev))
        if self.kernel == "log":
            w = self.order + 1
            fwd_a, fwd_b = (kept[1], kept[2]) if kept else self._log_locals(lists)
            mre = torch.empty((count, w), dtype=torch.float64, device=dev)
            mim = torch.empty_like(mre)
            wabs = torch.empty(count, dtype=torch.float64, device=dev)
            binom = self._binomial()
            self._log_moments_into(sw, sd, binom, wabs, mre, mim)
            adj_a, adj_b = self._log_locals(lists, moments=(mre, mim))
            kernel = _lib.KERNEL_LOG
        else:
            t = self._cartesian_tables()
            n_coef = _cartesian.size(self.order)
            n_m2l = lists["m2l"].shape[0]
            fwd_a = kept[1] if kept else self._cart_locals(
                lists["m2l_rows"], lists["m2l_partners"], n_m2l, self, softening)
            moments = torch.empty((count, n_coef), dtype=torch.float64, device=dev)
            _lib.call("td3_cart_moments_adjoint", levels.ctypes.data, len(levels) - 1,
                      self._sorted_pos.data_ptr(), sw.data_ptr(), sd.data_ptr(), n,
                      self.node_center.data_ptr(), self.node_start.data_ptr(),
                      self.node_end.data_ptr(), self.node_child.data_ptr(), t["ex"].data_ptr(),
                      t["ey"].data_ptr(), t["shift"].data_ptr(), t["shift_coef"].data_ptr(),
                      t["shift_start"].data_ptr(), n_coef, moments.data_ptr(), stream)
            adj_a = self._cart_locals(lists["m2l_rows"], lists["m2l_partners"], n_m2l, self,
                                      softening, moments=moments)
            fwd_b, adj_b = fwd_a, adj_a
            kernel = _lib.KERNEL_COULOMB
        if overlap:
            # the adjoint moments, M2L and L2L enqueued first; the near parts of qbar and
            # xbar on the second stream after the weights only, filling the SMs the
            # per-level launches leave idle
            side = _side_stream(dev)
            side.wait_event(ready)
            _lib.call("td3_fmm_adjoint_near_mixed",
                      _lib.KERNEL_LOG if self.kernel == "log" else _lib.KERNEL_COULOMB,
                      self._sorted_pos.data_ptr(), self._sorted_charge.data_ptr(),
                      self.perm.data_ptr(), n, self.node_center.data_ptr(),
                      self.node_start.data_ptr(), self.node_end.data_ptr(),
                      lists["p2p_partners"].data_ptr(), plan["seg_leaf"].data_ptr(),
                      plan["seg_range"].data_ptr(), plan["seg_out"].data_ptr(), plan["n_seg"],
                      partial.data_ptr(), sw.data_ptr(), sd.data_ptr(), float(softening),
                      self._unit, qbar.data_ptr(), xbar.data_ptr(), side.cuda_stream)
            near_done = torch.cuda.Event()
            near_done.record(side)
            torch.cuda.current_stream(dev).wait_event(near_done)
            _lib.call("td3_fmm_adjoint_far_mixed", kernel, self._sorted_pos.data_ptr(),
                      self._sorted_charge.data_ptr(), self.perm.data_ptr(), n,
                      self.node_center.data_ptr(), self.order, fwd_a.data_ptr(),
                      fwd_b.data_ptr(), adj_a.data_ptr(), adj_b.data_ptr(),
                      self._slot_leaves().data_ptr(), sw.data_ptr(), sd.data_ptr(),
                      efield.data_ptr(), qbar.data_ptr(), xbar.data_ptr(), stream)
            self._check_tensor_cores()
            return qbar, xbar
        plan = lists["plan"]
        partial = torch.empty(6 * max(plan["partial_len"], 1), dtype=torch.float64, device=dev)
        qbar = torch.zeros(n, dtype=torch.float64, device=dev)
        xbar = torch.zeros((2, n), dtype=torch.float64, device=dev)
        if self._mixed and NEAR_SPLIT:
            _lib.call("td3_fmm_adjoint_mixed", kernel, self._sorted_pos.data_ptr(),
                      self._sorted_charge.data_ptr(), self.perm.data_ptr(), n,
                      self.node_center.data_ptr(), self.node_start.data_ptr(),
                      self.node_end.data_ptr(), self.order, fwd_a.data_ptr(), fwd_b.data_ptr(),
                      adj_a.data_ptr(), adj_b.data_ptr(), self._slot_leaves().data_ptr(),
                      lists["p2p_partners"].data_ptr(), plan["seg_leaf"].data_ptr(),
                      plan["seg_range"].data_ptr(), plan["seg_out"].data_ptr(), plan["n_seg"],
                      partial.data_ptr(), sw.data_ptr(), sd.data_ptr(), efield.data_ptr(),
                      float(softening), self._unit, qbar.data_ptr(), xbar.data_ptr(), stream)
            self._check_tensor_cores()
            return qbar, xbar
        _lib.call("td3_fmm_adjoint", kernel, self._sorted_pos.data_ptr(),
                  self._sorted_charge.data_ptr(), self.perm.data_ptr(), n,
                  self.node_center.data_ptr(), self.node_start.data_ptr(), self.node_end.data_ptr(),
                  self.order, fwd_a.data_ptr(), fwd_b.data_ptr(), adj_a.data_ptr(),
                  adj_b.data_ptr(), lists["p2p_partners"].data_ptr(), plan["seg_leaf"].data_ptr(),
                  plan["seg_range"].data_ptr(), plan["seg_out"].data_ptr(), plan["n_seg"],
                  partial.data_ptr(), sw.data_ptr(), sd.data_ptr(), efield.data_ptr(),
                  float(softening), self._mixed, self._unit, qbar.data_ptr(), xbar.data_ptr(),
                  stream)
        self._check_tensor_cores()
        return qbar, xbar

    def _move_within_cells(self, positions) -> None:
        """New positions for the same particles in the same cells (the tree's topology
        and interaction lists stay): for derivatives of the expansions at fixed
        topology.  Raises if a particle leaves its leaf."""
        positions = _points(positions, "positions")
        sorted_pos = positions[:, self.perm].contiguous()
        # the non-empty leaves tile the slots 0..N-1 in the order of their starts
        leaves = torch.nonzero((self.node_child < 0) & (self.node_end > self.node_start)).flatten()
        leaves = leaves[torch.argsort(self.node_start[leaves])]
        leaf_of = torch.repeat_interleave(leaves, (self.node_end - self.node_start)[leaves])
        c = self.node_center[leaf_of]
        h = self.node_half[leaf_of]
        inside = (sorted_pos[0] >= c[:, 0] - h) & (sorted_pos[0] <= c[:, 0] + h) & \
                 (sorted_pos[1] >= c[:, 1] - h) & (sorted_pos[1] <= c[:, 1] + h)
        if not bool(inside.all()):
            raise ValueError("a particle left its cell; rebuild the tree")
        self.pos = positions.clone()
        self._sorted_pos = sorted_pos
        self._cart_moments = None
        self._moments()

    # ------------------------------------------------------------------ fmm_at
    def _dual_lists(self, tree: "FlatQuadtree", theta: float) -> dict:
        """ft:1086-1122: one-way M2L / P2P pairs (target cell, source cell) as rows by
        target cell, and the near-field plan of the target leaves."""
        dev = self.device
        capacity = np.array([16, 8, 12]) * (tree.node_count + self.node_count) + 64
        sizes = np.zeros(4, dtype=np.int64)
        while True:
            m2l = torch.empty((int(capacity[0]), 2), dtype=torch.int64, device=dev)
            p2p = torch.empty((int(capacity[1]), 2), dtype=torch.int64, device=dev)
            ws = _lib.workspace(_lib.query("td3_fmm_traverse_workspace_size", int(capacity[2]),
                                           tree.node_count + self.node_count), dev)
            rc = _lib.call(
                "td3_dual_traverse", tree.node_center.data_ptr(), tree.node_half.data_ptr(),
                tree.node_start.data_ptr(), tree.node_end.data_ptr(), tree.node_child.data_ptr(),
                tree.node_count, self.node_center.data_ptr(), self.node_half.data_ptr(),
                self.node_start.data_ptr(), self.node_end.data_ptr(), self.node_child.data_ptr(),
                self.node_count, float(theta),
                m2l.data_ptr(), int(capacity[0]), p2p.data_ptr(), int(capacity[1]),
                int(capacity[2]), sizes.ctypes.data, ws.data_ptr(), ws.numel(), _lib.stream(dev))
            if rc == _lib.OK:
                break
            capacity = np.maximum(2 * capacity, sizes[:3] + 64)
        m2l, p2p = m2l[: sizes[0]], p2p[: sizes[1]]
        m2l_rows, m2l_partners, m2l_entry = self._rows(m2l, mutual=False,
                                                       n_nodes=tree.node_count, entry_rows=True)
        p2p_rows, p2p_partners = self._rows(p2p, mutual=False, n_nodes=tree.node_count)
        return {
            "m2l": m2l, "p2p": p2p, "m2l_rows": m2l_rows, "m2l_partners": m2l_partners,
            "m2l_entry_row": m2l_entry, "p2p_rows": p2p_rows, "p2p_partners": p2p_partners,
            "plan": _nearfield_plan(p2p_rows, tree, p2p.shape[0]),
        }

    def _target_plan(self, targets: torch.Tensor, theta: float, leaf: int):
        """ft:1124-1149: the target tree and the dual lists, kept while the targets
        stay the same (repeated sums at the same points)."""
        key = ("targets", theta, leaf)
        cached = self._plans.get(key)
        if (cached is not None and cached[0].shape == targets.shape
                and torch.equal(cached[0], targets)):
            return cached[1], cached[2]
        m = targets.shape[1]
        lo = targets.amin(dim=1).tolist()
        hi = targets.amax(dim=1).tolist()
        centre = (0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]))
        half = 0.5 * max(hi[0] - lo[0], hi[1] - lo[1]) * (1 + 1e-12) + 1e-300
        tree = FlatQuadtree(targets, torch.zeros(m, dtype=torch.float64, device=self.device),
                            Quad(centre[0], centre[1], half), leaf_capacity=leaf,
                            max_depth=self.max_depth, kernel="coulomb")
        lists = self._dual_lists(tree, theta)
        self._plans[key] = (targets.clone(), tree, lists)
        return tree, lists

    @profile("flat_tree.fmm_at")
    def fmm_at(self, targets, *, exclude=None, theta: float = 0.5, softening: float = 0.0,
               potential: bool = True, leaf_capacity: int | None = None):
        """Potential (M,) and field (2, M) at ``targets`` (2, M) by the FMM, without
        ``k_e`` (ft:1151-1316): a tree of the targets (``leaf_capacity`` per leaf, by
        default the sources'), a one-way dual traversal against the source tree, M2L
        into the target cells, L2L down the target tree, L2P plus exact sums over the
        partner source leaves (skipping source ``exclude[i]``).  On the GPU."""
        theta = _finite("theta", theta, minimum=0)
        if not 0 < theta < 1:
            raise ValueError("FMM theta must lie in (0, 1)")
        softening = _finite("softening", softening, minimum=0)
        as_numpy = wants_numpy(targets)
        targets = _points(targets, "targets")
        if not bool(torch.isfinite(targets).all()):
            raise ValueError("targets must be finite")
        m, n, dev = targets.shape[1], self.pos.shape[1], self.device
        phi = torch.zeros(m, dtype=torch.float64, device=dev)
        field = torch.zeros((2, m), dtype=torch.float64, device=dev)
        if not m or not n:
            return out((phi, field), as_numpy)
        if exclude is None:
            exclude = torch.full((m,), -1, dtype=torch.int64, device=dev)
        exclude = _device(exclude, torch.int64).reshape(-1)
        leaf = self.leaf_capacity if leaf_capacity is None else int(leaf_capacity)
        tree, lists = self._target_plan(targets, theta, leaf)
        texclude = exclude[tree.perm].contiguous()
        stream = _lib.stream(dev)
        n_m2l = int(lists["m2l"].shape[0])
        if self.kernel == "log":
            w = self.order + 1
            local_a = torch.zeros((tree.node_count, w), dtype=torch.float64, device=dev)
            local_b = torch.zeros_like(local_a)
            if n_m2l:
                self._m2l_log(lists, tree, (self.moment_re, self.moment_im), local_a, local_b)
            tree._downward(local_a, local_b, self.order, self._binomial())
            kernel, with_pot = _lib.KERNEL_LOG, potential
        else:
            local_a = self._cart_locals(lists["m2l_rows"], lists["m2l_partners"], n_m2l, tree,
                                        softening)
            local_b = local_a
            kernel, with_pot = _lib.KERNEL_COULOMB, True
        plan = lists["plan"]
        status = status_word(dev)
        _lib.call(
            "td3_fmm_targets", kernel, tree._sorted_pos.data_ptr(), texclude.data_ptr(),
            tree.perm.data_ptr(), m, tree.node_center.data_ptr(), tree.node_start.data_ptr(),
            tree.node_end.data_ptr(), self.order, local_a.data_ptr(), local_b.data_ptr(),
            lists["p2p_partners"].data_ptr(), plan["seg_leaf"].data_ptr(),
            plan["seg_range"].data_ptr(), plan["seg_out"].data_ptr(), plan["n_seg"],
            plan["partial"].data_ptr(), self._sorted_pos.data_ptr(),
            self._sorted_charge.data_ptr(), self.perm.data_ptr(), n, self.node_start.data_ptr(),
            self.node_end.data_ptr(), float(softening), 1 if with_pot else 0, self._mixed,
            self._unit,
            phi.data_ptr(), field.data_ptr(), status.data_ptr(), stream)
        _check(status)
        self._check_tensor_cores()
        if not potential:
            phi.zero_()
        return out((phi, field), as_numpy)

    def _cart_locals(self, rows, partners, n_m2l, dst, softening, moments=None,
                     downward: bool = True):
        """Cartesian M2L from this tree's cells into the cells of ``dst`` (this tree for
        fmm, the target tree for fmm_at), then L2L down ``dst`` (ft:1371-1396); the M2L
        in FP32 on size-scaled expansions for ``precision="mixed"`` (orders up to 16)."""
        from tree_d_3d_b200 import _cartesian

        t = self._cartesian_tables()
        n_coef = _cartesian.size(self.order)
        stream = _lib.stream(self.device)
        if moments is None:
            moments = self._cartesian_moments()
        local = torch.zeros((dst.node_count, n_coef), dtype=torch.float64, device=self.device)
        if n_m2l and self.precision == "mixed" and self.order <= 16:
            _lib.call("td3_cart_m2l_mixed", rows.data_ptr(), partners.data_ptr(), dst.node_count,
                      dst.node_center.data_ptr(), dst.node_half.data_ptr(),
                      self.node_center.data_ptr(), self.node_half.data_ptr(),
                      moments.data_ptr(), self.order, float(softening), local.data_ptr(), stream)
        elif n_m2l:
            _lib.call("td3_cart_m2l", rows.data_ptr(), partners.data_ptr(), dst.node_count,
                      dst.node_center.data_ptr(), self.node_center.data_ptr(),
                      moments.data_ptr(), self.order, float(softening),
                      t["m2l_a"].data_ptr(), t["m2l_g"].data_ptr(), t["m2l_coef"].data_ptr(),
                      t["m2l_start32"].data_ptr(), local.data_ptr(), stream)
        if downward:
            self._cart_downward(dst, local)
        return local

    def _cart_downward(self, dst, local) -> None:
        """L2L of Cartesian locals of this tree's order down the cells of ``dst``, level
        by level (td3_cart_downward)."""
        t = self._cartesian_tables()
        levels = np.ascontiguousarray(dst.levels, dtype=np.int64)
        _lib.call("td3_cart_downward", levels.ctypes.data, len(levels) - 1,
                  dst.node_center.data_ptr(), dst.node_child.data_ptr(), self.order,
                  t["ex"].data_ptr(), t["ey"].data_ptr(), t["l2l_start"].data_ptr(),
                  t["l2l_g"].data_ptr(), t["l2l_d"].data_ptr(), t["l2l_coef"].data_ptr(),
                  local.data_ptr(), _lib.stream(self.device))

    # ------------------------------------------------------------------ ranks
    def _shard(self, theta: float, rank: int, world: int) -> dict:
        """Rank ``rank``'s share of the FMM of ``theta`` among ``world`` ranks, as the
        reference's _fmm_shares (ft:830-851): an even run of the M2L pairs (with the
        order the M2L kernel reads) and a run of leaves with about an even share of the
        near-field work (a near-field plan of those leaves only)."""
        key = (theta, rank, world)
        if key not in self._shard_cache:
            lists = self._lists(theta)
            m2l = lists["m2l"]
            pairs = _shards.share(torch.ones(m2l.shape[0], device=self.device), rank, world)
            mine = m2l[pairs]
            part = _Lists(self, m2l=mine)
            if self._grouped_m2l():
                part["groups"] = self._m2l_groups(mine, theta)
            else:
                part["m2l_rows"]  # the CSR rows of this run, made now
            work = _shards.leaf_work(self, lists["p2p_rows"], lists["p2p_partners"])
            leaves = _shards.share(work, rank, world)
            idx = torch.arange(self.node_count, device=self.device)
            inside = (idx >= leaves.start) & (idx < leaves.stop)
            end = torch.where(inside, self.node_end, self.node_start).contiguous()
            part["p2p"] = lists["p2p"]
            part["p2p_partners"] = lists["p2p_partners"]
            if self.precision == "mixed":
                # the far field of this share's leaves only (-1: another rank's slot)
                slot = self._slot_leaves()
                keep = (slot >= leaves.start) & (slot < leaves.stop)
                part["slot_leaf"] = torch.where(keep, slot, torch.full_like(slot, -1))
            part["plan"] = _nearfield_plan(lists["p2p_rows"], self, 2 * lists["p2p"].shape[0],
                                           end=end)
            part["pairs"], part["leaves"] = pairs, leaves
            self._shard_cache[key] = part
        return self._shard_cache[key]

    def _shard_locals(self, part: dict, softening: float):
        """The M2L of a share's pairs into zeroed locals (no L2L): the rank's part of
        the locals, completed by a sum over the ranks."""
        if self.kernel == "log":
            return self._log_locals(part, downward=False)
        local = self._cart_locals(part["m2l_rows"], part["m2l_partners"], part["m2l"].shape[0],
                                  self, softening, downward=False)
        return local, local

    def _shard_near(self, part: dict, local_a, local_b, softening, potential, phi, field,
                    status) -> None:
        """L2P + P2P of a share's leaves into phi and field (zero elsewhere)."""
        kernel = _lib.KERNEL_LOG if self.kernel == "log" else _lib.KERNEL_COULOMB
        with_pot = potential if self.kernel == "log" else True
        self._evaluate_near(part, kernel, local_a, local_b, softening, with_pot, phi, field,
                            status)

    def _full_downward(self, local_a, local_b) -> None:
        if self.kernel == "log":
            self._downward(local_a, local_b, self.order, self._binomial())
        else:
            self._cart_downward(self, local_a)

    def _fmm_sharded(self, theta, softening, potential, phi, field) -> None:
        """fmm over the ranks of ``comm`` (ft:1505-1539, :1600-1631): the same tree and
        lists on every rank; this rank's M2L pairs into its locals, summed over the
        ranks; L2L everywhere; this rank's leaves' near field, the potential and field
        summed over the ranks and the coincidence status maximised."""
        part = self._shard(theta, self._rank, self._world)
        local_a, local_b = self._shard_locals(part, softening)
        _shards.allsum(local_a, self.comm)
        if local_b is not local_a:
            _shards.allsum(local_b, self.comm)
        self._full_downward(local_a, local_b)
        status = status_word(self.device)
        self._shard_near(part, local_a, local_b, softening, potential, phi, field, status)
        _shards.allsum(phi, self.comm)
        _shards.allsum(field, self.comm)
        _shards.allmax(status, self.comm)
        _check(status)
        self._check_tensor_cores()
        self._fwd_locals = None
        lists = self._lists(theta)
        self.fmm_pairs = (int(lists["m2l"].shape[0]), int(lists["p2p"].shape[0]))
        if not potential:
            phi.zero_()

    def _coulomb_fmm(self, theta, softening, phi, field, status=None):
        """ft:1360-1428: the Coulomb FMM with Cartesian expansions (the potential is
        always computed, as in the reference); ``status`` as fmm's ``_status``."""
        lists = self._lists(theta)
        deferred = status is not None
        status = status_word(self.device) if status is None else status
        overlap = self._mixed and NEAR_SPLIT and NEAR_OVERLAP
        if overlap:  # as fmm's log kernel: the pair sums beside the M2L and L2L
            lists["m2l_rows"]
            ready = torch.cuda.Event()
            ready.record(torch.cuda.current_stream(self.device))
        local = self._cart_locals(lists["m2l_rows"], lists["m2l_partners"],
                                  lists["m2l"].shape[0], self, softening)
        self._fwd_locals = ((theta, softening), local, local)
        if overlap:
            done = self._near_part(lists, _lib.KERNEL_COULOMB, softening, True, phi, field,
                                   status, after=ready)
            torch.cuda.current_stream(self.device).wait_event(done)
            _lib.call("td3_fmm_far_mixed", _lib.KERNEL_COULOMB, self._sorted_pos.data_ptr(),
                      self.perm.data_ptr(), self.pos.shape[1], self.node_center.data_ptr(),
                      self.order, local.data_ptr(), local.data_ptr(),
                      self._slot_leaves().data_ptr(), 1, phi.data_ptr(), field.data_ptr(),
                      _lib.stream(self.device))
        else:
            self._evaluate_near(lists, _lib.KERNEL_COULOMB, local, local, softening, True,
                                phi, field, status)
        if not deferred:
            _check(status)
        self.fmm_pairs = (int(lists["m2l"].shape[0]), int(lists["p2p"].shape[0]))
