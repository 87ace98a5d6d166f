"""Host-side logic of the package, run without a GPU.

The C-ABI library must load and export every entry point that include/treed3d.h
declares (no compute calls here); argument validation, the Cartesian tables, the M2L
matrix and the binomial table must equal the reference's; the synthetic generators
must produce the documented distributions.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden


def test_library_exports_every_declared_entry_point():
    from tree_d_3d_b200 import _lib

    handle = _lib.lib()
    names = _lib.declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(handle, name), name
    assert handle.td3_version() >= 100
    # pure host size queries
    assert _lib.query("td3_direct_sum_workspace_size", 100, 10_000) > 0
    assert _lib.query("td3_quadtree_build_workspace_size", 1000, 4000) > 0
    assert _lib.query("td3_walk_workspace_size", 1000, 0) > 0
    assert _lib.query("td3_fmm_traverse_workspace_size", 1000, 500) > 0
    assert _lib.query("td3_pair_csr_workspace_size", 1000, 1, 500) > 0
    assert _lib.query("td3_nearfield_plan_workspace_size", 500) > 0


def test_library_rejects_bad_arguments_without_touching_the_gpu():
    from tree_d_3d_b200 import _lib

    handle = _lib.lib()
    null = ctypes.c_void_p(0)
    # negative sizes and unknown kernels are refused before any launch
    rc = handle.td3_direct_sum(7, null, 1, null, null, null, 1, 0.0, 1, null, null, null, null,
                               0, null)
    assert rc == _lib.EINVAL
    rc = handle.td3_direct_sum(0, null, -1, null, null, null, 1, 0.0, 1, null, null, null, null,
                               0, null)
    assert rc == _lib.EINVAL
    rc = handle.td3_fmm_m2l(null, null, -1, null, null, null, null, 12, null, null, null, null)
    assert rc == _lib.EINVAL
    rc = handle.td3_fmm_m2l(null, null, 10, null, null, null, null, 65, null, null, null, null)
    assert rc == _lib.EINVAL


def test_validation_messages_match_the_reference():
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    with pytest.raises(ValueError, match="kernel must be one of"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), kernel="yukawa")
    with pytest.raises(ValueError, match="order must be a positive integer"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), order=0)
    with pytest.raises(ValueError, match="order must be at most 64"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), order=65)
    with pytest.raises(ValueError, match="half_size must be positive"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 0))
    with pytest.raises(ValueError, match="leaf_capacity must be a positive integer"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), leaf_capacity=0)
    # comm is a torch.distributed process group; without an initialised group it is refused
    with pytest.raises(ValueError, match="comm must be a torch.distributed process group"):
        FlatQuadtree([[0.0], [0.0]], [1.0], Quad(0, 0, 1), comm=object())
    with pytest.raises(ValueError, match="kernel must be one of"):
        direct_field([[0.0], [0.0]], [[0.0], [0.0]], [1.0], kernel="yukawa")


def test_status_words_become_the_reference_exceptions():
    from tree_d_3d_b200._utils import _check_code

    _check_code(0)
    with pytest.raises(ValueError, match="Coincident charges require positive softening"):
        _check_code(17)
    with pytest.raises(RuntimeError, match="too deep"):
        _check_code(-1)


def test_cartesian_tables_equal_the_reference():
    from tree_d_3d_b200 import _cartesian

    data = golden("tables")
    for order in (4, 8, 12):
        t = _cartesian.tables(order)
        for name in ("ex", "ey", "mono_parent", "mono_dir", "rec", "grad", "m2l", "m2l_coef",
                     "shift", "shift_coef"):
            np.testing.assert_array_equal(t[name], data[f"p{order}/{name}"], err_msg=name)
        # the regrouped views cover every row once
        assert t["m2l_start32"][-1] == len(t["m2l"])
        assert t["l2l_start"][-1] == len(t["shift"])
        rows = sorted(zip(t["l2l_g"].tolist(), t["l2l_d"].tolist()))
        assert rows == sorted((int(g), int(d)) for g, _, d in t["shift"])


def test_m2l_matrix_and_binomials_equal_the_oracle(oracle):
    from tree_d_3d_b200.flat_tree import _binomial_table, _m2l_coefficients

    for size in (5, 25, 129):
        np.testing.assert_array_equal(_binomial_table(size), oracle.binomial_table(size))
    for order in (1, 6, 12, 40, 64):
        for symmetric in (False, True):
            np.testing.assert_array_equal(_m2l_coefficients(order, symmetric),
                                          oracle.m2l_coefficients(order, symmetric))


def test_synthetic_distributions():
    from tree_d_3d_b200 import synthetic

    pos, q = synthetic.mixture8(20_000, seed=3)
    assert pos.shape == (2, 20_000) and np.all(np.abs(pos) < 1)
    assert q.sum() == 0 and set(np.unique(q)) == {-1.0, 1.0}
    pos, q = synthetic.gaussian(5000, 0.3, seed=1)
    assert np.all(np.abs(pos) < 1) and pos.shape == (2, 5000)
    pos, q = synthetic.protons(3000)
    assert np.all(q == 1) and np.all(np.abs(pos) < 1)
    a = synthetic.mixture8(1000, seed=9)[0]
    b = synthetic.mixture8(1000, seed=9)[0]
    np.testing.assert_array_equal(a, b)


def test_strip_arguments_are_checked_like_the_reference():
    from tree_d_3d_b200.strip import GroundedStripField

    for width in (0.0, -1.0, float("inf")):
        with pytest.raises(ValueError, match="width must be finite and positive"):
            GroundedStripField(width)
    with pytest.raises(ValueError, match="method must be"):
        GroundedStripField(1.0, method="walk")
    with pytest.raises(ValueError, match="softening must be finite and nonnegative"):
        GroundedStripField(1.0, softening=-1.0)
    with pytest.raises(ValueError, match="cutoff must exceed 1"):
        GroundedStripField(1.0, cutoff=1.0)
    strip = GroundedStripField(2.0)
    assert (strip.order, strip.theta, strip.leaf_capacity, strip.cutoff) == (14, 0.5, 32, 6.0)


def test_trace_regions_follow_the_reference_names_and_are_off_by_default():
    """NVTX ranges named as the reference's scope-profiler regions
    (src/tree_d_3d/_profiling.py:10-13): off by default, nested when on."""
    from tree_d_3d_b200 import _trace

    was = _trace.enabled()
    _trace.opened.clear()
    try:
        _trace.enable(False)
        with _trace.region("flat_tree.fmm"):
            pass
        assert _trace.opened == []

        @_trace.profile("flat_tree.evaluate")
        def walk(x):
            with _trace.region("flat_tree.traverse"):
                return 2 * x

        _trace.enable(True)
        assert walk(3) == 6
        assert _trace.opened == ["tree_d_3d.flat_tree.evaluate", "tree_d_3d.flat_tree.traverse"]
    finally:
        _trace.enable(was)
        _trace.opened.clear()


def test_panel_tree_root_is_the_widened_bounding_square():
    """electrodes.py:1143-1146: centre of the bounding box, half the larger side times
    (1 + 1e-9) plus 1e-300."""
    import torch

    from tree_d_3d_b200.electrodes import FMM_AT_RATIO, FMM_AT_THETA, WALK_THETA, bounding_quad

    pts = torch.tensor([[-0.5, 0.25, 0.75], [0.1, -0.3, 0.2]], dtype=torch.float64)
    q = bounding_quad(pts)
    assert (q.xmid, q.ymid) == (0.125, -0.04999999999999999)
    assert q.half == 0.5 * 1.25 * (1 + 1e-9) + 1e-300
    assert (FMM_AT_THETA, FMM_AT_RATIO, WALK_THETA) == (0.5, 8, 0.7)
