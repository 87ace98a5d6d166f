"""The mixed-precision M2L with a group of 8 lanes per destination row
(td3_fmm_m2l_mixed_rows, the step's form) against the lane-per-translation form and
FP64 on the same lists and moments: the locals to FP32 accuracy, the same bits every
run, at every template order (rows above 96 entries, taken by a whole warp, included).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [3, 4, 8, 12, 16, 20])
def test_row_group_m2l_matches_lane_form_and_fp64(order, monkeypatch):
    from tree_d_3d_b200 import FlatQuadtree, Quad, flat_tree, synthetic

    monkeypatch.setattr(flat_tree, "M2L_GROUPED", False)
    pos, q = synthetic.mixture8(150_000, seed=60 + order)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    ref = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=order)
    fp64 = [t.cpu().numpy() for t in ref._log_locals(ref._lists(0.5))]
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=order, precision="mixed")
    lists = tree._lists(0.5)
    rows = lists["m2l_rows"].cpu().numpy()
    assert np.diff(rows).max() > 96  # the whole-warp rows are exercised
    runs = {}
    for form in (True, False):
        monkeypatch.setattr(flat_tree, "M2L_ROWS", form)
        runs[form] = [t.cpu().numpy() for t in tree._log_locals(lists)]
    monkeypatch.setattr(flat_tree, "M2L_ROWS", True)
    again = [t.cpu().numpy() for t in tree._log_locals(lists)]
    for part in (0, 1):
        assert relative(runs[True][part], fp64[part]) < 1e-6
        assert relative(runs[True][part], runs[False][part]) < 1e-6
        assert np.array_equal(again[part], runs[True][part])


def test_row_group_m2l_records_and_rejections():
    """The packed source records hold the centre, the scaled moments and h / unit; the
    entry points reject orders above 20 and non-positive units."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, _lib, synthetic

    pos, q = synthetic.uniform(5_000, seed=3)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=12, precision="mixed")
    rec = tree._source_records((tree.moment_re, tree.moment_im)).cpu().numpy()
    assert rec.shape[1] == _lib.lib().td3_m2l_record_floats(12) == 32
    centre = rec[:, :4].copy().view(np.float64)
    assert np.array_equal(centre, tree.node_center.cpu().numpy())
    half = tree.node_half.cpu().numpy()
    mre, mim = tree.moment_re.cpu().numpy(), tree.moment_im.cpu().numpy()
    k = np.arange(13)
    scale = (1.0 / half)[:, None] ** k[None, :]
    hat = rec[:, 4:30].reshape(-1, 13, 2)
    assert relative(hat[..., 0], (mre * scale).astype(np.float32)) < 1e-6
    assert relative(hat[..., 1], (mim * scale).astype(np.float32)) < 1e-6
    assert np.allclose(rec[:, 30], (half / tree._unit).astype(np.float32))
    assert _lib.lib().td3_m2l_record_floats(21) == _lib.EINVAL
    rc = _lib.lib().td3_pack_m2l_sources(1, 12, 0, 0, 0, 0, 0.0, 0, 0)
    assert rc == _lib.EINVAL
    rc = _lib.lib().td3_fmm_m2l_mixed_rows(0, 0, 1, 0, 0, 0, 21, 0, 1.0, 0, 0, 0)
    assert rc == _lib.EINVAL


def test_row_group_m2l_on_runs_of_empty_rows():
    """Rows of a real tree with a contiguous half emptied (the shape of fmm_at's target
    rows, where a run of empty or short rows once fell to one warp): the row-group form
    through the C ABI against the lane-per-entry form on the same rows, to FP32 accuracy,
    the same bits every run."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, _lib, synthetic
    from tree_d_3d_b200.flat_tree import _m2l_coefficients

    pos, q = synthetic.mixture8(150_000, seed=81)
    P, Q = torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda")
    tree = FlatQuadtree(P, Q, Quad(0, 0, 1), kernel="log", order=12, precision="mixed")
    lists = tree._lists(0.5)
    rows = lists["m2l_rows"].cpu().numpy()
    partners = lists["m2l_partners"].cpu().numpy()
    n = tree.node_count
    length = np.diff(rows)
    length[n // 4: 3 * n // 4] = 0  # half the rows emptied, in one run
    keep = np.repeat(np.diff(rows) == length, np.diff(rows))
    new_rows = np.concatenate(([0], np.cumsum(length))).astype(np.int64)
    new_partners = partners[: rows[-1]][keep]
    entry_row = np.repeat(np.arange(n, dtype=np.int32), length)
    dev = tree.device
    R = torch.tensor(new_rows, device=dev)
    S = torch.tensor(np.ascontiguousarray(new_partners), device=dev)
    E = torch.tensor(entry_row, device=dev)
    coeff = np.ascontiguousarray(_m2l_coefficients(tree.order, tree.symmetric))
    moments = (tree.moment_re, tree.moment_im)
    records = tree._source_records(moments)
    hat = tree._scaled_moments(moments)
    stream = _lib.stream(dev)

    def run(rows_form):
        lre = torch.zeros((n, 13), dtype=torch.float64, device=dev)
        lim = torch.zeros_like(lre)
        if rows_form:
            _lib.call("td3_fmm_m2l_mixed_rows", R.data_ptr(), S.data_ptr(), n,
                      tree.node_center.data_ptr(), tree.node_half.data_ptr(),
                      records.data_ptr(), 12, coeff.ctypes.data, tree._unit, lre.data_ptr(),
                      lim.data_ptr(), stream)
        else:
            _lib.call("td3_fmm_m2l_mixed", R.data_ptr(), E.data_ptr(), S.data_ptr(), n,
                      tree.node_center.data_ptr(), tree.node_half.data_ptr(),
                      tree.node_center.data_ptr(), tree.node_half.data_ptr(), hat.data_ptr(),
                      12, coeff.ctypes.data, tree._unit, 0, lre.data_ptr(), lim.data_ptr(), 0,
                      stream)
        return lre.cpu().numpy(), lim.cpu().numpy()

    a, b, c = run(True), run(True), run(False)
    for part in (0, 1):
        assert np.array_equal(a[part], b[part])
        assert relative(a[part], c[part]) < 1e-6
        assert not a[part][n // 4: 3 * n // 4].any()  # the emptied rows stay zero

