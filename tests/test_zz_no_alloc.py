"""td3_direct_sum_noalloc, the direct sum for callers that cannot allocate device memory.

Such callers (a host application that owns every device buffer and hands the solver
only inputs and outputs) get an entry point whose scratch is a fixed array inside the
library.  Called through the C ABI, it must give the results of td3_direct_sum with a
workspace, on two calls in a row (the second finds the first call's partial sums still
in the shared array), and refuse more targets than the array holds.  This file sorts
last, so a run that stops at the first failure has run every other test first.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _with_workspace(lib, kernel, targets, exclude, pos, q, eps):
    from tree_d_3d_b200 import _lib

    m, n = targets.shape[1], pos.shape[1]
    phi = torch.zeros(m, dtype=torch.float64, device="cuda")
    field = torch.zeros((2, m), dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = _lib.workspace(lib.td3_direct_sum_workspace_size(m, n), targets.device)
    rc = lib.td3_direct_sum(kernel, targets.data_ptr(), m, exclude.data_ptr(), pos.data_ptr(),
                            q.data_ptr(), n, eps, 1, phi.data_ptr(), field.data_ptr(),
                            status.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream())
    assert rc == 0
    return phi, field, status


def _without_allocation(lib, kernel, targets, exclude, pos, q, eps):
    from tree_d_3d_b200 import _lib

    m, n = targets.shape[1], pos.shape[1]
    phi = torch.zeros(m, dtype=torch.float64, device="cuda")
    field = torch.zeros((2, m), dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = lib.td3_direct_sum_noalloc(kernel, targets.data_ptr(), m, exclude.data_ptr(),
                                    pos.data_ptr(), q.data_ptr(), n, eps, 1, phi.data_ptr(),
                                    field.data_ptr(), status.data_ptr(), _lib.stream())
    assert rc == 0
    return phi, field, status


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("m,n", [(37, 5000), (3000, 200_000), (65536, 8192)])
def test_noalloc_direct_sum_matches_the_workspace_entry(kernel, m, n):
    from tree_d_3d_b200 import _lib

    lib = _lib.lib()
    rng = np.random.default_rng(kernel * 7 + m)
    dev = torch.device("cuda")
    targets = torch.tensor(rng.uniform(-1, 1, (2, m)), device=dev)
    pos = torch.tensor(rng.normal(0, 0.4, (2, n)), device=dev)
    q = torch.tensor(rng.choice([-1.0, 1.0], n), device=dev)
    exclude = torch.tensor(rng.integers(-1, n, m), device=dev)
    ref = _with_workspace(lib, kernel, targets, exclude, pos, q, 1e-3)
    for _ in range(2):
        got = _without_allocation(lib, kernel, targets, exclude, pos, q, 1e-3)
        torch.cuda.synchronize()
        assert int(got[2].item()) == int(ref[2].item()) == 0
        assert relative(got[0].cpu().numpy(), ref[0].cpu().numpy()) <= TOL
        assert relative(got[1].cpu().numpy(), ref[1].cpu().numpy()) <= TOL


def test_noalloc_direct_sum_refuses_more_targets_than_its_scratch():
    from tree_d_3d_b200 import _lib

    lib = _lib.lib()
    m = 65537
    dev = torch.device("cuda")
    targets = torch.zeros((2, m), dtype=torch.float64, device=dev)
    exclude = torch.full((m,), -1, dtype=torch.int64, device=dev)
    pos = torch.ones((2, 4), dtype=torch.float64, device=dev)
    q = torch.ones(4, dtype=torch.float64, device=dev)
    phi = torch.zeros(m, dtype=torch.float64, device=dev)
    field = torch.zeros((2, m), dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int64, device=dev)
    rc = lib.td3_direct_sum_noalloc(0, targets.data_ptr(), m, exclude.data_ptr(), pos.data_ptr(),
                                    q.data_ptr(), 4, 0.0, 1, phi.data_ptr(), field.data_ptr(),
                                    status.data_ptr(), _lib.stream())
    assert rc == _lib.ETOOLARGE
    assert b"TD3_DIRECT_NOALLOC_MAX_TARGETS" in lib.td3_last_error()
