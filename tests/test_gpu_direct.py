"""direct_field on the GPU against the oracle and the reference's golden vectors.

Tolerance: the CUDA sums use rsqrt / FMA and a different summation order, so they
match the reference's CPU sums to 1e-12 normwise, not bitwise.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, relative

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
@pytest.mark.parametrize("eps", [0.0, 0.01])
def test_direct_field_matches_golden(kernel, eps):
    from tree_d_3d_b200 import direct_field

    data = golden("direct")
    phi, field = direct_field(data["targets"], data["pos"], data["charge"], softening=eps,
                              exclude=data["exclude"], kernel=kernel)
    assert relative(phi, data[f"{kernel}/eps{eps}/phi"]) < TOL
    assert relative(field, data[f"{kernel}/eps{eps}/field"]) < TOL


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
@pytest.mark.parametrize("m,n", [(1, 1), (37, 5000), (4096, 200_000), (70_000, 300)])
def test_direct_field_matches_oracle(oracle, kernel, m, n):
    from tree_d_3d_b200 import direct_field

    rng = np.random.default_rng(m + n)
    targets = rng.uniform(-1, 1, (2, m))
    pos = rng.normal(0, 0.3, (2, n))
    q = rng.choice([-1.0, 1.0], n)
    q[::5] = 0.0
    exclude = rng.integers(-1, n, m)
    ref = oracle.direct_field(targets, pos, q, softening=1e-3, exclude=exclude, kernel=kernel)
    got = direct_field(torch.tensor(targets, device="cuda"), torch.tensor(pos, device="cuda"),
                       torch.tensor(q, device="cuda"), softening=1e-3,
                       exclude=torch.tensor(exclude, device="cuda"), kernel=kernel)
    assert isinstance(got[0], torch.Tensor) and got[0].is_cuda
    assert relative(got[0].cpu().numpy(), ref[0]) < TOL
    assert relative(got[1].cpu().numpy(), ref[1]) < TOL


def test_direct_field_config1_and_coincidence():
    from tree_d_3d_b200 import direct_field

    data = golden("evaluate")
    pos, charge = data["config1/pos"], data["config1/charge"]
    phi, field = direct_field(pos, pos, charge, softening=1e-3, exclude=np.arange(5000))
    assert relative(phi, data["config1/direct_phi"]) < TOL
    assert relative(field, data["config1/direct_field"]) < TOL
    pos = np.array([[0.1, 0.1, 0.5], [0.1, 0.1, -0.2]])
    with pytest.raises(ValueError, match="Coincident"):
        direct_field(pos, pos, np.ones(3), exclude=np.arange(3))
    # neutral coincident partners are skipped as sources
    phi, _ = direct_field(pos, pos, np.array([0.0, 0.0, 1.0]), exclude=np.arange(3))
    assert np.all(np.isfinite(phi))


def test_empty_inputs():
    from tree_d_3d_b200 import direct_field

    phi, field = direct_field(np.zeros((2, 0)), np.zeros((2, 3)), np.ones(3))
    assert phi.shape == (0,) and field.shape == (2, 0)
    phi, field = direct_field(np.zeros((2, 4)), np.zeros((2, 0)), np.ones(0))
    assert not np.any(phi) and field.shape == (2, 4)
