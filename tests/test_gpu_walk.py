"""The GPU Barnes-Hut walk against the reference's golden vectors and the oracle.

Each target gets exactly the terms of the reference's walk (the opening decisions
are evaluated with exactly rounded operations); the terms themselves use rsqrt and
FMA, so results match to 1e-12 normwise.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, relative

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
@pytest.mark.parametrize("leaf", [1, 8])
@pytest.mark.parametrize("theta", [0.0, 0.5, 1.2])
def test_walk_matches_golden(kernel, leaf, theta):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("evaluate")
    pos, charge = data["cloud/pos"], data["cloud/charge"]
    depth = 10 if leaf == 1 else 48
    tree = FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=leaf, max_depth=depth,
                        kernel=kernel)
    phi, field = tree.evaluate(pos, exclude=np.arange(pos.shape[1]), theta=theta,
                               softening=0.01)
    key = f"cloud/{kernel}/l{leaf}/t{theta}"
    assert relative(phi, data[f"{key}/phi"]) < TOL
    assert relative(field, data[f"{key}/field"]) < TOL


def test_walk_config1_and_probes():
    from tree_d_3d_b200 import FlatQuadtree, Quad

    data = golden("evaluate")
    pos, charge = data["config1/pos"], data["config1/charge"]
    tree = FlatQuadtree(pos, charge, Quad(0, 0, 1))
    phi, field = tree.evaluate(pos, exclude=np.arange(5000), theta=0.5, softening=1e-3)
    assert relative(phi, data["config1/phi"]) < TOL
    assert relative(field, data["config1/field"]) < TOL
    pos, q, probes = data["probes/pos"], data["probes/charge"], data["probes/targets"]
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=10)
    for potential in (True, False):
        phi, field = tree.evaluate(probes, theta=0.6, potential=potential)
        assert relative(field, data[f"probes/log/pot{int(potential)}/field"]) < TOL
        if potential:
            assert relative(phi, data["probes/log/pot1/phi"]) < TOL
        else:
            assert not np.any(phi)
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1))
    phi, field = tree.evaluate(probes, theta=0.6, softening=0.002)
    assert relative(phi, data["probes/coulomb/phi"]) < TOL
    assert relative(field, data["probes/coulomb/field"]) < TOL


@pytest.mark.parametrize("kernel", ["coulomb", "log"])
def test_walk_large_matches_oracle(oracle, kernel):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    rng = np.random.default_rng(31)
    n = 200_000
    pos = rng.normal(0, 0.3, (2, n))
    keep = np.all(np.abs(pos) < 1, axis=0)
    pos = pos[:, keep]
    n = pos.shape[1]
    q = rng.choice([-1.0, 1.0], n)
    probes = rng.uniform(-1, 1, (2, 20_000))
    order = 12 if kernel == "log" else None
    ref_tree = oracle.OracleTree(pos, q, (0, 0, 1), kernel=kernel, order=order)
    tree = FlatQuadtree(torch.tensor(pos, device="cuda"), torch.tensor(q, device="cuda"),
                        Quad(0, 0, 1), kernel=kernel, order=order)
    for targets, exclude in ((pos, np.arange(n)), (probes, None)):
        ref = ref_tree.evaluate(targets, exclude=exclude, theta=0.5, softening=1e-3)
        got = tree.evaluate(torch.tensor(targets, device="cuda"),
                            exclude=None if exclude is None else torch.tensor(exclude, device="cuda"),
                            theta=0.5, softening=1e-3)
        assert relative(got[0].cpu().numpy(), ref[0]) < TOL
        assert relative(got[1].cpu().numpy(), ref[1]) < TOL


def test_walk_theta_zero_is_the_direct_sum_and_coincidence_raises():
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    rng = np.random.default_rng(5)
    pos = rng.uniform(-0.9, 0.9, (2, 3000))
    q = rng.normal(size=3000)
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1), leaf_capacity=4)
    own = np.arange(3000)
    a = tree.evaluate(pos, exclude=own, theta=0.0, softening=0.01)
    b = direct_field(pos, pos, q, exclude=own, softening=0.01)
    assert relative(a[0], b[0]) < TOL and relative(a[1], b[1]) < TOL
    pos[:, 7] = pos[:, 3]
    tree = FlatQuadtree(pos, q, Quad(0, 0, 1))
    with pytest.raises(ValueError, match="Coincident"):
        tree.evaluate(pos, exclude=own)
    phi, _ = tree.evaluate(pos, exclude=own, softening=0.01)
    assert np.all(np.isfinite(phi))


def test_field_at_and_reference_radius():
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    tree = FlatQuadtree([[0.0], [0.0]], [2.0], Quad(0, 0, 1), kernel="log")
    phi, field = tree.field_at([[3.0], [4.0]], k_e=1.0, reference_radius=2.0)
    assert phi[0] == pytest.approx(-2 * 2.0 * np.log(5.0 / 2.0))
    np.testing.assert_allclose(field[:, 0], 2 * 2.0 * np.array([3.0, 4.0]) / 25)
    rng = np.random.default_rng(4)
    pos = rng.normal(0, 0.3, (2, 100)).clip(-0.99, 0.99)
    charge = rng.normal(size=100)
    tree = FlatQuadtree(pos, charge, Quad(0, 0, 1))
    probes = np.array([[3.0, 0.0], [0.0, -4.0]])
    phi, field = tree.field_at(probes, theta=0, k_e=2, softening=0.01)
    ref_phi, ref_field = direct_field(probes, pos, charge, softening=0.01)
    np.testing.assert_allclose(phi, 2 * ref_phi, rtol=1e-12)
    np.testing.assert_allclose(field, 2 * ref_field, rtol=1e-12)
