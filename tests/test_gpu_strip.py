"""GroundedStripField on the GPU against the reference's golden vectors and the strip's
closed forms.

The direct method is the reference's arithmetic up to summation order and the device's
exp / sin / cos in the map: 1e-12 normwise.  The FMM method builds its tree on the
mapped points, whose last bits come from those functions, so a point on a cell edge can
fall into another cell than in the reference: its fields agree to the FMM's truncation
error (the reference's own FMM and direct sums differ by 8e-10 here), checked at 1e-8.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, relative

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,tol", [("direct", 1e-12), ("fmm", 1e-8)])
@pytest.mark.parametrize("eps", [0.0, 0.02])
def test_strip_matches_golden(method, tol, eps):
    from tree_d_3d_b200.strip import GroundedStripField

    data = golden("strip")
    pos, charge, points = data["pos"], data["charge"], data["points"]
    strip = GroundedStripField(float(data["width"]), method=method, softening=eps)
    key = f"{method}/eps{eps}"
    phi, field = strip.field_at_charges(pos, charge)
    assert relative(phi, data[f"{key}/phi"]) < tol
    assert relative(field, data[f"{key}/field"]) < tol
    phi0, field0 = strip.field_at_charges(pos, charge, potential=False)
    assert not np.any(phi0)
    assert relative(field0, data[f"{key}/field_nopot"]) < tol
    pphi, pfield = strip.probe(pos, charge, points)
    assert relative(pphi, data[f"{key}/probe_phi"]) < tol
    assert relative(pfield, data[f"{key}/probe_field"]) < tol
    assert relative(strip.potential(pos, charge, points), pphi) == 0.0


def test_lone_charge_feels_the_image_force_of_the_plates():
    """E_x = -pi k q / L cot(pi x / L), E_y = 0 (strip.py:213-215), and the golden value."""
    from tree_d_3d_b200.strip import GroundedStripField

    data = golden("strip")
    width, q = 2.5, 1.5
    strip = GroundedStripField(width, k_e=1.0)
    for x in (0.3, 0.7, 1.25, 2.2):
        phi, field = strip.field_at_charges(np.array([[x], [0.3]]), np.array([q]))
        expect = -np.pi * q / width / np.tan(np.pi * x / width)
        assert abs(field[0, 0] - expect) <= 1e-12 * max(1.0, abs(expect))
        assert abs(field[1, 0]) < 1e-12
        if x == 0.7:
            assert relative(phi, data["lone/phi"]) < 1e-12
            assert relative(field, data["lone/field"]) < 1e-12


def test_probe_potential_is_the_strip_green_function():
    """phi = -k q ln[(sin^2((x - x0)/2a) + sinh^2((y - y0)/2a)) /
    (sin^2((x + x0)/2a) + sinh^2((y - y0)/2a))], a = L / pi (strip.py:55-68)."""
    from tree_d_3d_b200.strip import GroundedStripField

    rng = np.random.default_rng(3)
    width, q, k_e = 2.3, 0.8, 1.7
    src = np.array([[0.9], [0.2]])
    pts = np.stack((rng.uniform(0.1, 2.2, 50), rng.uniform(-1, 1, 50)))
    a = width / np.pi
    for method in ("fmm", "direct"):
        strip = GroundedStripField(width, k_e=k_e, method=method)
        phi = strip.potential(src, np.array([q]), pts)

        def sin2(re, im):
            return np.sin(re / (2 * a)) ** 2 + np.sinh(im / (2 * a)) ** 2

        x, y, x0, y0 = pts[0], pts[1], src[0, 0], src[1, 0]
        expect = -k_e * q * np.log(sin2(x - x0, y - y0) / sin2(x + x0, y - y0))
        assert relative(phi, expect) < 1e-11


def test_strip_fmm_matches_direct_at_scale_and_tensors_stay_on_device():
    """60k charges: the mapped points span several decades (|zeta| = exp(-pi y / L)), and
    the order-14 FMM stays within 1e-6 of the direct sum."""
    from tree_d_3d_b200.strip import GroundedStripField

    rng = np.random.default_rng(11)
    n, width = 60_000, 3.0
    pos = torch.tensor(np.stack((rng.uniform(0.01, 0.99, n) * width, rng.normal(0, 1.0, n))),
                       device="cuda")
    q = torch.tensor(rng.normal(size=n), device="cuda")
    fmm = GroundedStripField(width, softening=0.004).field_at_charges(pos, q)
    direct = GroundedStripField(width, method="direct", softening=0.004).field_at_charges(pos, q)
    for a, b in zip(fmm, direct):
        assert a.is_cuda
        assert relative(a.cpu().numpy(), b.cpu().numpy()) < 1e-6


def test_strip_errors():
    from tree_d_3d_b200.strip import GroundedStripField

    strip = GroundedStripField(2.0, softening=0.01)
    with pytest.raises(ValueError, match="strictly between the plates"):
        strip.field_at_charges(np.array([[2.0], [0.0]]), np.array([1.0]))
    with pytest.raises(ValueError, match="strictly between the plates"):
        strip.probe(np.array([[1.0], [0.0]]), np.array([1.0]), np.array([[-0.1], [0.0]]))
    with pytest.raises(ValueError, match="same length"):
        strip.field_at_charges(np.array([[1.0, 1.5], [0.0, 0.1]]), np.array([1.0]))
    with pytest.raises(ValueError, match="Coincident charges"):
        strip.field_at_charges(np.array([[1.0, 1.0], [0.2, 0.2]]), np.array([1.0, -1.0]))
    # a probe on a charge: the mapped-plane walk reports it first, as in the reference
    for method in ("fmm", "direct"):
        with pytest.raises(ValueError, match="Coincident charges"):
            GroundedStripField(2.0, softening=0.01, method=method).probe(
                np.array([[1.0], [0.2]]), np.array([1.0]), np.array([[1.0], [0.2]]))
    phi, field = strip.field_at_charges(np.zeros((2, 0)), np.zeros(0))
    assert phi.shape == (0,) and field.shape == (2, 0)
    assert np.allclose(np.abs(strip.to_plane(np.array([[0.5], [0.0]]))), 1.0)
