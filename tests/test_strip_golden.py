"""The strip fixtures (made by the reference's GroundedStripField) against the strip's
closed forms, on the CPU: the image force on a lone charge and the Green's function of
the grounded strip summed directly."""

from __future__ import annotations

import numpy as np

from conftest import golden, relative


def test_lone_charge_fixture_is_the_image_force():
    data = golden("strip")
    width, q, x = 2.5, 1.5, 0.7
    expect = -np.pi * q / width / np.tan(np.pi * x / width)
    assert abs(data["lone/field"][0, 0] - expect) <= 1e-12 * abs(expect)
    assert abs(data["lone/field"][1, 0]) < 1e-12


def test_direct_probe_fixture_is_the_strip_green_function():
    """phi(z) = -k sum_j q_j ln[(sin^2((x - x_j)/2a) + sinh^2((y - y_j)/2a)) /
    (sin^2((x + x_j)/2a) + sinh^2((y - y_j)/2a))], a = L / pi."""
    from tree_d_3d_b200.constants import K_E

    data = golden("strip")
    pos, q, pts = data["pos"], data["charge"], data["points"]
    a = float(data["width"]) / np.pi

    def sin2(re, im):
        return np.sin(re / (2 * a)) ** 2 + np.sinh(im / (2 * a)) ** 2

    x, y = pts[0][:, None], pts[1][:, None]
    xj, yj = pos[0][None, :], pos[1][None, :]
    phi = -K_E * (q[None, :] * np.log(sin2(x - xj, y - yj) / sin2(x + xj, y - yj))).sum(1)
    assert relative(data["direct/eps0.0/probe_phi"], phi) < 1e-12
