"""ElectrostaticSimulation on the GPU and its differentiable rollout.

The scheme is checked against a NumPy integration of the reference's step
(simulation.py:800-835) with the oracle's direct sums; the stepping behaviour against
the reference's own tests (one field evaluation per step, method selection, walls,
the exact cyclotron drift); the rollout's gradient against torch autograd through a
plain PyTorch FP64 direct-sum reference.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import relative

pytestmark = pytest.mark.gpu


def _cloud(n, seed=5):
    rng = np.random.default_rng(seed)
    pos = rng.normal(0, 0.3, (2, n)).clip(-0.95, 0.95)
    q = np.where(rng.random(n) < 0.5, -1.0, 1.0) * rng.uniform(0.5, 2, n)
    return pos, q


def _numpy_steps(oracle, pos, vel, q, m, dt, b_z, k_e, eps, steps):
    """The reference's step (simulation.py:800-835) with the oracle's direct fields."""
    pos, vel = pos.copy(), vel.copy()
    everyone = np.arange(pos.shape[1])

    def force(p):
        _, f = oracle.direct_field(p, p, q, softening=eps, exclude=everyone)
        return k_e * q * f

    e = force(pos)
    for _ in range(steps):
        vel = vel + 0.5 * dt * e / m
        angle = q / m * b_z * dt
        c, s = np.cos(angle), np.sin(angle)
        a = np.sinc(angle / np.pi)
        b = 0.5 * angle * np.sinc(angle / (2 * np.pi)) ** 2
        vx, vy = vel[0], vel[1]
        pos = pos + dt * np.stack((a * vx + b * vy, a * vy - b * vx))
        vel = np.stack((c * vx + s * vy, c * vy - s * vx))
        e = force(pos)
        vel = vel + 0.5 * dt * e / m
    return pos, vel


def test_direct_stepping_matches_a_numpy_integration(oracle):
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.simulation import ElectrostaticSimulation

    pos, q = _cloud(300)
    rng = np.random.default_rng(1)
    vel = rng.normal(0, 0.1, pos.shape)
    m = rng.uniform(1, 2, 300)
    sim = ElectrostaticSimulation(positions=pos, velocities=vel, charges=q, masses=m,
                                  bounds=Quad(0, 0, 1), k_e=1e-3, softening=0.01, dt=1e-2,
                                  B_z=2.0, method="direct")
    for _ in range(10):
        sim.step()
    ref_pos, ref_vel = _numpy_steps(oracle, pos, vel, q, m, 1e-2, 2.0, 1e-3, 0.01, 10)
    assert relative(sim.positions.cpu().numpy(), ref_pos) < 1e-12
    assert relative(sim.velocities.cpu().numpy(), ref_vel) < 1e-12


def test_one_field_evaluation_per_step_and_method_selection(monkeypatch):
    from tree_d_3d_b200 import FlatQuadtree, Quad, simulation
    from tree_d_3d_b200.simulation import ElectrostaticSimulation

    pos, q = _cloud(2000)
    sim = ElectrostaticSimulation(positions=pos, charges=q, bounds=Quad(0, 0, 1), k_e=1,
                                  softening=0.05, dt=1e-3)
    assert sim._resolve_method() == "fmm"
    calls = []
    fmm = FlatQuadtree.fmm
    monkeypatch.setattr(FlatQuadtree, "fmm", lambda *a, **k: calls.append(1) or fmm(*a, **k))
    sim.step()
    assert len(calls) == 2
    for _ in range(3):
        sim.step()
    assert len(calls) == 5
    small = ElectrostaticSimulation(positions=pos[:, :20], charges=q[:20], bounds=Quad(0, 0, 1))
    assert small._resolve_method() == "direct"
    assert ElectrostaticSimulation(positions=pos, charges=q, bounds=Quad(0, 0, 1),
                                   theta=1.2)._resolve_method() == "tree"
    with pytest.raises(ValueError, match="theta"):
        ElectrostaticSimulation(positions=pos, charges=q, bounds=Quad(0, 0, 1), method="fmm",
                                theta=1.0)


def test_exact_cyclotron_drift():
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.simulation import ElectrostaticSimulation

    # one particle, no field: a circle of radius v m / (q B) in closed form
    sim = ElectrostaticSimulation(positions=[[0.0], [0.0]], velocities=[[0.3], [0.0]],
                                  charges=[2.0], masses=[1.5], bounds=Quad(0, 0, 1), k_e=0,
                                  dt=0.37, B_z=0.9)
    for _ in range(7):
        sim.step()
    omega = 2.0 / 1.5 * 0.9
    t = 7 * 0.37
    x = 0.3 / omega * np.sin(omega * t)
    y = 0.3 / omega * (np.cos(omega * t) - 1.0)
    np.testing.assert_allclose(sim.positions.cpu().numpy()[:, 0], [x, y], atol=1e-14)


def test_absorbing_walls_remove_and_record():
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.simulation import ElectrostaticSimulation

    pos = np.array([[0.0, 0.5, -0.5], [0.0, 0.2, -0.1]])
    vel = np.array([[0.0, 10.0, -0.1], [0.0, 0.0, 0.0]])
    sim = ElectrostaticSimulation(positions=pos, velocities=vel, charges=[1.0, 1.0, 1.0],
                                  bounds=Quad(0, 0, 2), k_e=0, dt=0.1,
                                  absorbing_walls={"x_max": 1.0, "x_min": -1.0})
    sim.step()
    assert sim.num_particles == 2 and len(sim.absorbed) == 1
    assert sim.absorbed.counts() == {"x_max": 1}
    with pytest.raises(ValueError, match="inside the absorbing walls"):
        ElectrostaticSimulation(positions=[[2.0], [0.0]], charges=[1.0], bounds=Quad(0, 0, 4),
                                absorbing_walls={"x_max": 1.0})


def test_fmm_and_tree_stepping_track_direct_stepping():
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.simulation import ElectrostaticSimulation

    pos, q = _cloud(3000, seed=9)
    runs = {}
    for method, order in (("direct", None), ("fmm", 12), ("tree", None)):
        sim = ElectrostaticSimulation(positions=pos, charges=q, masses=np.ones(3000),
                                      bounds=Quad(0, 0, 1), k_e=1e-5, softening=1e-3, dt=0.02,
                                      method=method, order=order, theta=0.3)
        for _ in range(5):
            sim.step()
        runs[method] = sim.positions.cpu().numpy()
    assert relative(runs["fmm"], runs["direct"]) < 1e-8
    assert relative(runs["tree"], runs["direct"]) < 1e-4
    sim = ElectrostaticSimulation(positions=pos, charges=q, bounds=Quad(0, 0, 1), k_e=1,
                                  softening=0.01, method="direct")
    assert sim.get_potential_energy() == pytest.approx(sim.get_potential_energy(exact=True),
                                                       rel=1e-12)


def _torch_field(pos, q, eps):
    """plain PyTorch FP64 Coulomb field at every particle (own charge excluded)"""
    d = pos[:, :, None] - pos[:, None, :]
    r2 = d[0] ** 2 + d[1] ** 2 + eps * eps
    eye = torch.eye(pos.shape[1], dtype=torch.bool, device=pos.device)
    r2 = torch.where(eye, torch.ones_like(r2), r2)
    qj = torch.where(eye, torch.zeros_like(r2), q[None, :].expand_as(r2))
    inv = r2.rsqrt()
    return (qj * inv).sum(1), ((qj * inv**3)[None] * d).sum(2)


def test_rollout_gradient_matches_torch_autograd_of_direct_fields():
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.simulation import rollout_kinetic_energy

    rng = np.random.default_rng(3)
    n = 1500
    pos0 = rng.normal(0, 0.1, (2, n)).clip(-0.9, 0.9)
    q0 = rng.uniform(0.5, 1.5, n)
    grads = []
    for fmm in (True, False):
        pos = torch.tensor(pos0, device="cuda")
        q = torch.tensor(q0, device="cuda", requires_grad=True)
        vel = torch.zeros_like(pos)
        m = torch.ones(n, dtype=torch.float64, device="cuda")
        ke = rollout_kinetic_energy(
            pos, vel, q, m, 5, bounds=Quad(0, 0, 1), dt=1e-3, B_z=1.0, k_e=1e-2,
            softening=1e-3, order=14, theta=0.4, absorbing_walls={"x_max": 1.0},
            field_fn=None if fmm else (lambda p, c: _torch_field(p, c, 1e-3)))
        ke.backward()
        grads.append(q.grad.cpu().numpy())
    assert relative(grads[0], grads[1]) < 1e-6


def test_config5_shape_steps_and_checkpointed_gradient():
    """Config 5's workload shape at 200k protons: steps of the FMM simulation and the
    gradient of the mean kinetic energy through checkpointed steps."""
    from tree_d_3d_b200 import Quad, synthetic
    from tree_d_3d_b200.simulation import ElectrostaticSimulation, rollout_kinetic_energy

    pos, q = synthetic.protons(200_000, seed=1)
    walls = {"x_min": -1.0, "x_max": 1.0, "y_min": -1.0, "y_max": 1.0}
    sim = ElectrostaticSimulation(positions=pos, charges=q, bounds=Quad(0, 0, 1), k_e=1.0,
                                  B_z=1.0, dt=1e-4, absorbing_walls=walls)
    ke0 = sim.get_kinetic_energy()
    for _ in range(3):
        sim.step()
    assert sim.get_kinetic_energy() > ke0
    P = torch.tensor(pos, device="cuda")
    Q = torch.tensor(q, device="cuda", requires_grad=True)
    ke = rollout_kinetic_energy(P, torch.zeros_like(P), Q, torch.ones_like(Q).detach(), 3,
                                bounds=Quad(0, 0, 1), dt=1e-4, B_z=1.0, k_e=1.0,
                                absorbing_walls=walls)
    ke.backward()
    assert torch.isfinite(Q.grad).all() and float(Q.grad.abs().max()) > 0
