"""Time integration of charged particles in a plane, on the GPU, with fields from the
flat tree (the reference's ElectrostaticSimulation, src/tree_d_3d/simulation.py:224-940).

The state is tensors on the current CUDA device: positions and velocities (2, N),
charges, masses (N,) and a ``fixed`` mask.  One step is the reference's second-order
scheme (simulation.py:800-835): electric half kick, the exact drift of a uniform B_z
(sinc forms, velocity Verlet at B_z = 0), absorption at the walls, the end-of-step
fields (one field evaluation per step, cached), electric half kick.  ``method``
"auto" sums directly up to ``direct_threshold`` charged particles or at theta = 0,
and otherwise uses the FMM (theta < 1; both kernels run on the GPU here) or the tree
walk; the FMM's leaves hold 32 particles unless ``leaf_capacity`` says otherwise.
Absorbing objects (simgeometry shapes) and MPI sharing are not part of this port.

``rollout_kinetic_energy`` is the differentiable form: the mean kinetic energy after
some steps, with gradients to the initial state and charges through the FMM's
hand-written backward, each step checkpointed (its tree and expansions recomputed in
the backward, not stored).
"""

from __future__ import annotations

from collections.abc import Mapping

import numpy as np
import torch

from tree_d_3d_b200 import _lib
from tree_d_3d_b200._utils import _check, _device, _finite, _points, device, status_word
from tree_d_3d_b200.constants import K_E
from tree_d_3d_b200.flat_tree import COULOMB_ORDER, FlatQuadtree, _direct
from tree_d_3d_b200.quad import Quad

#: ``method="auto"`` sums pairs directly up to this many charged particles.
DIRECT_THRESHOLD = 1000
_METHODS = ("auto", "tree", "direct", "fmm")
#: name -> (axis, sign): beyond the wall when sign * (coordinate - wall) > 0
_WALLS = {"x_min": (0, -1), "x_max": (0, 1), "y_min": (1, -1), "y_max": (1, 1)}


def _parse_walls(walls: Mapping[str, float]):
    """simulation.py:36-53."""
    unknown = set(walls) - set(_WALLS)
    if unknown:
        raise ValueError(f"Unknown absorbing walls {sorted(unknown)}; use {list(_WALLS)}")
    parsed = [(name, *_WALLS[name], _finite(name, walls[name])) for name in _WALLS if name in walls]
    for low, high in (("x_min", "x_max"), ("y_min", "y_max")):
        if low in walls and high in walls and not walls[low] < walls[high]:
            raise ValueError(f"{low} must be below {high}")
    return parsed


class AbsorbedParticles:
    """Particles removed at the walls, in removal order (simulation.py:66-118): state
    just after the drift that crossed the wall, the wall's name and the step's end."""

    def __init__(self, dev: torch.device) -> None:
        f64 = torch.float64
        self.time = np.zeros(0)
        self.wall = np.zeros(0, dtype=str)
        self.position = torch.zeros((2, 0), dtype=f64, device=dev)
        self.velocity = torch.zeros((2, 0), dtype=f64, device=dev)
        self.mass = torch.zeros(0, dtype=f64, device=dev)
        self.charge = torch.zeros(0, dtype=f64, device=dev)

    def record(self, *, time, walls, positions, velocities, masses, charges):
        self.time = np.append(self.time, np.full(len(walls), time))
        self.wall = np.append(self.wall, np.asarray(walls, dtype=str))
        self.position = torch.cat((self.position, positions), dim=1)
        self.velocity = torch.cat((self.velocity, velocities), dim=1)
        self.mass = torch.cat((self.mass, masses))
        self.charge = torch.cat((self.charge, charges))

    @property
    def total_charge(self) -> float:
        return float(self.charge.sum())

    @property
    def kinetic_energy(self) -> float:
        return float(0.5 * (self.mass * (self.velocity**2).sum(0)).sum())

    def counts(self) -> dict:
        names, counts = np.unique(self.wall, return_counts=True)
        return {str(n): int(c) for n, c in zip(names, counts)}

    def __len__(self) -> int:
        return len(self.time)


def _drift(pos, vel, charges, masses, b_z, dt, mobile):
    """The exact B_z drift over dt (simulation.py:814-827): new positions, rotated
    velocities; ``mobile`` (float) freezes fixed particles."""
    angle = charges / masses * b_z * dt
    c, s = torch.cos(angle), torch.sin(angle)
    a = torch.sinc(angle / np.pi)
    b = 0.5 * angle * torch.sinc(angle / (2 * np.pi)) ** 2
    vx, vy = vel[0], vel[1]
    step = dt * torch.stack((a * vx + b * vy, a * vy - b * vx))
    rotated = torch.stack((c * vx + s * vy, c * vy - s * vx))
    pos = pos + step * mobile
    vel = torch.where(mobile.bool(), rotated, vel)
    return pos, vel


def _expanded_root(bounds: Quad, points: torch.Tensor) -> Quad:
    """The root enlarged to hold ``points`` (simulation.py:625-639)."""
    if not points.shape[1]:
        return bounds
    if not bool(torch.isfinite(points).all()):
        raise ValueError("Particle positions must be finite; reduce dt")
    b = bounds
    lo = points.amin(dim=1).tolist()
    hi = points.amax(dim=1).tolist()
    lo = [min(lo[0], b.xmid - b.half), min(lo[1], b.ymid - b.half)]
    hi = [max(hi[0], b.xmid + b.half), max(hi[1], b.ymid + b.half)]
    if (lo[0] < b.xmid - b.half or lo[1] < b.ymid - b.half or hi[0] > b.xmid + b.half
            or hi[1] > b.ymid + b.half):
        center = (lo[0] / 2 + hi[0] / 2, lo[1] / 2 + hi[1] / 2)
        half = max(hi[0] / 2 - lo[0] / 2, hi[1] / 2 - lo[1] / 2) * (1 + 1e-12)
        return Quad(float(center[0]), float(center[1]), float(half))
    return bounds


class ElectrostaticSimulation:
    """Electrostatic N-body dynamics of charges in a plane on one GPU.

    Arguments as the reference (simulation.py:416-495) with the particles given as
    tensors (``positions``, ``velocities`` (2, N), ``charges``, ``masses`` (N,),
    ``fixed``) instead of ChargedBody objects; ``bodies`` with ``pos``, ``vel``,
    ``charge``, ``mass`` and ``fixed`` attributes are accepted and copied.
    """

    def __init__(self, bodies=None, bounds: Quad | None = None, theta: float = 0.5,
                 k_e: float = K_E, softening: float = 0.0, dt: float = 1e-12, B_z: float = 0.0,
                 *, positions=None, velocities=None, charges=None, masses=None, fixed=None,
                 leaf_capacity: int | None = None, max_depth: int = 48, method: str = "auto",
                 direct_threshold: int = DIRECT_THRESHOLD, absorbing_walls=None,
                 kernel: str = "coulomb", order: int | None = None,
                 reference_radius: float = 1.0, symmetric: bool = False,
                 precision: str = "fp64") -> None:
        if bounds is None:
            raise ValueError("bounds (the root Quad) is required")
        if method not in _METHODS:
            raise ValueError(f"method must be one of {_METHODS}")
        if method == "fmm" and not 0 < theta < 1:
            raise ValueError("method='fmm' needs 0 < theta < 1")
        if kernel not in ("coulomb", "log"):
            raise ValueError("kernel must be one of ('coulomb', 'log')")
        if (isinstance(direct_threshold, bool) or int(direct_threshold) != direct_threshold
                or direct_threshold < 0):
            raise ValueError("direct_threshold must be a nonnegative integer")
        dev = device()
        if bodies is not None:
            bodies = list(bodies)
            positions = np.array([b.pos for b in bodies], dtype=float).reshape(-1, 2).T
            velocities = np.array([b.vel for b in bodies], dtype=float).reshape(-1, 2).T
            charges = [b.charge for b in bodies]
            masses = [b.mass for b in bodies]
            fixed = [bool(getattr(b, "fixed", False)) for b in bodies]
        self.positions = _points(positions, "positions").clone()
        n = self.positions.shape[1]
        self.velocities = (torch.zeros_like(self.positions) if velocities is None
                           else _points(velocities, "velocities").clone())
        self.charges = _device(charges).reshape(-1).clone()
        self.masses = (torch.ones(n, dtype=torch.float64, device=dev) if masses is None
                       else _device(masses).reshape(-1).clone())
        self.fixed = (torch.zeros(n, dtype=torch.bool, device=dev) if fixed is None
                      else _device(fixed, torch.int64).reshape(-1).bool())
        self.forces = torch.zeros_like(self.positions)
        self.kernel = kernel
        self.order = int(order if order is not None else (18 if kernel == "log" else COULOMB_ORDER))
        self.symmetric = bool(symmetric)
        self.reference_radius = _finite("reference_radius", reference_radius, positive=True)
        self.bounds = bounds
        self.theta = _finite("theta", theta, minimum=0)
        self.k_e = _finite("k_e", k_e, minimum=0)
        self.softening = _finite("softening", softening, minimum=0)
        self.dt = _finite("dt", dt, positive=True)
        self.B_z = _finite("B_z", B_z)
        self.leaf_capacity = leaf_capacity
        self.max_depth = max_depth
        self.method = method
        self.direct_threshold = int(direct_threshold)
        self.precision = precision
        self.current_time = 0.0
        self.iteration = 0
        self._walls = _parse_walls(absorbing_walls or {})
        self.absorbed = AbsorbedParticles(dev)
        self._electric = torch.zeros_like(self.positions)
        self._potential = torch.zeros(n, dtype=torch.float64, device=dev)
        self._potential_done = False
        self._field_state = None
        self._tree = None
        if bool(self._outside()[0].any()):
            raise ValueError("Particles must start inside the absorbing walls and outside the "
                             "absorbing objects")

    @property
    def num_particles(self) -> int:
        return self.positions.shape[1]

    # ------------------------------------------------------------------ walls
    def _outside(self):
        """Mask of particles beyond a wall and the index of the deepest wall crossed
        (simulation.py:473-495)."""
        n = self.num_particles
        depth = torch.zeros(n, dtype=torch.float64, device=self.positions.device)
        which = torch.full((n,), -1, dtype=torch.int64, device=self.positions.device)
        for k, (_, axis, sign, value) in enumerate(self._walls):
            beyond = sign * (self.positions[axis] - value)
            deeper = beyond > depth
            depth = torch.where(deeper, beyond, depth)
            which = torch.where(deeper, torch.full_like(which, k), which)
        return which >= 0, which

    def _absorb(self) -> None:
        """simulation.py:508-565: remove and record the particles beyond a wall."""
        if not self._walls:
            return
        outside, which = self._outside()
        if not bool(outside.any()):
            return
        names = [self._walls[int(k)][0] for k in which[outside].tolist()]
        self.absorbed.record(time=self.current_time + self.dt, walls=names,
                             positions=self.positions[:, outside],
                             velocities=self.velocities[:, outside],
                             masses=self.masses[outside], charges=self.charges[outside])
        keep = ~outside
        for name in ("positions", "velocities", "forces", "_electric"):
            setattr(self, name, getattr(self, name)[:, keep].contiguous())
        for name in ("masses", "charges", "fixed", "_potential"):
            setattr(self, name, getattr(self, name)[keep].contiguous())
        self._field_state = None
        self._tree = None

    # ------------------------------------------------------------------ fields
    def _resolve_method(self) -> str:
        """simulation.py:567-581 (the Coulomb FMM runs on the GPU here)."""
        if self.method != "auto":
            return self.method
        charged = int(torch.count_nonzero(self.charges))
        if self.theta == 0 or charged <= self.direct_threshold:
            return "direct"
        return "fmm" if self.theta < 1 else "tree"

    def _parameters(self) -> tuple:
        return (self.theta, self.softening, self.k_e, self.method, self.direct_threshold,
                self.leaf_capacity, self.max_depth, self.kernel, self.order,
                self.reference_radius, self.precision)

    def _fields_current(self) -> bool:
        state = self._field_state
        if state is None:
            return False
        pos, charge, fixed, params = state
        return (params == self._parameters() and torch.equal(pos, self.positions)
                and torch.equal(charge, self.charges) and torch.equal(fixed, self.fixed))

    def _make_tree(self, method: str) -> FlatQuadtree:
        leaf = self.leaf_capacity
        if leaf is None:
            leaf = 32 if method == "fmm" else 8
        return FlatQuadtree(self.positions, self.charges, self.bounds, leaf_capacity=leaf,
                            max_depth=self.max_depth, kernel=self.kernel, order=self.order,
                            symmetric=self.symmetric, precision=self.precision)

    def build_tree(self) -> FlatQuadtree:
        self.bounds = _expanded_root(self.bounds, self.positions)
        return self._make_tree(self._resolve_method())

    def _line_offset(self) -> torch.Tensor:
        return 2 * float(np.log(self.reference_radius)) * (self.charges.sum() - self.charges)

    def compute_fields(self, include_fixed: bool = True, potential: bool = True):
        """Electric force and potential on every particle, reused while the state is
        unchanged (simulation.py:704-798).  Returns the tree used (None: direct)."""
        want_potential = potential or self.kernel != "log"
        if want_potential and not self._potential_done and self._field_state is not None:
            self._field_state = None
        if self._fields_current():
            return self._tree
        n = self.num_particles
        self.bounds = _expanded_root(self.bounds, self.positions)
        method = self._resolve_method()
        self._potential_done = want_potential or method == "direct"
        self._tree = None
        phi = torch.zeros(n, dtype=torch.float64, device=self.positions.device)
        field = torch.zeros_like(self.positions)
        charged = self.charges != 0
        if self.k_e != 0 and n and bool(charged.any()):
            if method == "fmm":
                self._tree = self._make_tree(method)
                phi, field = self._tree.fmm(theta=self.theta, softening=self.softening,
                                            potential=self._potential_done)
            else:
                targets = torch.nonzero(charged & (include_fixed | ~self.fixed)).flatten()
                tpos = self.positions[:, targets].contiguous()
                if method == "tree":
                    self._tree = self._make_tree(method)
                    p, f = self._tree.evaluate(tpos, exclude=targets, theta=self.theta,
                                               softening=self.softening,
                                               potential=self._potential_done)
                else:
                    p, f = _direct(tpos, targets, self.positions, self.charges,
                                   self.softening, self.kernel)
                phi[targets] = p
                field[:, targets] = f
        if self._potential_done:
            if self.kernel == "log":
                phi = phi + self._line_offset()
            self._potential = self.k_e * phi
        self._electric = self.k_e * self.charges[None, :] * field
        self._field_state = (self.positions.clone(), self.charges.clone(), self.fixed.clone(),
                             self._parameters())
        return self._tree

    # ------------------------------------------------------------------ stepping
    def step(self, dt: float | None = None):
        """Electric half kick, exact cyclotron drift, absorption, electric half kick
        (simulation.py:800-835).  Returns the tree of the end-of-step forces."""
        self.dt = _finite("dt", self.dt if dt is None else dt, positive=True)
        self.compute_fields(include_fixed=False, potential=False)
        mobile = (~self.fixed).to(torch.float64)
        self.velocities = self.velocities + 0.5 * self.dt * self._electric / self.masses * mobile
        self.positions, self.velocities = _drift(self.positions, self.velocities, self.charges,
                                                 self.masses, self.B_z, self.dt, mobile)
        self._absorb()
        tree = self.compute_fields(include_fixed=False, potential=False)
        mobile = (~self.fixed).to(torch.float64)
        self.velocities = self.velocities + 0.5 * self.dt * self._electric / self.masses * mobile
        vx, vy = self.velocities
        self.forces = self._electric + self.charges * self.B_z * torch.stack((vy, -vx))
        self.current_time += self.dt
        self.iteration += 1
        return tree

    # ------------------------------------------------------------------ diagnostics
    def get_kinetic_energy(self) -> float:
        return float(0.5 * (self.masses * (self.velocities**2).sum(0)).sum())

    def get_potential_energy(self, exact: bool = False) -> float:
        """0.5 sum q phi from the field evaluation, or the exact pair sum
        (simulation.py:853-916)."""
        if self.k_e == 0 or not self.num_particles:
            return 0.0
        if not exact:
            self.compute_fields()
            return float(0.5 * (self.charges * self._potential).sum())
        n = self.num_particles
        if self.kernel == "log":
            everyone = torch.arange(n, device=self.positions.device)
            phi, _ = _direct(self.positions, everyone, self.positions, self.charges,
                             self.softening, "log")
            phi = phi + self._line_offset()
            return float(0.5 * self.k_e * (self.charges * phi).sum())
        dev = self.positions.device
        status = status_word(dev)
        energy = torch.zeros(1, dtype=torch.float64, device=dev)
        ws = _lib.workspace(_lib.query("td3_pair_energy_workspace_size", n), dev)
        _lib.call("td3_pair_energy", self.positions.data_ptr(), self.charges.data_ptr(), n,
                  float(self.softening), energy.data_ptr(), status.data_ptr(), ws.data_ptr(),
                  ws.numel(), _lib.stream(dev))
        _check(status)
        return float(self.k_e * energy.item())

    def get_total_energy(self, exact: bool = False) -> float:
        return self.get_kinetic_energy() + self.get_potential_energy(exact)

    def get_total_charge(self) -> float:
        return float(self.charges.sum())

    def get_momentum(self) -> np.ndarray:
        return (self.velocities @ self.masses).cpu().numpy()

    def get_center_of_mass(self) -> np.ndarray:
        total = float(self.masses.sum())
        if not total:
            return np.zeros(2)
        return (self.positions @ self.masses).cpu().numpy() / total

    def get_angular_momentum(self) -> float:
        x, y = self.positions
        vx, vy = self.velocities
        return float((self.masses * (x * vy - y * vx)).sum())


# ---------------------------------------------------------------------- differentiable
def rollout_kinetic_energy(positions: torch.Tensor, velocities: torch.Tensor,
                           charges: torch.Tensor, masses: torch.Tensor, steps: int, *,
                           bounds: Quad, dt: float, B_z: float = 0.0, k_e: float = 1.0,
                           theta: float = 0.5, softening: float = 0.0,
                           kernel: str = "coulomb", order: int | None = None,
                           leaf_capacity: int = 32, absorbing_walls=None,
                           precision: str = "fp64", checkpoint: bool = True,
                           field_fn=None) -> torch.Tensor:
    """Mean kinetic energy of the particles still inside the walls after ``steps``
    steps of the scheme of ElectrostaticSimulation.step with FMM fields, differentiable
    to the initial positions, velocities and charges.  Absorbed particles are masked
    (their charge stops acting, their state freezes); each step is checkpointed, so
    its trees and expansions are rebuilt in the backward instead of being stored.
    ``field_fn(pos, charge) -> (phi, E)`` replaces the FMM (for tests)."""
    from torch.utils.checkpoint import checkpoint as ckpt

    from tree_d_3d_b200.autograd import fmm_field

    walls = _parse_walls(absorbing_walls or {})
    if order is None:
        order = 18 if kernel == "log" else COULOMB_ORDER

    def fields(pos, charge):
        if field_fn is not None:
            return field_fn(pos, charge)
        root = _expanded_root(bounds, pos.detach())
        return fmm_field(pos, charge, root, kernel=kernel, order=order, theta=theta,
                         softening=softening, leaf_capacity=leaf_capacity, precision=precision)

    def inside(pos):
        alive = torch.ones(pos.shape[1], dtype=torch.float64, device=pos.device)
        for _, axis, sign, value in walls:
            alive = alive * (sign * (pos[axis].detach() - value) <= 0).to(torch.float64)
        return alive

    def step(pos, vel, force, alive):
        vel = vel + 0.5 * dt * force / masses * alive
        new_pos, new_vel = _drift(pos, vel, charges, masses, B_z, dt, alive)
        alive = alive * inside(new_pos)
        new_pos = torch.where(alive.bool(), new_pos, pos)
        _, field = fields(new_pos, charges * alive)
        force = k_e * charges * alive * field
        new_vel = new_vel + 0.5 * dt * force / masses * alive
        return new_pos, new_vel, force, alive

    alive = inside(positions)
    _, field = fields(positions, charges * alive)
    force = k_e * charges * alive * field
    pos, vel = positions, velocities
    for _ in range(steps):
        if checkpoint:
            pos, vel, force, alive = ckpt(step, pos, vel, force, alive, use_reentrant=False)
        else:
            pos, vel, force, alive = step(pos, vel, force, alive)
    ke = 0.5 * masses * (vel**2).sum(0) * alive
    return ke.sum() / alive.sum()
