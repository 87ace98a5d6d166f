"""Generate the golden fixtures of the field solver from the reference implementation.

Run where the reference package tree-d-3d is available: its ``src`` directory is
passed with ``--reference`` or, failing that, in the ``TD3_REFERENCE_SRC``
environment variable::

    python tests/golden/make_golden.py --reference <tree-d-3d checkout>/src

It imports the reference's own ``tree_d_3d.flat_tree`` unmodified, behind minimal
stand-ins for the packages it imports but does not need for one process on the CPU
(``cunumpy`` = NumPy, ``scope_profiler`` and ``methodcard`` as no-ops,
``maybempi.collectives`` as one process). Each kernel is the reference's Pyccel
source ``kernels/<name>/<name>_pyccel.py``, compiled by numba (``del`` statements
stripped; numba contracts no FMAs without ``fastmath``, like Pyccel's default
build) or run as plain Python with ``--python``.

The outputs are written to ``tests/golden/*.npz``; the tests read only those
files, never the reference.
"""

from __future__ import annotations

import argparse
import ast
import importlib
import importlib.util
import os
import sys
import textwrap
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


# --------------------------------------------------------------------------- stubs
class _KernelFunction:
    """A reference kernel: its Pyccel source, numba-compiled or plain Python."""

    def __init__(self, module_name: str, use_numba: bool) -> None:
        self.name = module_name.rsplit(".", 1)[-1]
        spec = importlib.util.find_spec(module_name)
        folder = Path(spec.origin).parent
        source = (folder / f"{self.name}_pyccel.py").read_text()
        self.source_path = folder / f"{self.name}_pyccel.py"
        self.python = self._load(source, strip_del=False)
        self.function = self.python
        if use_numba:
            import numba

            self.function = numba.njit(cache=False)(self._load(source, strip_del=True))

    def _load(self, source: str, strip_del: bool):
        tree = ast.parse(source)
        if strip_del:

            class StripDel(ast.NodeTransformer):
                def visit_Delete(self, node):  # noqa: N802
                    return ast.Pass()

            tree = ast.fix_missing_locations(StripDel().visit(tree))
        namespace: dict = {"__name__": f"_golden_{self.name}"}
        exec(compile(tree, str(self.source_path), "exec"), namespace)
        return namespace[self.name]

    def __call__(self, *args, n_threads=None):
        return self.function(*args)


def install_stubs(reference_src: Path, use_numba: bool) -> None:
    """Make ``import tree_d_3d.flat_tree`` load the reference behind stand-ins."""
    cunumpy = types.ModuleType("cunumpy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cunumpy, name, getattr(np, name))
    cunumpy.to_numpy = lambda a: np.asarray(a)
    cunumpy.get_backend = lambda: "numpy"
    cunumpy.cupy_available = lambda: False

    class KernelPackage:
        def __init__(self, name):
            self.name = name

        def from_folder(self, module_name):
            return _KernelFunction(module_name, use_numba)

    kernels_mod = types.ModuleType("cunumpy.kernels")
    kernels_mod.KernelPackage = KernelPackage
    kernels_mod.metal_available = lambda: False
    cunumpy.kernels = kernels_mod
    sys.modules["cunumpy"] = cunumpy
    sys.modules["cunumpy.kernels"] = kernels_mod

    sp = types.ModuleType("scope_profiler")

    def profile(*args, **kwargs):
        return lambda f: f

    class _Region:
        def __init__(self, *a, **k):
            pass

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

    sp.profile = profile
    sp.region = _Region
    sp.register_opt_in_tag = lambda *a, **k: None
    sys.modules["scope_profiler"] = sp

    mm = types.ModuleType("maybempi")
    coll = types.ModuleType("maybempi.collectives")
    coll.is_parallel = lambda comm: False
    mm.collectives = coll
    sys.modules["maybempi"] = mm
    sys.modules["maybempi.collectives"] = coll

    mc = types.ModuleType("methodcard")
    mc.method = lambda *a, **k: (lambda f: f)
    mc.Rule = lambda *a, **k: None
    mc.ConvergenceProblem = lambda *a, **k: None
    sys.modules["methodcard"] = mc

    # tree_d_3d as a namespace package on the reference sources, bypassing its
    # __init__ (which imports the electrode solver and its geometry package)
    pkg = types.ModuleType("tree_d_3d")
    pkg.__path__ = [str(reference_src / "tree_d_3d")]
    sys.modules["tree_d_3d"] = pkg


# --------------------------------------------------------------------------- data
def cloud_flat(n, seed=0, neutral_fraction=0.1):
    """A Gaussian cloud with a coincident clump and neutral markers (2, n)."""
    rng = np.random.default_rng(seed)
    pos = np.ascontiguousarray(rng.normal(0, 0.3, (n, 2)).T).clip(-0.99, 0.99)
    pos[:, : n // 10] = pos[:, :1]
    charge = np.where(rng.random(n) < 0.5, -1.0, 1.0) * rng.uniform(0.5, 2, n)
    charge[rng.random(n) < neutral_fraction] = 0.0
    return pos, charge


def cloud_fmm(n=3000, seed=0):
    rng = np.random.default_rng(seed)
    pos = np.concatenate(
        (
            rng.normal([[-0.3], [0.1]], 0.1, (2, n // 2)),
            rng.normal([[0.4], [-0.2]], 0.25, (2, n - n // 2)),
        ),
        axis=1,
    ).clip(-0.99, 0.99)
    return pos, rng.normal(0.3, 1, n)


def build_clouds():
    rng = np.random.default_rng(5)
    angle = rng.uniform(0, 2 * np.pi, 3000)
    return {
        "uniform": rng.uniform(-0.99, 0.99, (2, 4000)),
        "circle": 0.9 * np.stack((np.cos(angle), np.sin(angle))),
        "clustered": np.clip(rng.normal(0.3, 0.01, (2, 2000)), -1, 1),
        "lattice": np.stack(
            np.meshgrid(np.linspace(-0.5, 0.5, 33), np.linspace(-0.5, 0.5, 33))
        ).reshape(2, -1),
        "coincident": np.full((2, 40), 0.25),
    }


TREE_ARRAYS = (
    "perm",
    "node_center",
    "node_half",
    "node_start",
    "node_end",
    "node_child",
    "node_depth",
    "levels",
)


def tree_dict(tree, prefix):
    out = {f"{prefix}/{a}": np.asarray(getattr(tree, a)) for a in TREE_ARRAYS}
    out[f"{prefix}/node_count"] = np.asarray(tree.node_count)
    return out


# --------------------------------------------------------------------------- cases
def make_build(ft, Quad):
    out = {}
    for name, pos in build_clouds().items():
        q = np.ones(pos.shape[1])
        tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), leaf_capacity=6)
        out[f"{name}/pos"] = pos
        out.update(tree_dict(tree, name))
    # deep coincident chain
    pos = np.array([[0.3, 0.3, -0.5], [0.3, 0.3, 0.2]])
    tree = ft.FlatQuadtree(pos, [1, 1, -1], Quad(0, 0, 1), leaf_capacity=1, max_depth=48)
    out["chain/pos"] = pos
    out.update(tree_dict(tree, "chain"))
    # leaf 1 / depth 10 and leaf 8 / depth 48 on the cloud of the walk tests
    pos, charge = cloud_flat(300)
    for leaf, depth in ((1, 10), (8, 48)):
        tree = ft.FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=leaf, max_depth=depth)
        key = f"cloud300_l{leaf}_d{depth}"
        out[f"{key}/pos"] = pos
        out.update(tree_dict(tree, key))
    # a root that is not a dyadic square: the target tree of fmm_at
    rng = np.random.default_rng(21)
    targets = rng.uniform(-0.73, 0.91, (2, 2500))
    lo, hi = targets.min(axis=1), targets.max(axis=1)
    centre = 0.5 * (lo + hi)
    half = 0.5 * float(np.max(hi - lo)) * (1 + 1e-12) + 1e-300
    root = Quad(float(centre[0]), float(centre[1]), half)
    tree = ft.FlatQuadtree(targets, np.zeros(2500), root, leaf_capacity=16)
    out["offroot/pos"] = targets
    out["offroot/root"] = np.array([root.xmid, root.ymid, root.half])
    out.update(tree_dict(tree, "offroot"))
    return out


def make_moments(ft, Quad):
    out = {}
    pos, charge = cloud_flat(2000, seed=3)
    out["pos"], out["charge"] = pos, charge
    tree = ft.FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=8)
    for a in ("node_q", "node_qabs", "node_p", "node_s"):
        out[f"coulomb/{a}"] = np.asarray(getattr(tree, a))
    out.update(tree_dict(tree, "coulomb"))
    tree = ft.FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=8, kernel="log", order=12)
    for a in ("node_qabs", "moment_re", "moment_im", "node_q", "node_p"):
        out[f"log/{a}"] = np.asarray(getattr(tree, a))
    # Cartesian moments at orders 4 and 12
    for order in (4, 12):
        tree = ft.FlatQuadtree(pos, charge, Quad(0, 0, 1), leaf_capacity=8, order=order)
        out[f"cart{order}/moments"] = np.asarray(tree._cartesian_moments())
    return out


def make_evaluate(ft, Quad):
    out = {}
    pos, charge = cloud_flat(300)
    out["cloud/pos"], out["cloud/charge"] = pos, charge
    exclude = np.arange(pos.shape[1])
    for kernel in ("coulomb", "log"):
        for leaf, depth in ((1, 10), (8, 48)):
            tree = ft.FlatQuadtree(
                pos, charge, Quad(0, 0, 1), leaf_capacity=leaf, max_depth=depth, kernel=kernel
            )
            for theta in (0.0, 0.5, 1.2):
                phi, field = tree.evaluate(pos, exclude=exclude, theta=theta, softening=0.01)
                key = f"cloud/{kernel}/l{leaf}/t{theta}"
                out[f"{key}/phi"], out[f"{key}/field"] = phi, field
    # config 1: N=5000 uniform, charges +-1, Coulomb, theta 0.5, softening 1e-3
    rng = np.random.default_rng(1)
    pos = rng.uniform(-1, 1, (2, 5000))
    charge = rng.choice([-1.0, 1.0], 5000)
    tree = ft.FlatQuadtree(pos, charge, Quad(0, 0, 1))
    exclude = np.arange(5000)
    phi, field = tree.evaluate(pos, exclude=exclude, theta=0.5, softening=1e-3)
    dphi, dfield = ft.direct_field(pos, pos, charge, softening=1e-3, exclude=exclude)
    out["config1/pos"], out["config1/charge"] = pos, charge
    out["config1/phi"], out["config1/field"] = phi, field
    out["config1/direct_phi"], out["config1/direct_field"] = dphi, dfield
    # off-source probes, log kernel at order 10, potential on and off
    probes = np.random.default_rng(2).uniform(-1, 1, (2, 400))
    pos, q = cloud_fmm(2000, seed=7)
    tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=10)
    out["probes/pos"], out["probes/charge"], out["probes/targets"] = pos, q, probes
    for potential in (True, False):
        phi, field = tree.evaluate(probes, theta=0.6, softening=0.0, potential=potential)
        out[f"probes/log/pot{int(potential)}/phi"] = phi
        out[f"probes/log/pot{int(potential)}/field"] = field
    tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="coulomb")
    phi, field = tree.evaluate(probes, theta=0.6, softening=0.002)
    out["probes/coulomb/phi"], out["probes/coulomb/field"] = phi, field
    return out


def make_direct(ft, Quad):
    out = {}
    rng = np.random.default_rng(4)
    targets = rng.uniform(-1.2, 1.2, (2, 700))
    pos = rng.normal(0, 0.4, (2, 1500))
    charge = rng.normal(size=1500)
    charge[::9] = 0.0
    exclude = np.where(rng.random(700) < 0.3, rng.integers(0, 1500, 700), -1)
    out["targets"], out["pos"], out["charge"], out["exclude"] = targets, pos, charge, exclude
    for kernel in ("coulomb", "log"):
        for eps in (0.0, 0.01):
            phi, field = ft.direct_field(
                targets, pos, charge, softening=eps, exclude=exclude, kernel=kernel
            )
            out[f"{kernel}/eps{eps}/phi"], out[f"{kernel}/eps{eps}/field"] = phi, field
    return out


def make_fmm(ft, Quad):
    out = {}
    pos, q = cloud_fmm(3000, seed=0)
    out["log/pos"], out["log/charge"] = pos, q
    tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=12)
    phi, field = tree.fmm(theta=0.5)
    m2l, p2p, sizes = tree._traversals[0.5]
    out["log/phi"], out["log/field"] = phi, field
    out["log/m2l"] = np.asarray(m2l[: int(sizes[0])])
    out["log/p2p"] = np.asarray(p2p[: int(sizes[1])])
    out["log/sizes"] = np.asarray(sizes[:2])
    rows, partners = tree._m2l_rows(0.5, m2l, slice(0, int(sizes[0])))
    out["log/m2l_rows"], out["log/m2l_partners"] = rows, partners[: 2 * int(sizes[0])]
    phi, field = tree.fmm(theta=0.5, softening=0.005, potential=False)
    out["log/eps/phi"], out["log/eps/field"] = phi, field
    tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=12, symmetric=True)
    phi, field = tree.fmm(theta=0.4)
    out["log/sym/phi"], out["log/sym/field"] = phi, field
    tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), kernel="log", order=8, leaf_capacity=1)
    phi, field = tree.fmm(theta=0.6)
    out["log/leaf1/phi"], out["log/leaf1/field"] = phi, field
    # Coulomb (Cartesian) FMM
    rng = np.random.default_rng(11)
    pos = np.concatenate(
        (rng.uniform(-0.9, 0.9, (2, 1500)), rng.normal(0.3, 0.05, (2, 1500))), axis=1
    ).clip(-0.99, 0.99)
    q = rng.normal(size=pos.shape[1])
    out["coulomb/pos"], out["coulomb/charge"] = pos, q
    for order, eps in ((4, 0.0), (8, 0.02), (12, 0.001)):
        tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), order=order, leaf_capacity=16)
        phi, field = tree.fmm(theta=0.5, softening=eps)
        out[f"coulomb/p{order}/phi"], out[f"coulomb/p{order}/field"] = phi, field
        out[f"coulomb/p{order}/eps"] = np.asarray(eps)
    return out


def make_fmm_at(ft, Quad):
    out = {}
    rng = np.random.default_rng(13)
    pos, q = cloud_fmm(4000, seed=13)
    targets = np.concatenate((rng.uniform(-0.9, 0.9, (2, 1500)), pos[:, :500]), axis=1)
    exclude = np.concatenate((np.full(1500, -1), np.arange(500)))
    out["pos"], out["charge"], out["targets"], out["exclude"] = pos, q, targets, exclude
    for kernel in ("coulomb", "log"):
        order = 8 if kernel == "coulomb" else 16
        tree = ft.FlatQuadtree(pos, q, Quad(0, 0, 1), kernel=kernel, order=order, leaf_capacity=16)
        eps = 0.01 if kernel == "coulomb" else 0.0
        phi, field = tree.fmm_at(targets, exclude=exclude, theta=0.5, softening=eps)
        out[f"{kernel}/phi"], out[f"{kernel}/field"] = phi, field
        _, ttree, lists = tree._traversals[("targets", 0.5, 16)]
        (m2l_rows, m2l_partners, n_m2l), (p2p_rows, p2p_partners, n_p2p) = lists
        out[f"{kernel}/m2l_rows"] = m2l_rows
        out[f"{kernel}/m2l_partners"] = m2l_partners[:n_m2l]
        out[f"{kernel}/p2p_rows"] = p2p_rows
        out[f"{kernel}/p2p_partners"] = p2p_partners[:n_p2p]
        out.update(tree_dict(ttree, f"{kernel}/target_tree"))
    return out


def make_tables():
    from tree_d_3d import _cartesian

    out = {}
    for order in (4, 8, 12):
        for name, value in _cartesian.tables(order).items():
            out[f"p{order}/{name}"] = value
    return out


def make_energy(ft, Quad):
    from tree_d_3d.kernels import _kernels

    k = _kernels(True)
    pos, charge = cloud_fmm(1500, seed=9)
    status, energy = np.zeros(1, dtype=np.int64), np.zeros(1)
    k.pair_energy(pos, charge, 0.01, status, energy)
    return {"pos": pos, "charge": charge, "energy": energy, "status": status}


def make_strip():
    strip = importlib.import_module("tree_d_3d.strip")
    rng = np.random.default_rng(21)
    width = 2.0
    n = 1200
    pos = np.stack((rng.uniform(0.05, 0.95, n) * width, rng.normal(0, 0.6, n)))
    charge = np.where(rng.random(n) < 0.5, -1.0, 1.0) * rng.uniform(0.5, 1.5, n)
    points = np.stack((rng.uniform(0.02, 0.98, 400) * width, rng.normal(0, 0.8, 400)))
    out = {"pos": pos, "charge": charge, "points": points, "width": np.asarray(width)}
    for method in ("fmm", "direct"):
        for eps in (0.0, 0.02):
            field = strip.GroundedStripField(width, method=method, softening=eps)
            key = f"{method}/eps{eps}"
            out[f"{key}/phi"], out[f"{key}/field"] = field.field_at_charges(pos, charge)
            _, out[f"{key}/field_nopot"] = field.field_at_charges(pos, charge, potential=False)
            out[f"{key}/probe_phi"], out[f"{key}/probe_field"] = field.probe(pos, charge, points)
    # a lone charge: the image force of the plates
    lone = strip.GroundedStripField(2.5, k_e=1.0)
    out["lone/phi"], out["lone/field"] = lone.field_at_charges(np.array([[0.7], [0.3]]),
                                                               np.array([1.5]))
    return out


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("TD3_REFERENCE_SRC"),
                        help="the reference's src directory (default: $TD3_REFERENCE_SRC)")
    parser.add_argument("--python", action="store_true", help="plain Python kernels")
    parser.add_argument("--only", nargs="*", help="the fixture groups to write (default all)")
    args = parser.parse_args()
    if not args.reference:
        parser.error("the reference's src directory is required: pass --reference or set "
                     "TD3_REFERENCE_SRC")
    install_stubs(Path(args.reference), use_numba=not args.python)
    ft = importlib.import_module("tree_d_3d.flat_tree")
    from tree_d_3d.quad import Quad

    groups = {
        "build": lambda: make_build(ft, Quad),
        "moments": lambda: make_moments(ft, Quad),
        "direct": lambda: make_direct(ft, Quad),
        "evaluate": lambda: make_evaluate(ft, Quad),
        "fmm": lambda: make_fmm(ft, Quad),
        "fmm_at": lambda: make_fmm_at(ft, Quad),
        "tables": make_tables,
        "energy": lambda: make_energy(ft, Quad),
        "strip": make_strip,
    }
    for name, make in groups.items():
        if args.only and name not in args.only:
            continue
        data = make()
        np.savez_compressed(HERE / f"{name}.npz", **data)
        size = (HERE / f"{name}.npz").stat().st_size
        print(f"{name}.npz: {len(data)} arrays, {size / 1024:.0f} KiB", flush=True)


if __name__ == "__main__":
    main()
