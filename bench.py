"""Benchmark of the field solver: FMM particles/s at N = 1M, p = 12 on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one FMM field evaluation of a fresh tree of the workload: the tree build
with its moments, the traversal and interaction lists, M2L, L2L, and L2P + P2P at all
N particles (log kernel, order 12, theta 0.5, leaf 8, softening 1e-3), on the 1M
8-Gaussian mixture with +-1 charges of net zero (synthetic, seeded).  ``value`` is
whole-job particles/s with the inputs resident in HBM; ``e2e`` is the same through the
public API from pinned host buffers, host-device copies inside the timed region.

``--impl reference`` times the reference algorithm on the host cores: the C
restatement of the reference's CPU kernels (``oracle/``) with OpenMP on every core,
on a bounded sample of the same workload.  Under torchrun with N > 1 every rank runs
an independent replica (the path needs no exchange on one tree); rank 0 prints.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PARTICLES = 1_000_000
ORDER = 12
THETA = 0.5
LEAF = 8
SOFTENING = 1e-3
SEED = 3
CPU_SAMPLE = 250_000
L2_FLUSH_BYTES = 256 << 20
WORKLOAD = "log-kernel FMM, 1M particles, 8-Gaussian mixture, p=12, theta=0.5, leaf 8"


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--n", type=int, default=N_PARTICLES)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--trace-only", action="store_true",
                   help="timed steps only (no e2e, launch count or kernel timing): for ncu")
    return p.parse_args()


def _config(n):
    return {
        "workload": WORKLOAD,
        "n_particles": n,
        "kernel": "log",
        "order": ORDER,
        "theta": THETA,
        "leaf_capacity": LEAF,
        "softening": SOFTENING,
        "distribution": "mixture of 8 Gaussians (sigma 0.02-0.2), charges +-1, net zero",
        "l2": "flushed before every step (256 MiB write, outside the step's events)",
    }


# ----------------------------------------------------------------------------- CPU arm
def _cpu_fmm(pos, q):
    from oracle import flat_tree_oracle as oracle

    t0 = time.perf_counter()
    tree = oracle.OracleTree(pos, q, (0.0, 0.0, 1.0), kernel="log", order=ORDER, leaf_capacity=LEAF)
    tree.fmm(theta=THETA, softening=SOFTENING)
    return time.perf_counter() - t0


def cpu_baseline(repeats=2):
    """The oracle (C restatement of the reference's CPU kernels, OpenMP on all cores)
    on a bounded sample of the workload; particles/s."""
    from oracle import flat_tree_oracle as oracle
    from tree_d_3d_b200 import synthetic

    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    pos, q = synthetic.mixture8(CPU_SAMPLE, seed=SEED)
    _cpu_fmm(pos, q)
    best = min(_cpu_fmm(pos, q) for _ in range(repeats))
    return {
        "value": CPU_SAMPLE / best,
        "unit": "particles/s",
        "cores": cores,
        "kind": "port",
        "sample": f"{CPU_SAMPLE} particles of the same distribution, build + FMM per run, best of {repeats}",
    }


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import flat_tree_oracle as oracle
    from tree_d_3d_b200 import synthetic

    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    pos, q = synthetic.mixture8(CPU_SAMPLE, seed=SEED)
    for _ in range(max(args.warmup, 1)):
        _cpu_fmm(pos, q)
    times = [_cpu_fmm(pos, q) for _ in range(args.steps)]
    total = sum(times)
    value = CPU_SAMPLE * args.steps / total
    line = {
        "impl": "reference",
        "metric": "FMM particles/s at N=1M p=12",
        "value": value,
        "unit": "particles/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": _config(N_PARTICLES),
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": cores, "kind": "port",
                         "sample": f"{CPU_SAMPLE} particles of the workload's distribution per step"},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- GPU arm
class ClockSampler:
    """nvidia-smi samples of SM clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=5)
            self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self):
        rows = []
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[3:]))
            except (ValueError, IndexError):
                continue
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags)
                          if i < len(names) and f.lower() == "active"})
        sm = sorted(r[0] for r in rows)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's ``value`` (the job's time is its slowest rank's)."""
    import torch

    if dist is None:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gpu_step(pos, q, torch):
    from tree_d_3d_b200 import FlatQuadtree, Quad

    tree = FlatQuadtree(pos, q, Quad(0.0, 0.0, 1.0), kernel="log", order=ORDER, leaf_capacity=LEAF)
    phi, field = tree.fmm(theta=THETA, softening=SOFTENING)
    return tree, phi, field


def count_our_launches(fn, torch):
    """Kernels of libtreed3d.so launched by one call of fn (CUPTI trace via torch.profiler)."""
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    ours = re.compile(r"(^|::)k_\w+")
    counts = {}
    for ev in prof.events():
        if ev.device_type is not None and "CUDA" in str(ev.device_type) and ours.search(ev.name):
            key = ours.search(ev.name).group(0).lstrip(":")
            counts[key] = counts.get(key, 0) + 1
    return counts


def time_m2l(tree, torch, reps):
    """The M2L kernel alone (CUDA events on its stream), average ms per launch."""
    from tree_d_3d_b200 import _lib

    lists = tree._lists(THETA)
    count, w = tree.node_count, tree.order + 1
    lre = torch.zeros((count, w), dtype=torch.float64, device=tree.device)
    lim = torch.zeros_like(lre)
    args = (lists["m2l_rows"].data_ptr(), lists["m2l_partners"].data_ptr(), count,
            tree.node_center.data_ptr(), tree.node_center.data_ptr(), tree.moment_re.data_ptr(),
            tree.moment_im.data_ptr(), tree.order, tree._m2l_matrix().data_ptr(),
            lre.data_ptr(), lim.data_ptr(), _lib.stream(tree.device))
    _lib.call("td3_fmm_m2l", *args)
    stream = torch.cuda.current_stream()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(reps):
        _lib.call("td3_fmm_m2l", *args)
    stop.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(stop) / reps, int(lists["m2l"].shape[0])


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from tree_d_3d_b200 import synthetic

    dev = torch.device("cuda", local)
    n = args.n
    pos_np, q_np = synthetic.mixture8(n, seed=SEED)
    pos = torch.tensor(pos_np, device=dev)
    q = torch.tensor(q_np, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        gpu_step(pos, q, torch)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    stream = torch.cuda.current_stream()
    total_ms = 0.0
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            gpu_step(pos, q, torch)
            b.record(stream)
            b.synchronize()
            total_ms += a.elapsed_time(b)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = max_over_ranks(total_ms, dist, dev)
    ms_per_step = total_ms / args.steps
    value = world * n * args.steps / (total_ms / 1e3)

    if args.trace_only:
        if dist:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"trace_only": True, "ms_per_step": ms_per_step}), flush=True)
        return 0

    # end to end through the public API: pinned host inputs in, host results out
    from tree_d_3d_b200 import FlatQuadtree, Quad

    pos_h = torch.tensor(pos_np).pin_memory()
    q_h = torch.tensor(q_np).pin_memory()
    phi_h = torch.empty(n, dtype=torch.float64).pin_memory()
    field_h = torch.empty((2, n), dtype=torch.float64).pin_memory()

    def e2e_step():
        p = pos_h.to(dev, non_blocking=True)
        c = q_h.to(dev, non_blocking=True)
        tree = FlatQuadtree(p, c, Quad(0.0, 0.0, 1.0), kernel="log", order=ORDER, leaf_capacity=LEAF)
        phi, field = tree.fmm(theta=THETA, softening=SOFTENING)
        phi_h.copy_(phi, non_blocking=True)
        field_h.copy_(field, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
    e2e_ms = max_over_ranks(e2e_ms, dist, dev)
    e2e_value = world * n * args.steps / (e2e_ms / 1e3)

    # launches of our kernels per step, and the dominant kernel's roofline
    launches = count_our_launches(lambda: gpu_step(pos, q, torch), torch)
    tree, _, _ = gpu_step(pos, q, torch)
    m2l_ms, n_m2l = time_m2l(tree, torch, reps=5)
    w = ORDER + 1
    flops = 2 * n_m2l * 8 * w * w  # directed translations x 8 (p + 1)^2
    achieved = flops / (m2l_ms * 1e-3) / 1e12
    fp64_peak = 37.0  # nominal B200 FP64 (no measured FP64 peak is available)
    roofline = {
        "kernel": "k_m2l_log (FP64 M2L)",
        "bound": "fp64",
        "achieved": achieved,
        "peak": fp64_peak,
        "unit": "TFLOP/s",
        "frac": achieved / fp64_peak,
        "peak_source": "nominal B200 FP64 FMA rate; MEASURED_PEAKS.json has no FP64 figure",
        "traffic": None,
        "ms_per_launch": m2l_ms,
        "flop_per_launch": flops,
    }
    clock = clocks.summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "FMM particles/s at N=1M p=12",
        "value": value,
        "unit": "particles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {**_config(n), "parallelism": f"replicas x{world}", "precision": "fp64",
                   "pipeline": "build + moments + traverse + M2L + L2L + L2P/P2P per step"},
        "e2e": {"value": e2e_value, "unit": "particles/s",
                "h2d_bytes_per_step": 3 * 8 * n, "d2h_bytes_per_step": 3 * 8 * n},
        "gpu_launches": int(sum(launches.values()) * args.steps),
        "launches_per_step": launches,
        "roofline": roofline,
        "clocks": clock,
        "fmm_pairs": list(tree.fmm_pairs),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = _args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
