"""Benchmark of the field solver: FMM particles/s at N = 1M, p = 12, mixed precision vs
FP64, field plus backward, on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step takes the 1M particles of the workload (8-Gaussian mixture, +-1 charges of net
zero; log kernel, order 12, theta 0.5, leaf 8, unsoftened), builds a fresh tree
(build, moments, traversal, interaction lists) and evaluates the FMM potential and
field at every particle in mixed precision (FP32 near field with compensated sums,
FP32 M2L on size-scaled expansions, FP64 M2M / L2L / L2P), then runs the hand-written
backward of L = sum w phi + sum e . E (fixed seeded w, e) to dL/dq and dL/dx.
``value`` is whole-job particles/s with the inputs resident in HBM; the same step in
the plain FP64 form is timed beside it (``fp64``), and the mixed field error against
the FP64 direct sum on 4096 sampled particles is reported (``rel_err_field``).
``e2e`` is the mixed step through the public API from pinned host buffers, with the
host-device copies of every step's inputs and results inside the timed region (on a copy
stream: step k + 1's inputs come in and step k's results go out while step k computes).

``--impl reference`` times the reference algorithm on the host cores: the C
restatement of the reference's CPU kernels (``oracle/``) with OpenMP on every core, on
the same 1M particles (field only, FP64: the reference has no backward and no mixed
form), with one single-threaded step beside it.
Under torchrun with N > 1 every rank runs an independent replica; rank 0 prints.
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
#: nominal FP32 FMA rate of a B200 at its max SM clock, TFLOP/s (148 SM x 128 lanes x 2)
FP32_PEAK = 148 * 128 * 2 * 1.965e9 / 1e12
ORDER = 12
THETA = 0.5
LEAF = 8
#: the log kernel softens the near field only (the reference's convention); the error
#: against the direct sum is defined for the unsoftened kernel
SOFTENING = 0.0
SEED = 3
L2_FLUSH_BYTES = 256 << 20
METRIC = "FMM particles/s at N=1M p=12: mixed-prec vs FP64 GPU at rel err<=1e-6, +backward"
WORKLOAD = ("log-kernel FMM field + backward, 1M particles, 8-Gaussian mixture, p=12, "
            "theta=0.5, leaf 8, fresh tree per step")


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--n", type=int, default=N_PARTICLES)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--suite", action="store_true",
                   help="every workload configuration (one JSON line per case) instead of "
                        "the headline line")
    p.add_argument("--trace-only", action="store_true",
                   help="timed mixed steps only (no e2e, FP64 arm, counts or errors): for ncu")
    p.add_argument("--kernel", choices=("log", "coulomb"), default="log",
                   help="the kernel of the --trace-only steps (the headline is the log kernel)")
    p.add_argument("--precision", choices=("mixed", "fp64"), default="mixed",
                   help="the precision of the --trace-only steps")
    p.add_argument("--m2l", choices=("rows", "lanes", "grouped"), default="rows",
                   help="the mixed log M2L form of the --trace-only steps on the CUDA cores: "
                        "8 lanes per destination row (the step's) or a lane per translation; "
                        "or tensor-core products grouped by translation")
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
        "loss": "L = sum w phi + sum e.E, w and e seeded N(0, 1)",
        "l2": "flushed before every step (256 MiB write, outside the step's events)",
    }


# ----------------------------------------------------------------------------- CPU arm
#: what the CPU arm runs, against the GPU arm's step
CPU_DIFFERS = ("forward only: build + FP64 FMM field at every particle (the reference has no "
               "backward and no mixed-precision form); same particles, kernel, order, theta, "
               "leaf capacity and softening as the GPU arm")


def _cpu_fmm(pos, q):
    from oracle import flat_tree_oracle as oracle

    t0 = time.perf_counter()
    tree = oracle.OracleTree(pos, q, (0.0, 0.0, 1.0), kernel="log", order=ORDER, leaf_capacity=LEAF)
    tree.fmm(theta=THETA, softening=SOFTENING)
    return time.perf_counter() - t0


def _cpu_config(n):
    return {**_config(n), "backward": False, "precision": "fp64", "differs": CPU_DIFFERS,
            "implementation": ("the oracle: C restatement of the reference's CPU kernels "
                               "(K/*/<name>_pyccel.py) driven as the reference's flat_tree.py, "
                               "OpenMP on the loops the reference parallelises")}


def _single_thread(pos, q, cores):
    """One step of the same workload on one thread (the reference's unmodified,
    single-threaded kernels), then the thread count back to ``cores``."""
    from oracle import flat_tree_oracle as oracle

    oracle.set_threads(1)
    try:
        seconds = _cpu_fmm(pos, q)
    finally:
        oracle.set_threads(cores)
    return {"value": pos.shape[1] / seconds, "unit": "particles/s", "cores": 1,
            "ms_per_step": 1e3 * seconds}


def cpu_baseline(repeats=2):
    """The oracle on the host cores, on the full 1M workload, field only: particles/s
    on every core (best of ``repeats`` after one warm-up) and on one thread."""
    from oracle import flat_tree_oracle as oracle
    from tree_d_3d_b200 import synthetic

    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    pos, q = synthetic.mixture8(N_PARTICLES, seed=SEED)
    _cpu_fmm(pos, q)
    best = min(_cpu_fmm(pos, q) for _ in range(repeats))
    return {
        "value": N_PARTICLES / best,
        "unit": "particles/s",
        "cores": cores,
        "kind": "port",
        "sample": (f"the full workload ({N_PARTICLES} particles), {CPU_DIFFERS}; best of "
                   f"{repeats}"),
        "single_thread": _single_thread(pos, q, cores),
    }


def run_reference(args):
    """The reference's CPU algorithm (the oracle) on the host cores, on the same 1M
    particles as the GPU arm; rank 0 alone runs it under torchrun."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import flat_tree_oracle as oracle
    from tree_d_3d_b200 import synthetic

    n = args.n
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    pos, q = synthetic.mixture8(n, seed=SEED)
    for _ in range(max(args.warmup, 1)):
        _cpu_fmm(pos, q)
    times = [_cpu_fmm(pos, q) for _ in range(args.steps)]
    total = sum(times)
    value = n * args.steps / total
    sample = f"{n} particles per step (the full workload), {CPU_DIFFERS}"
    line = {
        "impl": "reference",
        "metric": METRIC,
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
        "config": _cpu_config(n),
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": cores, "kind": "port",
                         "sample": sample, "single_thread": _single_thread(pos, q, cores)},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- GPU arm
class ClockSampler:
    """SM clocks and throttle reasons sampled while the timed region runs: NVML read every
    5 ms from a thread (reads only; no setting is touched), or nvidia-smi every 200 ms
    where NVML is not importable."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self, nvml):
        """This process's CUDA device in NVML, found by its PCI address (CUDA and NVML
        may number the GPUs differently), else by index."""
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_loop(self, nvml, handle):
        bits = [nvml.nvmlClocksEventReasonHwSlowdown, nvml.nvmlClocksEventReasonHwThermalSlowdown,
                nvml.nvmlClocksEventReasonSwThermalSlowdown, nvml.nvmlClocksEventReasonSwPowerCap]
        top = nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                why = nvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                self.rows.append((float(sm), float(top),
                                  ["Active" if why & b else "Not Active" for b in bits]))
            except Exception:  # a failed read drops one sample
                pass
            self.stop.wait(0.005)

    def __enter__(self):
        import threading

        try:
            import pynvml as nvml

            nvml.nvmlInit()
            handle = self._nvml_handle(nvml)
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nvml, handle),
                                           daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            return False
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=5)
            for ln in out.splitlines():
                parts = [p.strip() for p in ln.split(",")]
                try:
                    self.rows.append((float(parts[0]), float(parts[1]), parts[3:]))
                except (ValueError, IndexError):
                    continue
        return False

    def summary(self):
        rows = self.rows
        if not rows:
            return None
        reasons = sorted({self.NAMES[i] for _, _, flags in rows for i, f in enumerate(flags)
                          if i < len(self.NAMES) and f.lower() == "active"})
        sm = sorted(r[0] for r in rows)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows),
                "source": "nvml every 5 ms" if self.thread is not None else "nvidia-smi every 200 ms"}


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's ``value`` (the job's time is its slowest rank's)."""
    import torch

    if dist is None:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


#: the Coulomb kernel's softening in its workload line (config 3)
COULOMB_SOFTENING = 1e-3


def gpu_step(pos, q, w, e, precision, backward=True, kernel="log"):
    """One step: a fresh tree, the FMM field at every particle and its backward."""
    from tree_d_3d_b200 import Quad
    from tree_d_3d_b200.autograd import fmm_field

    p = pos.detach().requires_grad_(backward)
    c = q.detach().requires_grad_(backward)
    eps = SOFTENING if kernel == "log" else COULOMB_SOFTENING
    phi, field = fmm_field(p, c, Quad(0.0, 0.0, 1.0), kernel=kernel, order=ORDER, theta=THETA,
                           softening=eps, leaf_capacity=LEAF, precision=precision)
    if backward:
        ((w * phi).sum() + (e * field).sum()).backward()
    return phi.detach(), field.detach(), p.grad, c.grad


def time_steps(fn, steps, flush, torch):
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(steps):
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b)
    return total


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


def time_m2l_mixed(tree, torch, reps, form="grouped"):
    """One mixed M2L form alone (CUDA events on its stream), average ms per launch:
    "rows" the FP32 CUDA-core form with 8 lanes per destination row (the step's form),
    "lanes" the FP32 CUDA-core form with a lane per translation, "grouped"
    the tensor-core products grouped by translation, "tile" the per-translation
    tensor-core form."""
    from tree_d_3d_b200 import _lib
    from tree_d_3d_b200.flat_tree import _m2l_coefficients

    lists = tree._lists(THETA)
    count, w = tree.node_count, tree.order + 1
    lre = torch.zeros((count, w), dtype=torch.float64, device=tree.device)
    lim = torch.zeros_like(lre)
    hat = tree._scaled_moments((tree.moment_re, tree.moment_im))
    stream = _lib.stream(tree.device)
    status = tree._tensor_status()
    if form == "grouped":
        groups = lists.get("groups") or tree._m2l_groups(lists["m2l"], THETA)

        def launch():
            tree._m2l_grouped(groups, hat, lre, lim)
    elif form == "rows":
        coeff = np.ascontiguousarray(_m2l_coefficients(tree.order, tree.symmetric))
        records = tree._source_records((tree.moment_re, tree.moment_im))
        args = (lists["m2l_rows"].data_ptr(), lists["m2l_partners"].data_ptr(), count,
                tree.node_center.data_ptr(), tree.node_half.data_ptr(), records.data_ptr(),
                tree.order, coeff.ctypes.data, tree._unit, lre.data_ptr(), lim.data_ptr(),
                stream)

        def launch():
            _lib.call("td3_fmm_m2l_mixed_rows", *args)
    else:
        coeff = np.ascontiguousarray(_m2l_coefficients(tree.order, tree.symmetric))
        args = (lists["m2l_rows"].data_ptr(), lists["m2l_entry_row"].data_ptr(),
                lists["m2l_partners"].data_ptr(), count,
                tree.node_center.data_ptr(), tree.node_half.data_ptr(), tree.node_center.data_ptr(),
                tree.node_half.data_ptr(), hat.data_ptr(), tree.order, coeff.ctypes.data,
                tree._unit, 1 if form == "tile" else 0, lre.data_ptr(), lim.data_ptr(),
                status.data_ptr(), stream)

        def launch():
            _lib.call("td3_fmm_m2l_mixed", *args)
    launch()
    cur = torch.cuda.current_stream()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(cur)
    for _ in range(reps):
        launch()
    stop.record(cur)
    torch.cuda.synchronize()
    tree._check_tensor_cores()
    return start.elapsed_time(stop) / reps, int(lists["m2l"].shape[0])


def _peaks():
    """Measured peaks of this pool (MEASURED_PEAKS.json) or the stated fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            data = json.load(f)
        bf16 = float(data.get("bf16_tflops") or data.get("bf16_tflops_burst"))
        return bf16, "of measured (MEASURED_PEAKS.json bf16_tflops)"
    except (OSError, ValueError, TypeError):
        return 1590.0, "of fallback (1.59 PFLOP/s bf16, no MEASURED_PEAKS.json)"


def field_error(pos, q, precision, torch, n_sample=4096, kernel="log"):
    """Normwise relative field error against the FP64 direct sum on sampled particles."""
    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field

    eps = SOFTENING if kernel == "log" else COULOMB_SOFTENING
    tree = FlatQuadtree(pos, q, Quad(0.0, 0.0, 1.0), kernel=kernel, order=ORDER,
                        leaf_capacity=LEAF, precision=precision)
    _, field = tree.fmm(theta=THETA, softening=eps)
    idx = torch.tensor(np.random.default_rng(0).choice(pos.shape[1], n_sample, replace=False),
                       device=pos.device)
    _, ref = direct_field(pos[:, idx], pos, q, softening=eps, exclude=idx, kernel=kernel)
    diff = (field[:, idx] - ref).abs().max() / ref.abs().max()
    return float(diff), tree


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        from datetime import timedelta

        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from tree_d_3d_b200 import synthetic

    dev = torch.device("cuda", local)
    n = args.n
    pos_np, q_np = synthetic.mixture8(n, seed=SEED)
    rng = np.random.default_rng(SEED + 1)
    w_np, e_np = rng.normal(size=n), rng.normal(size=(2, n))
    pos = torch.tensor(pos_np, device=dev)
    q = torch.tensor(q_np, device=dev)
    w = torch.tensor(w_np, device=dev)
    e = torch.tensor(e_np, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    kernel, precision = ("log", "mixed")
    if args.trace_only:
        from tree_d_3d_b200 import flat_tree

        kernel, precision = args.kernel, args.precision
        flat_tree.M2L_GROUPED = args.m2l == "grouped"
        flat_tree.M2L_ROWS = args.m2l == "rows"
    for _ in range(args.warmup):
        gpu_step(pos, q, w, e, precision, kernel=kernel)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        total_ms = time_steps(lambda: gpu_step(pos, q, w, e, precision, kernel=kernel),
                              args.steps, flush, torch)
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

    # the plain FP64 form of the same step
    for _ in range(max(1, args.warmup // 2)):
        gpu_step(pos, q, w, e, "fp64")
    fp64_ms = max_over_ranks(time_steps(lambda: gpu_step(pos, q, w, e, "fp64"), args.steps,
                                        flush, torch), dist, dev)
    fp64_value = world * n * args.steps / (fp64_ms / 1e3)
    fwd_mixed = time_steps(lambda: gpu_step(pos, q, w, e, "mixed", backward=False), 3, flush,
                           torch) / 3
    fwd_fp64 = time_steps(lambda: gpu_step(pos, q, w, e, "fp64", backward=False), 3, flush,
                          torch) / 3

    # the same step with the Coulomb kernel (config 3's kernel; softening 1e-3): mixed and
    # FP64, and the mixed field error against the FP64 direct sum
    coulomb = {}
    for prec in ("mixed", "fp64"):
        gpu_step(pos, q, w, e, prec, kernel="coulomb")
        reps = 3
        c_ms = max_over_ranks(time_steps(lambda: gpu_step(pos, q, w, e, prec, kernel="coulomb"),
                                         reps, flush, torch), dist, dev) / reps
        coulomb[prec] = {"ms_per_step": c_ms, "value": world * n / (c_ms / 1e3)}
    coulomb["speedup_mixed_over_fp64"] = coulomb["mixed"]["value"] / coulomb["fp64"]["value"]
    coulomb["softening"] = COULOMB_SOFTENING

    # end to end through the public API: pinned host inputs in, host results out
    pos_h, q_h = torch.tensor(pos_np).pin_memory(), torch.tensor(q_np).pin_memory()
    w_h, e_h = torch.tensor(w_np).pin_memory(), torch.tensor(e_np).pin_memory()
    outs = [torch.empty(n, dtype=torch.float64).pin_memory(),
            torch.empty((2, n), dtype=torch.float64).pin_memory(),
            torch.empty((2, n), dtype=torch.float64).pin_memory(),
            torch.empty(n, dtype=torch.float64).pin_memory()]

    host_in = (pos_h, q_h, w_h, e_h)
    dev_in = [tuple(torch.empty(h.shape, dtype=h.dtype, device=dev) for h in host_in)
              for _ in range(2)]
    copy_stream = torch.cuda.Stream(device=dev)

    def e2e_run(steps):
        """`steps` steps back to back, each with its inputs copied in from pinned host
        memory and its results copied out: the copies run on a copy stream, step k + 1's
        inputs (into the other of two device buffers) and step k's results while step k
        computes; the L2 flush before every step runs on the compute stream.  Device time
        of the whole run (CUDA events; the copy stream joins before the end event)."""
        cur = torch.cuda.current_stream()
        ready = [torch.cuda.Event() for _ in range(steps)]
        done = [torch.cuda.Event() for _ in range(steps)]
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(cur)
        copy_stream.wait_stream(cur)

        def fetch(k):
            with torch.cuda.stream(copy_stream):
                if k >= 2:
                    copy_stream.wait_event(done[k - 2])  # step k - 2 has read this buffer
                for d, h in zip(dev_in[k % 2], host_in):
                    d.copy_(h, non_blocking=True)
                ready[k].record(copy_stream)

        fetch(0)
        for k in range(steps):
            if k + 1 < steps:
                fetch(k + 1)
            flush.fill_(1.0)
            cur.wait_event(ready[k])
            results = gpu_step(*dev_in[k % 2], "mixed")
            done[k].record(cur)
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(done[k])
                for host, r in zip(outs, results):
                    host.copy_(r, non_blocking=True)
                    r.record_stream(copy_stream)
        cur.wait_stream(copy_stream)
        stop.record(cur)
        stop.synchronize()
        return start.elapsed_time(stop)

    e2e_run(2)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e2e_run(args.steps), dist, dev)
    e2e_value = world * n * args.steps / (e2e_ms / 1e3)

    launches = count_our_launches(lambda: gpu_step(pos, q, w, e, "mixed"), torch)
    err_mixed, tree = field_error(pos, q, "mixed", torch)
    err_fp64, _ = field_error(pos, q, "fp64", torch)
    for prec in ("mixed", "fp64"):
        coulomb[prec]["rel_err_field"], _ = field_error(pos, q, prec, torch, kernel="coulomb")
    # the step's M2L form (FP32 on the CUDA cores, a lane per translation); the tensor-core
    # forms (products grouped by translation; per translation) are timed beside it
    m2l_ms, n_m2l = time_m2l_mixed(tree, torch, reps=5, form="rows")
    m2l_lanes_ms, _ = time_m2l_mixed(tree, torch, reps=5, form="lanes")
    m2l_grouped_ms, _ = time_m2l_mixed(tree, torch, reps=5, form="grouped")
    m2l_tile_ms, _ = time_m2l_mixed(tree, torch, reps=5, form="tile")
    groups = tree._m2l_groups(tree._lists(THETA)["m2l"], THETA)
    n_runs = int(groups["tile_run"][-1].item())
    width = ORDER + 1
    flops = 2 * n_m2l * 8 * width * width  # directed translations x 8 (p + 1)^2
    achieved = flops / (m2l_ms * 1e-3) / 1e12
    bf16, peak_note = _peaks()
    tf32 = bf16 / 2  # dense TF32 runs at half the BF16 rate on the tensor cores
    # per run: D[128 x 64] += A_hi [128 x 32] B^T and D[128 x 32] += A_lo B_hi^T
    issued = n_runs * 2 * 128 * 32 * (64 + 32)
    roofline = {
        "kernel": "k_m2l_mixed_rows<12> (FP32 M2L, 8 lanes per destination row, forward)",
        "bound": "fp32",
        "achieved": achieved,
        "peak": FP32_PEAK,
        "unit": "TFLOP/s",
        "frac": achieved / FP32_PEAK,
        "peak_source": ("nominal FP32 FMA rate at the max SM clock (148 SM x 128 lanes x 2 x "
                        "1965 MHz); MEASURED_PEAKS.json has no FP32 CUDA-core figure"),
        "algorithmic": "8 (p + 1)^2 flop per directed translation (the reference's count)",
        # dram read + write of one ncu capture of this kernel at 300k particles (72.8 MB
        # for 3.745M translations), scaled by the translations of this launch
        "traffic": 72.8e6 * (2 * n_m2l) / 3.745e6,
        "traffic_unit": "bytes per launch (scaled from a 300k-particle ncu capture)",
        "ms_per_launch": m2l_ms,
        "flop_per_launch": flops,
        "grouped_tensor_form": {
            "kernel": "k_m2l_grouped<12> (3xTF32 tcgen05 products grouped by translation)",
            "ms_per_launch": m2l_grouped_ms,
            "runs_per_launch": n_runs,
            "issued_tensor_tflops": issued / (m2l_grouped_ms * 1e-3) / 1e12,
            "issued_frac": issued / (m2l_grouped_ms * 1e-3) / 1e12 / tf32,
            "peak_source": f"dense TF32 = half the BF16 tensor rate, {peak_note}",
        },
        "tile_form_ms_per_launch": m2l_tile_ms,
        "lane_form_ms_per_launch": m2l_lanes_ms,
    }
    clock = clocks.summary()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "particles/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64 mixed",
        "data": "synthetic",
        "config": {**_config(n), "parallelism": f"replicas x{world}", "precision": "mixed",
                   "backward": True},
        "fp64": {"value": fp64_value, "ms_per_step": fp64_ms / args.steps,
                 "speedup_mixed_over_fp64": value / fp64_value,
                 "rel_err_field": err_fp64},
        "rel_err_field": err_mixed,
        "forward_only_ms": {"mixed": fwd_mixed, "fp64": fwd_fp64},
        "coulomb": coulomb,
        "e2e": {"value": e2e_value, "unit": "particles/s",
                "h2d_bytes_per_step": 8 * n * (2 + 1 + 1 + 2),
                "d2h_bytes_per_step": 8 * n * (1 + 2 + 2 + 1)},
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


# ----------------------------------------------------------------------------- suite
def _event_ms(fn, torch, reps=5, warm=2):
    """Median CUDA-event time of fn() in ms (inputs resident; no L2 flush: repeated work
    on the same data, as an application that steps the same particles)."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    return float(np.median(times))


def _sample_error(torch, pos, q, field, kernel, eps, n_sample=4096, targets=None, tfield=None):
    """Normwise relative field error against the FP64 direct sum on sampled points."""
    from tree_d_3d_b200 import direct_field

    if targets is None:
        idx = torch.tensor(np.random.default_rng(0).choice(pos.shape[1], n_sample, replace=False),
                           device=pos.device)
        _, ref = direct_field(pos[:, idx], pos, q, softening=eps, exclude=idx, kernel=kernel)
        got = field[:, idx]
    else:
        idx = torch.tensor(np.random.default_rng(0).choice(targets.shape[1], n_sample,
                                                           replace=False), device=pos.device)
        _, ref = direct_field(targets[:, idx], pos, q, softening=eps, kernel=kernel)
        got = tfield[:, idx]
    return float((got - ref).abs().max() / ref.abs().max())


def run_suite(args):
    """Every workload configuration of the solver on one GPU, one JSON line per case:
    config 1 (5000 uniform charges: walk and direct sum), config 2 (200k Gaussian line
    charges: FMM p = 12), config 3 (1M 8-Gaussian mixture: walk at theta 0.3 / 0.5 / 0.7,
    FMM at p = 8 / 12 / 16 for both kernels, fmm_at at 1M uniform targets), config 4
    (100k uniform, N(0, 1) charges: energy and its backward), config 5 (1M protons: 100
    simulation steps, gradient of the final kinetic energy through 20 checkpointed
    steps).  Tree builds are inside the timed FMM cases (a fresh tree per call)."""
    import torch

    from tree_d_3d_b200 import FlatQuadtree, Quad, direct_field, synthetic
    from tree_d_3d_b200.autograd import fmm_energy
    from tree_d_3d_b200.simulation import ElectrostaticSimulation, rollout_kinetic_energy

    dev = torch.device("cuda", 0)
    root = Quad(0.0, 0.0, 1.0)

    def emit(config, case, ms, n, unit="particles/s", **extra):
        print(json.dumps({"suite": config, "case": case, "ms": round(ms, 4),
                          "value": n / (ms / 1e3), "unit": unit, **extra}), flush=True)

    # config 1
    rng = np.random.default_rng(SEED)
    p1 = torch.tensor(rng.uniform(-1, 1, (2, 5000)), device=dev)
    q1 = torch.tensor(rng.choice([-1.0, 1.0], 5000), device=dev)
    idx1 = torch.arange(5000, device=dev)
    for prec in ("fp64", "mixed"):
        tree = FlatQuadtree(p1, q1, root, precision=prec)
        ms = _event_ms(lambda: tree.evaluate(p1, exclude=idx1, theta=0.5, softening=1e-3), torch)
        _, f = tree.evaluate(p1, exclude=idx1, theta=0.5, softening=1e-3)
        _, ref = direct_field(p1, p1, q1, softening=1e-3, exclude=idx1)
        err = float((f - ref).abs().max() / ref.abs().max())
        emit("1", f"walk coulomb theta=0.5 {prec}", ms, 5000, "targets/s", rel_err_vs_direct=err)
    ms = _event_ms(lambda: direct_field(p1, p1, q1, softening=1e-3, exclude=idx1), torch)
    emit("1", "direct coulomb", ms, 5000 * 5000, "pairs/s")

    # config 2
    p2, q2 = (torch.tensor(a, device=dev) for a in synthetic.gaussian(200_000, 0.3, seed=2))
    for prec in ("fp64", "mixed"):
        def run2():
            return FlatQuadtree(p2, q2, root, kernel="log", order=12, precision=prec).fmm(theta=0.5)
        ms = _event_ms(run2, torch)
        err = _sample_error(torch, p2, q2, run2()[1], "log", 0.0)
        emit("2", f"fmm log p=12 {prec}", ms, 200_000, rel_err_vs_direct=err)

    # config 3
    p3, q3 = (torch.tensor(a, device=dev) for a in synthetic.mixture8(1_000_000, seed=SEED))
    idx3 = torch.arange(1_000_000, device=dev)
    for prec in ("fp64", "mixed"):
        tree = FlatQuadtree(p3, q3, root, kernel="coulomb", precision=prec)
        for theta in (0.3, 0.5, 0.7):
            ms = _event_ms(lambda: tree.evaluate(p3, exclude=idx3, theta=theta, softening=1e-3),
                           torch, reps=3)
            f = tree.evaluate(p3, exclude=idx3, theta=theta, softening=1e-3)[1]
            err = _sample_error(torch, p3, q3, f, "coulomb", 1e-3)
            emit("3", f"walk coulomb theta={theta} {prec}", ms, 1_000_000, "targets/s",
                 rel_err_vs_direct=err)
    for kernel, eps in (("coulomb", 1e-3), ("log", 0.0)):
        for order in (8, 12, 16):
            for prec in ("fp64", "mixed"):
                def run3():
                    return FlatQuadtree(p3, q3, root, kernel=kernel, order=order,
                                        precision=prec).fmm(theta=0.5, softening=eps)
                ms = _event_ms(run3, torch, reps=3)
                err = _sample_error(torch, p3, q3, run3()[1], kernel, eps)
                emit("3", f"fmm {kernel} p={order} {prec}", ms, 1_000_000,
                     rel_err_vs_direct=err)
    targets = torch.tensor(np.random.default_rng(SEED + 2).uniform(-1, 1, (2, 1_000_000)),
                           device=dev)
    for kernel, eps in (("coulomb", 1e-3), ("log", 0.0)):
        for prec in ("fp64", "mixed"):
            tree = FlatQuadtree(p3, q3, root, kernel=kernel, order=12, precision=prec)
            tree.fmm_at(targets, theta=0.5, softening=eps)  # target tree and lists, kept
            ms = _event_ms(lambda: tree.fmm_at(targets, theta=0.5, softening=eps), torch, reps=3)
            err = _sample_error(torch, p3, q3, None, kernel, eps, targets=targets,
                                tfield=tree.fmm_at(targets, theta=0.5, softening=eps)[1])
            emit("3", f"fmm_at {kernel} p=12 1M targets {prec} (plan kept)", ms, 1_000_000,
                 "targets/s", rel_err_vs_direct=err)

    # config 4
    rng = np.random.default_rng(SEED + 4)
    p4 = torch.tensor(rng.uniform(-1, 1, (2, 100_000)), device=dev)
    q4 = torch.tensor(rng.normal(size=100_000), device=dev)
    for kernel, eps in (("log", 0.0), ("coulomb", 1e-3)):
        for prec in ("fp64", "mixed"):
            def run4():
                P = p4.detach().requires_grad_(True)
                Q = q4.detach().requires_grad_(True)
                fmm_energy(P, Q, root, kernel=kernel, order=12, softening=eps,
                           precision=prec).backward()
                return P.grad, Q.grad
            ms = _event_ms(run4, torch)
            emit("4", f"energy + backward {kernel} p=12 {prec}", ms, 100_000)

    # config 5
    p5, q5 = synthetic.protons(1_000_000, seed=SEED)
    walls = {"x_min": -1.0, "x_max": 1.0, "y_min": -1.0, "y_max": 1.0}
    def new_sim():
        return ElectrostaticSimulation(positions=p5, charges=q5, bounds=root, k_e=1.0, B_z=1.0,
                                       dt=1e-4, absorbing_walls=walls)
    # one step of the full 1M cloud (fields at the start and at the end of the step)
    ms = _event_ms(lambda: new_sim().step(), torch, reps=3, warm=1)
    emit("5", f"first step of 1M protons (method {new_sim()._resolve_method()})", ms,
         1_000_000, "particle-steps/s")
    # 100 steps: the like charges fly apart and the walls absorb most of them, so the
    # later steps hold few particles (the method follows the particle count)
    sim = new_sim()
    sim.step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(100):
        sim.step()
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b)
    emit("5", "100 simulation steps after the first", ms, 100, "steps/s",
         particles_left=int(sim.num_particles), method_at_end=sim._resolve_method(),
         wall_s=time.perf_counter() - t0)
    P = torch.tensor(p5, device=dev)
    Q = torch.tensor(q5, device=dev)

    def run5():
        Qg = Q.detach().requires_grad_(True)
        ke = rollout_kinetic_energy(P, torch.zeros_like(P), Qg, torch.ones_like(Q), 20,
                                    bounds=root, dt=1e-4, B_z=1.0, k_e=1.0,
                                    absorbing_walls=walls)
        ke.backward()
        return Qg.grad
    ms = _event_ms(run5, torch, reps=2, warm=1)
    emit("5", "gradient of the final kinetic energy through 20 checkpointed steps", ms,
         20 * 1_000_000, "particle-steps/s")
    return 0


def main():
    args = _args()
    if args.impl == "reference":
        return run_reference(args)
    if args.suite:
        return run_suite(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
