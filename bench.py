"""Benchmark: G pair-interactions/s of the Hermite-4 step on one B200.

Workload (default, the headline): Plummer sphere N = 65536 (Henon units, seed
1), softening eps = 1e-2, shared fixed dt = 1/1024; one step = predict + acc/jerk
of all N^2 pairs + correct, replayed from the engine's captured CUDA graph.
The headline `value` is the mixed-precision path (FP32 pair loop, FP64
accumulation and integration) with the automatic mixed kernel, tiled by the
autotuner; the plain FP64 path runs on the same input and is reported beside
it.  Both run on to one N-body time unit for |dE/E|.

At N = 1 the same JSON line also carries
  accuracy_t0    per-body acc/jerk error at t = 0 of the mixed kernel families
                 (near/far tile-relative, hi/lo, plain tile-relative) against
                 FP64, and of the reference's own _F32 arithmetic on sampled bodies
  tuning         the autotuner's tiling and pair time next to the heuristic's
  large_n        N = 262144 (seed 2, eps = 4e-3, dt = 1/2048): mixed and FP64
                 G interactions/s, their ratio, acc error, |dE/E| over one time unit
  ensemble       512 Plummer clusters (seed 3): one persistent launch per step
                 against one launch per cluster (serial and concurrent)
  cpu_baseline   the reference's FP64 CPU build on this host's cores, whole
                 force_calculation calls

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own FP64 CPU code (compiled from its
sources into oracle/_ref) on this host's cores: every step is one complete
fixed-dt Hermite step of the same workload (prediction, force_calculation over
all rows, snapandcrackle, correction); the input comes from the oracle's own
Plummer sampler, so that arm loads no library of the product.

Multi-GPU (torchrun): replicas only - every rank runs the same independent
system on its own GPU with no data exchange; value = ranks x N^2 / max time.
"""
from __future__ import annotations

import os

# The reference CPU force loop keeps OpenMP private copies of its six output
# arrays on each thread's stack (array-section reductions, src/kernel.cpp:1180):
# 48 bytes per body per thread.  Worker stacks are sized before anything loads
# libgomp; the calling thread gets its own large stack (cpu_call below).
os.environ.setdefault("OMP_STACKSIZE", "256M")

import argparse
import json
import statistics
import subprocess
import sys
import threading
import time
import traceback
from dataclasses import dataclass

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "n-body-code_b200"))

METRIC = "Gpair-interactions/s at N=65536: mixed-prec vs FP64 GPU, equal energy error"
FLOP_PER_INTERACTION = 60
L2_FLUSH_BYTES = 256 << 20

# Instructions per pair interaction of each pair kernel, counted from its
# source (csrc/pair.cuh): FP32 (or FP64) pipe lane-operations and MUFU
# operations.  record_format -> (pipe, lane ops, mufu ops).  The near/far
# kernel (format 3) issues 25 lane-ops on a far tile and 31 on a near one
# (double-single separation): roofline() weights them by the measured share.
ISSUED_OPS = {
    0: ("fp64", 31, 1),   # pair_fp64_kernel: rsqrt.approx.f64 + one Householder step
    1: ("fp32", 32, 1),   # pair_mixed_kernel: scalar hi/lo, y^2 by multiply
    2: ("fp32", 31, 2),   # pair_mixed_x2_kernel: packed hi/lo, rsqrt + rcp on MUFU
    3: ("fp32", 25, 2),   # pair_mixed_nf_kernel, far tiles: one add per separation component
}
NEAR_EXTRA_OPS = 6        # near tiles: three adds per component instead of one
KERNEL_NAMES = {0: "pair_fp64_kernel", 1: "pair_mixed_kernel", 2: "pair_mixed_x2_kernel",
                3: "pair_mixed_nf_kernel"}
VARIANT_NAMES = {1: "scalar hi/lo (pair_variant 1)", 2: "packed hi/lo (pair_variant 2)",
                 3: "packed hi/lo (pair_variant 3)",
                 4: "near/far tile-relative (pair_variant 4): far tiles one add per separation "
                    "component, near tiles double-single separations",
                 5: "tile-relative with every tile taken as far (pair_variant 5): one add per "
                    "separation component for all pairs"}


@dataclass
class Workload:
    n: int
    seed: int
    eps: float
    dt: float

    @property
    def eps2(self):
        return self.eps ** 2

    def name(self, precision):
        return (f"Hermite-4 shared fixed step, Plummer N={self.n} seed {self.seed} (Henon units), "
                f"eps={self.eps:g}, dt=1/{round(1 / self.dt)}, {precision}")


LARGE_N = Workload(262144, 2, 4e-3, 1.0 / 2048)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--eps", type=float, default=1e-2)
    ap.add_argument("--dt", type=float, default=1.0 / 1024)
    ap.add_argument("--precision", default="mixed", choices=("mixed", "fp64"))
    ap.add_argument("--no-fp64-arm", action="store_true", help="skip the FP64 comparison arm")
    ap.add_argument("--heuristic", action="store_true",
                    help="tile the pair kernels by the heuristic instead of the autotuner")
    ap.add_argument("--variant", type=int, default=0,
                    help="mixed pair kernel (nbody_config.pair_variant): 0 = automatic (near/far "
                         "tile-relative from 16384 bodies), 1 = scalar hi/lo, 2/3 = packed hi/lo, "
                         "4 = near/far tile-relative, 5 = plain tile-relative; ensembles: 4 = "
                         "near/far, 5 = plain tile-relative, else packed hi/lo")
    ap.add_argument("--time-units", type=float, default=1.0,
                    help="integrate to this model time in total (timed steps included, untimed "
                         "beyond them) and report |dE/E| there")
    ap.add_argument("--large-n-time-units", type=float, default=1.0,
                    help="model time of the N=262144 energy runs (0 = skip them)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the accuracy, tuning, N=262144 and ensemble sections")
    ap.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--kernels-only", action="store_true",
                    help="time the main arm only (no peaks, e2e, CPU baseline): the profiling case")
    ap.add_argument("--ensemble", action="store_true",
                    help="batched-ensemble workload: Plummer clusters (seed 3), N log-uniform in "
                         "[256, 8192], eps = 4/N, dt = 1/512, vs one launch per cluster")
    ap.add_argument("--clusters", type=int, default=512)
    ap.add_argument("--adjoint", action="store_true",
                    help="gradient workload: Plummer N=4096 (seed 4), eps=1e-2, dt=1/256, 256 steps, "
                         "checkpoint every 16; forward and backward times")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.p = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.p is not None:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[4:8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for _, _, r in rows for k, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def traffic_per_launch(kernel):
    """DRAM bytes per pair-kernel launch (the headline workload) from the
    committed ncu summary, by kernel name."""
    path = os.path.join(ROOT, "profiles", "pair_kernel_dram.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel)
    except (OSError, ValueError):
        return None


def run_arm(w, precision, state, torch, dist, world, dev, steps, warmup, variant=0, tune=True,
            time_units=0.0, flush_l2=True):
    """K timed Hermite steps of workload w (CUDA events on the engine's stream,
    L2 flushed between steps), then untimed steps up to `time_units` of model
    time for |dE/E|."""
    import nbody_b200 as nb
    clk = ClockSampler(dev).__enter__()  # sampling starts before the warm-up so the timed region is covered
    e = nb.Engine(w.n, eps2=w.eps2, precision=precision, device=dev, dt=w.dt, tune=tune,
                  pair_variant=variant if precision == "mixed" else 0)
    e.set_state(state)
    e.force_calculation()
    T0, U0 = e.energy()
    stream = torch.cuda.ExternalStream(e.stream, device=f"cuda:{dev}")
    flush = torch.empty(L2_FLUSH_BYTES if flush_l2 else 1, dtype=torch.uint8, device=f"cuda:{dev}")
    e.timestepping(warmup)
    e.synchronize()
    reorders0 = e.timers()["reorders"]
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    pair_ms, pred_ms, corr_ms = [], [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        for k in range(steps):
            if flush_l2:
                flush.zero_()                   # evict L2 between timed steps
            starts[k].record(stream)
            e.timestepping(1)
            ends[k].record(stream)
            ends[k].synchronize()
            t = e.timers()                      # graph-internal events of this step
            pred_ms.append(t["pred_ms"]); pair_ms.append(t["eval_ms"]); corr_ms.append(t["corr_ms"])
    torch.cuda.synchronize(dev)
    clk.__exit__(None, None, None)
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(t) for s, t in zip(starts, ends)]
    tm = e.timers()  # near_tile_fraction: the last timed step's pair pass
    # kernels of the timed steps: the captured step graph each step, plus the
    # captured Hilbert re-ordering where one ran (tile-relative kernel)
    launches = tm["step_kernels"] * steps + tm["order_kernels"] * (tm["reorders"] - reorders0)
    if time_units > 0:  # carry on (untimed) to the requested model time
        rest = int(round(time_units / w.dt)) - warmup - steps
        while rest > 0:
            k = min(rest, 256)
            e.timestepping(k)
            e.synchronize()
            rest -= k
    t_end = e.timers()["t"]
    T1, U1 = e.energy()
    de = abs((T1 + U1) - (T0 + U0)) / abs(T0 + U0)
    e.close()
    return {
        "ms_per_step": float(np.mean(step_ms)),
        "pair_ms": float(np.mean(pair_ms)),
        "pred_ms": float(np.mean(pred_ms)),
        "corr_ms": float(np.mean(corr_ms)),
        "dE_over_E": de,
        "t_end": t_end,
        "E0": T0 + U0,
        "tiling": {k: tm[k] for k in ("threads", "i_per_thread", "j_tile", "split_j", "j_cluster")},
        "tiling_source": {1: "heuristic", 2: "autotuned", 3: "autotuned (cached)"}.get(tm["tiling_source"]),
        "clocks": clk.summary(),
        "launches": int(launches),
        "record_format": tm["record_format"],
        "near_tile_fraction": tm["near_tile_fraction"],
    }


def run_e2e(w, precision, state, torch, steps):
    """End to end through the drop-in C-ABI call (the reference's
    force_calculation contract): pinned host arrays in, host arrays out,
    host<->device copies inside every timed call."""
    import nbody_b200 as nb
    n = w.n
    pinned = {k: torch.from_numpy(np.ascontiguousarray(state[k])).pin_memory() for k in nb.FIELDS}
    host = {k: v.numpy() for k, v in pinned.items()}
    out_t = torch.empty((6, n), dtype=torch.float64).pin_memory()
    import ctypes as C
    from nbody_b200 import _lib
    L = _lib.load()
    ptrs = [C.c_void_p(host[k].ctypes.data) for k in nb.FIELDS]
    outs = [C.c_void_p(out_t[k].data_ptr()) for k in range(6)]
    prec = 1 if precision == "mixed" else 0

    def call():
        _lib.check(L.nbody_force_calculation(n, w.eps2, prec, 0, n, *ptrs, *outs),
                   "nbody_force_calculation")

    # once per system size, untimed: the drop-in's autotuner (reuses the choice
    # of the arm's tuned engine when it holds the same size and format)
    nb.force_calculation_tune(host, w.eps2, precision)
    for _ in range(2):
        call()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        call()
        ts.append(time.perf_counter() - t0)
    nb.release_force_cache()
    s = float(np.mean(ts))
    return {"value": n * n / s / 1e9, "unit": "Gint/s", "h2d_bytes_per_step": 7 * 8 * n,
            "d2h_bytes_per_step": 6 * 8 * n, "ms_per_call": s * 1e3,
            "what": "nbody_force_calculation (drop-in for force_calculation), pinned host buffers; "
                    "tiling from nbody_force_calculation_tune (untimed, once per size)"}


def roofline(peaks, w, arm, prec):
    """60-flop convention against the measured FMA peak, plus the issued
    lane-operations of the kernel against the same pipe's lane-op peak."""
    inter = float(w.n) * w.n
    fmt = arm["record_format"]
    peak = peaks["fp32_tflops"] if prec == "mixed" else peaks["fp64_tflops"]
    achieved = FLOP_PER_INTERACTION * inter / (arm["pair_ms"] * 1e-3) / 1e12
    pipe, lane_ops, mufu_ops = ISSUED_OPS[fmt]
    near = arm.get("near_tile_fraction", 0.0) if fmt == 3 else 0.0
    lane_ops = lane_ops + NEAR_EXTRA_OPS * near
    lane_peak = (max(peaks["fp32_tflops"], peaks["fp32x2_tflops"]) if pipe == "fp32"
                 else peaks["fp64_tflops"]) / 2 * 1e12       # FMA = 2 flop = 1 lane-op
    rate = inter / (arm["pair_ms"] * 1e-3)
    return {"bound": pipe, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic_per_launch(KERNEL_NAMES[fmt]),
            "kernel": KERNEL_NAMES[fmt],
            "peak_source": "measured live by nbody_measure_peaks (FMA microkernel, this GPU)",
            "flop_per_interaction": FLOP_PER_INTERACTION,
            "issued_frac": rate * lane_ops / lane_peak,
            "issued": {"lane_ops_per_interaction": lane_ops, "mufu_ops_per_interaction": mufu_ops,
                       "near_tile_fraction": near if fmt == 3 else None,
                       "lane_op_peak_per_s": lane_peak,
                       "mufu_frac": rate * mufu_ops / (peaks["mufu_rsqrt_gops"] * 1e9)}}


# ---------------------------------------------------------------------------
# accuracy at t = 0
# ---------------------------------------------------------------------------
def _stats(e):
    return {"median": float(np.median(e)), "p99": float(np.quantile(e, 0.99)), "max": float(e.max())}


def _vec_rel(a, b):
    return np.sqrt(((a - b) ** 2).sum(0)) / np.sqrt((b ** 2).sum(0))


def engine_derivs(w, state, precision, dev, variant=0):
    import nbody_b200 as nb
    with nb.Engine(w.n, eps2=w.eps2, precision=precision, device=dev, dt=w.dt,
                   pair_variant=variant if precision == "mixed" else 0) as e:
        e.set_state(state)
        e.force_calculation()
        return e.get_derivs(), e.timers()["record_format"]


def accuracy_block(w, state, dev, sample_rows=2048):
    """Per-body acc/jerk error at t = 0 of the mixed kernel families against the
    FP64 engine (all bodies), and - on evenly spaced sampled bodies - of the same
    kernels and of the reference's _F32 arithmetic (oracle restatement,
    src/kernel.cpp:1101-1163) against FP64 direct sums; the FP64 engine itself
    against those direct sums."""
    O = _oracle()
    d64, _ = engine_derivs(w, state, "fp64", dev)
    rows = np.linspace(0, w.n - 1, min(sample_rows, w.n)).astype(np.int64)
    ref = O.force_rows(state, w.eps2, rows)
    f32 = O.force_rows(state, w.eps2, rows, "f32")
    out = {"fp64_engine_vs_direct_sums_max": {
               "acc": float(_vec_rel(d64[:3, rows], ref[:3]).max()),
               "jerk": float(_vec_rel(d64[3:, rows], ref[3:]).max())},
           "all_bodies_vs_fp64_engine": {}, "sampled_vs_fp64": {},
           "sampled_rows": int(rows.size)}
    keys = ((4, "tile_relative"), (3, "hilo"), (5, "plain_tile_relative"))
    for v, key in keys:
        dm, fmt = engine_derivs(w, state, "mixed", dev, v)
        out["all_bodies_vs_fp64_engine"][key] = {"acc": _stats(_vec_rel(dm[:3], d64[:3])),
                                                 "jerk": _stats(_vec_rel(dm[3:], d64[3:])),
                                                 "kernel": KERNEL_NAMES[fmt]}
        out["sampled_vs_fp64"][key] = {"acc": _stats(_vec_rel(dm[:3, rows], ref[:3])),
                                       "jerk": _stats(_vec_rel(dm[3:, rows], ref[3:]))}
    out["sampled_vs_fp64"]["reference_f32"] = {"acc": _stats(_vec_rel(f32[:3], ref[:3])),
                                               "jerk": _stats(_vec_rel(f32[3:], ref[3:]))}
    rf = out["sampled_vs_fp64"]["reference_f32"]["acc"]
    out["acc_err_over_reference_f32"] = {
        key: {q: out["sampled_vs_fp64"][key]["acc"][q] / rf[q] for q in ("median", "p99", "max")}
        for _, key in keys}
    out["kernels"] = {key: VARIANT_NAMES[v] for v, key in keys}
    return out


# ---------------------------------------------------------------------------
# CPU: the reference's own code (oracle/_ref) or, if absent, the oracle port
# ---------------------------------------------------------------------------
def cpu_call(fn, *args):
    """Runs fn on a thread with a 1 GiB stack (the OpenMP master thread of the
    reference's force loop needs 48 bytes of stack per body)."""
    out = {}

    def body():
        try:
            out["r"] = fn(*args)
        except BaseException as exc:  # re-raised in the caller
            out["e"] = exc
    old = threading.stack_size(1 << 30)
    try:
        th = threading.Thread(target=body)
        th.start()
        th.join()
    finally:
        threading.stack_size(old)
    if "e" in out:
        raise out["e"]
    return out.get("r")


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_state(w):
    """The workload's bodies from the oracle's Plummer sampler (equal, value
    for value, to the engine's), from the reference build's library when it
    exists so that the reference arm maps nothing else."""
    O = _oracle()
    return O.plummer(w.n, w.seed, from_reference_build=O.have_reference())


def cpu_reference_steps(w, state, warmup, steps=None, seconds=None):
    """Complete fixed-dt Hermite steps of the reference's FP64 build on all
    host cores: prediction, force_calculation over all rows, snapandcrackle,
    correction (oracle/ref_harness.cpp ref_bench_step with one rank).  Runs
    `warmup` untimed steps, then `steps` timed ones, or timed ones until
    `seconds` have passed (at least two)."""
    O = _oracle()
    if not O.have_reference():
        return None
    lib = O.ref()
    cores = lib.ref_max_threads()
    arrs = [np.ascontiguousarray(state[k]) for k in ("x", "y", "z", "m", "vx", "vy", "vz")]
    P = O._p
    h = lib.ref_bench_create(w.n, w.dt, 1, *map(P, arrs))
    t3 = np.zeros(3)
    for _ in range(warmup):
        lib.ref_bench_step(h, P(t3))
    per = []
    while True:
        lib.ref_bench_step(h, P(t3))
        per.append(float(t3.sum()))
        if steps is not None and len(per) >= steps:
            break
        if steps is None and len(per) >= 2 and sum(per) >= seconds:
            break
    lib.ref_bench_destroy(h)
    return {"per_step_s": np.array(per), "cores": cores, "kind": "reference",
            "sample": (f"reference FP64 CPU build (oracle/_ref), N={w.n}, {len(per)} complete "
                       f"fixed-dt Hermite steps: prediction + full force_calculation (all rows, "
                       f"one rank) + snapandcrackle + correction, OpenMP on {cores} threads")}


def cpu_port_steps(w, state, steps, seconds_per_step):
    """Fallback when the reference build is absent: the oracle's direct row
    sums on a sample of rows, scaled to all rows (one thread)."""
    O = _oracle()
    n = w.n
    rows_per_s = 2e8 / n  # rough single-thread rate of the direct row sum
    nrows = int(max(8, min(n, rows_per_s * seconds_per_step)))
    rows = np.linspace(0, n - 1, nrows).astype(np.int32)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.force_rows(state, w.eps2, rows)
        ts.append(time.perf_counter() - t0)
    per = np.array(ts) * (n / nrows)
    return {"per_step_s": per, "cores": 1, "kind": "port",
            "sample": f"oracle direct row sums on {nrows} of {n} rows per step, scaled by N/rows"}


def cpu_baseline(a, w):
    state = cpu_state(w)
    r = cpu_call(cpu_reference_steps, w, state, 1, None, a.cpu_sample_seconds)
    if r is None:
        r = cpu_call(cpu_port_steps, w, state, 3, a.cpu_sample_seconds / 3)
    v = w.n * w.n / float(np.mean(r["per_step_s"])) / 1e9
    return {"value": v, "unit": "Gint/s", "cores": r["cores"], "kind": r["kind"], "sample": r["sample"]}


# ---------------------------------------------------------------------------
def max_over_ranks_fn(world, dist, device):
    """x -> max of x over all ranks (all-reduce MAX on `device`; NCCL on GPUs,
    gloo on CPU)."""
    if world == 1:
        return lambda x: x
    import torch

    def f(x):
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return f


def arms_over_ranks(max_fn, main_arm, other):
    """Slowest-rank step and pair times of both arms (other may be None).
    Every rank calls this, with the same arms, in the same order."""
    main_arm["ms_per_step"] = max_fn(main_arm["ms_per_step"])
    main_arm["pair_ms"] = max_fn(main_arm["pair_ms"])
    if other is not None:
        other["ms_per_step"] = max_fn(other["ms_per_step"])
        other["pair_ms"] = max_fn(other["pair_ms"])


def e2e_over_ranks(max_fn, world, n, e2e):
    """Whole-job e2e value from the slowest rank's drop-in call time."""
    e2e["ms_per_call"] = max_fn(e2e["ms_per_call"])
    e2e["value"] = world * float(n) * n / (e2e["ms_per_call"] * 1e-3) / 1e9
    return e2e


def replica_value(world, interactions_per_replica, ms_per_step):
    """Whole-job G interactions/s of `world` independent replicas timed at the
    slowest rank's step time."""
    return world * interactions_per_replica / (ms_per_step * 1e-3) / 1e9


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def main_reference(a):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    w = Workload(a.n, a.seed, a.eps, a.dt)
    state = cpu_state(w)
    r = cpu_call(cpu_reference_steps, w, state, a.warmup, a.steps)
    if r is None:
        per_step_budget = min(2.0, max(0.2, 150.0 / max(a.steps + a.warmup, 1)))
        r = cpu_call(cpu_port_steps, w, state, a.steps + a.warmup, per_step_budget)
        r["per_step_s"] = r["per_step_s"][a.warmup:]
    s = float(np.mean(r["per_step_s"]))
    v = w.n * w.n / s / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gint/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Plummer sphere)",
        "config": {"workload": w.name("FP64 CPU (reference)"), "n": w.n, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": v, "unit": "Gint/s", "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"]},
        "e2e": {"value": v, "unit": "Gint/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def shard_clusters(sizes, world, rank):
    """Cluster indices of `rank` when the clusters are shared out over `world`
    GPUs: largest N^2 first, each to the rank with the least work so far.
    Deterministic, so every rank computes the same assignment."""
    load = [0.0] * world
    owner = np.empty(len(sizes), dtype=np.int64)
    for c in sorted(range(len(sizes)), key=lambda c: (-int(sizes[c]) ** 2, c)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[c] = r
        load[r] += float(sizes[c]) ** 2
    return np.flatnonzero(owner == rank)


def run_ensemble(a, torch, world, rank, dist, dev, steps, warmup, time_units):
    """Batched ensemble of this rank's clusters: one persistent launch per step,
    then the same clusters as single-system engines (one launch per cluster),
    stepped one at a time and all at once on their own streams."""
    import nbody_b200 as nb
    sizes_all, eps2_all, state_all = nb.plummer_ensemble(a.clusters, 3)
    mine = shard_clusters(sizes_all, world, rank)
    off_all = np.concatenate([[0], np.cumsum(sizes_all)])
    sizes, eps2 = sizes_all[mine], eps2_all[mine]
    state = {k: np.concatenate([state_all[k][off_all[c]:off_all[c + 1]] for c in mine])
             for k in nb.FIELDS}
    dt = 1.0 / 512
    inter = float((sizes_all.astype(np.float64) ** 2).sum())
    variant = a.variant if a.precision == "mixed" and a.variant in (3, 4, 5) else 0
    ens = nb.Ensemble(sizes, eps2, dt, precision=a.precision, tune=True, pair_variant=variant)
    ens.set_state(state)
    ens.force_calculation()
    T0, U0 = ens.energy()
    stream = torch.cuda.ExternalStream(ens.stream, device=f"cuda:{dev}")
    ens.timestepping(warmup)
    ens.synchronize()
    reorders0 = ens.info()["reorders"]
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream), ClockSampler(dev) as clk:
        for k in range(steps):
            ev[k][0].record(stream)
            ens.timestepping(1)
            ev[k][1].record(stream)
        ens.synchronize()
    ms = float(np.mean([s.elapsed_time(t) for s, t in ev]))
    info = ens.info()
    launches = info["step_kernels"] * steps + info["order_kernels"] * (info["reorders"] - reorders0)
    de_run = None
    if time_units > 0:
        nsteps = int(round(time_units / dt)) - warmup - steps
        ens.timestepping(max(nsteps, 0))
        ens.synchronize()
        T1, U1 = ens.energy()
        de = np.abs((T1 + U1) - (T0 + U0)) / np.abs(T0 + U0)
        de_run = {"time_units": time_units, "median": float(np.median(de)), "max": float(de.max())}
    ens.close()
    # baseline: every cluster its own single-system engine (own stream, its
    # own captured step graph), all clusters issued per step, then one sync
    engines = []
    off = np.concatenate([[0], np.cumsum(sizes)])
    for c, n in enumerate(sizes):
        # the single-system engines use their fastest kernel at these sizes
        # (256-8192 bodies): packed hi/lo for mixed (measured 163 vs 123 Gint/s
        # serial for tile-relative engines, whose record building is a larger
        # share of a small system's step)
        e = nb.Engine(int(n), eps2=float(eps2[c]), precision=a.precision, dt=dt,
                      pair_variant=3 if a.precision == "mixed" else 0)
        e.set_state({k: state[k][off[c]:off[c + 1]] for k in nb.FIELDS})
        e.force_calculation()
        e.timestepping(1)
        engines.append(e)
    for e in engines:
        e.synchronize()
    # serialized: one cluster at a time; its step's device time from the
    # event nodes inside its graph (predict + pair + correct)
    serial_ms = 0.0
    for e in engines:
        e.timestepping(1)
        t = e.timers()
        serial_ms += t["pred_ms"] + t["eval_ms"] + t["corr_ms"]
    base_steps = max(3, min(steps, 10))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(base_steps):
        for e in engines:
            e.timestepping(1)
    for e in engines:
        e.synchronize()
    base_ms = (time.perf_counter() - t0) / base_steps * 1e3
    for e in engines:
        e.close()
    return {"ms": ms, "serial_ms": serial_ms, "base_ms": base_ms, "de_run": de_run, "info": info,
            "launches": int(launches), "inter": inter, "bodies": int(sizes_all.sum()),
            "clusters_here": int(len(sizes)), "clocks": clk.summary()}


def ensemble_summary(a, r):
    inter, ms, serial_ms, base_ms = r["inter"], r["ms"], r["serial_ms"], r["base_ms"]
    return {
        "workload": f"{a.clusters} Plummer clusters (seed 3), N log-uniform in [256, 8192], "
                    f"eps = 4/N, dt = 1/512, {a.precision}",
        "bodies": r["bodies"], "interactions_per_step": inter,
        "value": inter / (ms * 1e-3) / 1e9, "unit": "Gint/s", "ms_per_step": ms,
        "kernel": {k: r["info"][k] for k in ("items", "tiles_per_item", "j_tile", "threads", "grid",
                                             "padded_rows", "record_format")},
        "launch_per_cluster_serial": {
            "ms_per_step": serial_ms, "value": inter / (serial_ms * 1e-3) / 1e9,
            "how": "one single-system engine per cluster stepped one at a time; sum of each "
                   "cluster's step device time (CUDA events in its graph)"},
        "launch_per_cluster_concurrent": {
            "ms_per_step": base_ms, "value": inter / (base_ms * 1e-3) / 1e9,
            "how": f"one single-system engine per cluster, all {r['clusters_here']} of a GPU stepping "
                   "their graphs on their own streams at once; wall clock per step"},
        "speedup_vs_launch_per_cluster_serial": serial_ms / ms,
        "speedup_vs_launch_per_cluster_concurrent": base_ms / ms,
        "energy_error": r["de_run"],
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }


def main_ensemble(a):
    """Batched ensemble: one persistent launch per step vs one launch per
    cluster.  Under torchrun the clusters are sharded over the GPUs (one
    ensemble per rank, no communication but the timing reduction)."""
    import torch
    world, rank, local = dist_setup()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    dev = local
    torch.cuda.set_device(dev)
    r = run_ensemble(a, torch, world, rank, dist, dev, a.steps, a.warmup, a.time_units)
    # the slowest rank sets every time (same reductions, same order, on all ranks)
    mx = max_over_ranks_fn(world, dist, f"cuda:{dev}")
    r["ms"], r["serial_ms"], r["base_ms"] = mx(r["ms"]), mx(r["serial_ms"]), mx(r["base_ms"])
    if r["de_run"] is not None:
        r["de_run"]["max"] = mx(r["de_run"]["max"])
    if world > 1:
        dist.barrier()
        if rank != 0:
            dist.destroy_process_group()
            return 0
    s = ensemble_summary(a, r)
    line = {
        "metric": "Gpair-interactions/s, batched ensemble (one persistent launch per step)",
        "value": s["value"], "unit": "Gint/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": s["ms_per_step"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64" if a.precision == "mixed" else "f64",
        "data": "synthetic (seeded Plummer clusters, Henon units)",
        "config": {"workload": s["workload"], "bodies": s["bodies"],
                   "interactions_per_step": s["interactions_per_step"],
                   "parallelism": f"clusters sharded over {world} GPUs" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (no flush)"},
        **{k: s[k] for k in ("launch_per_cluster_serial", "launch_per_cluster_concurrent",
                             "speedup_vs_launch_per_cluster_serial",
                             "speedup_vs_launch_per_cluster_concurrent", "energy_error", "clocks",
                             "gpu_launches")},
        "ensemble": s["kernel"],
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main_adjoint(a):
    """Checkpointed adjoint: time of the forward run and of the backward
    sweep (segment recompute + reverse steps) on the torch stream."""
    import torch
    import nbody_b200 as nb
    n, eps2, dt, nsteps, k = 4096, 1e-4, 1.0 / 256, 256, 16
    s = nb.plummer(n, 4)
    rng = np.random.default_rng(4)
    sel = torch.tensor(np.sort(rng.choice(n, 64, replace=False)), device="cuda")
    X = torch.tensor(np.stack([s["x"], s["y"], s["z"]]), dtype=torch.float64, device="cuda")
    V = torch.tensor(np.stack([s["vx"], s["vy"], s["vz"]]), dtype=torch.float64, device="cuda")
    m = torch.tensor(s["m"], dtype=torch.float64, device="cuda")
    out = {"metric": "checkpointed adjoint of a fixed-dt Hermite-4 run (gradients w.r.t. x0, v0, m)",
           "config": {"workload": "Plummer N=4096 seed 4, eps=1e-2, dt=1/256, 256 steps, checkpoint 16, "
                                  "loss = sum |x_final - target|^2 over 64 seeded bodies"},
           "unit": "ms", "higher_is_better": False}
    for prec in ("fp64", "mixed"):
        adj = nb.Adjoint(n, eps2, dt, nsteps, k, precision=prec)
        fw, bw = [], []
        for rep in range(a.warmup + a.steps):
            x0 = X.clone().requires_grad_()
            v0 = V.clone().requires_grad_()
            mm = m.clone().requires_grad_()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            x1, v1 = nb.hermite_rollout(x0, v0, mm, eps2, dt, nsteps, k, prec, adjoint=adj)
            e1.record()
            target = x1.detach()[:, sel] + 1e-3
            ((x1[:, sel] - target) ** 2).sum().backward()
            e2.record()
            torch.cuda.synchronize()
            if rep >= a.warmup:
                fw.append(e0.elapsed_time(e1))
                bw.append(e1.elapsed_time(e2))
        adj.close()
        inter = float(n) * n * (nsteps + 1)
        out[prec] = {"forward_ms": float(np.mean(fw)), "backward_ms": float(np.mean(bw)),
                     "forward_Gint_s": inter / (np.mean(fw) * 1e-3) / 1e9}
    out["value"] = out["fp64"]["forward_ms"] + out["fp64"]["backward_ms"]
    print(json.dumps(out), flush=True)
    return 0


def section(name, fn, *args):
    """An extra section of the N = 1 line: its result, or the error that
    stopped it (the headline line is printed either way)."""
    t0 = time.perf_counter()
    try:
        r = fn(*args)
    except Exception as exc:  # noqa: BLE001 - reported in the line, not fatal
        traceback.print_exc()
        r = {"error": f"{type(exc).__name__}: {exc}"}
    if isinstance(r, dict):
        r["section_seconds"] = time.perf_counter() - t0
    print(f"[bench] {name}: {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
    return r


def tuning_block(w, state, torch, dev, tuned):
    """The heuristic tiling (wave model) timed beside the autotuner's."""
    out = {}
    for prec in ("mixed", "fp64"):
        h = run_arm(w, prec, state, torch, None, 1, dev, 10, 3, tune=False)
        t = tuned.get(prec)
        out[prec] = {"autotuned": {"tiling": t["tiling"], "pair_ms": t["pair_ms"],
                                   "source": t["tiling_source"]} if t else None,
                     "heuristic": {"tiling": h["tiling"], "pair_ms": h["pair_ms"]}}
        if t:
            out[prec]["heuristic_over_autotuned"] = h["pair_ms"] / t["pair_ms"]
    return out


def large_n_block(a, peaks, torch, dev):
    """N = 262144 Plummer (seed 2, eps = 4e-3, dt = 1/2048): the mixed path
    (automatic kernel, and the hi/lo kernel) against FP64 over timed steps;
    acc error at t = 0; |dE/E| of the mixed and FP64 runs at one time unit."""
    import nbody_b200 as nb
    w = LARGE_N
    state = nb.plummer(w.n, w.seed)
    tu = a.large_n_time_units
    arms = {"mixed": run_arm(w, "mixed", state, torch, None, 1, dev, 10, 3, time_units=tu),
            "fp64": run_arm(w, "fp64", state, torch, None, 1, dev, 10, 3, time_units=tu),
            "mixed_hilo": run_arm(w, "mixed", state, torch, None, 1, dev, 10, 3, variant=3)}
    inter = float(w.n) * w.n
    out = {"workload": w.name("mixed vs FP64"), "n": w.n, "timed_steps": 10}
    for k, arm in arms.items():
        prec = "fp64" if k == "fp64" else "mixed"
        out[k] = {"value": inter / (arm["ms_per_step"] * 1e-3) / 1e9, "unit": "Gint/s",
                  "ms_per_step": arm["ms_per_step"], "steps_per_s": 1e3 / arm["ms_per_step"],
                  "pair_ms": arm["pair_ms"],
                  "kernel": KERNEL_NAMES[arm["record_format"]], "tiling": arm["tiling"],
                  "tiling_source": arm["tiling_source"], "roofline": roofline(peaks, w, arm, prec),
                  "clocks": arm["clocks"]}
        if k != "mixed_hilo" and tu > 0:
            out[k]["dE_over_E"] = arm["dE_over_E"]
            out[k]["t_end"] = arm["t_end"]
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed_hilo_over_fp64"] = out["mixed_hilo"]["value"] / out["fp64"]["value"]
    if tu > 0:
        out["energy_error_ratio_mixed_over_fp64"] = out["mixed"]["dE_over_E"] / out["fp64"]["dE_over_E"]
    out["accuracy_t0"] = accuracy_block(w, state, dev, sample_rows=256)
    return out


def main():
    a = parse()
    if a.impl == "reference":
        return main_reference(a)
    if a.ensemble:
        return main_ensemble(a)
    if a.adjoint:
        return main_adjoint(a)
    import torch
    world, rank, local = dist_setup()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    dev = local
    torch.cuda.set_device(dev)
    import nbody_b200 as nb
    w = Workload(a.n, a.seed, a.eps, a.dt)
    state = nb.plummer(w.n, w.seed)
    tune = not a.heuristic
    if a.kernels_only:
        arm = run_arm(w, a.precision, state, torch, dist, world, dev, a.steps, a.warmup, a.variant, tune)
        if rank == 0:
            print(json.dumps({"kernels_only": True, "precision": a.precision, "n": w.n, **arm}))
        if world > 1:
            dist.destroy_process_group()
        return 0
    peaks = nb.measure_peaks(dev)
    # the energy runs go on to one time unit at N = 1 only (replica runs stay short)
    tu = a.time_units if world == 1 else 0.0
    main_arm = run_arm(w, a.precision, state, torch, dist, world, dev, a.steps, a.warmup, a.variant,
                       tune, time_units=tu)
    other = None
    other_prec = "fp64" if a.precision == "mixed" else "mixed"
    if not a.no_fp64_arm:
        other = run_arm(w, other_prec, state, torch, dist, world, dev, a.steps, a.warmup, a.variant,
                        tune, time_units=tu)

    max_over_ranks = max_over_ranks_fn(world, dist, f"cuda:{dev}")
    # every cross-rank reduction happens here, on all ranks, before the
    # non-zero ranks leave
    arms_over_ranks(max_over_ranks, main_arm, other)
    ms, pair_ms = main_arm["ms_per_step"], main_arm["pair_ms"]
    if world > 1:
        dist.barrier()
    e2e = e2e_over_ranks(max_over_ranks, world, w.n,
                         run_e2e(w, a.precision, state, torch, max(3, min(a.steps, 20))))
    if world > 1:
        dist.barrier()
    if rank != 0:
        dist.destroy_process_group()
        return 0
    cpu = None
    extras = {}
    if world == 1:
        if not a.no_cpu_baseline:
            cpu = section("cpu_baseline", cpu_baseline, a, w)
        if not a.no_extras:
            extras["accuracy_t0"] = section("accuracy_t0", accuracy_block, w, state, dev)
            tuned = {a.precision: main_arm, **({other_prec: other} if other else {})}
            extras["tuning"] = section("tuning", tuning_block, w, state, torch, dev, tuned)
            extras["large_n"] = section("large_n", large_n_block, a, peaks, torch, dev)
            extras["ensemble"] = section(
                "ensemble", lambda: ensemble_summary(a, run_ensemble(a, torch, 1, 0, None, dev, 10, 3, 1.0)))
    inter = float(w.n) * w.n
    value = replica_value(world, inter, ms)
    main_arm["pair_ms"] = pair_ms
    variant_used = {3: 4, 2: 3, 1: 1, 0: 0}[main_arm["record_format"]]
    if variant_used == 4 and a.variant == 5:
        variant_used = 5
    line = {
        "metric": METRIC, "value": value, "unit": "Gint/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "steps_per_s": 1e3 / ms, "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
        "data": "synthetic (seeded Plummer sphere, Henon units)",
        "config": {"workload": w.name(a.precision), "n": w.n, "eps": w.eps, "dt": w.dt,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MiB write, untimed)",
                   "mixed_kernel": VARIANT_NAMES.get(variant_used, "FP64") if a.precision == "mixed"
                   else "FP64",
                   "tiling": main_arm["tiling_source"]},
        "roofline": roofline(peaks, w, main_arm, a.precision),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": main_arm["launches"],
        "clocks": main_arm["clocks"],
        "phases_ms": {"pred": main_arm["pred_ms"], "eval": main_arm["pair_ms"], "corr": main_arm["corr_ms"]},
        "tiling": main_arm["tiling"],
        "energy_error": {a.precision: main_arm["dE_over_E"], "t_end": main_arm["t_end"]},
        "peaks_measured": peaks,
    }
    if other is not None:
        ov = replica_value(world, inter, other["ms_per_step"])
        line[other_prec] = {"value": ov, "ms_per_step": other["ms_per_step"],
                            "steps_per_s": 1e3 / other["ms_per_step"], "pair_ms": other["pair_ms"],
                            "roofline": roofline(peaks, w, other, other_prec), "tiling": other["tiling"],
                            "tiling_source": other["tiling_source"], "clocks": other["clocks"]}
        line["energy_error"][other_prec] = other["dE_over_E"]
        line["mixed_over_fp64"] = (value / ov) if a.precision == "mixed" else (ov / value)
    line.update(extras)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
