"""Benchmark: G pair-interactions/s of the Hermite-4 step on one B200.

Workload (default): Plummer sphere N = 65536 (Henon units, seed 1), softening
eps = 1e-2, shared fixed dt = 1/1024; one step = predict + acc/jerk of all N^2
pairs + correct, replayed from the engine's captured CUDA graph.  The headline
`value` is the mixed-precision path (FP32 pair loop on hi/lo positions, FP64
accumulation and integration); the plain FP64 path runs on the same input
and is reported beside it with both runs' |dE/E|.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own FP64 CPU code (compiled from its
sources into oracle/_ref) on this host's cores: each step is one fixed-dt
Hermite step whose force evaluation computes the share of i-rows that rank 0
of an S-rank job owns (the reference's own decomposition, src/kernel.cpp:1185),
with S sized to bound the run; the full-step time is S x that force time plus
the unsampled O(N) phases.

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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "n-body-code_b200"))

METRIC = "Gpair-interactions/s at N=65536: mixed-prec vs FP64 GPU, equal energy error"
FLOP_PER_INTERACTION = 60
L2_FLUSH_BYTES = 256 << 20


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
    ap.add_argument("--tune", action="store_true", help="autotune pair-kernel tiling first")
    ap.add_argument("--variant", type=int, default=0,
                    help="mixed pair kernel (nbody_config.pair_variant): 0 = automatic (tile-relative "
                         "from 8192 bodies), 1 = scalar hi/lo, 2/3 = packed hi/lo, 4 = tile-relative; "
                         "ensembles: 3 = packed hi/lo, else tile-relative")
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
    ap.add_argument("--time-units", type=float, default=0.0,
                    help="also integrate this many N-body time units (untimed) and report |dE/E|")
    ap.add_argument("--accuracy", action="store_true",
                    help="report the mixed path's per-body acc/jerk error against FP64 at t = 0")
    return ap.parse_args()


def workload_name(a, precision):
    return (f"Hermite-4 shared fixed step, Plummer N={a.n} seed {a.seed} (Henon units), "
            f"eps={a.eps:g}, dt=1/{round(1 / a.dt)}, {precision}")


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


def run_arm(a, precision, state, torch, dist, rank, world, dev):
    import nbody_b200 as nb
    n = a.n
    clk = ClockSampler(dev).__enter__()  # sampling starts before the warm-up so the timed region is covered
    e = nb.Engine(n, eps2=a.eps ** 2, precision=precision, device=dev, dt=a.dt, tune=a.tune,
                  pair_variant=a.variant if precision == "mixed" else 0)
    e.set_state(state)
    e.force_calculation()
    T0, U0 = e.energy()
    stream = torch.cuda.ExternalStream(e.stream, device=f"cuda:{dev}")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{dev}")
    e.timestepping(a.warmup)
    e.synchronize()
    reorders0 = e.timers()["reorders"]
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    pair_ms, pred_ms, corr_ms = [], [], []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        for k in range(a.steps):
            flush.zero_()                       # evict L2 between timed steps
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
    tm = e.timers()
    # kernels of the timed steps: the captured step graph each step, plus the
    # captured Morton re-ordering where one ran (tile-relative kernel)
    launches = tm["step_kernels"] * a.steps + tm["order_kernels"] * (tm["reorders"] - reorders0)
    if a.time_units > 0:  # carry on (untimed) to the requested model time
        rest = int(round(a.time_units / a.dt)) - a.warmup - a.steps
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
        "tiling": {k: tm[k] for k in ("threads", "i_per_thread", "j_tile", "split_j")},
        "clocks": clk.summary(),
        "launches": int(launches),
        "record_format": tm["record_format"],
    }


def run_e2e(a, precision, state, torch, steps):
    """End to end through the drop-in C-ABI call (the reference's
    force_calculation contract): pinned host arrays in, host arrays out,
    host<->device copies inside every timed call."""
    import nbody_b200 as nb
    n = a.n
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
        _lib.check(L.nbody_force_calculation(n, a.eps ** 2, prec, 0, n, *ptrs, *outs),
                   "nbody_force_calculation")

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
            "what": "nbody_force_calculation (drop-in for force_calculation), pinned host buffers"}


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


def cpu_reference_steps(a, state, nsteps, seconds_per_step):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n = a.n
    if not O.have_reference():
        return None
    lib = O.ref()
    cores = lib.ref_max_threads()
    arrs = [np.ascontiguousarray(state[k]) for k in ("x", "y", "z", "m", "vx", "vy", "vz")]
    P = O._p
    # calibrate the sample: one step with a small share, then size S
    s_cal = 4096
    h = lib.ref_bench_create(n, a.dt, s_cal, *map(P, arrs))
    t3 = np.zeros(3)
    lib.ref_bench_step(h, P(t3))
    lib.ref_bench_destroy(h)
    full_force = max(t3[1] * s_cal, 1e-6)
    S = int(min(4096, max(1, round(full_force / seconds_per_step))))
    h = lib.ref_bench_create(n, a.dt, S, *map(P, arrs))
    steps = []
    for _ in range(nsteps):
        lib.ref_bench_step(h, P(t3))
        steps.append(t3.copy())
    lib.ref_bench_destroy(h)
    st = np.array(steps)
    step_s = st[:, 0] + S * st[:, 1] + st[:, 2]
    return {"per_step_s": step_s, "force_sample_s": st[:, 1], "S": S, "cores": cores,
            "kind": "reference",
            "sample": (f"reference FP64 CPU build (oracle/_ref), N={n}: each step = prediction + "
                       f"force_calculation on rank 0's 1/{S} share of i-rows (src/kernel.cpp:1185) "
                       f"+ snapandcrackle + correction; full step = pred + {S} x force + corr")}


def cpu_port_steps(a, state, nsteps, seconds_per_step):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n = a.n
    rows_per_s = 2e8 / n  # rough single-thread rate of the direct row sum
    nrows = int(max(8, min(n, rows_per_s * seconds_per_step)))
    rows = np.linspace(0, n - 1, nrows).astype(np.int32)
    ts = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        O.force_rows(state, a.eps ** 2, rows)
        ts.append(time.perf_counter() - t0)
    per = np.array(ts) * (n / nrows)
    return {"per_step_s": per, "S": n / nrows, "cores": 1, "kind": "port",
            "sample": f"oracle direct row sums on {nrows} of {n} rows per step, scaled by N/rows"}


def cpu_baseline(a, state):
    r = cpu_call(cpu_reference_steps, a, state, 3, a.cpu_sample_seconds / 3) or \
        cpu_call(cpu_port_steps, a, state, 3, a.cpu_sample_seconds / 3)
    v = a.n * a.n / float(np.mean(r["per_step_s"])) / 1e9
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
    import nbody_b200 as nb  # host-only: the Plummer generator
    state = nb.plummer(a.n, a.seed)
    total = a.steps + a.warmup
    per_step_budget = min(2.0, max(0.2, 150.0 / max(total, 1)))
    r = cpu_call(cpu_reference_steps, a, state, total, per_step_budget)
    if r is None:
        r = cpu_call(cpu_port_steps, a, state, total, per_step_budget)
    timed = r["per_step_s"][a.warmup:]
    s = float(np.mean(timed))
    v = a.n * a.n / s / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gint/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Plummer sphere)",
        "config": {"workload": workload_name(a, "FP64 CPU (reference)"), "n": a.n,
                   "l2": "n/a (CPU)"},
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


def main_ensemble(a):
    """Batched ensemble: one persistent launch per step vs one launch per
    cluster.  Under torchrun the clusters are sharded over the GPUs (one
    ensemble per rank, no communication but the timing reduction)."""
    import torch
    import nbody_b200 as nb
    world, rank, local = dist_setup()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    dev = local
    torch.cuda.set_device(dev)
    sizes_all, eps2_all, state_all = nb.plummer_ensemble(a.clusters, 3)
    mine = shard_clusters(sizes_all, world, rank)
    off_all = np.concatenate([[0], np.cumsum(sizes_all)])
    sizes, eps2 = sizes_all[mine], eps2_all[mine]
    state = {k: np.concatenate([state_all[k][off_all[c]:off_all[c + 1]] for c in mine])
             for k in nb.FIELDS}
    dt = 1.0 / 512
    inter = float((sizes_all.astype(np.float64) ** 2).sum())
    variant = 3 if a.precision == "mixed" and a.variant in (1, 2, 3) else 0
    ens = nb.Ensemble(sizes, eps2, dt, precision=a.precision, tune=True, pair_variant=variant)
    ens.set_state(state)
    ens.force_calculation()
    T0, U0 = ens.energy()
    stream = torch.cuda.ExternalStream(ens.stream, device=f"cuda:{dev}")
    ens.timestepping(a.warmup)
    ens.synchronize()
    reorders0 = ens.info()["reorders"]
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    with torch.cuda.stream(stream), ClockSampler(dev) as clk:
        for k in range(a.steps):
            ev[k][0].record(stream)
            ens.timestepping(1)
            ev[k][1].record(stream)
        ens.synchronize()
    ms = float(np.mean([s.elapsed_time(t) for s, t in ev]))
    info = ens.info()
    launches = info["step_kernels"] * a.steps + info["order_kernels"] * (info["reorders"] - reorders0)
    de_run = None
    if a.time_units > 0:
        nsteps = int(round(a.time_units / dt)) - a.warmup - a.steps
        ens.timestepping(max(nsteps, 0))
        ens.synchronize()
        T1, U1 = ens.energy()
        de = np.abs((T1 + U1) - (T0 + U0)) / np.abs(T0 + U0)
        de_run = {"time_units": a.time_units, "median": float(np.median(de)), "max": float(de.max())}
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
    base_steps = max(3, min(a.steps, 10))
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
    # the slowest rank sets every time (same reductions, same order, on all ranks)
    mx = max_over_ranks_fn(world, dist, f"cuda:{dev}")
    ms, serial_ms, base_ms = mx(ms), mx(serial_ms), mx(base_ms)
    if de_run is not None:
        de_run["max"] = mx(de_run["max"])
    if world > 1:
        dist.barrier()
        if rank != 0:
            dist.destroy_process_group()
            return 0
    line = {
        "metric": "Gpair-interactions/s, batched ensemble (one persistent launch per step)",
        "value": inter / (ms * 1e-3) / 1e9, "unit": "Gint/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
        "data": "synthetic (seeded Plummer clusters, Henon units)",
        "config": {"workload": f"{a.clusters} Plummer clusters (seed 3), N log-uniform in [256, 8192], "
                               f"eps = 4/N, dt = 1/512, {a.precision}",
                   "bodies": int(sizes_all.sum()), "interactions_per_step": inter,
                   "parallelism": f"clusters sharded over {world} GPUs" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (no flush)"},
        "ensemble": {k: info[k] for k in ("items", "tiles_per_item", "j_tile", "threads", "grid", "padded_rows",
                                          "record_format")},
        "launch_per_cluster_serial": {
            "ms_per_step": serial_ms, "value": inter / (serial_ms * 1e-3) / 1e9,
            "how": "one single-system engine per cluster stepped one at a time; sum of each "
                   "cluster's step device time (CUDA events in its graph)"},
        "launch_per_cluster_concurrent": {
            "ms_per_step": base_ms, "value": inter / (base_ms * 1e-3) / 1e9,
            "how": f"one single-system engine per cluster, all {len(sizes)} of a GPU stepping their "
                   "graphs on their own streams at once; wall clock per step"},
        "speedup_vs_launch_per_cluster_serial": serial_ms / ms,
        "speedup_vs_launch_per_cluster_concurrent": base_ms / ms,
        "energy_error": de_run,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
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
    state = nb.plummer(a.n, a.seed)
    if a.kernels_only:
        arm = run_arm(a, a.precision, state, torch, dist, rank, world, dev)
        if rank == 0:
            print(json.dumps({"kernels_only": True, "precision": a.precision, "n": a.n, **arm}))
        if world > 1:
            dist.destroy_process_group()
        return 0
    peaks = nb.measure_peaks(dev)
    main_arm = run_arm(a, a.precision, state, torch, dist, rank, world, dev)
    other = None
    other_prec = "fp64" if a.precision == "mixed" else "mixed"
    if not a.no_fp64_arm:
        other = run_arm(a, other_prec, state, torch, dist, rank, world, dev)

    max_over_ranks = max_over_ranks_fn(world, dist, f"cuda:{dev}")

    accuracy = None
    if a.accuracy and rank == 0:
        d = {}
        for prec in ("fp64", "mixed"):
            with nb.Engine(a.n, eps2=a.eps ** 2, precision=prec, device=dev, dt=a.dt,
                           pair_variant=a.variant if prec == "mixed" else 0) as e:
                e.set_state(state)
                e.force_calculation()
                d[prec] = e.get_derivs()

        def rel(blk):
            num = np.sqrt(((d["mixed"][blk] - d["fp64"][blk]) ** 2).sum(0))
            return num / np.sqrt((d["fp64"][blk] ** 2).sum(0))
        ea, ej = rel(slice(0, 3)), rel(slice(3, 6))
        accuracy = {"acc_rel_err_vs_fp64": {"median": float(np.median(ea)), "p99": float(np.quantile(ea, 0.99)),
                                            "max": float(ea.max())},
                    "jerk_rel_err_vs_fp64": {"median": float(np.median(ej)), "p99": float(np.quantile(ej, 0.99)),
                                             "max": float(ej.max())}}
    # every cross-rank reduction happens here, on all ranks, before the
    # non-zero ranks leave
    arms_over_ranks(max_over_ranks, main_arm, other)
    ms, pair_ms = main_arm["ms_per_step"], main_arm["pair_ms"]
    if world > 1:
        dist.barrier()
    e2e = e2e_over_ranks(max_over_ranks, world, a.n,
                         run_e2e(a, a.precision, state, torch, max(3, min(a.steps, 20))))
    cpu = cpu_baseline(a, state) if (rank == 0 and world == 1 and not a.no_cpu_baseline) else None
    if world > 1:
        dist.barrier()
    if rank != 0:
        dist.destroy_process_group()
        return 0
    inter = float(a.n) * a.n
    value = replica_value(world, inter, ms)

    kernel_names = {0: "pair_fp64_kernel", 1: "pair_mixed_kernel", 2: "pair_mixed_x2_kernel",
                    3: "pair_mixed_rel_kernel"}

    def roofline(arm, prec):
        peak = peaks["fp32_tflops"] if prec == "mixed" else peaks["fp64_tflops"]
        achieved = FLOP_PER_INTERACTION * inter / (arm["pair_ms"] * 1e-3) / 1e12
        return {"bound": "fp32" if prec == "mixed" else "fp64", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic_per_launch(kernel_names[arm["record_format"]]),
                "kernel": kernel_names[arm["record_format"]],
                "peak_source": "measured live by nbody_measure_peaks (FMA microkernel, this GPU)",
                "flop_per_interaction": FLOP_PER_INTERACTION}

    main_arm["pair_ms"] = pair_ms
    line = {
        "metric": METRIC, "value": value, "unit": "Gint/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
        "data": "synthetic (seeded Plummer sphere, Henon units)",
        "config": {"workload": workload_name(a, a.precision), "n": a.n, "eps": a.eps, "dt": a.dt,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": f"flushed between timed steps ({L2_FLUSH_BYTES >> 20} MiB write, untimed)"},
        "roofline": roofline(main_arm, a.precision),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": main_arm["launches"],
        "clocks": main_arm["clocks"],
        "phases_ms": {"pred": main_arm["pred_ms"], "eval": main_arm["pair_ms"], "corr": main_arm["corr_ms"]},
        "tiling": main_arm["tiling"],
        "energy_error": {a.precision: main_arm["dE_over_E"], "t_end": main_arm["t_end"]},
        "accuracy_t0": accuracy,
        "peaks_measured": peaks,
    }
    if other is not None:
        ov = replica_value(world, inter, other["ms_per_step"])
        line[other_prec] = {"value": ov, "ms_per_step": other["ms_per_step"], "pair_ms": other["pair_ms"],
                            "roofline": roofline(other, other_prec), "tiling": other["tiling"],
                            "clocks": other["clocks"]}
        line["energy_error"][other_prec] = other["dE_over_E"]
        line["mixed_over_fp64"] = (value / ov) if a.precision == "mixed" else (ov / value)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
