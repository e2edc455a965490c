#!/usr/bin/env python
"""Benchmark of the all-pairs softened gravity path on B200.

Workload (the single-large-system configuration): Plummer sphere, N = 262144,
seed 2, eps = 1e-3, KDK leapfrog dt = 5e-4, FP32-compensated pair arithmetic.
A "step" is one leapfrog step = one force evaluation (N(N-1) ordered pairs)
plus the fused kick/drift.  Metric: GPairs/s = pairs evaluated / device time.

Output: ONE JSON line on stdout (rank 0).  Keys beyond the base contract:
  roofline      the force kernel against the FP32 FMA-pipe roofline
                (16 FMA-pipe operations per pair, 128 FP32 lanes per SM);
  cpu_baseline  the reference's own CPU kernel on this host's cores;
  fp64          the plain FP64 kernel's GPairs/s in the same run (the FP32C /
                FP64 ratio), and the FP64 default's (fp64.default: the
                Newton-3 FP64 kernel at this size);
  accuracy      FP32C vs FP64 per-particle force error and energy drift;
  e2e           the same metric through the C ABI with host buffers
                (upload, one step, download per step);
  clocks        nvidia-smi samples taken during the timed region.

--impl reference times the reference's CPU implementation instead (rank 0).
--gpus N (under torchrun) shards the receivers of the one system over N GPUs
with an NCCL all-gather of positions per step (--shard takes that path on
one GPU too).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "n-body-ring-solver_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

METRIC = "GPairs/s FP32-compensated vs FP64 on 1 B200 at median force rel err <=1e-6"
UNIT = "GPairs/s"
# SM count of the device (set in run_ours / run_sharded from the device
# properties; 148 on B200).
SMS = 148
FMA_OPS_PER_PAIR = 16
# The Newton-3 kernel evaluates each unordered pair once: the 16 operations of
# the pair plus 5 for the reaction (receiver-mass correction, its product, 3
# accumulations), i.e. 10.5 per ordered pair of the N(N-1) the metric counts.
REACTION_OPS = 5
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "force_fp32c_plummer262144.json")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=262144)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--eps", type=float, default=1e-3)
    p.add_argument("--dt", type=float, default=5e-4)
    p.add_argument("--precision", choices=["fp32c", "fp64"], default="fp32c")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-accuracy", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the N=2048 (100 KDK steps) and N=1048576 (5 steps) lines")
    p.add_argument("--no-config-accuracy", action="store_true",
                   help="skip the cold-collapse and two-component accuracy runs")
    p.add_argument("--shard", action="store_true",
                   help="use the multi-GPU i-partition path even on one GPU (process group of 1)")
    return p.parse_args()


def workload_config(a, extra=None):
    cfg = {"workload": f"plummer_n{a.n}_seed{a.seed}_eps{a.eps:g}_kdk_dt{a.dt:g}",
           "n": a.n, "ic": "plummer", "seed": a.seed, "eps": a.eps, "dt": a.dt,
           "scheme": "kdk", "pairs_per_step": a.n * (a.n - 1),
           "l2": f"flushed between timed steps (256 MiB write); j-stream {48 * a.n / 1e6:.1f} MB "
                 "is L2-resident within a step"}
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [t.strip() for t in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [v for v in sm if v >= 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


# ------------------------------------------------------------ CPU baseline --
# The reference's CPU solver (oracle/_ref, compiled from its sources) is timed
# in two legs, both on this host's cores with every OpenMP thread, FP64,
# unsoftened (the reference has no softening; the pair count is the same):
#   * force only: its fastest kernel (AVX-512 rsqrt 4i; AVX2 blocked without
#     AVX-512), on rank 0's share of its own ring decomposition
#     (hybrid_ring_solver) of one force evaluation -- the counterpart of our
#     force kernel;
#   * end to end: reduced_solver_omp_lf (CPU/omp_solver.cpp:257-456), the
#     solver behind main.cpp's -i lf: DKD leapfrog order 2 with the AVX2 blocked
#     kernel, whole steps of the whole system -- the counterpart of our C-ABI
#     step.  Throughput = steps x N(N-1) / seconds (the reference's own
#     effective-pair count, CPU/omp_solver.cpp:745-752).
# Inputs come from the oracle's samplers (bit-identical to the product's), so
# a process timing the reference never loads the product library.

def _reference():
    sys.path.insert(0, ORACLE)
    from oracle import Oracle, Reference, reference_available
    if not reference_available():
        return None, None
    ref = Reference()
    ref.set_threads(os.cpu_count() or 1)
    return ref, Oracle()


def _ref_kernel_name(ref):
    return "AVX512-RSQRT-4I" if ref.has_avx512 else "AVX2-blocked"


def ref_force_leg(ref, s, per_call_s, target_s, max_s, warmup=0, calls=None):
    """Force-only leg: the rank-0 share (1/comm_sz of one N-particle force
    evaluation) whose time is at most per_call_s, repeated until target_s
    (or exactly `calls` times)."""
    n = len(s["x"])
    comm = 1
    while comm < n and n % (comm * 2) == 0 and comm < 1024:
        comm *= 2
    t = ref.ring_share(s, comm)
    while comm > 1 and t * 2 <= per_call_s:
        comm //= 2
        t = ref.ring_share(s, comm)
    for _ in range(warmup):
        ref.ring_share(s, comm)
    secs = []
    while (calls is None and (sum(secs) < target_s and sum(secs) + t <= max_s or not secs)) or \
            (calls is not None and len(secs) < calls):
        secs.append(ref.ring_share(s, comm))
    total = sum(secs)
    value = len(secs) * n * (n - 1) / comm / total / 1e9
    kernel = _ref_kernel_name(ref)
    return {"value": value, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
            "seconds": total, "calls": len(secs), "comm_sz": comm, "kernel": kernel,
            "sample": f"{len(secs)} x rank-0 share (1/{comm}) of one N={n} force evaluation of the "
                      f"reference's {kernel} kernel (hybrid_ring_solver's ring decomposition), eps=0, "
                      f"FP64, {ref.threads()} OpenMP threads"}, secs


def ref_e2e_leg(ref, s, dt, target_s, max_steps):
    """End-to-end leg: reduced_solver_omp_lf (DKD order 2, AVX2 blocked FP64)
    on the whole system: one untimed step, then as many whole steps as fit in
    about target_s (at least one, at most max_steps) in one solver call."""
    n = len(s["x"])
    _, t1 = ref.lf(s, dt, 1, order=2)
    k = int(max(1, min(max_steps, target_s // max(t1, 1e-9))))
    _, secs = ref.lf(s, dt, k, order=2)
    return {"value": k * n * (n - 1) / secs / 1e9, "unit": UNIT, "cores": ref.threads(),
            "kind": "reference", "steps": k, "seconds": secs, "steps_per_s": k / secs,
            "ms_per_step": 1e3 * secs / k,
            "sample": f"{k} whole DKD steps (order 2, dt={dt:g}) of the N={n} system through the "
                      f"reference's reduced_solver_omp_lf (AVX2 blocked FP64 kernel, eps=0), "
                      f"{ref.threads()} OpenMP threads, after one untimed step"}


def ref_config0_leg(ref, orc, steps=100):
    """The small-system configuration on the reference's solver:
    reduced_solver_omp_lf on Plummer N = 2048 (seed 0), DKD order 2, dt 1e-3,
    100 steps (eps=0)."""
    s = orc.plummer(2048, 0)
    ref.lf(s, 1e-3, 5, order=2)
    _, secs = ref.lf(s, 1e-3, steps, order=2)
    return {"steps_per_s": steps / secs, "gpairs": steps * 2048 * 2047 / secs / 1e9,
            "seconds": secs, "cores": ref.threads(),
            "sample": f"{steps} DKD steps (order 2, dt=1e-3) of Plummer N=2048 seed 0 through "
                      f"reduced_solver_omp_lf (AVX2 blocked FP64, eps=0), {ref.threads()} threads"}


def cpu_reference_sample(n, seed, dt, target_s=10.0, max_s=30.0):
    """cpu_baseline of our line: both legs on a bounded sample (about 10 s
    each) plus the small-system configuration."""
    ref, orc = _reference()
    if ref is None:
        return None
    s = orc.plummer(n, seed)
    force, _ = ref_force_leg(ref, s, per_call_s=target_s, target_s=target_s, max_s=max_s)
    e2e = ref_e2e_leg(ref, s, dt, target_s=target_s, max_steps=50)
    out = dict(force)
    out["legs"] = {"force_only": force, "end_to_end": e2e, "config0": ref_config0_leg(ref, orc)}
    return out


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref, orc = _reference()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU solver (oracle/_ref) was not built here"}))
        return
    n = a.n
    s = orc.plummer(n, a.seed)
    # per-step budget so that warmup + steps end within about two minutes
    per_step = min(3.0, 120.0 / max(1, a.steps + a.warmup))
    force, secs = ref_force_leg(ref, s, per_call_s=per_step, target_s=0, max_s=0, warmup=a.warmup,
                                calls=a.steps)
    total = sum(secs)
    value = force["value"]
    e2e = ref_e2e_leg(ref, s, a.dt, target_s=20.0, max_steps=a.steps)
    cfg0 = ref_config0_leg(ref, orc)
    cpu = dict(force)
    cpu["sample"] = ("each step: " + force["sample"])
    cpu["legs"] = {"force_only": force, "end_to_end": e2e, "config0": cfg0}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * total / a.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(a),
            "reference_run": {"force_kernel": force["kernel"], "comm_sz": force["comm_sz"],
                              "eps": 0.0, "scheme_e2e": "dkd order 2",
                              "note": "the reference has no softening and no KDK scheme: it runs "
                                      "the same Plummer system unsoftened (same pair count, one "
                                      "add fewer per pair) with its own DKD leapfrog"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0, "steps_per_s": e2e["steps_per_s"],
                    "ms_per_step": e2e["ms_per_step"], "steps": e2e["steps"],
                    "solver": "reduced_solver_omp_lf (DKD order 2, AVX2 blocked FP64), whole steps"},
            "config0": cfg0}
    print(json.dumps(line))


# -------------------------------------------------------------------- ours --
def measured_hbm_gbs():
    """The measured copy bandwidth of this pool's B200s (MEASURED_PEAKS.json,
    written beside bench.py), else the recipe's earlier measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError, TypeError):
        return 6650.0, "fallback"


def profile_traffic():
    try:
        with open(PROFILE_SUMMARY) as f:
            return json.load(f).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def run_ours(a):
    import numpy as np
    import torch
    import nbr

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 or a.shard:
        return run_sharded(a, rank, world, local)
    torch.cuda.set_device(local)
    global SMS
    SMS = torch.cuda.get_device_properties(local).multi_processor_count
    prec = nbr.FP32C if a.precision == "fp32c" else nbr.FP64
    eps2 = a.eps * a.eps
    n = a.n
    pairs = float(n) * float(n - 1)
    s = nbr.plummer(n, a.seed)
    ctx = nbr.Context(local)
    ctx.upload(s)
    ext = torch.cuda.ExternalStream(ctx.stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")

    def l2_flush():
        flush.zero_()
        torch.cuda.synchronize()

    def time_kernel(p, launches):
        ctx.forces_device(p, eps2=eps2)  # pack + warm
        ctx.forces_device(p, eps2=eps2)
        ctx.synchronize()
        ts = []
        for _ in range(launches):
            l2_flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            ctx.forces_device(p, eps2=eps2)
            e1.record(ext)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        return ts

    # ---- kernel-level timing (roofline) for both precisions
    k32 = time_kernel(nbr.FP32C, 5)
    a32 = ctx.forces_download()
    # The plain FP64 kernel (every ordered pair), the one the FP32C / FP64
    # ratio is defined on, then the FP64 default for this size (the Newton-3
    # FP64 kernel from 16384 to 2^20 particles).
    ctx.set_force_config(nbr.FP64, 4, 4, 0)
    cfg64 = ctx.get_force_config(nbr.FP64, eps2)
    k64 = time_kernel(nbr.FP64, 3)
    a64 = ctx.forces_download()
    ctx.set_force_config(nbr.FP64, 0)
    cfg64d = ctx.get_force_config(nbr.FP64, eps2)
    k64n3 = time_kernel(nbr.FP64, 3)
    a64n3 = ctx.forces_download()
    num = np.linalg.norm(a32 - a64, axis=0)
    den = np.linalg.norm(a64, axis=0)
    rel = num / np.where(den > 0, den, 1.0)

    # ---- timed leapfrog steps
    ctx.upload(s)
    d0 = ctx.diagnostics(eps2=eps2)
    for _ in range(a.warmup):
        ctx.run(prec, nbr.KDK, 2, a.dt, 1, eps2=eps2)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    step_s, launches = [], 0
    torch.cuda.synchronize()
    t_wall0 = time.perf_counter()
    for _ in range(a.steps):
        l2_flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        st = ctx.run(prec, nbr.KDK, 2, a.dt, 1, eps2=eps2)
        e1.record(ext)
        e1.synchronize()
        step_s.append(e0.elapsed_time(e1) * 1e-3)
        launches += int(st["kernels"])
        assert st["force_evals"] == 1
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    d1 = ctx.diagnostics(eps2=eps2)
    t_total = sum(step_s)
    value = a.steps * pairs / t_total / 1e9

    # ---- energy drift of the same number of steps in FP64 (comparison)
    acc = {"fp32c_vs_fp64_force_median_rel_err": float(np.median(rel)),
           "fp32c_vs_fp64_force_max_rel_err": float(rel.max()),
           "energy_drift": abs(d1["E"] - d0["E"]) / abs(d0["E"]),
           "energy_drift_steps": a.warmup + a.steps}
    if not a.no_accuracy and prec == nbr.FP32C:
        ctx.upload(s)
        for _ in range(a.warmup + a.steps):
            ctx.run(nbr.FP64, nbr.KDK, 2, a.dt, 1, eps2=eps2)
        d64 = ctx.diagnostics(eps2=eps2)
        acc["energy_drift_fp64"] = abs(d64["E"] - d0["E"]) / abs(d0["E"])

    # ---- end to end through the C ABI with pinned host buffers
    host = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in nbr.KEYS}
    for k in nbr.KEYS:
        host[k][:] = s[k]
    e2e_s = []
    for i in range(a.warmup + a.steps):
        l2_flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        ctx.upload_raw(n, *[host[k] for k in nbr.KEYS])
        st = ctx.run(prec, nbr.DKD, 2, a.dt, 1, eps2=eps2)
        ctx.download_raw(*[host[k] for k in nbr.KEYS[:6]])
        e1.record(ext)
        e1.synchronize()
        if i >= a.warmup:
            e2e_s.append(e0.elapsed_time(e1) * 1e-3)
            launches += 0
    e2e_value = a.steps * pairs / sum(e2e_s) / 1e9

    # ---- roofline of the force kernel
    t_k = statistics.mean(k32)
    achieved = pairs / t_k / 1e9
    mhz = clk.get("sm_mhz") or 1965.0
    cfg = ctx.get_force_config(nbr.FP32C, eps2)
    newton3 = cfg[0] == 3
    ops = (FMA_OPS_PER_PAIR + REACTION_OPS) / 2 if newton3 else FMA_OPS_PER_PAIR
    peak = SMS * 128 * mhz * 1e6 / ops / 1e9
    roofline = {"bound": "fp32_fma_pipe", "achieved": achieved, "peak": peak, "unit": UNIT,
                "frac": achieved / peak, "traffic": profile_traffic(),
                "algorithmic_bytes": 96 * n,
                "kernel": ("k_force_n3_f32c + k_n3_reduce (Newton-3: each unordered pair evaluated once)"
                           if newton3 else f"k_force_f32c<{cfg[0]},{cfg[1]}> split {cfg[2]}"),
                "fma_ops_per_ordered_pair": ops,
                "traffic_note": "dram bytes per launch of the pair kernel from "
                                "profiles/force_fp32c_plummer262144.json",
                "peak_source": f"{SMS} SMs x 128 FP32 lanes x median SM clock sampled in the timed region "
                               f"/ {ops:g} FMA-pipe ops per ordered pair (MEASURED_PEAKS.json has no "
                               "FP32-pipe figure)",
                "frac_at_max_clock": achieved / (SMS * 128 * 1965e6 / ops / 1e9),
                "frac_of_16op_roofline": achieved / (SMS * 128 * mhz * 1e6 / FMA_OPS_PER_PAIR / 1e9),
                "kernel_ms": 1e3 * t_k, "mufu_peak": SMS * 16 * mhz * 1e6 / 1e9}
    traffic = roofline["traffic"]
    hbm_peak, hbm_src = measured_hbm_gbs()
    if traffic:
        # The HBM roofline for comparison: the kernel's DRAM bytes per launch
        # (ncu) over its live launch time, against the measured copy bandwidth.
        gbs = traffic / t_k / 1e9
        roofline["hbm_view"] = {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                                "frac": gbs / hbm_peak, "peak_source": hbm_src}
    fp64 = {"value": pairs / statistics.mean(k64) / 1e9, "unit": UNIT, "kernel_ms": 1e3 * statistics.mean(k64),
            "kernel": f"k_force_f64<{cfg64[0]},{cfg64[1]}> split {cfg64[2]} (the plain FP64 kernel: "
                      "every ordered pair)"}
    fp64["fp32c_over_fp64"] = achieved / fp64["value"]
    d64 = np.linalg.norm(a64n3 - a64, axis=0) / np.where(den > 0, den, 1.0)
    n3v = pairs / statistics.mean(k64n3) / 1e9
    fp64["default"] = {"value": n3v, "unit": UNIT, "kernel_ms": 1e3 * statistics.mean(k64n3),
                       "kernel": ("k_force_n3_f64 + k_n3_reduce (Newton-3: each unordered pair "
                                  "evaluated once)" if cfg64d[0] == 3 else
                                  f"config {cfg64d}"),
                       "over_plain": n3v / fp64["value"], "fp32c_over_fp64_default": achieved / n3v,
                       "max_rel_diff_vs_plain": float(d64.max())}

    config0 = None if a.no_configs else measure_config0(ctx, l2_flush, mhz)
    large = None if a.no_configs else measure_large(ctx, l2_flush, mhz)
    batched = None if a.no_batch else measure_batch(ctx, eps2, value)
    config_acc = None if a.no_config_accuracy else measure_config_accuracy(ctx)

    cpu = None
    if not a.no_cpu_baseline and rank == 0:
        try:
            cpu = cpu_reference_sample(n, a.seed, a.dt)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"error": str(ex)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * t_total / a.steps,
            "steps_per_s": a.steps / t_total, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec == nbr.FP32C else "f64",
            "precision": a.precision, "data": "synthetic", "config": workload_config(a),
            "gpu_launches": launches, "wall_s_timed": t_wall,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 7 * 8 * n,
                    "d2h_bytes_per_step": 6 * 8 * n, "scheme": "dkd order 2 (reduced_solver_omp_lf's)",
                    "ms_per_step": 1e3 * sum(e2e_s) / a.steps},
            "roofline": roofline, "fp64": fp64, "accuracy": acc, "clocks": clk,
            "config0": config0, "n1048576": large, "batched": batched,
            "config_accuracy": config_acc, "cpu_baseline": cpu}
    print(json.dumps(line))
    ctx.close()


def measure_batch(ctx, eps2, single_value, steps=100, nsys=4096, seed=3):
    """The batched workload: 4096 Plummer systems, sizes log-uniform in
    [64, 4096] (seed 3, system s seeded by index), KDK dt = 1e-3 for 100 steps,
    one persistent work-queue launch per step, the step loop in one CUDA graph.
    The time is the graph launch alone (nbr_run_stats.gpu_ms: CUDA events on
    the context stream around cudaGraphLaunch), capture and instantiation
    excluded."""
    import nbr
    off, st = nbr.batch_plummer(nsys, seed)
    out = {"workload": f"{nsys} Plummer systems, N log-uniform in [64, 4096], seed {seed}, "
                       f"eps 1e-3, KDK dt 1e-3, {steps} steps", "systems": nsys,
           "particles": int(off[-1])}
    for prec, name in ((nbr.FP32C, "fp32c"), (nbr.FP64, "fp64")):
        ctx.batch_upload(off, st)
        ctx.batch_run(prec, dt=1e-3, steps=2, eps2=eps2)  # warm-up (and FSAL)
        r = ctx.batch_run(prec, dt=1e-3, steps=steps, eps2=eps2)
        t = r["gpu_ms"] * 1e-3
        out[name] = {"gpairs": r["pairs"] / t / 1e9, "systems_steps_per_s": nsys * steps / t,
                     "ms_per_step": 1e3 * t / steps, "steps": steps, "force_evals": r["force_evals"],
                     "kernels": r["kernels"]}
    out["fp32c"]["frac_of_single_system"] = out["fp32c"]["gpairs"] / single_value
    return out


def fp64_peak(mhz, ops=FMA_OPS_PER_PAIR):
    """Pairs/s of the FP64 pipe: SMs x 64 FP64 lanes x clock / ops per pair."""
    return SMS * 64 * mhz * 1e6 / ops / 1e9


def measure_config0(ctx, l2_flush, mhz, n=2048, steps=100):
    """The small-system configuration: Plummer N = 2048 (seed 0), eps = 1e-3,
    KDK dt = 1e-3 for 100 steps, FP64 (and FP32C beside it): one nbr_run call,
    whose 100 steps run as one CUDA graph launch; time = nbr_run_stats.gpu_ms
    (events around the graph launch; the first call's capture is untimed)."""
    import nbr
    s = nbr.plummer(n, 0)
    eps2 = 1e-6
    out = {"workload": f"plummer_n{n}_seed0_eps0.001_kdk_dt0.001_{steps}steps"}
    for prec, name in ((nbr.FP64, "fp64"), (nbr.FP32C, "fp32c")):
        times = []
        for rep in range(4):
            ctx.upload(s)
            l2_flush()
            r = ctx.run(prec, nbr.KDK, 2, 1e-3, steps, eps2=eps2)
            if rep > 0:
                times.append(r["gpu_ms"] * 1e-3)
        t = min(times)
        cfg = ctx.get_force_config(prec, eps2)
        gp = r["pairs"] / t / 1e9
        persistent = r["kernels"] == 1
        out[name] = {"steps_per_s": steps / t, "ms_per_step": 1e3 * t / steps, "gpairs": gp,
                     "force_evals": r["force_evals"], "kernels_per_run": r["kernels"],
                     "path": ("k_run_small_f64: all steps in one cooperative launch" if persistent
                              else f"one graph of per-step launches, force config {list(cfg)}"),
                     "runs_timed": len(times),
                     "time": "best of 3 runs (events around the launch)"}
    out["fp64"]["frac_of_fp64_16op_roofline"] = out["fp64"]["gpairs"] / fp64_peak(mhz)
    out["fp32c"]["frac_of_fp32_16op_roofline"] = out["fp32c"]["gpairs"] / (
        SMS * 128 * mhz * 1e6 / FMA_OPS_PER_PAIR / 1e9)
    out["reference_published_steps_per_s"] = {
        "value": 3866, "hardware": "2x Xeon Gold 6148, 40 cores, AVX512-RSQRT-4I, Euler, eps=0",
        "source": "final_results/single_node_combined.csv:10"}
    return out


def measure_large(ctx, l2_flush, mhz, n=1048576, steps=5, seed=2):
    """The large single system: Plummer N = 1048576 (seed 2), eps = 1e-3, KDK
    dt = 5e-4 for 5 steps, FP32C and FP64 (each the default kernel for this
    size), plus the FP32C force error against FP64 on all particles."""
    import numpy as np
    import nbr
    s = nbr.plummer(n, seed)
    eps2 = 1e-6
    pairs = float(n) * float(n - 1)
    out = {"workload": f"plummer_n{n}_seed{seed}_eps0.001_kdk_dt0.0005_{steps}steps"}
    for prec, name in ((nbr.FP32C, "fp32c"), (nbr.FP64, "fp64")):
        ctx.upload(s)
        ctx.run(prec, nbr.KDK, 2, 5e-4, steps, eps2=eps2)  # capture + warm-up
        ctx.upload(s)
        l2_flush()
        r = ctx.run(prec, nbr.KDK, 2, 5e-4, steps, eps2=eps2)
        t = r["gpu_ms"] * 1e-3
        cfg = ctx.get_force_config(prec, eps2)
        out[name] = {"gpairs": r["pairs"] / t / 1e9, "steps_per_s": steps / t,
                     "ms_per_step": 1e3 * t / steps, "force_evals": r["force_evals"],
                     "config": list(cfg)}
    ctx.upload(s)
    a32 = ctx.forces(nbr.FP32C, eps2=eps2)
    a64 = ctx.forces(nbr.FP64, eps2=eps2)
    e = _rel(a32, a64)
    out["fp32c_over_fp64"] = out["fp32c"]["gpairs"] / out["fp64"]["gpairs"]
    out["fp32c_vs_fp64_force_median_rel_err"] = float(np.median(e))
    out["fp32c_vs_fp64_force_max_rel_err"] = float(e.max())
    out["fp32c"]["frac_of_16op_roofline"] = out["fp32c"]["gpairs"] / (
        SMS * 128 * mhz * 1e6 / FMA_OPS_PER_PAIR / 1e9)
    del a32, a64
    return out


def _rel(a, b):
    import numpy as np
    num = np.linalg.norm(a - b, axis=0)
    den = np.linalg.norm(b, axis=0)
    return num / np.where(den > 0, den, 1.0)


def _drift(ctx, prec, s, dt, steps, eps2):
    ctx.upload(s)
    st = ctx.run(prec, 0, 2, dt, steps, eps2=eps2, diag=True)
    e0, e1 = st["diag"]
    return abs(e1["E"] - e0["E"]) / abs(e0["E"])


def measure_config_accuracy(ctx):
    """The two accuracy workloads beside the throughput one, FP32C against
    the FP64 kernel on identical inputs:
      * cold collapse: uniform ball N = 32768 (seed 1), zero velocities,
        eps = 1e-2, KDK dt = 1e-4 for 200 steps;
      * two-component stress test: N = 131072 Plummer (seed 4), 1 % heavy
        particles 1000x heavier, eps = 1e-3, KDK dt = 2e-4 for 500 steps, with
        the force error stratified by receiver and source mass class (each
        class of sources evaluated separately through nbr_accel_ij)."""
    import numpy as np
    import nbr
    out = {}
    s = nbr.uniform_ball(32768, 1)
    eps2 = 1e-4
    ctx.upload(s)
    a32 = ctx.forces(nbr.FP32C, eps2=eps2)
    a64 = ctx.forces(nbr.FP64, eps2=eps2)
    e = _rel(a32, a64)
    out["uniform_ball_n32768"] = {
        "force_median_rel_err": float(np.median(e)), "force_max_rel_err": float(e.max()),
        "energy_drift_fp32c": _drift(ctx, nbr.FP32C, s, 1e-4, 200, eps2),
        "energy_drift_fp64": _drift(ctx, nbr.FP64, s, 1e-4, 200, eps2), "steps": 200}
    n, nh = 131072, 1311
    s = nbr.two_component(n, nh, 1000.0, 4)
    eps2 = 1e-6
    heavy = np.zeros(n, dtype=bool)
    heavy[:nh] = True
    strat = {}
    for src_name, src in (("heavy", heavy), ("light", ~heavy)):
        res = {}
        for prec in (nbr.FP32C, nbr.FP64):
            res[prec] = ctx.accel_ij(s["x"], s["y"], s["z"], s["x"][src], s["y"][src], s["z"][src],
                                     s["m"][src], precision=prec, eps2=eps2)
        e = _rel(res[nbr.FP32C], res[nbr.FP64])
        for rcv_name, rcv in (("heavy", heavy), ("light", ~heavy)):
            strat[f"{rcv_name}<-{src_name}"] = {"median_rel_err": float(np.median(e[rcv])),
                                                "max_rel_err": float(e[rcv].max())}
    ctx.upload(s)
    a32 = ctx.forces(nbr.FP32C, eps2=eps2)
    a64 = ctx.forces(nbr.FP64, eps2=eps2)
    e = _rel(a32, a64)
    out["two_component_n131072"] = {
        "stratified_receiver<-source": strat,
        "force_median_rel_err": float(np.median(e)), "force_max_rel_err": float(e.max()),
        "energy_drift_fp32c": _drift(ctx, nbr.FP32C, s, 2e-4, 500, eps2),
        "energy_drift_fp64": _drift(ctx, nbr.FP64, s, 2e-4, 500, eps2), "steps": 500}
    return out


def run_sharded(a, rank, world, local):
    """--gpus N under torchrun: the one system over the N GPUs with Newton-3
    across them (nbr_shard.ShardedSystem, method "newton3": each GPU computes
    its slices of the pair triangle for every particle, an NCCL all-to-all
    hands each GPU the partial forces of its own receivers, added in slice
    order, then an NCCL all-gather of positions per step).  Strong scaling:
    N(N-1) pairs per step in total."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    import nbr
    from nbr_shard import ShardedSystem

    torch.cuda.set_device(local)
    global SMS
    SMS = torch.cuda.get_device_properties(local).multi_processor_count
    for k, v in (("MASTER_ADDR", "127.0.0.1"), ("MASTER_PORT", "29533"), ("RANK", str(rank)),
                 ("WORLD_SIZE", str(world))):
        os.environ.setdefault(k, v)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    try:
        prec = nbr.FP32C if a.precision == "fp32c" else nbr.FP64
        eps2 = a.eps * a.eps
        n = a.n
        pairs = float(n) * float(n - 1)
        s = nbr.plummer(n, a.seed)
        ctx = nbr.Context(local)
        sh = ShardedSystem(ctx, method="newton3", slices=max(8, world))
        sh.upload(s)
        ext = torch.cuda.ExternalStream(ctx.stream)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")

        def l2_flush():
            with torch.cuda.stream(ext):
                flush.zero_()

        def timed(fn):
            l2_flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            fn()
            e1.record(ext)
            e1.synchronize()
            return e0.elapsed_time(e1) * 1e-3

        def step():
            sh.step(prec, nbr.KDK, a.dt, a.dt, 1.0, eps2)

        def max_over_ranks(v):
            t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        # kernel-only: this GPU's Newton-3 slices (state unchanged); one untimed
        # call first (scratch, the slice-width choice)
        def my_slices():
            ctx.n3_slice_accel(prec, eps2, sh.v0, sh.slices, sh._mine, slice_end=sh.v1)
        my_slices()
        ctx.synchronize()
        k_s = [timed(my_slices) for _ in range(3)]
        for _ in range(a.warmup):
            step()
        ctx.synchronize()
        clocks = ClockSampler(local) if rank == 0 else None
        if clocks:
            clocks.start()
            time.sleep(0.5)
        dist.barrier()
        torch.cuda.synchronize()
        step_s = [timed(step) for _ in range(a.steps)]
        dist.barrier()
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        t_total = max_over_ranks(sum(step_s))
        ctx.synchronize()  # surfaces a bounded-wait timeout of any step
        value = a.steps * pairs / t_total / 1e9

        # end to end: host state in (pinned), one sharded step, positions out
        host = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in nbr.KEYS}
        for k in nbr.KEYS:
            host[k][:] = s[k]
        e2e_s = []
        for i in range(a.warmup + a.steps):
            def e2e_step():
                ctx.upload_raw(n, *[host[k] for k in nbr.KEYS])
                sh.step(prec, nbr.KDK, a.dt, a.dt, 1.0, eps2)
                ctx.download_raw(host["x"], host["y"], host["z"], None, None, None)
            t = timed(e2e_step)
            if i >= a.warmup:
                e2e_s.append(t)
        e2e_total = max_over_ranks(sum(e2e_s))
        k_t = statistics.median(k_s) if k_s else 0.0
        k_max = max_over_ranks(k_t)
        if rank == 0:
            mhz = (clk or {}).get("sm_mhz") or 1965.0
            ops = (FMA_OPS_PER_PAIR + REACTION_OPS) / 2  # Newton-3: per ordered pair
            peak = world * SMS * 128 * mhz * 1e6 / ops / 1e9
            achieved = pairs / k_max / 1e9 if k_max > 0 else None
            line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                    "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t_total / a.steps,
                    "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                    "dtype": "f32" if prec == nbr.FP32C else "f64", "data": "synthetic",
                    "config": workload_config(a, {"precision": a.precision,
                                                  "parallelism": f"Newton-3 slices x{world} GPUs "
                                                                 f"({sh.slices} slices), NCCL all-to-all "
                                                                 "of partial forces + all-gather of "
                                                                 "positions per step",
                                                  "shard": sh.count}),
                    "gpu_launches": a.steps * (2 + (sh.v1 - sh.v0)),
                    "e2e": {"value": a.steps * pairs / e2e_total / 1e9, "unit": UNIT,
                            "h2d_bytes_per_step": 7 * 8 * n, "d2h_bytes_per_step": 3 * 8 * n,
                            "scheme": "kdk, whole state uploaded and positions downloaded per step"},
                    "roofline": {"bound": "fp32_fma_pipe", "achieved": achieved, "peak": peak,
                                 "unit": UNIT, "frac": achieved / peak if achieved else None,
                                 "traffic": None,
                                 "peak_source": f"{world} GPUs x {SMS} SMs x 128 FP32 lanes x rank-0 "
                                                f"median SM clock / {ops:g} FMA-pipe ops per ordered "
                                                "pair (Newton-3)",
                                 "kernel_ms_max_over_ranks": 1e3 * k_max},
                    "clocks": clk, "cpu_baseline": None,
                    "collectives_per_step": "1 all-to-all + 3 in-place all-gathers"}
            print(json.dumps(line))
        ctx.synchronize()
        ctx.close()
    finally:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
