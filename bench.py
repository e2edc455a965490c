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
def cpu_reference_sample(n, seed, target_s, max_s):
    """The reference's fastest CPU force kernel (AVX-512 rsqrt 4i, or AVX2
    blocked on a host without AVX-512) on this host's cores, on rank 0's share
    of its own ring decomposition (hybrid_ring_solver) of one N-particle force
    evaluation: N(N-1)/comm_sz effective pairs per share.  comm_sz is the
    smallest power of two whose share takes at most target_s."""
    sys.path.insert(0, ORACLE)
    import nbr
    from oracle import Reference, reference_available
    if not reference_available():
        return None
    ref = Reference()
    ref.set_threads(os.cpu_count() or 1)
    s = nbr.plummer(n, seed)
    # calibrate on a small share
    comm = 1
    while comm < n and n % (comm * 2) == 0 and comm < 256:
        comm *= 2
    t = ref.ring_share(s, comm)
    while comm > 1 and t * 2 <= target_s:
        comm //= 2
        t = ref.ring_share(s, comm)
    reps, total, pairs = 0, 0.0, 0.0
    while total < target_s and total + t <= max_s or reps == 0:
        tt = ref.ring_share(s, comm)
        total += tt
        pairs += n * (n - 1) / comm
        reps += 1
        if total >= target_s:
            break
    kernel = "AVX512-RSQRT-4I" if ref.has_avx512 else "AVX2-blocked"
    return {"value": pairs / total / 1e9, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
            "seconds": total,
            "sample": f"{reps} x rank-0 share (1/{comm}) of one N={n} force evaluation of the reference's "
                      f"{kernel} kernel (ring decomposition of hybrid_ring_solver, eps=0, FP64), "
                      f"{ref.threads()} OpenMP threads"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, ORACLE)
    from oracle import reference_available
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU solver (oracle/_ref) was not built here"}))
        return
    import nbr
    from oracle import Reference
    ref = Reference()
    ref.set_threads(os.cpu_count() or 1)
    n = a.n
    s = nbr.plummer(n, a.seed)
    # per-step budget so that warmup + steps end within about two minutes
    per_step = min(3.0, 120.0 / max(1, a.steps + a.warmup))
    comm = 1
    while comm < n and n % (comm * 2) == 0 and comm < 1024:
        comm *= 2
    t = ref.ring_share(s, comm)
    while comm > 1 and t * 2 <= per_step:
        comm //= 2
        t = ref.ring_share(s, comm)
    for _ in range(a.warmup):
        ref.ring_share(s, comm)
    secs = [ref.ring_share(s, comm) for _ in range(a.steps)]
    total = sum(secs)
    pairs = a.steps * n * (n - 1) / comm
    value = pairs / total / 1e9
    kernel = "AVX512-RSQRT-4I" if ref.has_avx512 else "AVX2-blocked"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * total / a.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(a, {"reference_kernel": kernel,
                                                               "comm_sz": comm}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
                             "sample": f"each step: rank-0 share (1/{comm}) of one N={n} force evaluation "
                                       f"of the reference's {kernel} kernel (hybrid_ring_solver's ring "
                                       f"decomposition), eps=0 FP64, {ref.threads()} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
                "peak_source": f"148 SMs x 128 FP32 lanes x median SM clock sampled in the timed region "
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

    batched = None if a.no_batch else measure_batch(ctx, ext, eps2, value)
    config_acc = None if a.no_config_accuracy else measure_config_accuracy(ctx)

    cpu = None
    if not a.no_cpu_baseline and rank == 0:
        try:
            cpu = cpu_reference_sample(n, a.seed, target_s=10.0, max_s=30.0)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"error": str(ex)}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * t_total / a.steps,
            "steps_per_s": a.steps / t_total, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec == nbr.FP32C else "f64",
            "data": "synthetic", "config": workload_config(a, {"precision": a.precision}),
            "gpu_launches": launches, "wall_s_timed": t_wall,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 7 * 8 * n,
                    "d2h_bytes_per_step": 6 * 8 * n, "scheme": "dkd order 2 (reduced_solver_omp_lf's)",
                    "ms_per_step": 1e3 * sum(e2e_s) / a.steps},
            "roofline": roofline, "fp64": fp64, "accuracy": acc, "clocks": clk,
            "batched": batched, "config_accuracy": config_acc, "cpu_baseline": cpu}
    print(json.dumps(line))
    ctx.close()


def measure_batch(ctx, ext, eps2, single_value, steps=10, nsys=4096, seed=3):
    """The batched workload: 4096 Plummer systems, sizes log-uniform in
    [64, 4096] (seed 3, system s seeded by index), KDK dt = 1e-3, one persistent
    work-queue launch per step, the step loop in one CUDA graph."""
    import torch
    import nbr
    off, st = nbr.batch_plummer(nsys, seed)
    ctx.batch_upload(off, st)
    out = {"workload": f"{nsys} Plummer systems, N log-uniform in [64, 4096], seed {seed}, "
                       f"eps 1e-3, KDK dt 1e-3", "systems": nsys, "particles": int(off[-1])}
    for prec, name in ((nbr.FP32C, "fp32c"), (nbr.FP64, "fp64")):
        ctx.batch_upload(off, st)
        ctx.batch_run(prec, dt=1e-3, steps=2, eps2=eps2)  # warm-up (and FSAL)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        r = ctx.batch_run(prec, dt=1e-3, steps=steps, eps2=eps2)
        e1.record(ext)
        e1.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        out[name] = {"gpairs": r["pairs"] / t / 1e9, "systems_steps_per_s": nsys * steps / t,
                     "ms_per_step": 1e3 * t / steps, "force_evals": r["force_evals"],
                     "kernels": r["kernels"]}
    out["fp32c"]["frac_of_single_system"] = out["fp32c"]["gpairs"] / single_value
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
    """--gpus N under torchrun: the one system split by receivers over the N
    GPUs (nbr_shard.ShardedSystem: owned slice against all sources, then an
    NCCL all-gather of positions per step, as hybrid_full_solver does with
    MPI_Allgather).  Strong scaling: N(N-1) pairs per step in total."""
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    import nbr
    from nbr_shard import ShardedSystem

    torch.cuda.set_device(local)
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
        sh = ShardedSystem(ctx)
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

        # kernel-only: the owned slice's evaluation with kick = drift = 0
        # (state unchanged), then an exchange to refill the other slices
        k_s = []
        for _ in range(3):
            if sh.owned:
                k_s.append(timed(lambda: ctx.step_range(prec, nbr.KDK, sh.i0, sh.owned, 0.0, 0.0,
                                                        1.0, eps2)))
            sh.exchange_positions()
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
        k_t = statistics.mean(k_s) if k_s else 0.0
        k_max = max_over_ranks(k_t)
        if rank == 0:
            mhz = (clk or {}).get("sm_mhz") or 1965.0
            peak = world * SMS * 128 * mhz * 1e6 / FMA_OPS_PER_PAIR / 1e9
            achieved = pairs / k_max / 1e9 if k_max > 0 else None
            line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                    "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t_total / a.steps,
                    "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                    "dtype": "f32" if prec == nbr.FP32C else "f64", "data": "synthetic",
                    "config": workload_config(a, {"precision": a.precision,
                                                  "parallelism": f"i-partition x{world}, NCCL "
                                                                 "all-gather of positions per step",
                                                  "shard": sh.count}),
                    "gpu_launches": 2 * a.steps,
                    "e2e": {"value": a.steps * pairs / e2e_total / 1e9, "unit": UNIT,
                            "h2d_bytes_per_step": 7 * 8 * n, "d2h_bytes_per_step": 3 * 8 * n,
                            "scheme": "kdk, whole state uploaded and positions downloaded per step"},
                    "roofline": {"bound": "fp32_fma_pipe", "achieved": achieved, "peak": peak,
                                 "unit": UNIT, "frac": achieved / peak if achieved else None,
                                 "traffic": None,
                                 "peak_source": f"{world} GPUs x 148 SMs x 128 FP32 lanes x rank-0 "
                                                "median SM clock / 16 FMA-pipe ops per pair",
                                 "kernel_ms_max_over_ranks": 1e3 * k_max},
                    "clocks": clk, "cpu_baseline": None, "collectives_per_step": 1}
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
