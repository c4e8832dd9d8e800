"""Benchmark: KPM density of states on the 5x5 square lattice (N=25, full
2^25 basis, 1024 Chebyshev moments, 32 Rademacher probes).

One step = one complete KPM DOS solve: spectral bounds (FP64 Lanczos on the
device), the moment recurrence (FP32 vectors, FP64 moments, doubling
identities) and the Jackson-kernel DOS on 400 energies.  The metric is
solves/s over all ranks; the roofline entry is the tiled KPM pass kernel
(one Chebyshev step per launch) against measured HBM bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

--impl reference times the CPU restatement of the reference recurrence
(oracle/el_oracle.c, OpenMP over all host cores) on a bounded sample of the
same workload and extrapolates linearly in moments x probes.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Sector H·v GB/s; solves/s & grads/s, chosen vs plain FP64 B200 at fixed error"
NUM, NVEC, CHUNK = 1024, 32, 32
WORKLOAD = "kpm_dos_square25"


def workload():
    from energy_level_b200 import configs
    cfg = configs.square25()
    return cfg


def config_dict(cfg, extra=None):
    d = {"workload": WORKLOAD, "lattice": "5x5 square a=6um", "n_sites": 25, "basis": "full 2^25",
         "dim": 1 << 25, "moments": NUM, "probes": NVEC, "probe_block": CHUNK,
         "vectors": "float32", "moment_accumulation": "float64",
         "recurrence": "Chebyshev doubling (T2n=2Tn^2-T0)",
         "l2": "inputs larger than L2 (probe block 4.3 GB per vector)"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """dram bytes per pass launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "kpm_pass_square25.md")
    try:
        for line in open(path, encoding="utf-8"):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- CPU side

def cpu_sample(cfg, moments=8, probes=2):
    """Time the C oracle's direct KPM recurrence on a bounded sample of the
    workload; return (seconds per probe-moment, threads, description)."""
    from oracle import build as ob
    n = cfg["n"]
    pairs = [(p["i"], p["j"], p["V"]) for p in cfg["calib"]["pairs"]]
    d = ob.diag_full(n, cfg["delta"], pairs)
    from energy_level_b200.probes import rademacher_host
    z = rademacher_host(seed=cfg["probe_seed"], probe0=0, nvec=probes, dim=1 << n)
    # a rigorous interval: diagonal range widened by sum |Omega_i| / 2
    half = 0.5 * float(np.sum(np.abs(cfg["Om"])))
    lo, hi = float(d.min()) - half, float(d.max()) + half
    c, r = 0.5 * (lo + hi), 0.5 * (hi - lo) * (1.0 + 1e-3)
    lib = ob.load()
    t0 = time.perf_counter()
    ob.kpm_full(n, cfg["Om"], d, c, r, moments, z)
    dt = time.perf_counter() - t0
    return dt / (moments * probes), int(lib.oracle_threads()), \
        "N=25 full basis, %d probes x %d moments (direct recurrence, FP64)" % (probes, moments)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = workload()
    times = []
    for i in range(args.warmup + args.steps):
        tpm, threads, desc = cpu_sample(cfg)
        if i >= args.warmup:
            times.append(tpm)
    tpm = float(np.mean(times))
    solve_s = tpm * NUM * NVEC
    value = 1.0 / solve_s
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice, counter-based probes)",
            "config": config_dict(cfg, {"sample": desc}),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": desc + "; extrapolated linearly to 1024 moments x 32 probes"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU side

def run_native(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA 不可用")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from energy_level_b200.build import build
    build()
    from energy_level_b200 import kpm as bkpm, solvers
    from energy_level_b200.core import Context, Basis, Hamiltonian

    cfg = workload()
    n = cfg["n"]
    pairs = [(p["i"], p["j"], p["V"]) for p in cfg["calib"]["pairs"]]
    ctx = Context(local)
    basis = Basis(ctx, n, "full")
    ham = Hamiltonian(ctx, basis, cfg["Om"], cfg["delta"], pairs)
    seed = cfg["probe_seed"] + 1000 * rank          # replicas draw distinct probes
    stream = torch.cuda.current_stream()

    def solve(dtype="float32"):
        lo, hi = solvers.bounds(ham, max_iter=300, tol=1e-12, seed=0)
        c, r = solvers.kpm_scale(lo, hi)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        mu = solvers.kpm_moments(ham, NUM, NVEC, c, r, dtype=dtype, chunk=CHUNK, seed=seed,
                                 mode="doubling")
        ev1.record(stream)
        span = max(hi - lo, 1e-9)
        energies = np.linspace(lo + span * 1e-6, hi - span * 1e-6, 400)
        rho = bkpm.dos_from_moments(mu, c, r, energies, NUM)
        return mu, rho, (lo, hi, c, r), (ev0, ev1)

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = ctx.launches
    kpm_events = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            mu, rho, scal, evs = solve()
            kpm_events.append(evs)
        t1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    launches = ctx.launches - launches0
    elapsed = t0.elapsed_time(t1) / 1e3
    kpm_s = sum(a.elapsed_time(b) for a, b in kpm_events) / 1e3
    if dist:
        tt = torch.tensor([elapsed, kpm_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed, kpm_s = float(tt[0]), float(tt[1])
    value = world * args.steps / elapsed

    # roofline of the dominant kernel: one tiled pass = one Chebyshev step
    passes = (NUM + 1) // 2 + 1                    # prologue + M passes per probe block
    launch_s = kpm_s / (args.steps * passes)
    dim = 1 << n
    alg_bytes = dim * (3 * NVEC * 4 + 4)           # read t_n, t_n-1, write t_n+1, read d
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / launch_s / 1e9
    traffic = profiled_traffic()

    # plain FP64 comparator (same probes) and the error of the chosen form
    mu64, rho64, _, evs64 = solve("float64")
    torch.cuda.synchronize()
    fp64_s = evs64[0].elapsed_time(evs64[1]) / 1e3
    err_mu = float(np.max(np.abs(mu - mu64)))
    err_dos = float(np.max(np.abs(rho - rho64)) / max(np.max(np.abs(rho64)), 1e-300))

    # end to end through the public API with host inputs (pinned) each step
    e2e_value, h2d, d2h = None, None, None
    if rank == 0 or world > 1:
        from energy_level_b200.core import default_context
        system = {"calib": cfg["calib"], "Om": cfg["Om"], "delta": cfg["delta"], "terms": ["I1"]}
        e2e_ctx = default_context(local)
        reps = max(1, min(args.steps, 2))
        bkpm.kpm_dos_b200(system, num=NUM, nvec=NVEC, seed=seed, dtype="float32", chunk=CHUNK,
                          device="cuda:%d" % local)          # warm the public path once
        torch.cuda.synchronize()
        b0 = e2e_ctx.copied_bytes
        te = time.perf_counter()
        for _ in range(reps):
            out = bkpm.kpm_dos_b200(system, num=NUM, nvec=NVEC, seed=seed, dtype="float32", chunk=CHUNK,
                                    device="cuda:%d" % local)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - te) / reps
        b1 = e2e_ctx.copied_bytes
        e2e_value = world / e2e_s
        h2d = (b1[0] - b0[0]) // reps          # parameters copied in (Omega, delta, V table)
        d2h = (b1[1] - b0[1]) // reps          # scalars and moments copied out

    # CPU baseline on the host cores (rank 0, single GPU only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        tpm, threads, desc = cpu_sample(cfg)
        cpu = {"value": 1.0 / (tpm * NUM * NVEC), "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": desc + "; extrapolated linearly to 1024 moments x 32 probes"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 5x5 lattice, C6/r^6 couplings, counter-based Rademacher probes)",
            "config": config_dict(cfg, {"parallelism": "replicas" if world > 1 else "single GPU"}),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_kpm_pass (one Chebyshev step of 32 probes over 2^25 rows)",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": launch_s * 1e3,
                         "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "plain_fp64": {"solves_per_s": 1.0 / (fp64_s + (elapsed / args.steps - kpm_s / args.steps)),
                           "moments_ms": fp64_s * 1e3, "form": "FP64 vectors, same tiled recurrence"},
            "error_vs_fp64": {"max_abs_moment": err_mu, "max_rel_dos": err_dos},
            "hv_gbs": achieved,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_native(args)


if __name__ == "__main__":
    sys.exit(main())
