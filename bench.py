#!/usr/bin/env python
"""Throughput of the fused LBM step on B200 (MLUPS and HBM-roofline fraction).

Default workload: D3Q27 MRT lid-driven cavity 256^3 (Gram-Schmidt moment basis, lid 0.05 on the
z-top face, shear rate from Re 1000, other rates 1.2), FP16-shifted storage as the headline value
and FP32 plain storage beside it.  One bench step = one lattice time step (one kernel launch over
all 16.8M cells); the populations (0.85 GB FP16 / 1.7 GB FP32 per buffer) are larger than L2, so
no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Under torchrun (N > 1) every rank advances its own replica lattice (weak scaling, no data-path
collective); the reported time is the max over ranks.  `--impl reference` times the CPU
restatement of the reference's loop (the reference's ArrayFire CPU backend is not installed).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "lbm-arrayfire_b200"))

METRIC = "MLUPS & HBM-roofline %: FP16-shifted vs FP32 plain at <=1e-3 rel L2 vs FP64"
FALLBACK_HBM_GBS = 6650.0

# ---------------------------------------------------------------------------------------------
# workloads (the engine side); each returns (desc, mask, F0 or None = rest state)
# ---------------------------------------------------------------------------------------------


def cube(n):
    return tuple(n) if isinstance(n, (tuple, list)) else (n, n, n)


def wl_mrt256(lb, storage, n=256):
    """D3Q27 MRT lid cavity n^3 (or nx x ny x nz), Gram-Schmidt basis, lid 0.05, sv from Re 1000 at L=256."""
    sv = 1.0 / (3.0 * (0.05 * 256 / 1000.0) + 0.5)
    d = lb.make_desc(lb.D3Q27, lb.MRT, storage, cube(n), mrt_s=lb.mrt_rates(sv, 1.2),
                     mrt_basis=lb.MRT_GRAM_SCHMIDT)
    m = lb.setup_cavity3d(d, 0.05)
    return d, m


def wl_channel(lb, storage, n=None):
    """D2Q9 channel 1024x256, circle d=40 at (200,128), inlet 0.04, zero-gradient outlet, Re 200."""
    nu = 0.04 * 40 / 200.0
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (1024, 256), omega=1.0 / (3 * nu + 0.5))
    m = lb.setup_channel2d(d, 0.04, 200, 128, 20, True)
    return d, m


def wl_cavity128(lb, storage, n=None):
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (128, 128), omega=lb.omega_from_re(0.1, 128, 100.0, 0))
    m = lb.setup_cavity2d(d, 0.1)
    return d, m


def wl_sc1024(lb, storage, n=None):
    d = lb.make_desc(lb.D2Q9, lb.SHANCHEN, storage, tuple(n) if n else (1024, 1024), omega=1.0, sc_G=-5.5)
    return d, None


def wl_bgk3d(lb, storage, n=256):
    d = lb.make_desc(lb.D3Q27, lb.BGK, storage, cube(n), omega=lb.omega_from_re(0.05, cube(n)[0], 1000.0, 0))
    m = lb.setup_cavity3d(d, 0.05)
    return d, m


def wl_cavity2d_big(lb, storage, n=8192):
    d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (n, n), omega=lb.omega_from_re(0.1, n, 1000.0, 1))
    m = lb.setup_cavity2d(d, 0.1)
    return d, m


WORKLOADS = {
    "d3q27_mrt_gs_lid_256": (wl_mrt256, "D3Q27 MRT (Gram-Schmidt) lid cavity 256^3, lid 0.05 z-top, Re 1000"),
    "d2q9_channel_1024x256": (wl_channel, "D2Q9 BGK channel 1024x256, cylinder d=40, inlet 0.04, Re 200"),
    "d2q9_lid_128": (wl_cavity128, "D2Q9 BGK lid cavity 128^2, lid 0.1, Re 100"),
    "d2q9_shanchen_1024": (wl_sc1024, "D2Q9 Shan-Chen 1024^2 periodic, G=-5.5, tau=1"),
    "d3q27_bgk_lid_256": (wl_bgk3d, "D3Q27 BGK lid cavity 256^3"),
    "d2q9_lid_8192": (wl_cavity2d_big, "D2Q9 BGK lid cavity 8192^2"),
    "ensemble_config5": (None, "48 D2Q9 BGK lids L in {64..1024} Re in [100,1000] + 16 D3Q27 BGK channels "
                               "(4L,L,L) L in {64..192} with sphere d=L/4, inlet 0.04, seed 3"),
}

STORAGE_NAMES = {0: "f32", 1: "f16s", 2: "bf16s", 3: "f64"}


def storage_bytes(storage):
    return {0: 4, 1: 2, 2: 2, 3: 8}[storage]


def algorithmic_bytes_per_cell(d):
    """2 Q s (read + write of every population); Shan-Chen adds the psi write and read (8 B)."""
    b = 2 * d.q * storage_bytes(d.storage)
    if d.collision == 2:
        b += 8
    return b


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            j = json.loads(p.read_text())
            return float(j["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def dram_traffic(workload, storage):
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "dram_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and not line.startswith("#") and parts[0] == workload and parts[1] == STORAGE_NAMES[storage]:
            return float(parts[2])
    return None


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            return None
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            cols = [c.strip() for c in line.split(",")]
            if len(cols) < 8:
                continue
            try:
                sm.append(float(cols[0]))
                smax.append(float(cols[1]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if cols[4 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_id_for_smi(torch, dev):
    try:
        u = torch.cuda.get_device_properties(dev).uuid
        return f"GPU-{u}"
    except Exception:
        return str(dev)


# ---------------------------------------------------------------------------------------------
# CPU restatement (oracle) timings: the cpu_baseline object and the reference arm
# ---------------------------------------------------------------------------------------------
def oracle_problem_for(workload, n_side):
    """The workload's problem for the CPU restatement, built on the oracle side only (oracle/problems.py
    restates the reference drivers' set-up): the reference arm never loads the engine library.
    n_side: cube side of a D3Q27 sample (None: the configuration's own size)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import problems as P

    if workload == "d3q27_mrt_gs_lid_256":
        return P.config_mrt_lid((n_side or 256,) * 3)
    if workload == "d3q27_bgk_lid_256":
        return P.config_bgk_lid3d((n_side or 256,) * 3)
    if workload == "d2q9_channel_1024x256":
        return P.config_channel()
    if workload == "d2q9_lid_128":
        return P.config_lid128()
    if workload == "d2q9_shanchen_1024":
        return P.config_shanchen()
    if workload == "d2q9_lid_8192":
        return P.cavity2d(8192, 8192, 0.1, P.omega_from_re(0.1, 8192, 1000.0, 1))
    raise KeyError(workload)


def oracle_mlups(workload, target_s, cube=None):
    """Time the oracle (FP32, all host threads) on a sample of the workload for ~target_s seconds."""
    import oracle as O

    side = cube or 64
    p = oracle_problem_for(workload, side)
    F0 = O.init_equilibrium(p)
    t = time.perf_counter()
    O.run(p, F0, 1, dtype=np.float32)
    t1 = max(time.perf_counter() - t, 1e-4)
    steps = max(2, int(target_s / t1))
    t = time.perf_counter()
    O.run(p, F0, steps, dtype=np.float32)
    dt = time.perf_counter() - t
    cells = p.n
    return cells * steps / dt / 1e6, cells, steps, p.shape


def threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_reference(args, rank, world):
    """The reference arm: the CPU restatement of the reference loop, on rank 0 only."""
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.lib()
    if args.workload == "ensemble_config5":
        return run_reference_ensemble(args, world, O)
    # calibrate, then pick a sample lattice so that W + K steps end within the budget (default 150 s)
    mlups0, _, _, _ = oracle_mlups(args.workload, 1.0)
    budget_cells = mlups0 * 1e6 * args.ref_seconds / max(1, args.steps + args.warmup)
    if args.workload.startswith("d3q27"):
        side = int(max(8, min(256, math.floor(budget_cells ** (1 / 3)))))
        p = oracle_problem_for(args.workload, side)
    else:
        p = oracle_problem_for(args.workload, None)
    F = O.init_equilibrium(p)
    if args.warmup:
        F, _, _ = O.run(p, F, args.warmup, dtype=np.float32)
    t = time.perf_counter()
    O.run(p, F, args.steps, dtype=np.float32)
    dt = time.perf_counter() - t
    value = p.n * args.steps / dt / 1e6
    sample = f"{'x'.join(map(str, p.shape))} lattice of the same workload, {args.steps} timed steps, FP32, " \
             f"{threads()} threads on {cpu_model()}"
    return {
        "metric": METRIC, "value": value, "unit": "MLUPS", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload][1], "sample_shape": list(p.shape)},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": threads(), "kind": "port", "sample": sample,
                         "note": "ArrayFire CPU backend unavailable on this box; C restatement of the reference loop"},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference_ensemble(args, world, O):
    """Reference arm of config 5: the CPU restatement on the smallest member of each lattice family
    (a D2Q9 lid and a D3Q27 channel of the ensemble), K steps each; MLUPS = cells x steps / time.  The
    members come from oracle/problems.py (the same seeded list the engine side draws)."""
    import problems as P

    spec = P.ensemble_spec(3)
    picks = []
    for fam in ("d2q9", "d3q27"):
        name, shape, omega = min((s for s in spec if s[0].startswith(fam)), key=lambda s: int(np.prod(s[1])))
        picks.append((P.ensemble_problem(name, shape, omega), name, shape))
    cells = 0
    dt = 0.0
    for p, _, _ in picks:
        F = O.init_equilibrium(p)
        if args.warmup:
            F, _, _ = O.run(p, F, args.warmup, dtype=np.float32)
        t = time.perf_counter()
        O.run(p, F, args.steps, dtype=np.float32)
        dt += time.perf_counter() - t
        cells += p.n
    value = cells * args.steps / dt / 1e6
    sample = " + ".join(f"{name} {'x'.join(map(str, shp))}" for _, name, shp in picks) + \
        f", {args.steps} timed steps each, FP32, {threads()} threads on {cpu_model()}"
    return {
        "metric": METRIC, "value": value, "unit": "MLUPS", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload][1]},
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": threads(), "kind": "port", "sample": sample,
                         "note": "ArrayFire CPU backend unavailable on this box; C restatement of the reference loop"},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------
def timed_steps(torch, lat, steps, dev):
    """Device time of `steps` lattice steps on the context's stream (CUDA events)."""
    s = torch.cuda.ExternalStream(lat.stream(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    lat.step(steps)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def build_workload(lb, args, storage):
    fn = WORKLOADS[args.workload][0]
    if args.dims and (args.workload.startswith("d3q27") or args.workload == "d2q9_shanchen_1024"):
        d, m = fn(lb, storage, tuple(int(v) for v in args.dims.lower().split("x")))
    elif args.size and (args.workload.startswith("d3q27") or args.workload == "d2q9_lid_8192"):
        d, m = fn(lb, storage, args.size)
    else:
        d, m = fn(lb, storage)
    if getattr(args, "rounding", "stochastic") == "nearest":
        d.rounding = lb.ROUND_NEAREST
    return d, m


def apply_kernel_choice(lb, lat, args):
    if args.kernel != "auto":
        lat.set_kernel({"plain": lb.KERNEL_PLAIN, "rows": lb.KERNEL_ROWS, "cluster": lb.KERNEL_CLUSTER}[args.kernel])
    if args.block:
        lat.set_block(args.block)


KERNEL_NAMES = {1: "plain", 2: "rows", 3: "cluster"}


def measure(torch, lb, args, storage, dev, world, sample_clocks=False):
    d, m = build_workload(lb, args, storage)
    d.device = dev
    lat = lb.Lattice(d, m)
    apply_kernel_choice(lb, lat, args)
    lat.step(args.warmup if args.warmup > 0 else 1)   # includes the block-width autotune
    lat.sync()
    torch.cuda.synchronize(dev)
    barrier(torch, world)
    sampler = ClockSampler(gpu_id_for_smi(torch, dev)) if sample_clocks else None
    if sampler:
        time.sleep(0.3)
    elapsed = timed_steps(torch, lat, args.steps, dev)
    clocks = sampler.stop() if sampler else None
    torch.cuda.synchronize(dev)
    barrier(torch, world)
    elapsed_max = reduce_max(torch, elapsed, dev, world)
    return d, lat, elapsed_max, clocks


def e2e_measure(torch, lb, args, storage, dev, world):
    """Through the public API with host buffers: pinned H2D of the start populations, K steps,
    D2H of the macroscopic fields, all inside the timed region."""
    d, m = build_workload(lb, args, storage)
    d.device = dev
    lat = lb.Lattice(d, m)
    apply_kernel_choice(lb, lat, args)
    N, Q = d.cells, d.q
    _, _, _, w, _ = lb.velocities(d.lattice)
    F_host = torch.empty(N * Q, dtype=torch.float32, pin_memory=True)
    F_host.view(Q, N).copy_(torch.tensor(w, dtype=torch.float32)[:, None].expand(Q, N))
    rho_host = torch.empty(N, dtype=torch.float32, pin_memory=True)
    u_host = torch.empty(d.dim * N, dtype=torch.float32, pin_memory=True)
    lat.step(2)  # autotune + graph build outside the timed region
    lat.sync()
    torch.cuda.synchronize(dev)
    barrier(torch, world)
    s = torch.cuda.ExternalStream(lat.stream(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    lat.set_populations(F_host)
    lat.step(args.steps)
    lat.macros_into(rho_host, u_host)
    e1.record(s)
    e1.synchronize()
    elapsed = e0.elapsed_time(e1) / 1e3
    elapsed = reduce_max(torch, elapsed, dev, world)
    h2d = N * Q * 4
    d2h = N * (1 + d.dim) * 4
    lat.close()
    return {"value": world * N * args.steps / elapsed / 1e6, "unit": "MLUPS",
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "api": "lbm_set_populations (pinned host F32) + lbm_step(K) + lbm_get_macros (pinned host F32)"}


# ---------------------------------------------------------------------------------------------
# accuracy of FP32 and 16-bit storage against the FP64 run of the same kernels, every configuration
# ---------------------------------------------------------------------------------------------
def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def solid_cells(lb, d, m):
    """Cells whose class bounces back (the reference's ON nodes)."""
    if m is None:
        return np.zeros(d.cells, dtype=bool)
    flags = np.array([c[0] for c in lb.classes_of(d)])
    return (flags[np.asarray(m).ravel()] & lb.BOUNCE) != 0


def start_channel(lb, lat, d, m, u_in=0.04, seed=1, noise=1e-4):
    """Config 2's start: equilibrium of rho = 1, u = (u_in + U(-noise, noise), 0) in the fluid (numpy
    PCG64 seeded), rho = u = 0 in solid cells."""
    solid = solid_cells(lb, d, m)
    rng = np.random.default_rng(seed)
    ux = np.where(solid, 0.0, u_in + rng.uniform(-noise, noise, d.cells))
    lat.init_equilibrium(np.where(solid, 0.0, 1.0), np.concatenate([ux, np.zeros(d.cells)]))


def start_shanchen(lb, lat, d, m, rho0=0.693, amp=0.01, seed=2):
    """Config 3's start: rho = rho0 + U(-amp, amp) per cell (numpy PCG64 seeded), u = 0."""
    rng = np.random.default_rng(seed)
    lat.init_equilibrium(rho0 + rng.uniform(-amp, amp, d.cells))


def acc_run(lb, wl, storage, steps, start=None, shape=None, hook=None, nearest=False):
    """One run of a workload from its start state; returns fields, FP64 mass before/after, family.
    nearest: 16-bit storage rounds to nearest instead of stochastically (the default)."""
    fn = WORKLOADS[wl][0]
    d, m = fn(lb, storage, shape) if shape is not None else fn(lb, storage)
    if nearest:
        d.rounding = lb.ROUND_NEAREST
    with lb.Lattice(d, m) as lat:
        if start:
            start(lb, lat, d, m)
        m0 = lat.sums()[0]
        extra = hook(lat, steps) if hook else lat.step(steps)
        lat.sync()
        rho, u = lat.macros()
        m1 = lat.sums()[0]
        fam = KERNEL_NAMES.get(lat.kernel(), "unknown")
    return {"d": d, "m": m, "rho": rho, "u": u, "mass0": m0, "mass1": m1, "family": fam, "extra": extra}


def field_errors(lb, runs, ref, names):
    """rel. L2 of u and rho (non-solid cells) of each run against the reference run, and the FP64
    mass drift of each run over its steps."""
    d, m = runs[ref]["d"], runs[ref]["m"]
    keep = ~solid_cells(lb, d, m)
    n = d.cells
    vel = lambda u: np.concatenate([u[k * n:(k + 1) * n][keep] for k in range(d.dim)])  # noqa: E731
    out = {}
    for name in names:
        r = runs[name]
        out[f"rel_l2_u_{name}_vs_f64"] = rel_l2(vel(r["u"]), vel(runs[ref]["u"]))
        out[f"rel_l2_rho_{name}_vs_f64"] = rel_l2(r["rho"][keep], runs[ref]["rho"][keep])
    for name, r in runs.items():
        out[f"mass_drift_{name}"] = (r["mass1"] - r["mass0"]) / r["mass0"]
    out["kernel_family"] = {name: r["family"] for name, r in runs.items()}
    return out


def acc_cavity128(lb):
    """Config 1: D2Q9 lid 128^2, Re 100, 10,000 steps from rest; also the reference's own FP32
    arithmetic (ABSOLUTE mode) against the same FP64 run."""
    runs = {}
    for name, st in (("f64", lb.F64), ("f32", lb.F32), ("f16s", lb.F16S)):
        runs[name] = acc_run(lb, "d2q9_lid_128", st, 10000)
    runs["f16s_nearest"] = acc_run(lb, "d2q9_lid_128", lb.F16S, 10000, nearest=True)
    d, m = wl_cavity128(lb, lb.F32)
    d.arithmetic = lb.ARITH_ABSOLUTE
    with lb.Lattice(d, m) as lat:
        m0 = lat.sums()[0]
        lat.step(10000)
        rho, u = lat.macros()
        runs["f32_reference_arithmetic"] = {"d": d, "m": m, "rho": rho, "u": u, "mass0": m0,
                                            "mass1": lat.sums()[0], "family": "plain"}
    out = field_errors(lb, runs, "f64", ["f32", "f16s", "f16s_nearest", "f32_reference_arithmetic"])
    out["steps"] = 10000
    return out


def channel_hook(probe, avg_steps=20000, every=100):
    """Steps to the end; over the last avg_steps samples u every `every` steps: the time-averaged
    velocity field and u_y at a probe point behind the cylinder (the shedding signal)."""
    def hook(lat, steps):
        lat.step(steps - avg_steps)
        acc = None
        sig = []
        for _ in range(avg_steps // every):
            lat.step(every)
            _, u = lat.macros()
            acc = u.copy() if acc is None else acc + u
            sig.append(u[lat.n + probe])
        return {"u_mean": acc / (avg_steps // every), "probe": np.array(sig), "every": every}
    return hook


def shedding_period(sig, every):
    """Mean spacing of the upward zero crossings of the mean-free signal (linear interpolation), in
    steps; None with fewer than two crossings."""
    x = sig - sig.mean()
    t = [k + x[k] / (x[k] - x[k + 1]) for k in range(len(x) - 1) if x[k] < 0 <= x[k + 1]]
    if len(t) < 2:
        return None
    return float((t[-1] - t[0]) / (len(t) - 1) * every)


def acc_channel(lb, steps=50000):
    """Config 2: D2Q9 channel 1024x256, 50,000 steps from the seeded start.  The vortex street is a limit
    cycle whose phase depends on every rounding since the start, so beside the instantaneous fields it
    compares what the flow settles into: the velocity field averaged over the last 20,000 steps and the
    shedding frequency (Strouhal number St = f d / U) at a probe 100 cells behind the cylinder on the
    centre line."""
    probe = 128 * 1024 + 300
    runs = {}
    for name, st in (("f64", lb.F64), ("f32", lb.F32), ("f16s", lb.F16S)):
        runs[name] = acc_run(lb, "d2q9_channel_1024x256", st, steps, start=start_channel, hook=channel_hook(probe))
    runs["f16s_nearest"] = acc_run(lb, "d2q9_channel_1024x256", lb.F16S, steps, start=start_channel,
                                   hook=channel_hook(probe), nearest=True)
    out = field_errors(lb, runs, "f64", ["f32", "f16s", "f16s_nearest"])
    d, m = runs["f64"]["d"], runs["f64"]["m"]
    keep = np.tile(~solid_cells(lb, d, m), 2)
    ref = runs["f64"]["extra"]["u_mean"][keep]
    for name in ("f32", "f16s", "f16s_nearest"):
        out[f"rel_l2_u_mean_{name}_vs_f64"] = rel_l2(runs[name]["extra"]["u_mean"][keep], ref)
    for name, r in runs.items():
        T = shedding_period(r["extra"]["probe"], r["extra"]["every"])
        out[f"strouhal_{name}"] = None if T is None else 40.0 / (T * 0.04)
        out[f"probe_uy_rms_{name}"] = float(np.std(r["extra"]["probe"]))
    out["steps"] = steps
    out["note"] = ("u_mean: velocity averaged over the last 20,000 steps; Strouhal from the u_y zero crossings "
                   "at (300, 128)")
    return out


def sc_statistics(rho, n):
    """Phase-separation statistics of a density field: the mean densities of the dense and the light
    phase (cells above / below the global mean), the dense-phase fraction, and the domain length
    2 pi sum S(k) / sum |k| S(k) from the structure factor of the density."""
    r = rho.reshape(n, n)
    mean = r.mean()
    dense = r > mean
    S = np.abs(np.fft.fft2(r - mean)) ** 2
    k = 2 * np.pi * np.fft.fftfreq(n)
    kk = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
    S[0, 0] = 0.0
    return {"rho_dense": float(r[dense].mean()), "rho_light": float(r[~dense].mean()),
            "dense_fraction": float(dense.mean()), "domain_length": float(2 * np.pi * S.sum() / (kk * S).sum())}


def acc_shanchen(lb, steps=20000):
    """Config 3: D2Q9 Shan-Chen 1024^2, 20,000 steps from the seeded start.  Spinodal decomposition
    amplifies every rounding difference (the pattern of domains differs in each run), so beside the
    pointwise error the phases' statistics are compared: dense/light densities, dense fraction and
    domain length; the FP64 mass drift of each run is its conservation error."""
    runs = {}
    for name, st in (("f64", lb.F64), ("f32", lb.F32), ("bf16s", lb.BF16S)):
        runs[name] = acc_run(lb, "d2q9_shanchen_1024", st, steps, start=start_shanchen)
    runs["bf16s_nearest"] = acc_run(lb, "d2q9_shanchen_1024", lb.BF16S, steps, start=start_shanchen, nearest=True)
    out = field_errors(lb, runs, "f64", ["f32", "bf16s", "bf16s_nearest"])
    for name, r in runs.items():
        out[f"stats_{name}"] = sc_statistics(r["rho"], 1024)
    out["steps"] = steps
    return out


def acc_mrt256(lb, steps=5000, shape=(256, 256, 256)):
    """Config 4: D3Q27 MRT (Gram-Schmidt) lid cavity 256^3, 5,000 steps from rest."""
    runs = {}
    for name, st in (("f64", lb.F64), ("f32", lb.F32), ("f16s", lb.F16S)):
        runs[name] = acc_run(lb, "d3q27_mrt_gs_lid_256", st, steps, shape=shape)
    runs["f16s_nearest"] = acc_run(lb, "d3q27_mrt_gs_lid_256", lb.F16S, steps, shape=shape, nearest=True)
    out = field_errors(lb, runs, "f64", ["f32", "f16s", "f16s_nearest"])
    out["steps"] = steps
    out["lattice"] = "x".join(map(str, shape))
    return out


def acc_ensemble(lb, steps=1000):
    """Config 5: the F16S batch (one launch per step over every member) against each member's FP64 run
    (stepped alone), after `steps` steps: per-member rel. L2 of u; max, median and the pooled value over
    the members whose FP64 run stays finite (a member that blows up in FP64 too is under-resolved, not a
    storage error, and is listed instead)."""
    members = ensemble_members(lb, lb.F16S)
    batch = lb.Batch([d for d, _, _ in members], [m for _, m, _ in members])
    batch.step(steps)
    batch.sync()
    members64 = ensemble_members(lb, lb.F64)
    errs, num, den, diverged, worst = [], 0.0, 0.0, [], (0.0, "")
    for k, (d, m, name) in enumerate(members):
        _, u16 = batch.macros(k)
        dd, mm, _ = members64[k]
        with lb.Lattice(dd, mm) as lat:
            lat.step(steps)
            _, u64 = lat.macros()
        keep = np.tile(~solid_cells(lb, dd, mm), d.dim)
        if not np.all(np.isfinite(u64[keep])):
            diverged.append(f"{name} (member {k}, tau {1.0 / d.omega:.4f}, FP64 {'and F16S ' if not np.all(np.isfinite(u16[keep])) else ''}non-finite)")
            continue
        e = rel_l2(u16[keep], u64[keep])
        errs.append(e)
        worst = max(worst, (e, name))
        num += float(np.sum((u16[keep] - u64[keep]) ** 2))
        den += float(np.sum(u64[keep] ** 2))
    batch.close()
    return {"rel_l2_u_f16s_vs_f64_max": max(errs), "rel_l2_u_f16s_vs_f64_median": float(np.median(errs)),
            "rel_l2_u_f16s_vs_f64_pooled": float(np.sqrt(num / den)), "members": len(members),
            "members_compared": len(errs), "diverged_in_fp64": diverged, "steps": steps, "worst_member": worst[1]}


ACCURACY = {
    "d2q9_lid_128": acc_cavity128,
    "d2q9_channel_1024x256": acc_channel,
    "d2q9_shanchen_1024": acc_shanchen,
    "d3q27_mrt_gs_lid_256": acc_mrt256,
    "ensemble_config5": acc_ensemble,
}


def accuracy_all(lb, which):
    """Accuracy block of the default run: every configuration at its own size and step count."""
    out = {}
    for name in which:
        t = time.perf_counter()
        out[name] = ACCURACY[name](lb)
        out[name]["seconds"] = time.perf_counter() - t
    return out


def barrier(torch, world):
    if world > 1:
        torch.distributed.barrier()


def reduce_max(torch, value, dev, world):
    """Max over ranks (the job takes as long as its slowest rank)."""
    from lbm_b200.shard import max_over_ranks

    if world <= 1:
        return value
    return max_over_ranks(value, device=f"cuda:{dev}")


# ---------------------------------------------------------------------------------------------
# config 5: batched ensemble
# ---------------------------------------------------------------------------------------------
def ensemble_members(lb, storage, seed=3):
    """48 D2Q9 BGK lid cavities (L uniform in {64, 128, ..., 1024}, Re uniform in [100, 1000], lid 0.1,
    the Rust examples' viscosity rule nu = u 2 L / Re, rust/examples/d2q9_bgk_lid.rs:52) and 16 D3Q27 BGK
    channels (4L, L, L), L uniform in {64, 96, 128, 160, 192}, sphere of diameter L/4 centred in the
    channel, equilibrium inlet 0.04, zero-gradient outlet, nu from Re = 100 on the sphere diameter.  numpy
    PCG64 seeded with `seed`.  (With the C++ rule nu = u L / Re four of the lids -- L = 64 and 128 at
    Re 450-840, tau 0.52-0.55 -- are under-resolved and blow up in FP64 too; with the Rust rule one is.)"""
    rng = np.random.default_rng(seed)
    members = []
    for _ in range(48):
        L = int(rng.integers(1, 17)) * 64
        re = float(rng.uniform(100.0, 1000.0))
        d = lb.make_desc(lb.D2Q9, lb.BGK, storage, (L, L), omega=lb.omega_from_re(0.1, L, re, 1))
        members.append((d, lb.setup_cavity2d(d, 0.1), f"d2q9_lid_{L}"))
    for _ in range(16):
        L = int(rng.choice([64, 96, 128, 160, 192]))
        diam = L / 4.0
        nu = 0.04 * diam / 100.0
        d = lb.make_desc(lb.D3Q27, lb.BGK, storage, (4 * L, L, L), omega=1.0 / (3.0 * nu + 0.5))
        members.append((d, lb.setup_duct3d(d, 0.04, 2.0 * L, L / 2.0, L / 2.0, diam / 2.0), f"d3q27_channel_{L}"))
    return members


def run_ensemble(args, rank, world, local_rank):
    """Config 5: every rank advances its LPT share of the ensemble as one batch (one launch per lattice
    family per step, CUDA graphs); aggregate MLUPS = all cells x steps / max-over-ranks time.  Beside it,
    the same members stepped one lattice at a time with the plain single-lattice path."""
    import torch

    import lbm_b200 as lb
    from lbm_b200.shard import lpt_assign

    dev = local_rank
    torch.cuda.set_device(dev)
    storage = {"f16s": lb.F16S, "f32": lb.F32, "bf16s": lb.BF16S, "f64": lb.F64}[args.storage]
    peak, peak_kind = peaks()
    members = ensemble_members(lb, storage)
    bytes_upd = [algorithmic_bytes_per_cell(d) * d.cells for d, _, _ in members]
    parts = lpt_assign(bytes_upd, world)
    mine = [members[k] for k in parts[rank]]
    total_cells = sum(d.cells for d, _, _ in members)
    total_bytes = sum(bytes_upd)
    my_cells = sum(d.cells for d, _, _ in mine)

    def events_time(stream_handle, fn):
        st = torch.cuda.ExternalStream(stream_handle, device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    batch = lb.Batch([d for d, _, _ in mine], [m for _, m, _ in mine])
    batch.step(max(args.warmup, 1))  # tile autotune + graph capture
    batch.sync()
    torch.cuda.synchronize(dev)
    barrier(torch, world)
    sampler = ClockSampler(gpu_id_for_smi(torch, dev)) if rank == 0 else None
    if sampler:
        time.sleep(0.3)
    el = events_time(batch.stream(), lambda: batch.step(args.steps))
    clocks = sampler.stop() if sampler else None
    torch.cuda.synchronize(dev)
    barrier(torch, world)
    el_max = reduce_max(torch, el, dev, world)
    tile = batch.tile_info()
    mode = {lb.BATCH_TILES: "tiles", lb.BATCH_ROWS: "rows, one launch for both families",
            lb.BATCH_ROWS_PER_FAMILY: "rows, one launch per family"}.get(batch.mode(), "auto")
    launches, group2, group3 = batch.plan()
    batch.close()
    del batch

    # the same members one lattice at a time (plain single-lattice path, autotuned, graphs)
    seq = 0.0
    if not args.no_compare:
        for d, m, _ in mine:
            d.device = dev
            with lb.Lattice(d, m) as lat:
                lat.step(max(args.warmup, 1))
                lat.sync()
                seq += events_time(lat.stream(), lambda: lat.step(args.steps))
        seq = reduce_max(torch, seq, dev, world)

    # the same ensemble in FP32 storage, batched the same way
    el32 = 0.0
    if not args.no_compare and storage != lb.F32:
        mem32 = ensemble_members(lb, lb.F32)
        mine32 = [mem32[k] for k in parts[rank]]
        b32 = lb.Batch([d for d, _, _ in mine32], [m for _, m, _ in mine32])
        b32.step(max(args.warmup, 1))
        b32.sync()
        el32 = reduce_max(torch, events_time(b32.stream(), lambda: b32.step(args.steps)), dev, world)
        b32.close()
        del b32

    value = total_cells * args.steps / el_max / 1e6
    achieved = total_bytes * args.steps / el_max / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el_max * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "ensemble_config5", "description": WORKLOADS["ensemble_config5"][1],
                   "members": len(members), "cells": total_cells, "storage": STORAGE_NAMES[storage],
                   "l2": f"inputs larger than L2: {total_bytes / 2 / 1e9:.2f} GB of populations per buffer set",
                   "parallelism": f"LPT shards x{world}" if world > 1 else "single GPU",
                   "members_per_rank": [len(p) for p in parts], "cells_this_rank": my_cells,
                   "batch_mode": mode, "launches_per_step": launches,
                   "row_group_bytes": {"d2q9": group2, "d3q27": group3}, "tile_width": tile[0], "tiles": tile[1]},
        "roofline": {"bound": "hbm", "achieved": achieved / world, "peak": peak, "unit": "GB/s",
                     "frac": achieved / world / peak, "traffic": None,
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s",
                     "kernel": {"tiles": "k_batch_bgk<D2Q9> + k_batch_bgk<D3Q27>",
                                "rows, one launch for both families": "k_batch_rows_mix",
                                "rows, one launch per family": "k_batch_rows<D2Q9> + k_batch_rows<D3Q27>"}.get(mode, mode),
                     "note": "achieved per GPU: algorithmic bytes of all members / max-over-ranks time / ranks"},
        "gpu_launches": args.steps * launches,
        "clocks": clocks,
    }
    if el32 > 0:
        out["fp32_batched"] = {"value": total_cells * args.steps / el32 / 1e6, "unit": "MLUPS",
                               "ms_per_step": el32 * 1e3 / args.steps}
        out[f"speedup_{STORAGE_NAMES[storage]}_vs_f32"] = el32 / el_max
    if seq > 0:
        out["sequential_plain"] = {"value": total_cells * args.steps / seq / 1e6, "unit": "MLUPS",
                                   "seconds": seq, "note": "each member alone through lbm_step, summed"}
        out["speedup_batched_vs_sequential"] = seq / el_max
    return out


# ---------------------------------------------------------------------------------------------
# the other configurations' throughput (lines beside the headline)
# ---------------------------------------------------------------------------------------------
STORAGES = {"f16s": 1, "f32": 0, "bf16s": 2, "f64": 3}

# (workload, 16-bit storage of the configuration, timed steps)
SMALL_CONFIGS = (("d2q9_lid_128", "f16s", 20000), ("d2q9_channel_1024x256", "f16s", 4000),
                 ("d2q9_shanchen_1024", "bf16s", 2000))


def config_lines(torch, lb, args, dev, world):
    """MLUPS of configs 1-3 (16-bit storage and FP32) and of the config-5 ensemble, each timed like the
    headline (CUDA events on the lattice's stream after warm-up).  Configs 1-3 are L2-resident (their
    populations fit the 126 MB L2), so no HBM roofline applies to them; their achieved GB/s is stated
    against the algorithmic bytes."""
    import copy

    out = {}
    for wl, st16, steps in SMALL_CONFIGS:
        rec = {}
        for stn in (st16, "f32"):
            a = copy.copy(args)
            a.workload, a.steps, a.warmup = wl, steps, max(args.warmup, 3)
            a.kernel, a.block, a.dims, a.size = "auto", 0, "", 0
            d, lat, el, _ = measure(torch, lb, a, STORAGES[stn], dev, world)
            fam = KERNEL_NAMES.get(lat.kernel(), "unknown")
            lat.close()
            del lat
            rec[stn] = {"value": d.cells * steps / el / 1e6, "unit": "MLUPS", "ms_per_step": el * 1e3 / steps,
                        "kernel_family": fam,
                        "achieved_gbs": algorithmic_bytes_per_cell(d) * d.cells * steps / el / 1e9}
            rec["lattice"] = list(d.shape)
            mb = d.cells * d.q * storage_bytes(STORAGES[stn]) * 2 / 1e6
            rec["l2"] = (f"L2-resident ({mb:.1f} MB of populations in both buffers at {stn}); no flush"
                         if fam != "cluster" else
                         f"resident in one thread-block cluster's shared memory ({mb:.1f} MB at {stn}) for up "
                         f"to 4096 steps per launch; HBM/L2 only at launch start and end")
        rec[f"speedup_{st16}_vs_f32"] = rec[st16]["value"] / rec["f32"]["value"]
        rec["steps"] = steps
        out[wl] = rec
    a = copy.copy(args)
    a.workload, a.storage = "ensemble_config5", "f16s"
    e = run_ensemble(a, 0, world, dev)
    keep = ("value", "unit", "ms_per_step", "roofline", "fp32_batched", "speedup_f16s_vs_f32", "sequential_plain",
            "speedup_batched_vs_sequential", "clocks", "gpu_launches", "steps")
    out["ensemble_config5"] = {k: e[k] for k in keep if k in e}
    out["ensemble_config5"]["config"] = {k: e["config"][k] for k in ("members", "cells", "storage", "l2", "batch_mode",
                                                                      "launches_per_step", "row_group_bytes")}
    return out


def run_ours(args, rank, world, local_rank):
    import torch

    import lbm_b200 as lb

    dev = local_rank
    torch.cuda.set_device(dev)
    head_storage = {"f16s": lb.F16S, "f32": lb.F32, "bf16s": lb.BF16S, "f64": lb.F64}[args.storage]
    peak, peak_kind = peaks()

    d, lat, el, clocks = measure(torch, lb, args, head_storage, dev, world, sample_clocks=(rank == 0))
    N = d.cells
    # Shan-Chen: two launches per step, one with the one-pass kernel (the single-pass family); the
    # cluster-resident family: one launch per 4096 steps
    launches_per_step = 2 if d.collision == 2 and lat.kernel() != lb.KERNEL_ROWS else 1
    if lat.kernel() == lb.KERNEL_CLUSTER:
        launches_per_step = -(-args.steps // 4096) / args.steps
    bytes_cell = algorithmic_bytes_per_cell(d)
    value = world * N * args.steps / el / 1e6
    avg_launch_s = el / (args.steps * launches_per_step)
    achieved = bytes_cell * N / launches_per_step / avg_launch_s / 1e9
    traffic = dram_traffic(args.workload, head_storage)
    kernel_family = KERNEL_NAMES.get(lat.kernel(), "unknown")
    block_used = lat.block()
    lat.close()
    del lat

    out = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if head_storage != lb.F64 else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload][1],
                   "lattice": list(d.shape), "cells": N, "storage": STORAGE_NAMES[head_storage],
                   "bytes_per_cell_update": bytes_cell,
                   "l2": f"inputs larger than L2: {N * d.q * storage_bytes(head_storage) / 1e9:.2f} GB per population buffer"
                   if N * d.q * storage_bytes(head_storage) > 126e6 else
                   ("lattice resident in one thread-block cluster's shared memory for up to 4096 steps per launch"
                    if kernel_family == "cluster" else "lattice is L2-resident (no flush)"),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "kernel_family": kernel_family, "block": block_used},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "kernel": ("k_step_sc_window" if d.collision == 2 else "k_step_rows") if kernel_family == "rows"
                     else "k_step_cluster" if kernel_family == "cluster"
                     else {0: "k_step_bgk", 1: "k_step_mrt", 2: "k_step_sc + k_sc_psi"}[d.collision],
                     "bytes_per_launch": bytes_cell * N / launches_per_step},
        "gpu_launches": round(args.steps * launches_per_step),
        "clocks": clocks,
    }
    # FP32 plain beside the 16-bit headline
    if head_storage != lb.F32 and not args.no_compare:
        d32, lat32, el32, clocks32 = measure(torch, lb, args, lb.F32, dev, world, sample_clocks=(rank == 0))
        family32 = KERNEL_NAMES.get(lat32.kernel(), "unknown")
        lat32.close()
        del lat32
        v32 = world * N * args.steps / el32 / 1e6
        b32 = algorithmic_bytes_per_cell(d32)
        a32 = b32 * N / launches_per_step / (el32 / (args.steps * launches_per_step)) / 1e9
        out["fp32_plain"] = {"value": v32, "unit": "MLUPS", "ms_per_step": el32 * 1e3 / args.steps,
                             "kernel_family": family32, "clocks": clocks32,
                             "roofline": {"achieved": a32, "peak": peak, "frac": a32 / peak,
                                          "traffic": dram_traffic(args.workload, lb.F32)}}
        out[f"speedup_{STORAGE_NAMES[head_storage]}_vs_f32"] = value / v32
    if not args.no_e2e:
        out["e2e"] = e2e_measure(torch, lb, args, head_storage, dev, world)
    if rank == 0 and world == 1 and not args.no_configs:
        out["configs"] = config_lines(torch, lb, args, dev, world)
    if rank == 0 and world == 1 and not args.no_accuracy:
        out["accuracy"] = accuracy_all(lb, args.accuracy.split(",") if args.accuracy else list(ACCURACY))
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        O.lib()
        side = 64 if args.workload.startswith("d3q27") else None
        mlups, cells, steps, shape = oracle_mlups(args.workload, args.cpu_seconds, side)
        out["cpu_baseline"] = {"value": mlups, "unit": "MLUPS", "cores": threads(), "kind": "port",
                               "sample": f"{'x'.join(map(str, shape))} lattice of the same workload, {steps} steps, "
                                         f"FP32, {threads()} threads on {cpu_model()}"}
    return out


def run_slab(args, rank, world, local_rank):
    """The workload's lattice split into `world` slabs along its slowest axis (lbm_b200.slab.Slab, one
    rank per GPU, faces over NCCL; with one rank the faces wrap onto the rank itself).  Times the
    overlapped step (interior planes beside the boundary planes and the face exchange) and the
    sequential one (step, then exchange) with CUDA events on the slab's stream, max over ranks, and
    the undivided lattice at one rank.  Strong scaling: the global lattice is fixed."""
    import torch

    import lbm_b200 as lb
    from lbm_b200.slab import Slab

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    storage = STORAGES[args.storage]
    d, m = build_workload(lb, args, storage)
    d.device = local_rank
    _, _, _, w, _ = lb.velocities(d.lattice)
    F0 = np.repeat(np.asarray(w, dtype=np.float32), d.cells)  # rest state

    def timed(slab):
        slab.step(max(args.warmup, 1))
        torch.cuda.synchronize(dev)
        barrier(torch, world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(slab.stream)
        slab.step(args.steps)
        e1.record(slab.stream)
        e1.synchronize()
        el = reduce_max(torch, e0.elapsed_time(e1) / 1e3, dev, world)
        barrier(torch, world)
        return el

    out = {}
    for overlap in (True, False):
        slab = Slab(d, m, F0, rank, world, device=dev, overlap=overlap)
        out[overlap] = (timed(slab), slab.overlap)
        slab.close()
    whole = None
    if world == 1:
        with lb.Lattice(d, m) as lat:
            lat.set_populations(F0)
            lat.step(max(args.warmup, 1))
            lat.sync()
            whole = timed_steps(torch, lat, args.steps, dev)
    el, used = out[True]
    return {
        "metric": METRIC, "value": d.cells * args.steps / el / 1e6, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (rest state)",
        "config": {"workload": args.workload, "storage": args.storage, "shape": list(d.shape),
                   "parallelism": f"slab x{world}", "overlap": used, "reserved_sms": 8,
                   "exchange": "nccl p2p" if world > 1 else "faces wrap onto the one rank",
                   "l2": "inputs larger than L2"},
        "sequential_ms_per_step": out[False][0] / args.steps * 1e3,
        "undivided_ms_per_step": whole / args.steps * 1e3 if whole else None,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="d3q27_mrt_gs_lid_256", choices=sorted(WORKLOADS))
    ap.add_argument("--storage", default="f16s", choices=["f16s", "f32", "bf16s", "f64"])
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--accuracy", default="", help="comma-separated configurations of the accuracy block "
                    f"(default: all of {','.join(ACCURACY)})")
    ap.add_argument("--accuracy-only", action="store_true", help="print the accuracy block alone and exit")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' throughput lines")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=150.0, help="time budget of the reference arm")
    ap.add_argument("--size", type=int, default=0,
                    help="cube side for D3Q27 workloads, square side for d2q9_lid_8192 (default: the config's)")
    ap.add_argument("--dims", default="", help="NXxNYxNZ for D3Q27 workloads, NXxNY for the Shan-Chen one")
    ap.add_argument("--kernel", default="auto", choices=["auto", "plain", "rows", "cluster"], help="step-kernel family")
    ap.add_argument("--rounding", default="stochastic", choices=["stochastic", "nearest"],
                    help="rounding of 16-bit storage in the timed runs")
    ap.add_argument("--block", type=int, default=0, help="fixed block width (default: autotune)")
    ap.add_argument("--slab", action="store_true",
                    help="slab decomposition of the workload over the ranks (overlapped and sequential exchange)")
    args = ap.parse_args()
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit("steps must be >= 1 and warmup >= 0")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    import torch

    if args.accuracy_only:
        import lbm_b200 as lb

        torch.cuda.set_device(local_rank)
        print(json.dumps(accuracy_all(lb, args.accuracy.split(",") if args.accuracy else list(ACCURACY))),
              flush=True)
        return
    if world > 1:
        import datetime

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device(f"cuda:{local_rank}"))
    try:
        if args.slab:
            out = run_slab(args, rank, world, local_rank)
        else:
            out = (run_ensemble if args.workload == "ensemble_config5" else run_ours)(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
