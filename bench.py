#!/usr/bin/env python
"""Throughput of the LES time step on B200: Mpts*steps/s at 256^3.

Headline arm: the mixed-precision step (FP32 fields, FFTs, convection and
SGS; FP64 tridiagonal pressure solve, mean mode and compensated diagnostics)
with the learned SGS closure (8 features -> 64 -> 64 -> Cs^2 on the tcgen05
tensor cores, trained on the GPU from Lagrangian scale-dependent dynamic
(LASD) pairs of the first 30 steps, untimed; the 8 levels next to the wall
keep the LASD procedure, LASD fallback for columns outside the training
range and an LASD check of the closure every 10 updates).
Beside it, the same step with the LASD closure and the plain FP64 GPU step
(LASD) of the same seed: their throughputs and the velocity error between
the headline and FP64 runs are part of the JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one 256^3 domain per GPU, no data-path
collective): weak scaling.  The reference arm (--impl reference) times the
CPU FP64 restatement of the reference algorithm on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpts*steps/s at 256^3 (LES time step, FP32 + learned SGS closure vs plain FP64 GPU)"
UNIT = "Mpts*steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--grid-n", dest="n", type=int, default=256, help="grid nx = ny (= nz unless --nz)")
    ap.add_argument("--nz", type=int, default=None, help="vertical levels (default: --n)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--closure", default="mlp", choices=["mlp", "lasd"], help="SGS closure of the headline arm")
    ap.add_argument("--train-steps", type=int, default=30, help="LASD steps that produce the training pairs")
    ap.add_argument("--train-epochs", type=int, default=4)
    ap.add_argument("--wall-levels", type=int, default=8,
                    help="levels next to the wall that keep the LASD procedure under the learned closure")
    ap.add_argument("--train-batch-tiles", type=int, default=16, help="training batch = 128 x this")
    ap.add_argument("--pressure-slabs", type=int, default=1,
                    help="solve the pressure columns by the partition method over this many row blocks")
    ap.add_argument("--train-protocol", default="short", choices=["short", "long"],
                    help="short: pairs of the first --train-steps LASD steps (default); long: the learned-closure "
                         "configuration's protocol, ~5e7 (invariant, Cs^2) pairs (10 %% held out) drawn evenly "
                         "from 2000 LASD steps")
    ap.add_argument("--case", default="abl", choices=["abl", "scalar", "cbl"],
                    help="abl: the headline (neutral channel, 256^3); scalar: config 2 (FP64, passive scalar "
                         "with the dynamic Prandtl model, 128^3); cbl: config 5 (convective boundary layer, "
                         "512x512x256: heat flux, inversion, buoyancy, sponge)")
    a = ap.parse_args()
    CASES = {"abl": {}, "scalar": dict(n=128, precision="fp64", closure="lasd", no_fp64=True),
             "cbl": dict(n=512, nz=256)}
    for k, v in CASES[a.case].items():
        if k in ("n", "nz") and getattr(a, k) not in (None, 256):
            continue  # explicit grid sizes win
        setattr(a, k, v)
    if not hasattr(a, "precision"):
        a.precision = "mixed"
    return a


# ----------------------------------------------------------------- helpers
def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [x.strip() for x in l.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 0, 1
    import datetime

    import torch
    import torch.distributed as dist

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = "nccl" if args.impl == "ours" else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600),
                            **({"device_id": torch.device("cuda", local)} if backend == "nccl" else {}))
    return dist, rank, local, ws


def max_over_ranks(dist, x: float, local: int) -> float:
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local):
    if dist is not None:
        import torch

        if dist.get_backend() == "nccl":
            dist.barrier(device_ids=[local])
        else:
            dist.barrier()


def cs2_clip(p) -> float:
    """Upper clip of the dynamic Cs^2 on grids with 512-point rows: from the
    synthetic start the LASD coefficient near the nearly laminar lid grows
    without bound there (the reference has no clip) and the explicit SGS
    diffusion loses stability within ~100 steps; 0.25 (Cs <= 0.5) keeps it."""
    return 0.25 if max(p.nx, p.ny) >= 512 else 0.0


def setup_case(les, p, args, seed: int):
    """Initial state of a bench case: the log-law velocity with seeded noise,
    and for the scalar cases theta, its model and the forcing."""
    from new_repo_b200 import inversion_noise, log_law_noise, scalar_linear_noise

    les.set_initial_conditions(*log_law_noise(p, seed=seed))
    if args.pressure_slabs > 1:
        les.set_pressure_slabs(args.pressure_slabs)
    if cs2_clip(p):
        les.set_cs2_max(cs2_clip(p))
    if args.case == "scalar":
        # config 2: passive scalar on a linear profile (+-0.01 noise), zero wall
        # flux, the profile's gradient at the lid, dynamic Prandtl model
        les.scalar_init(surface_flux=0.0, top_gradient=1.0, buoyancy=0.0, sgs="dynamic")
        les.scalar_set_initial(scalar_linear_noise(p, seed=seed))
    elif args.case == "cbl":
        # config 5: surface heat flux 0.24, inversion of 0.01 K/m above z = 0.5
        # (10 K per unit height with z_i = 1000 m), +-0.1 K noise below z = 0.1,
        # buoyancy g z_i / (theta_0 u*^2) with theta_0 = 300 K, sponge in the
        # top 20 % (sponge_damping.f90 profile)
        les.scalar_init(surface_flux=0.24, top_gradient=10.0, buoyancy=9.81 * 1000.0 / 300.0, sgs="dynamic")
        les.scalar_set_initial(inversion_noise(p, seed=seed))
        les.sponge_init(0.8)


def run_params(n: int, nz: int | None = None):
    from new_repo_b200 import RunParams

    # 2pi x 2pi x 1 channel, log-law wall (z0 = 1e-4), dp/dx = -1, LASD SGS
    # (cs_count = 5; the dynamic procedure starts at step 5), 3/2 dealiasing
    return RunParams(nx=n, ny=n, nz=nz or n, dt=1e-4, lbc_dz0=1e-4, pfx=1.0, sgs_model="dyn_LagScaleDep",
                     cs_count=5, dyn_init=5, lbc_special="wall_law", wall_model="wall_filter", dealias="padd")


# --------------------------------------------------------------- our arm
def timed_steps(les, k: int) -> float:
    les.sync()
    les.event_record(0)
    les.step(k)
    les.event_record(1)
    return les.event_elapsed(0, 1)


def run_ours(args, dist, rank, local, ws):
    import numpy as np

    from new_repo_b200 import LES, log_law_noise

    p = run_params(args.n, args.nz)
    npts = p.nx * p.ny * p.nz
    K, W = args.steps, max(args.warmup, 3)
    out = {}

    # ---- headline: mixed precision, learned closure trained on the GPU ----
    les = LES(p, precision=args.precision, device=local)
    setup_case(les, p, args, rank)
    T = args.train_steps if args.closure == "mlp" else 0
    if T and args.train_protocol == "long":
        T = 2000
    train = (train_closure(les, p, T, args.train_epochs, args.train_batch_tiles,
                           target_pairs=5e7 if args.train_protocol == "long" else None) if T else None)
    if T:
        les.mlp_set_wall_levels(args.wall_levels)
        train["wall_levels"] = args.wall_levels
    les.step(W)
    les.sync()
    barrier(dist, local)
    n0 = les.launch_count()
    with ClockSampler(local) as clk:
        ms = timed_steps(les, K)
    n1 = les.launch_count()
    barrier(dist, local)
    ms = max_over_ranks(dist, ms, local)
    value = npts * K * ws / (ms / 1e3) / 1e6
    # ---- a second timed pass of K steps with per-launch events on the
    #      state's stream: the dominant kernel's roofline and the per-kernel
    #      breakdown (the headline above ran without the events) ----
    les.profile(True)
    ms_prof = timed_steps(les, K)
    prof = les.profile_report()
    les.profile(False)
    status = les.status()
    top = max(prof.items(), key=lambda kv: kv[1]["ms"])
    label, rec = top
    avg_ms = rec["ms"] / rec["launches"]
    achieved = rec["bytes_per_launch"] / (avg_ms / 1e3) / 1e9
    pk, pk_kind = peaks()
    roof = {"kernel": label, "bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
            "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4), "peak_source": pk_kind,
            "traffic": ncu_traffic(label), "avg_launch_ms": round(avg_ms, 4),
            "algorithmic_bytes_per_launch": rec["bytes_per_launch"], "share_of_step": round(rec["ms"] / ms_prof, 4),
            "timed_in": f"a second pass of {K} steps with per-launch CUDA events ({ms_prof / K:.4f} ms/step)"}
    # step-level: algorithmic bytes per step (105 F + 28 F / cs_count, F = N * 4 B)
    F = npts * (8.0 if args.precision == "fp64" else 4.0)
    step_bytes = (105.0 + 28.0 / p.cs_count) * F
    prof_top = sorted(({"kernel": k, "ms_per_step": round(v["ms"] / K, 4), "launches_per_step": v["launches"] / K,
                        "gbs": round(v["bytes_per_launch"] * v["launches"] / (v["ms"] / 1e3) / 1e9, 1)}
                       for k, v in prof.items()), key=lambda d: -d["ms_per_step"])[:12]
    step_roof = {"algorithmic_bytes_per_step": step_bytes,
                 "achieved_gbs": round(step_bytes / (ms / K / 1e3) / 1e9, 1),
                 "frac": round(step_bytes / (ms / K / 1e3) / 1e9 / pk["hbm_gbs"], 4)}
    # ---- untimed continuation to the comparison step (>= 100 steps); the
    #      closure's LASD check (every 10 updates = 50 steps) also runs at the
    #      last update of the continuation ----
    S = max(100, T + W + 2 * K)
    done = T + W + 2 * K
    if args.no_fp64 and train is None:
        S = done  # nothing is compared at step S
    if train is not None:
        upd = [j for j in range(done + 1, S + 1) if j >= p.dyn_init and j % p.cs_count == 0]
        if upd:
            les.step(upd[-1] - done - 1)
            les.mlp_set_check_every(1)
            les.step(1)
            les.mlp_set_check_every(10)
            done = upd[-1]
    les.step(S - done)
    snap = snapshot(les, p) if not args.no_fp64 else None
    if train is not None:
        train.update(les.mlp_info())
        prof_chk = les.mlp_check_profile()
        nb = min(args.wall_levels, len(prof_chk) - 1)
        kmax = nb + int(np.argmax(prof_chk[nb:]))
        # levels 1..wall_levels run LASD: their entries are the closure's
        # error where it is not used (why the band exists)
        train["check_profile_max_above_wall_band"] = {"level": kmax + 1,
                                                      "rms_log_error": round(float(prof_chk[kmax]), 4)}
        train["check_profile_levels_1_12"] = [round(float(x), 4) for x in prof_chk[:12]]
        train["check_profile_top_12"] = [round(float(x), 4) for x in prof_chk[-12:]]
        train["check_after_steps"] = S

    # ---- end to end through the public API with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(les, p, min(K, 20), local)
    les.close()

    # ---- the same step with the LASD closure (mixed precision) ----
    lasd = None
    snap_l = None
    if args.closure == "mlp" and not args.no_fp64:
        ll = LES(p, precision="mixed", device=local)
        setup_case(ll, p, args, rank)
        ll.step(T + W)
        ll.sync()
        msl = max_over_ranks(dist, timed_steps(ll, K), local)
        ll.step(S - (T + W + K))
        snap_l = snapshot(ll, p)
        ll.close()
        lasd = {"value": round(npts * K * ws / (msl / 1e3) / 1e6, 2), "ms_per_step": round(msl / K, 4),
                "speedup_of_headline": round(msl / ms, 3)}

    # ---- plain FP64 GPU step (LASD), same seed, compared at step S ----
    fp64 = None
    if not args.no_fp64:
        l64 = LES(p, precision="fp64", device=local)
        setup_case(l64, p, args, rank)
        l64.step(T + W)
        l64.sync()
        ms64 = timed_steps(l64, K)
        l64.step(S - (T + W + K))
        snap64 = snapshot(l64, p)
        l64.close()
        ms64 = max_over_ranks(dist, ms64, local)
        vel = ("u", "v", "w")
        num = sum(float(((snap[n] - snap64[n]) ** 2).sum()) for n in vel)
        den = sum(float((snap64[n] ** 2).sum()) for n in vel)
        prof_m = snap["u"].mean(axis=(1, 2))
        prof_r = snap64["u"].mean(axis=(1, 2))
        fp64 = {"value": round(npts * K * ws / (ms64 / 1e3) / 1e6, 2), "ms_per_step": round(ms64 / K, 4),
                "speedup_of_headline": round(ms64 / ms, 3),
                "velocity_rms_rel_error": float(math.sqrt(num / den)),
                "mean_profile_drift": float(np.abs(prof_m - prof_r).max() / np.abs(prof_r).max()),
                "after_steps": S,
                "per_field_error_of_headline": field_errors(snap, snap64),
                "velocity_error_by_level_band": level_band_errors(snap, snap64)}
        if snap_l is not None:
            lasd["per_field_error_vs_fp64"] = field_errors(snap_l, snap64)
            lasd["after_steps"] = S

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_sample(args.n)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f64" if args.precision == "fp64" else
                      "f32 (fields, FFTs, convection, SGS) + f64 (pressure solve, mean mode, diagnostics)"),
            "data": "synthetic: log-law profile + seeded uniform +-0.1 noise (counter-based hash)"
                    + {"abl": "", "scalar": "; scalar: linear profile + seeded +-0.01 noise",
                       "cbl": "; temperature: inversion above z = 0.5 + seeded +-0.1 K noise below z = 0.1"}[args.case],
            "config": {"workload": f"LES time step {p.nx}x{p.ny}x{p.nz}, 3/2 dealiasing, "
                                   + (f"learned SGS closure above level {args.wall_levels} (LASD on the "
                                      f"{args.wall_levels} wall levels, LASD fallback/check)" if T else "LASD SGS")
                                   + " (cs_count 5, closure update every 5th step), log-law wall, "
                                   + ("FP64" if args.precision == "fp64" else "FP32+FP64-pressure")
                                   + {"abl": "", "scalar": ", passive scalar with the dynamic Prandtl model",
                                      "cbl": ", convective boundary layer: surface heat flux 0.24, capping "
                                             "inversion, buoyancy, top-20 % sponge, dynamic Prandtl model"}[args.case],
                       "case": args.case, "grid": [p.nx, p.ny, p.nz], "dt": p.dt_nd, "cs2_max": cs2_clip(p) or None,
                       "pressure_slabs": args.pressure_slabs,
                       "sgs_model": "mlp" if T else p.sgs_model,
                       "precision": args.precision, "parallelism": f"replicas x{ws}",
                       "l2": "inputs larger than L2 (>= 9 GB of fields per step)"},
            "roofline": roof, "step_roofline": step_roof, "profile_top": prof_top,
            "e2e": e2e, "gpu_launches": n1 - n0, "fp64_gpu": fp64, "lasd_mixed": lasd, "closure_training": train,
            "cpu_baseline": cpu,
            "clocks": clk.summary(), "status_bits": status,
        }
        print(json.dumps(line), flush=True)


COMPARED = ("u", "v", "w", "p", "cs_opt2", "txz", "rhsx")


def snapshot(les, p) -> dict:
    """Interior levels 1..nz of the fields the precision comparison reports."""
    return {n: les.download(n, 1, p.nz) for n in COMPARED}


def field_errors(a: dict, b: dict) -> dict:
    """Per field: RMS and max of a - b relative to the RMS / max of b."""
    import numpy as np

    out = {}
    for n in COMPARED:
        d = a[n] - b[n]
        out[n] = {"rms_rel": float(np.sqrt((d * d).mean() / max((b[n] * b[n]).mean(), 1e-300))),
                  "max_rel": float(np.abs(d).max() / max(np.abs(b[n]).max(), 1e-300))}
    return out


def level_band_errors(a: dict, b: dict, nbands: int = 8) -> dict:
    """Where the velocity differs: RMS of a - b over each of nbands equal bands
    of levels (1..nz, bottom to top), relative to the RMS of b over all
    levels, for u, v, w."""
    import numpy as np

    out = {}
    for n in ("u", "v", "w"):
        ref = max(float((b[n] * b[n]).mean()), 1e-300)
        bands = np.array_split(np.arange(b[n].shape[0]), nbands)
        out[n] = [round(float(np.sqrt(((a[n][k] - b[n][k]) ** 2).mean() / ref)), 5) for k in bands]
    return out


def train_closure(les, p, T: int, epochs: int = 4, tiles: int = 16, target_pairs: float | None = None) -> dict:
    """Untimed: T LASD steps; the (features, log Cs^2) pairs of consecutive
    update steps (the first update only records the coefficient) train the
    closure on the GPU; the state then continues with the learned closure.
    Short protocol: one point in 8, every point of the 8 lowest levels, the
    two wall levels 4 times.  With target_pairs: one point in a stride that
    spreads ~target_pairs (train + 10 % validation) evenly over the updates."""
    les.mlp_init(0)
    nupd = sum(1 for j in range(1, T + 1) if j >= p.dyn_init and j % p.cs_count == 0) - 1
    if target_pairs:
        npts = p.nx * p.ny * (p.nz + 1)
        stride = max(1, int(math.ceil(nupd * npts / target_pairs)))
        collect = dict(stride=stride, dense_levels=0, wall_repeat=1)
        les.mlp_reset_data(int(target_pairs * 1.02))
    else:
        collect = dict(stride=8, dense_levels=8, wall_repeat=4)
        les.mlp_reset_data(1 << 24)
    t0 = time.perf_counter()
    for _ in range(T):
        les.step(1)
        if les.jt_total >= p.dyn_init and les.jt_total % p.cs_count == 0:  # consecutive updates
            les.mlp_collect(seed=les.jt_total, **collect)
    les.sync()
    t1 = time.perf_counter()
    ntr, nva = les.mlp_counts()
    les.mlp_fit_stats()
    losses, val = les.mlp_train(epochs=epochs, tiles_per_step=tiles, lr=2e-3)
    les.sync()
    t2 = time.perf_counter()
    les.set_sgs_model("mlp")
    return {"lasd_steps": T, "collect": collect, "train_pairs": ntr, "validation_pairs": nva, "epochs": epochs,
            "batch": tiles * 128, "train_loss": [round(float(x), 4) for x in losses],
            "validation_loss": round(val, 4), "collect_s": round(t1 - t0, 3), "train_s": round(t2 - t1, 3)}


def ncu_traffic(label: str):
    """dram bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "traffic.json"
    try:
        d = json.loads(f.read_text())
        return d.get(label)
    except Exception:
        return None


def run_e2e(les, p, K: int, local: int):
    """K steps through the public API with the velocity state held in
    page-locked host memory (the drop-in boundary: the host arrays stay
    authoritative): per step H2D u,v,w -> les_step -> D2H u,v,w + diagnostics,
    one les_step_host call per step (the copies back of a step and the copies
    in of the next overlap, one per direction of the host link)."""
    import torch

    L = p.nz + 2
    shape = (L, p.ny, p.nx)
    host = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    diag = torch.empty(4, dtype=torch.float64, pin_memory=True)
    names = ("u", "v", "w")
    for h, n in zip(host, names):
        les.download_async(n, h.data_ptr())
    les.sync()
    les.event_record(2)
    t0 = time.perf_counter()
    les.step_host(host[0].data_ptr(), host[1].data_ptr(), host[2].data_ptr(), diag.data_ptr(), n=K)
    les.event_record(3)  # ordered after the last copies back
    les.sync()
    wall = time.perf_counter() - t0
    ms = les.event_elapsed(2, 3)
    npts = p.nx * p.ny * p.nz
    bytes_io = 3 * L * p.ny * p.nx * 8
    return {"value": round(npts * K / (ms / 1e3) / 1e6, 2), "unit": UNIT, "h2d_bytes_per_step": bytes_io,
            "d2h_bytes_per_step": bytes_io + 32, "steps": K, "ms_per_step": round(ms / K, 4),
            "host_wall_ms_per_step": round(wall * 1e3 / K, 4)}


# --------------------------------------------------------- CPU baseline
def cpu_sample(n: int):
    """The compiled FP64 oracle (oracle/cpu_step.cpp, OpenMP on every host
    core) on one plain step and one dynamic-update step of an n x n x 32 slab
    of the workload, amortised over cs_count = 5."""
    from oracle import cpu_step as CS
    from oracle import les_oracle as O

    cores = os.cpu_count() or 1
    p = O.Params(nx=n, ny=n, nz=32, dt=1e-4, dyn_init=1, cs_count=2)
    cs = CS.CpuStep(p, threads=cores)
    cs.mirror(O.make_state(p))
    t = []
    for _ in range(4):  # plain, F-initialising update, plain, interpolating update
        t0 = time.perf_counter()
        cs.step()
        t.append(time.perf_counter() - t0)
    cs.close()
    t_plain = 0.5 * (t[0] + t[2])
    t_upd = t[3]
    per_step = (4 * t_plain + t_upd) / 5.0
    pts = p.nx * p.ny * p.nz
    return {"value": round(pts / per_step / 1e6, 4), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"C++ FP64 port of the oracle (oracle/cpu_step.cpp, OpenMP, {cores} threads), "
                      f"{n}x{n}x32 slab: plain step {t_plain:.3f} s, dynamic-update step {t_upd:.3f} s, "
                      f"amortised 4:1 (cs_count 5)"}


# -------------------------------------------------------- reference arm
def run_reference(args, dist, rank, ws):
    """The reference's algorithm on the host cores: the compiled FP64 port
    (oracle/cpu_step.cpp, OpenMP on every core) stepping an n x n x 32 slab of
    the workload (one eighth of the 256^3 grid's levels)."""
    if rank != 0:
        return
    from oracle import cpu_step as CS
    from oracle import les_oracle as O

    cores = os.cpu_count() or 1
    n = args.n
    nz = 32
    p = O.Params(nx=n, ny=n, nz=nz, dt=1e-4, dyn_init=5, cs_count=5)
    cs = CS.CpuStep(p, threads=cores)
    cs.mirror(O.make_state(p))
    W, K = max(args.warmup, 3), args.steps
    cs.step(W)
    t0 = time.perf_counter()
    cs.step(K)
    dt = time.perf_counter() - t0
    cs.close()
    pts = p.nx * p.ny * p.nz
    v = pts * K / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": ws,
            "steps": K, "warmup": W, "ms_per_step": round(dt * 1e3 / K, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"LES time step, {n}x{n}x{nz} slab of the {n}^3 workload per sample step",
                       "grid": [n, n, nz]},
            "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"full time steps of a {n}x{n}x{nz} slab (LASD update every 5th step), "
                                       f"C++ FP64 port of the oracle with OpenMP on {cores} threads; the Fortran "
                                       "reference cannot be built here (no Fortran compiler, MPI, FFTW or "
                                       "2DECOMP&FFT)"},
            "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    dist, rank, local, ws = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, dist, rank, ws)
        else:
            run_ours(args, dist, rank, local, ws)
    finally:
        if dist is not None:
            barrier(dist, local)
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
