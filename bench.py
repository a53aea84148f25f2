#!/usr/bin/env python
"""Throughput of the PLM/minmod + HLLC + SSP-RK2 hydro step on B200.

Workload: 3D 256^3 periodic box (16,777,216 cells), seeded smooth random state,
gamma = 5/3, CFL 0.4; each step is one SSP-RK2 step with the CFL dt recomputed
on the device from the new state.  Metric: Mcell-updates/s (cells x steps / s),
whole job.  Both precision modes run: VB_MIXED (float32 reconstruction and
HLLC, float64 state) is the headline `value`; VB_FP64 (bit-identical to the
reference's float64 arithmetic) is reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 the script runs under torchrun, one rank per GPU; every rank
integrates its own independent 256^3 instance (weak scaling, no data-path
collective) and rank 0 prints the max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "vespa.jl_b200")]

METRIC = ("Mcell-updates/s 3D 256³ PLM+HLLC RK2 (fp64 vs fp32/fp64 split); %HBM; adj/fwd")
UNIT = "Mcell-updates/s"
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_CELL_STAGE = {1: 80, 2: 120}  # 5 float64 fields: stage 1 R(U)+W(U1), stage 2 R(U1)+R(U)+W(U)


def workload(n: int) -> str:
    """The headline workload's name, printed identically by both arms."""
    return (f"3D {n}^3 periodic PLM/minmod+HLLC SSP-RK2, gamma 5/3, CFL 0.4, "
            "dt recomputed each step")


DATA = ("synthetic: seeded smooth random periodic state (rho = 1 + 0.3 x mean of 8 random sine "
        "modes, velocity components uniform in [-0.5, 0.5], p = 1 + 0.2 U[-1, 1]); no dataset")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256, help="cells per axis of the cube")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plane", action="store_true",
                    help="skip the 2D 4096^2 throughput run")
    ap.add_argument("--no-amr", action="store_true",
                    help="skip the Sedov 48^2 AMR run")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the KH 512^2 adjoint timing and finite-difference check")
    ap.add_argument("--no-gravity", action="store_true",
                    help="skip the 256^3 self-gravity run")
    ap.add_argument("--no-bflux", action="store_true",
                    help="skip the 256^3 boundary-flux recording run")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 64-box batch run")
    ap.add_argument("--no-muscl", action="store_true",
                    help="skip the 256^3 PPMKernels MUSCL run")
    ap.add_argument("--workload", choices=["cube", "batch64", "slab", "plane", "adjoint", "amr",
                                           "gravity", "muscl"],
                    default="cube",
                    help="cube: the 256^3 headline line (with the plane, adjoint, AMR, gravity "
                         "and MUSCL sections); batch64: 64 uneven Riemann boxes in one batch; "
                         "slab: one grid split in z slabs across the ranks (strong scaling); "
                         "plane, adjoint, amr, gravity, muscl: that section alone")
    return ap.parse_args()


# ----------------------------------------------------------------- ranks
class Ranks:
    """One process per GPU (torchrun env vars).  NCCL on GPUs; gloo (CPU
    tensors) when no GPU is present, which the multi-rank host tests use."""

    def __init__(self, n_gpus: int, backend: str | None = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = f"cuda:{self.local}"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.dist = dist
            self.torch = torch

    def barrier(self):
        if self.dist:
            if self.device == "cpu":
                self.dist.barrier()
            else:
                self.dist.barrier(device_ids=[self.local])

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


def weak_scaling_value(cells_per_rank: int, world: int, steps: int, ms_max: float) -> float:
    """Whole-job Mcell-updates/s: all ranks' cells x steps over the slowest
    rank's device time."""
    return cells_per_rank * world * steps / (ms_max / 1e3) / 1e6


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel: str, cells: int):
    """Per-launch DRAM traffic of `kernel` scaled to `cells`: the
    `traffic_bytes_per_cell <kernel> <B>` line of a committed ncu summary
    under profiles/ (dram__bytes_read.sum + dram__bytes_write.sum of one
    captured launch divided by its cells), or None."""
    import glob
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        try:
            with open(p) as f:
                for ln in f:
                    parts = ln.split()
                    if len(parts) == 3 and parts[0] == "traffic_bytes_per_cell" \
                            and parts[1] == kernel:
                        return round(float(parts[2]) * cells)
        except (OSError, ValueError):
            continue
    return None


# ----------------------------------------------------------------- CPU baseline
def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def oracle_rate(n: int, steps: int, budget_s: float, nthreads: int):
    """Oracle (per-cell gather, OpenMP) Mcell-updates/s on an n^3 sample of the
    benchmark's generator; runs up to `steps` RK2 steps or until `budget_s`."""
    from oracle import oracle as O
    import vespa_b200 as vb
    prob = vb.smooth_random_problem((n, n, n))
    U = vb.initial_state(prob)
    g = O.grid_from_problem(prob)
    done, t0 = 0, time.perf_counter()
    while done < steps:
        dt = O.compute_dt(g, U)
        O.step(g, U, dt, mode=1, nthreads=nthreads)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return n ** 3 * done / el / 1e6, done, el


def choose_sample(nthreads: int, target_s: float):
    """Largest cube from the ladder whose single step fits target_s."""
    from oracle import oracle as O
    O.build()
    rate, _, _ = oracle_rate(32, 1, 60.0, nthreads)  # Mcell-updates/s estimate
    n = 32
    for cand in (48, 64, 96, 128, 192, 256):
        if cand ** 3 / (rate * 1e6) <= target_s:
            n = cand
    return n, rate


def oracle_rate_serial(dims, budget_s: float):
    """The oracle's faithful serial path (face enumeration in the reference's
    order, one thread, like the reference's loop): Mcell-updates/s."""
    from oracle import oracle as O
    import vespa_b200 as vb
    prob = vb.smooth_random_problem(dims)
    U = vb.initial_state(prob)
    g = O.grid_from_problem(prob)
    done, t0 = 0, time.perf_counter()
    while True:
        O.step(g, U, O.compute_dt(g, U), mode=0)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return prob.ncell * done / el / 1e6, done, el


def cpu_baseline(nthreads: int) -> dict:
    n, _ = choose_sample(nthreads, 6.0)
    rate, done, el = oracle_rate(n, 64, 15.0, nthreads)
    ser, sdone, sel = oracle_rate_serial((64, 64, 64), 3.0)
    ser2, s2done, s2el = oracle_rate_serial((512, 512), 3.0)
    return {"value": round(rate, 3), "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{done} RK2 step(s) of a {n}^3 periodic box from the same generator "
                      f"({el:.1f} s), C oracle per-cell gather with OpenMP",
            "serial": {"value": round(ser, 3), "cores": 1,
                       "sample": f"{sdone} step(s) of 64^3, faithful serial face loop ({sel:.1f} s)"},
            "serial_2d": {"value": round(ser2, 3), "cores": 1,
                          "sample": f"{s2done} step(s) of 512^2 (the 4096^2 plane's generator), "
                                    f"faithful serial face loop ({s2el:.1f} s)"}}


def run_reference(args, ranks: Ranks):
    """--impl reference: the CPU restatement of the reference's algorithm (the
    reference's Julia path cannot run on this box) on all host cores."""
    if ranks.rank != 0:
        return
    nthreads = cpu_threads()
    n, rate0 = choose_sample(nthreads, 4.0)
    from oracle import oracle as O
    import vespa_b200 as vb
    prob = vb.smooth_random_problem((n, n, n))
    U = vb.initial_state(prob)
    g = O.grid_from_problem(prob)
    for _ in range(args.warmup):
        O.step(g, U, O.compute_dt(g, U), mode=1, nthreads=nthreads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.step(g, U, O.compute_dt(g, U), mode=1, nthreads=nthreads)
    el = time.perf_counter() - t0
    value = n ** 3 * args.steps / el / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(el / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": {"workload": workload(args.n),
                   "sample": f"each timed step advances a {n}^3 box of the same generator "
                             f"(CPU-bounded sample of the {args.n}^3 workload)",
                   "cells_per_step": n ** 3, "parallelism": f"{nthreads} host threads"},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": nthreads,
                         "kind": "port",
                         "sample": f"{args.steps} timed RK2 steps of a {n}^3 box; the "
                                   "reference's Julia path cannot run here (no Julia), so the "
                                   "C restatement of its algorithm stands in"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- our arm
def run_ours(args, ranks: Ranks):
    import numpy as np
    import vespa_b200 as vb

    n = args.n
    cells = n ** 3
    K, W = args.steps, args.warmup
    ctx = vb.Context(ranks.local)
    prob = vb.smooth_random_problem((n, n, n), seed=vb.problem.DEFAULT_SEED + ranks.rank)
    U0 = vb.initial_state(prob)
    mesh = vb.B200Mesh(prob.dims, prob.domain)
    out = {}
    clocks = None
    finals = {}
    sampler = ClockSampler(ranks.local)  # spans both precisions' timed regions
    # started ahead of the timed regions: the sampler's own start-up (process
    # launch, NVML initialisation) once fell inside the short fp64 region and
    # stretched it by up to 2x
    sampler.start()
    # GPU warm-up ahead of the autotuner and the timed regions: in a fresh
    # process the first few hundred milliseconds of stepping ran up to 15 %
    # slower (float64 256^3: 4.34 against 3.82 ms per step for the same
    # configuration measured right after), which skewed both the autotuner's
    # choice and the first timed region
    warm = vb.Simulation(mesh, prob, precision="fp64", ctx=ctx, initial=U0)
    t_end = time.perf_counter() + 2.0
    while time.perf_counter() < t_end:
        vb.run_steps_async(warm, 8)
        ctx.synchronize()
    warm.close()
    drift = {}
    for prec in ("fp64", "mixed"):
        sim = vb.Simulation(mesh, prob, precision=prec, ctx=ctx, initial=U0)
        tot0 = np.array(vb.conserved_totals(sim))
        kz, _ = sim.autotune(3)  # setup: pick the z-chunk; state and clock restored
        vb.run_steps_async(sim, W)
        ctx.synchronize()
        ranks.barrier()
        l0 = ctx.launch_count
        ctx.mark(0)
        vb.run_steps_async(sim, K)
        ctx.mark(1)
        ms = ctx.elapsed_ms(0, 1)
        launches = ctx.launch_count - l0
        if prec == "mixed":
            clocks = sampler.stop()
        ranks.barrier()
        ms_max = ranks.max(ms)
        finals[prec] = sim.state()[0]  # density after W + K steps, for the L1 check
        # conservation over the W + K steps of this periodic box: relative
        # drift of mass and energy (the momenta start near zero)
        tot1 = np.array(vb.conserved_totals(sim))
        drift[prec] = {"mass": float(abs(tot1[0] - tot0[0]) / abs(tot0[0])),
                       "energy": float(abs(tot1[4] - tot0[4]) / abs(tot0[4]))}
        out[prec] = {"ms": ms_max, "launches": launches, "kernel": sim.kernel, "kz": kz,
                     "taper": sim.taper, **sim.profile_step(5)}
        sim.close()
    # accuracy statement: density L1 of the mixed path against float64
    l1_mixed = float(np.sum(np.abs(finals["mixed"] - finals["fp64"])) /
                     np.sum(np.abs(finals["fp64"])))
    del finals

    # end to end through the public API: pinned host state in, K steps, state out
    import torch
    h_in = torch.empty((5, cells), dtype=torch.float64, pin_memory=True)
    h_out = torch.empty((5, cells), dtype=torch.float64, pin_memory=True)
    h_in.numpy()[...] = U0
    sim = vb.Simulation(mesh, prob, precision="mixed", ctx=ctx, initial=U0)
    ranks.barrier()
    ctx.mark(2)
    sim.upload(h_in.numpy())
    vb.evolve(sim, tfinal=math.inf, max_steps=K)
    sim.state(out=h_out.numpy())
    ctx.mark(3)
    e2e_ms = ranks.max(ctx.elapsed_ms(2, 3))
    sim.close()

    hbm, hbm_kind = measured_hbm()
    mixed = out["mixed"]
    total_cells = cells * ranks.world
    value = weak_scaling_value(cells, ranks.world, K, mixed["ms"])
    fp64_value = weak_scaling_value(cells, ranks.world, K, out["fp64"]["ms"])

    def roofline(d, kname):
        bytes_launch = BYTES_PER_CELL_STAGE[2] * cells
        achieved = bytes_launch / (d["ms_stage2"] / 1e3) / 1e9
        traffic = ncu_traffic(kname, cells)
        b1 = BYTES_PER_CELL_STAGE[1] * cells
        a1 = b1 / (d["ms_stage1"] / 1e3) / 1e9
        return {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_source": hbm_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_launch,
                "step_hbm_frac": round(200 * cells / (d["ms"] / K / 1e3) / 1e9 / hbm, 4),
                "stage1": {"kernel": kname.replace("stage2", "stage1"),
                           "achieved": round(a1, 1), "frac": round(a1 / hbm, 4),
                           "algorithmic_bytes_per_launch": b1,
                           "traffic": ncu_traffic(kname.replace("stage2", "stage1"), cells)}}

    # the latency-bound AMR run goes before the adjoint's host-bound
    # finite-difference loop, after which it measured up to 2x slower
    batch64 = None if args.no_batch else batch64_section(ctx, ranks, K, W)
    amr = None if args.no_amr else amr_section(ctx, ranks)
    adjoint = None if args.no_adjoint else adjoint_section(ctx, ranks)
    plane = None if args.no_plane else plane_section(ctx, ranks, K, W)
    bflux = None if args.no_bflux else bflux_section(ctx, ranks, min(K, 20), W)
    gravity = None if args.no_gravity else gravity_section(ctx, ranks, min(K, 20), W)
    muscl = None if args.no_muscl else muscl_section(ctx, ranks, min(K, 20), W)

    cpu = None
    if ranks.world == 1 and ranks.rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cpu_threads())

    if ranks.rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ranks.world,
        "steps": K, "warmup": W, "ms_per_step": round(mixed["ms"] / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 reconstruction+HLLC / f64 state, accumulation, reductions",
        "data": DATA,
        "config": {"workload": workload(n),
                   "cells_per_gpu": cells, "precision": "mixed", "kernel": mixed["kernel"],
                   "tile": f"16x16 columns, z chunk {mixed['kz']}, "
                           f"{'tapered' if mixed['taper'] else 'uniform'} work queue (autotuned)",
                   "l2": "inputs larger than L2 (671 MB per state buffer)",
                   "parallelism": f"one independent instance per GPU x{ranks.world}"},
        "accuracy": {"l1_rho_mixed_vs_fp64_rel": l1_mixed, "after_steps": W + K,
                     "bound": 1e-6, "conservation_drift_rel": drift},
        "fp64": {"value": round(fp64_value, 1), "unit": UNIT,
                 "ms_per_step": round(out["fp64"]["ms"] / K, 4),
                 "tile": f"16x16 columns, z chunk {out['fp64']['kz']}, "
                         f"{'tapered' if out['fp64']['taper'] else 'uniform'} work queue (autotuned)",
                 "speedup_mixed_over_fp64": round(value / fp64_value, 3),
                 "roofline": roofline(out["fp64"], "stage2_fp64")},
        "roofline": roofline(mixed, "stage2_mixed"),
        "kernels_ms": {p: {k: round(v, 4) for k, v in out[p].items() if k.startswith("ms_")}
                       for p in out},
        "e2e": {"value": round(total_cells * K / (e2e_ms / 1e3) / 1e6, 1), "unit": UNIT,
                "h2d_bytes_per_step": int(5 * 8 * cells / K),
                "d2h_bytes_per_step": int(5 * 8 * cells / K),
                "what": f"vb_grid_upload of the state from pinned host memory, vb_evolve of {K} "
                        "steps, vb_grid_download; device time of the whole sequence"},
        "gpu_launches": mixed["launches"],
        "clocks": clocks,
    }
    if batch64:
        line["batch64"] = batch64
    if adjoint:
        line["adjoint"] = adjoint
    if amr:
        line["amr"] = amr
    if plane:
        line["plane2d"] = plane
    if bflux:
        line["bflux"] = bflux
    if gravity is not None:
        line["gravity"] = gravity
    if muscl is not None:
        line["muscl"] = muscl
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def adjoint_section(ctx, ranks: Ranks, n=512, nsteps=200, every=20, fd_cells=32, h_rel=1e-6):
    """KH n^2 float64: forward evolve! of nsteps vs the checkpointed adjoint
    (forward with checkpoints, reverse sweep = segment recompute + adjoint
    stages), all timed with CUDA events; then d(int rho^2)/d rho_0 against
    central differences of the forward path at fd_cells random cells (dt
    sequence held fixed), on the KH state with a 1e-2 texture and as
    specified (exactly uniform bands: limiter ties, no derivative there)."""
    import numpy as np
    import vespa_b200 as vb

    def fd_check(sim, U0, grad, dts):
        V = sim.backend.cell_volume()
        errs = []
        for c in np.random.default_rng(3).choice(sim.ncell, size=fd_cells, replace=False):
            h = h_rel * U0[0, c]
            Up = U0.copy(); Up[0, c] += h
            Um = U0.copy(); Um[0, c] -= h
            r = []
            for Ux in (Up, Um):
                sim.upload(Ux)
                for dt in dts:
                    vb.step(sim, float(dt))
                r.append(sim.state()[0])
            fd = float(np.sum((r[0] - r[1]) * (r[0] + r[1])) * V) / (2.0 * h)
            errs.append(abs(fd - grad[0, c]) / abs(grad[0, c]))
        errs = np.array(errs)
        return {"cells": fd_cells, "h_rel": h_rel, "median_rel_err": float(np.median(errs)),
                "max_rel_err": float(errs.max()), "frac_within_1e-6": float(np.mean(errs <= 1e-6))}

    res = {}
    for tex in (1e-2, 0.0):
        prob = vb.kelvin_helmholtz_problem(n=n, texture=tex)
        mesh = vb.B200Mesh(prob.dims, prob.domain)
        sim = vb.Simulation(mesh, prob, precision="fp64", ctx=ctx)
        U0 = sim.state()
        fwd = []
        for _ in range(3):
            sim.upload(U0)
            sim.set_time(0.0, 0)
            ctx.mark(4)
            vb.evolve(sim, max_steps=nsteps)
            ctx.mark(5)
            fwd.append(ctx.elapsed_ms(4, 5))
        fwd_ms = ranks.max(min(fwd[1:]))
        sim.upload(U0)
        sim.set_time(0.0, 0)
        adj = vb.Adjoint(sim, nsteps, every)
        adj.forward(max_steps=nsteps)
        lam = vb.rho2_seed(sim, sim.state())
        dts = adj.dts()
        adj.backward(lam)
        grad = adj.backward(lam)
        tm = adj.timing()
        entry = {"texture": tex, "fd": fd_check(sim, U0, grad, dts)}
        if tex > 0:
            fwd_ckpt = ranks.max(tm["forward_ms"])
            re_ms = ranks.max(tm["recompute_ms"])
            adj_ms = ranks.max(tm["adjoint_ms"])
            entry.update({
                "forward_ms": round(fwd_ms, 3), "forward_with_checkpoints_ms": round(fwd_ckpt, 3),
                "recompute_ms": round(re_ms, 3), "adjoint_stages_ms": round(adj_ms, 3),
                "adj_step_over_fwd_step": round((re_ms + adj_ms) / fwd_ms, 3),
                "adj_stages_over_fwd": round(adj_ms / fwd_ms, 3),
                "gradient_over_forward": round((fwd_ckpt + re_ms + adj_ms) / fwd_ms, 3)})
            # the same gradient from a tape of every step's two states (no recompute)
            adj.close()
            sim.upload(U0)
            sim.set_time(0.0, 0)
            adj = vb.Adjoint(sim, nsteps, 1)
            adj.forward(max_steps=nsteps)
            adj.backward(lam)
            grad_t = adj.backward(lam)
            tt = adj.timing()
            fwd_tape = ranks.max(tt["forward_ms"])
            adj_tape = ranks.max(tt["adjoint_ms"])
            entry["tape"] = {
                "what": "checkpoint every step: the forward run keeps both states of every "
                        "step (2 x 200 x 10.5 MB in HBM), the reverse sweep recomputes nothing",
                "forward_with_tape_ms": round(fwd_tape, 3), "adjoint_stages_ms": round(adj_tape, 3),
                "gradient_over_forward": round((fwd_tape + adj_tape) / fwd_ms, 3),
                "same_gradient_bits": bool(np.array_equal(grad_t, grad))}
        res["textured" if tex > 0 else "as_specified"] = entry
        adj.close()
        sim.close()
    return {"config": f"2D Kelvin-Helmholtz {n}^2 periodic, gamma 1.4, float64, {nsteps} "
                      f"CFL-limited RK2 steps, checkpoints every {every}; J = int rho^2 at "
                      "t_end, gradient w.r.t. the initial conserved density",
            "adj_step": "reverse sweep per step (segment recompute + two adjoint stages) "
                        "over the forward step (evolve!)",
            **res}


def plane_section(ctx, ranks: Ranks, K: int, W: int, n=4096):
    """2D 4096^2 periodic throughput (the reference's '2D uniform throughput
    step' configuration, same generator as the cube), both precisions, tiled
    2D kernel with the autotuned row chunk; K timed CFL steps after W warm-up."""
    import vespa_b200 as vb
    prob = vb.smooth_random_problem((n, n), seed=vb.problem.DEFAULT_SEED + ranks.rank)
    U0 = vb.initial_state(prob)
    mesh = vb.B200Mesh(prob.dims, prob.domain)
    out = {"config": f"2D {n}^2 periodic, gamma 5/3, CFL 0.4, 5 float64 fields "
                     "(z momentum stays 0), inputs larger than L2 (134 MB per buffer)"}
    for prec in ("fp64", "mixed"):
        sim = vb.Simulation(mesh, prob, precision=prec, ctx=ctx, initial=U0)
        ky, _ = sim.autotune(3)
        vb.run_steps_async(sim, W)
        ctx.synchronize()
        ranks.barrier()
        ctx.mark(8)
        vb.run_steps_async(sim, K)
        ctx.mark(9)
        ms = ranks.max(ctx.elapsed_ms(8, 9))
        prof = sim.profile_step(3)
        hbm, _ = measured_hbm()
        s2 = 120 * n * n / (prof["ms_stage2"] / 1e3) / 1e9
        out[prec] = {"value": round(n * n * ranks.world * K / (ms / 1e3) / 1e6, 1), "unit": UNIT,
                     "ms_per_step": round(ms / K, 4), "kernel": sim.kernel, "row_chunk": ky,
                     "stage2_hbm_frac": round(s2 / hbm, 4)}
        sim.close()
    return out


def bflux_section(ctx, ranks: Ranks, K: int, W: int, n=256):
    """The cube's generator on an outflow 256^3 box, both precisions, with and
    without the boundary-flux register recording the domain faces
    (BoundaryFluxRegister, src/reflux.jl:113-132): the tiled kernels record
    them in place, so the step keeps its speed."""
    import vespa_b200 as vb
    prob = vb.smooth_random_problem((n, n, n), seed=vb.problem.DEFAULT_SEED + ranks.rank)
    prob.bcs = vb.problem.Outflow
    U0 = vb.initial_state(prob)
    mesh = vb.B200Mesh(prob.dims, prob.domain)
    out = {"config": f"3D {n}^3, outflow on all six sides, gamma 5/3, CFL 0.4; the register "
                     "records (0.5 dt F) area at every domain face in both RK2 stages"}
    for prec in ("fp64", "mixed"):
        res = {}
        for on in (False, True):
            sim = vb.Simulation(mesh, prob, precision=prec, ctx=ctx, initial=U0)
            sim.bflux_enable(on)
            vb.run_steps_async(sim, W)
            ctx.synchronize()
            ranks.barrier()
            ctx.mark(8)
            vb.run_steps_async(sim, K)
            ctx.mark(9)
            ms = ranks.max(ctx.elapsed_ms(8, 9))
            res["on" if on else "off"] = {
                "value": round(n ** 3 * ranks.world * K / (ms / 1e3) / 1e6, 1), "unit": UNIT,
                "ms_per_step": round(ms / K, 4), "kernel": sim.kernel, "kz": sim.kz}
            sim.close()
        res["on_over_off_time"] = round(res["on"]["ms_per_step"] / res["off"]["ms_per_step"], 4)
        out[prec] = res
    return out


def gravity_section(ctx, ranks: Ranks, K: int, W: int, n=256, cpu_n=64):
    """Self-gravity (src/gravity.jl) on the 256^3 cube: (a) a cold Poisson solve
    (phi = 0, tol 1e-8) of a white-noise density with plain CG (the reference's
    default), whose iterations stream 88 B/cell (matvec r p w Ap, update r phi
    p r Ap w phi r, direction r p w p), and with the multigrid preconditioner
    (precond = :mg, ext/mg_pcg.jl); (b) K evolve! steps with gravity after W
    warm-up steps (one warm-started solve per step, stages on the tiled
    kernels with the source): both precisions with the preconditioner, float64
    with plain CG.
    CPU: the oracle's plain CG on a cpu_n^3 sample of (a), serial."""
    import numpy as np
    import vespa_b200 as vb
    prob = vb.smooth_random_problem((n, n, n), seed=vb.problem.DEFAULT_SEED + ranks.rank)
    U0 = vb.initial_state(prob)
    mesh = vb.B200Mesh(prob.dims, prob.domain)
    rng = np.random.default_rng(20261203 + ranks.rank)
    Un = U0.copy()
    Un[0] = 0.5 + rng.random(n ** 3)
    out = {"config": f"3D {n}^3 periodic, G = 1, phi periodic with the mean projected out; "
                     "(a) cold solve of a white-noise density U[0.5, 1.5), tol 1e-8; "
                     "(b) the cube's smooth random state, CFL 0.4, solve per step (tol 1e-8)"}
    hbm, _ = measured_hbm()
    for pc in ("mg", "none"):
        sim = vb.Simulation(mesh, prob, precision="fp64", ctx=ctx, initial=Un)
        grav = vb.enable_gravity(sim, G=1.0, tol=1e-8, maxiter=5000, precond=pc)
        vb.solve_poisson(sim, grav)  # warm-up (captures the iteration graph)
        grav.phi = np.zeros(n ** 3)
        ctx.synchronize()
        ranks.barrier()
        ctx.mark(10)
        its, rr = vb.solve_poisson(sim, grav)
        ctx.mark(11)
        ms = ranks.max(ctx.elapsed_ms(10, 11))
        per_it = ms / its
        rec = {"iters": its, "relres": rr, "ms": round(ms, 3), "ms_per_iteration": round(per_it, 4)}
        if pc == "none":
            bw = 88 * n ** 3 / (per_it / 1e3) / 1e9
            rec.update({"Mcell_iterations_per_s": round(n ** 3 / (per_it / 1e3) / 1e6, 1),
                        "achieved_gbs": round(bw, 1), "hbm_frac": round(bw / hbm, 4),
                        "bytes_per_cell_iteration": 88})
        out[f"cold_solve_{pc}"] = rec
        sim.close()
    for prec, pc in (("fp64", "mg"), ("mixed", "mg"), ("fp64", "none")):
        sim = vb.Simulation(mesh, prob, precision=prec, ctx=ctx, initial=U0)
        vb.enable_gravity(sim, G=1.0, precond=pc)
        vb.evolve(sim, tfinal=math.inf, max_steps=W)
        ctx.synchronize()
        ranks.barrier()
        ctx.mark(12)
        vb.evolve(sim, tfinal=math.inf, max_steps=K)
        ctx.mark(13)
        ms = ranks.max(ctx.elapsed_ms(12, 13))
        out[f"{prec}_{pc}"] = {"value": round(n ** 3 * ranks.world * K / (ms / 1e3) / 1e6, 1),
                               "unit": UNIT, "ms_per_step": round(ms / K, 4), "steps": K,
                               "stages": f"{sim.kernel} kernel with the gravity source"}
        sim.close()
    if ranks.rank == 0:
        from oracle import oracle as O
        O.build()
        cprob = vb.smooth_random_problem((cpu_n,) * 3)
        Uc = vb.initial_state(cprob)
        Uc[0] = 0.5 + rng.random(cpu_n ** 3)
        g = O.grid_from_problem(cprob)
        Pg = O.make_gravity(1.0, (1, 1, 1), (1, 1, 1), 5000, 1e-8, True)
        phi = np.zeros(cpu_n ** 3)
        t0 = time.perf_counter()
        cits, _ = O.grav_solve(g, Pg, Uc, phi)
        cs = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(cpu_n ** 3 * cits / cs / 1e6, 2),
                               "unit": "Mcell-CG-iterations/s", "cores": 1, "kind": "port",
                               "sample": f"cold plain-CG solve of a {cpu_n}^3 white-noise density, "
                                         f"tol 1e-8 ({cits} iterations, {cs:.2f} s), serial C oracle"}
    return out


def muscl_section(ctx, ranks: Ranks, K: int, W: int, n=256, ng=3, cpu_n=48):
    """lib/PPMKernels unsplit MUSCL (muscl_step_3d!, Enzo HydroMethod=3) on an
    n^3 active region with ng ghost zones per side (periodic fill), the cube's
    generator for the state, dt from CFL 0.4 of the initial state; K timed
    steps after W warm-up steps.  Bytes the kernels move per cell and step:
    first preparation pass (read U, write U0 and the primitives: 120), stage 1
    (prim, U0, write U: 120), second preparation pass (read U, write the
    primitives: 80), stage 2 (prim, U0, U, write U: 160) = 480 B (ghost fills
    add a few percent).  CPU: the oracle's serial restatement on a cpu_n^3
    sample."""
    import numpy as np
    import vespa_b200 as vb
    m = n + 2 * ng
    dims = (m, m, m)
    gamma = 5.0 / 3.0
    prob = vb.smooth_random_problem((m, m, m), seed=vb.problem.DEFAULT_SEED + ranks.rank)
    W5 = vb.problem.initial_primitive(prob)
    rho, vel, p = W5[0], W5[1:4], W5[4]
    etot = p / ((gamma - 1.0) * rho) + 0.5 * (vel ** 2).sum(axis=0)
    U0 = np.ascontiguousarray(np.array([rho, rho * vel[0], rho * vel[1], rho * vel[2], rho * etot]))
    cs = np.sqrt(gamma * p / rho)
    dx = 1.0 / n
    dt = 0.4 * dx / float(np.max(np.abs(vel).max(axis=0) + cs))
    g = vb.MusclGrid(dims, ng, ctx=ctx)
    g.upload(U0)
    kw = dict(dt=dt, gamma=gamma, dx=dx, bc="periodic")
    g.run_async(W, **kw)
    ctx.synchronize()
    ranks.barrier()
    ctx.mark(14)
    g.run_async(K, **kw)
    ctx.mark(15)
    ms = ranks.max(ctx.elapsed_ms(14, 15))
    hbm, _ = measured_hbm()
    gbs = 480 * m ** 3 / (ms / K / 1e3) / 1e9
    out = {"config": f"3D {n}^3 active cells + {ng} periodic ghost zones per side, gamma 5/3, "
                     f"theta 1.5, HLL, fixed dt = CFL 0.4 of the initial state",
           "value": round(n ** 3 * ranks.world * K / (ms / 1e3) / 1e6, 1), "unit": UNIT,
           "ms_per_step": round(ms / K, 4), "steps": K,
           "achieved_gbs": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4),
           "bytes_per_cell_step": 480}
    g.close()
    if ranks.rank == 0:
        from oracle import oracle as O
        O.build()
        mc = cpu_n + 2 * ng
        Uc = np.ascontiguousarray(U0.reshape(5, m, m, m)[:, :mc, :mc, :mc].reshape(5, -1))
        t0 = time.perf_counter()
        O.muscl_step((mc, mc, mc), ng, Uc, dt, gamma, 1.5, dx, bc=1)
        cs_ = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(cpu_n ** 3 / cs_ / 1e6, 3), "unit": UNIT, "cores": 1,
                               "kind": "port", "sample": f"one step of a {cpu_n}^3 (+ghosts) "
                                                         f"sample ({cs_:.2f} s), serial C oracle"}
    return out


def amr_section(ctx, ranks: Ranks, cpu_steps=60):
    """2D Sedov blast on the composite AMR mesh: 48^2 base, E = 1 in a 3-cell
    hot spot, reflecting walls, regrid every 4 steps refining above a density
    jump of 0.2 up to 4 levels, float64, to t = 0.05.  Single-rate (one global
    dt) and subcycled (per-level dt with flux registers), each after a warm-up
    of its first steps on a throwaway mesh.  Device time of the whole run
    (regrids, with their few host reads of counts, included); leaf-updates =
    sum over steps of the leaves stepped."""
    import numpy as np
    import vespa_b200 as vb
    from vespa_b200 import amr as A
    prob = vb.sedov_problem(n=48, r0=3.0 / 48, tfinal=0.05)
    pol = A.RefinementPolicy(0.2, 4, 4)
    out = {"config": "2D Sedov 48^2 base, r0 = 3 cells, gamma 1.4, reflecting, CFL 0.3, "
                     "RefinementPolicy(refine_above=0.2, max_level=4, every=4), t_end = 0.05, float64"}
    import gc
    gc.collect()
    gc.disable()  # the host drives this run: no collector pauses inside it
    sampler = ClockSampler(ranks.local)
    sampler.start()
    for sub in (False, True):
        # warm-up: the first steps and regrids of the same run on a throwaway mesh
        warm = A.AmrSimulation(A.AmrMesh(prob.dims, prob.domain), prob, ctx=ctx)
        A.evolve(warm, policy=pol, subcycle=sub, max_steps=3 if sub else 12)
        warm.close()
        ctx.synchronize()
        sim = A.AmrSimulation(A.AmrMesh(prob.dims, prob.domain), prob, ctx=ctx)
        t0 = A.conserved_totals(sim)
        ms = 0.0
        updates = 0
        regrid_ms = 0.0
        while sim.t < prob.tfinal * (1 - 1e-12):
            s0 = sim.step
            ctx.mark(6)
            A.evolve(sim, policy=pol, subcycle=sub, max_steps=4 if not sub else 1)
            ctx.mark(7)
            ms += ctx.elapsed_ms(6, 7)
            regrid_ms += sim.regrid_ms()
            if not sub:
                updates += (sim.step - s0) * sim.nleaf
        t1 = A.conserved_totals(sim)
        entry = {"steps": sim.step, "leaves_final": sim.nleaf, "max_level": sim.max_level,
                 "faces_final": sim.nface, "ms": round(ranks.max(ms), 3),
                 "regrid_ms": round(regrid_ms, 3),
                 "mass_drift_rel": abs(t1.mass - t0.mass) / t0.mass,
                 "energy_drift_rel": abs(t1.energy - t0.energy) / t0.energy}
        if not sub:
            entry["leaf_updates"] = updates
            entry["value"] = round(updates / (entry["ms"] / 1e3) / 1e6, 2)
            entry["unit"] = "Mleaf-updates/s"
        out["subcycled" if sub else "single_rate"] = entry
        sim.close()
    out["clocks"] = sampler.stop()
    gc.enable()
    # the oracle on the first cpu_steps steps of the same run (host, 1 thread)
    if ranks.rank == 0:
        from oracle import oracle as O
        ora = O.Amr(O.grid_from_problem(prob))
        ora.set_state(vb.initial_state(prob))
        upd, t_cpu, done = 0, 0.0, 0
        while done < cpu_steps:
            ts = time.perf_counter()
            ora.evolve(prob.tfinal, max_steps=4, refine_above=0.2, max_level=4, every=4)
            t_cpu += time.perf_counter() - ts
            upd += 4 * ora.nleaf
            done += 4
        out["cpu_oracle"] = {"value": round(upd / t_cpu / 1e6, 3), "unit": "Mleaf-updates/s",
                             "cores": 1, "kind": "port",
                             "sample": f"first {cpu_steps} single-rate steps of the same run, "
                                       "C oracle (serial, like the reference's loop)"}
    return out


BATCH_DATA = ("synthetic: 64 seeded planar two-state Riemann problems, rho in [0.1, 10], "
              "|u| <= 2, p in [0.01, 10], gamma 1.4, outflow; cube sides from "
              "{32,48,64,96,128,192,256}")


def batch64_section(ctx, ranks: Ranks, K: int, W: int):
    """64 independent 3D Riemann boxes (cube sides drawn from {32..256}), mixed
    precision, stepped as one batch: one persistent launch per stage for all
    boxes, the K timed steps replayed as one CUDA graph."""
    import vespa_b200 as vb
    from vespa_b200 import problem as P
    probs = [P.riemann_box_problem(i, seed=P.DEFAULT_SEED + 1000 * ranks.rank) for i in range(64)]
    batch = vb.Batch(probs, precision="mixed", ctx=ctx)
    cells = batch.ncell()
    cap, _ = batch.autotune(3)  # work-item depth; states and clocks restored
    batch.run_steps(W)
    batch.run_steps_async(K)  # capture the K-step graph once, outside the timing
    ctx.synchronize()
    ranks.barrier()
    l0 = ctx.launch_count
    ctx.mark(0)
    batch.run_steps_async(K)
    ctx.mark(1)
    ms = ranks.max(ctx.elapsed_ms(0, 1))
    launches = ctx.launch_count - l0
    total = ranks.sum(float(cells))
    batch.close()
    hbm, hbm_kind = measured_hbm()
    return {"value": round(total * K / (ms / 1e3) / 1e6, 1), "unit": UNIT,
            "ms_per_step": round(ms / K, 4), "steps": K, "warmup": W,
            "cells_per_gpu": cells, "boxes": 64,
            "items": "16x16 column tiles, " + ("each box's default z chunk" if cap == 0 else
                                                f"z chunks capped at {cap} planes") + " (autotuned)",
            "sides": sorted({p.dims[0] for p in probs}),
            "step_hbm_frac": round(200 * cells / (ms / K / 1e3) / 1e9 / hbm, 4),
            "hbm_peak_gbs": hbm, "hbm_peak_source": hbm_kind, "gpu_launches": launches,
            "precision": "mixed", "data": BATCH_DATA,
            "what": "per-box CFL dt; finalise, stage 1, stage 2 and advance per step for all "
                    "boxes; the K timed steps replay one CUDA graph; work-item depth picked by "
                    "vb_batch_autotune"}


def run_batch64(args, ranks: Ranks):
    """--workload batch64: the batch section alone, as its own JSON line."""
    import vespa_b200 as vb
    K, W = args.steps, args.warmup
    ctx = vb.Context(ranks.local)
    sec = batch64_section(ctx, ranks, K, W)
    if ranks.rank != 0:
        return
    line = {
        "metric": "Mcell-updates/s, 64 uneven 3D Riemann boxes batched, PLM+HLLC RK2, mixed",
        "value": sec["value"], "unit": UNIT, "n_gpus": ranks.world, "steps": K, "warmup": W,
        "ms_per_step": sec["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 reconstruction+HLLC / f64 state",
        "data": BATCH_DATA,
        "config": {"workload": "batch of 64 uneven boxes, per-box CFL dt, CUDA-graph replay",
                   "cells_per_gpu": sec["cells_per_gpu"], "boxes": 64,
                   "parallelism": f"independent batch per GPU x{ranks.world}"},
        "step_hbm_frac": sec["step_hbm_frac"], "hbm_peak_gbs": sec["hbm_peak_gbs"],
        "hbm_peak_source": sec["hbm_peak_source"], "gpu_launches": sec["gpu_launches"],
    }
    print(json.dumps(line), flush=True)


def run_slab(args, ranks: Ranks):
    """--workload slab: ONE n^3 periodic grid (the headline's generator) split
    along z across the ranks, two ghost planes exchanged per RK2 stage over
    NCCL and the CFL maximum all-reduced (strong scaling: the total work is
    fixed as N grows).  The result equals the single grid bit for bit."""
    import torch
    import vespa_b200 as vb
    from vespa_b200 import slab as S
    n = args.n
    K, W = args.steps, args.warmup
    ctx = vb.Context(ranks.local)
    prob = vb.smooth_random_problem((n, n, n), seed=vb.problem.DEFAULT_SEED)
    U0 = vb.initial_state(prob)
    out = {}
    for prec in ("fp64", "mixed"):
        sl = S.SlabSimulation(prob, precision=prec, ctx=ctx, initial=U0)
        sl.step(W)
        ctx.synchronize()
        ranks.barrier()
        ctx.mark(0)
        sl.step(K)
        ctx.mark(1)
        ms = ranks.max(ctx.elapsed_ms(0, 1))
        out[prec] = {"value": round(n ** 3 * K / (ms / 1e3) / 1e6, 1), "unit": UNIT,
                     "ms_per_step": round(ms / K, 4), "planes_per_rank": sl.halo.nact,
                     "ghost_planes": sl.halo.g_lo + sl.halo.g_hi}
        sl.close()
    if ranks.rank != 0:
        return
    line = {
        "metric": f"Mcell-updates/s 3D {n}^3 PLM+HLLC RK2, one grid split in z slabs",
        "value": out["mixed"]["value"], "unit": UNIT, "n_gpus": ranks.world, "steps": K,
        "warmup": W, "ms_per_step": out["mixed"]["ms_per_step"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 reconstruction+HLLC / f64 state", "data": DATA,
        "config": {"workload": workload(n) + ", one grid in z slabs",
                   "parallelism": f"z slabs x{ranks.world}, 2 ghost planes per side, NCCL "
                                  "send/recv per stage, CFL all-reduce (max)"},
        "fp64": out["fp64"],
    }
    print(json.dumps(line), flush=True)


def run_section(args, ranks: Ranks):
    """One of the secondary workloads alone, printed as its own JSON line."""
    import vespa_b200 as vb
    ctx = vb.Context(ranks.local)
    if args.workload == "plane":
        sec = plane_section(ctx, ranks, args.steps, args.warmup)
        metric, value = "Mcell-updates/s 2D 4096^2 PLM+HLLC RK2 (mixed)", sec["mixed"]["value"]
    elif args.workload == "adjoint":
        sec = adjoint_section(ctx, ranks)
        metric, value = ("adjoint step / forward step, KH 512^2 float64",
                         sec["textured"]["adj_step_over_fwd_step"])
    elif args.workload == "muscl":
        sec = muscl_section(ctx, ranks, args.steps, args.warmup, n=args.n)
        metric, value = (f"Mcell-updates/s 3D {args.n}^3 PPMKernels unsplit MUSCL-HLL RK2 (fp64)",
                         sec["value"])
    elif args.workload == "gravity":
        sec = gravity_section(ctx, ranks, min(args.steps, 20), args.warmup, n=args.n)
        metric, value = (f"Mcell-updates/s 3D {args.n}^3 with self-gravity (fp64, multigrid-preconditioned CG)",
                         sec["fp64_mg"]["value"])
    else:
        sec = amr_section(ctx, ranks)
        metric, value = ("Mleaf-updates/s, Sedov 48^2 AMR single rate",
                         sec["single_rate"]["value"])
    if ranks.rank == 0:
        print(json.dumps({"metric": metric, "value": value, "n_gpus": ranks.world,
                          "workload": args.workload, args.workload: sec}), flush=True)


def main():
    args = parse()
    ranks = Ranks(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, ranks)
        elif args.workload == "batch64":
            run_batch64(args, ranks)
        elif args.workload == "slab":
            run_slab(args, ranks)
        elif args.workload in ("plane", "adjoint", "amr", "gravity", "muscl"):
            run_section(args, ranks)
        else:
            run_ours(args, ranks)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
