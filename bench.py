"""Benchmark of the TORCH full step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload hii|sedov|batch] [--n 256] [--precision both|fp32|fp64]
    python bench.py --validate 1000 [--workload hii] [--n 256]   (accuracy, not timing)

Default workload: the 256^3 HII-region expansion (side 2 pc, star at the
centre with Q = 1e49 photons/s, lognormal density with mean 1e3 cm^-3,
sigma_ln 0.5 and a k^-11/3 spectrum from seed 12345, T = 100 K, radiation
and cooling on).  A step is one Torch::fullStep over the whole grid (hydro,
radiative transfer, heating/cooling, the time-step reduction); the metric is
cell updates per second (cells x full steps / time).  The head number is the
FP32 form (FP32 hydro, FP64 ionisation solve and reductions); the plain FP64
form is timed beside it on the same input (`plain_fp64`) and the FP32 form's
density and pressure error against it after the same steps is reported
(`error_vs_fp64`).  `--workload sedov` is the 256^3 hydro-only Sedov blast.
Inputs (7 x 256^3 cells) are far larger than the 126 MB L2, so no flush is
needed between steps.

One JSON line on rank 0.  Under torchrun (N > 1) every rank advances its own
replica of the workload on its own GPU (the step does not shard in this
build: "replicas only"), times are max-reduced over ranks, and value is the
whole-job rate.  --impl reference times the reference's own CPU code (the
unmodified reference build oracle/_ref/torch_ref, or the C restatement when
that binary is absent) on the host cores, on a bounded sample of the same
workload.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s/GPU full step 256\u00b3: learned+FP32 vs plain FP64, at stated error"
UNIT = "cell-updates/s"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def build_workload(name, n):
    from torch_b200 import workloads
    if name == "sedov":
        return workloads.sedov(n=n)
    if name == "hii":
        return workloads.hii_region(n=n)
    if name == "blister":  # the shipped 2-D cylindrical setup (150 x 200), whatever n
        return workloads.blister()
    raise ValueError(name)


def workload_config(name, n, precision, replicas):
    base = {"workload": f"{name} {n}^3", "cells": n ** 3, "precision": precision,
            "parallelism": f"replicas x{replicas}", "l2": "inputs larger than L2 (no flush)"}
    if name == "blister":
        base.update({"workload": "blister 150x200 (2-D cylindrical, the shipped setup)", "cells": 30000,
                     "l2": "inputs smaller than L2", "setup": "config/torch-config.lua + torch-setup.lua values",
                     "time": "operator split H/T/R"})
        return base
    if name == "sedov":
        base.update({"setup": "hydro-only Sedov blast, rho 1e-20, P 1e-12, E 1e51 erg in r<=3dx, outflow",
                     "reconstruction": "piecewise-linear albada (spatial_order 1)", "riemann": "RotatedHLLC",
                     "time": "RK2 midpoint", "gamma": 1.67, "side_pc": 2.0})
    else:
        base.update({"setup": "HII region, lognormal n (mean 1e3, sigma_ln 0.5, k^-11/3, seed 12345), "
                              "Q=1e49/s star at centre, radiation+cooling, T=100 K",
                     "time": "operator split H/T/R", "side_pc": 2.0})
    return base


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        # only samples taken while the GPU was busy (utilization >= 50 %) count as
        # "under load"; the sampler runs from before the first timed step to after the last
        sm, smax, reasons, idle = [], None, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                util = float(parts[9])
                clk = float(parts[1])
                smax = float(parts[2])
            except ValueError:
                continue
            if util < 50:
                idle += 1
                continue
            sm.append(clk)
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "idle_samples_dropped": idle}


def dist_setup(backend="nccl"):
    """One process per GPU under torchrun (RANK/LOCAL_RANK/WORLD_SIZE/MASTER_*
    from the environment); the ranks only synchronise and max-reduce times."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, value, local):
    if pg is None:
        return value
    import torch
    dev = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- CPU legs
def _write_case(d, tp, ic):
    from torch_b200 import config
    pp = os.path.join(d, "params.lua")
    with open(pp, "w") as f:
        f.write(config.to_lua(tp))
    icp = os.path.join(d, "ic_000.txt")
    config.write_initial_conditions(icp, ic.ncells, ic.dx, ic.den, ic.pre, ic.hii, ic.vel)
    return pp, icp


def cpu_sample(workload, n_sample, steps, procs):
    """Times the reference CPU code on `procs` independent replicas of a bounded
    sample (n_sample^3 cells, `steps` full steps each) on the host cores.
    Returns (cell-updates/s, kind, cores, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    tp, ic = build_workload(workload, n_sample)
    ref_bin = oracle.REF_BIN if os.path.exists(oracle.REF_BIN) else None
    cells = int(np.prod(ic.ncells))
    with tempfile.TemporaryDirectory() as d:
        pp, icp = _write_case(d, tp, ic)
        if ref_bin:
            t0 = time.perf_counter()
            ps = [subprocess.Popen([ref_bin, f"--params={pp}", f"--ic={icp}", f"--steps={steps}"],
                                   cwd=d, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for _ in range(procs)]
            rcs = [p.wait() for p in ps]
            wall = time.perf_counter() - t0
            if any(rcs):
                raise RuntimeError(f"reference sample failed: {rcs}")
            kind = "reference"
        else:
            from torch_b200 import config
            ic2 = config.read_initial_conditions(icp)
            t0 = time.perf_counter()
            o = oracle.Oracle(tp, ic2)
            for _ in range(steps):
                o.full_step()
            wall = time.perf_counter() - t0
            procs = 1
            kind = "port"
    rate = cells * steps * procs / wall
    desc = (f"{workload} {n_sample}^3, {steps} full steps x {procs} independent single-rank processes "
            f"({'reference build, MPI absent: one rank each' if kind == 'reference' else 'C restatement'}); "
            f"includes set-up")
    return rate, kind, procs, desc


def cpu_sample_batch(cases, steps):
    """The reference build on a sample of batch grids, one single-rank process
    per grid, all at once on the host cores: cell-updates/s of the sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not os.path.exists(oracle.REF_BIN):
        raise FileNotFoundError("reference build unavailable")
    cells = sum(int(np.prod(ic.ncells)) for _, ic in cases)
    with tempfile.TemporaryDirectory() as d:
        cmds = []
        for i, (tp, ic) in enumerate(cases):
            di = os.path.join(d, f"g{i}")
            os.makedirs(di)
            pp, icp = _write_case(di, tp, ic)
            cmds.append(([oracle.REF_BIN, f"--params={pp}", f"--ic={icp}", f"--steps={steps}"], di))
        t0 = time.perf_counter()
        ps = [subprocess.Popen(c, cwd=di, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for c, di in cmds]
        rcs = [p.wait() for p in ps]
        wall = time.perf_counter() - t0
    if any(rcs):
        raise RuntimeError(f"reference sample failed: {rcs}")
    return {"value": cells * steps / wall, "unit": UNIT, "cores": min(len(cases), os.cpu_count() or 1),
            "kind": "reference",
            "sample": f"the first {len(cases)} grids of the batch, {steps} full steps, one single-rank reference "
                      f"process per grid (MPI absent), run together; includes set-up"}


def run_reference_arm(args, rank):
    if rank != 0:
        return 0
    procs = max(1, min(os.cpu_count() or 1, 16))
    n_sample = 48 if args.workload == "sedov" else 32
    per_step = []
    total_steps = args.warmup + args.steps
    t0 = time.perf_counter()
    rate, kind, cores, desc = cpu_sample(args.workload, n_sample, max(1, total_steps), procs)
    wall = time.perf_counter() - t0
    config = workload_config(args.workload, args.n, "fp64", 1)
    # the rate is the metric of the named workload; the CPU time is measured
    # on a bounded sample of it (independent single-rank processes, no MPI)
    config["workload"] = (f"{args.workload} {args.n}^3 rate, timed on a sample: {cores} independent "
                          f"{n_sample}^3 grids, one single-rank reference process each")
    config["sample_cells"] = n_sample ** 3 * cores
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(1, total_steps),
        "ms_per_step_of": f"the sample ({cores} x {n_sample}^3 cells), not a {args.n}^3 step",
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU leg
def time_form(args, precision, tp, ic, local, pg, profile_names):
    """Times K full steps of one precision form; returns (ms, launches, prof, sim)."""
    import torch
    import torch_b200
    sim = torch_b200.Torch(tp, ic, precision=precision, device=local)
    if precision == torch_b200.PRECISION_FP32 and getattr(args, "fp32_contrast", None) is not None and tp.radiation_on:
        sim.fp32_contrast(args.fp32_contrast)
    if getattr(args, "thermo_queue", 0) and tp.cooling_on:
        sim.thermo_queue(args.thermo_queue)
    if getattr(args, "tile_z", 0):
        sim.tile = (sim.set_tile(args.tile_z), None)
    else:
        sim.tile = sim.autotune()
    dt_next = sim.dt_max
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=f"cuda:{local}")
    sim.run_steps(args.warmup)  # the first step is the reference's dt_max*1e-20 start step
    launches0 = sim.kernel_launches()
    sim.profile(True)
    barrier(pg)
    torch.cuda.synchronize(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sim.enqueue_steps(args.steps, dt_next)
    ev1.record(stream)
    sim.synchronize()
    torch.cuda.synchronize(local)
    barrier(pg)
    ms = ev0.elapsed_time(ev1)
    launches = sim.kernel_launches() - launches0
    prof = {}
    for name in profile_names:
        t, c = sim.profile_read(name)
        if c:
            prof[name] = (t, c)
    sim.profile(False)
    return ms, launches, prof, sim


PROFILE_NAMES = ("k_hydro_stage_fp32", "k_faces_fp64", "k_hydro_update_fp64", "k_q_from_u", "k_dt_reduce",
                 "k_dt_finalize", "k_dt_reset", "k_time_advance", "graph_rad_sweep", "graph_colden_sweep",
                 "k_rad_shell", "k_colden_shell", "k_thermo", "k_rad_heating", "k_rad_update", "k_rad_wind",
                 "k_rad_no_star")


def _conserved(sim):
    import torch_b200
    U = np.empty((7, sim.N), dtype=np.float64)
    rc = sim.lib.trg_get_state(sim.ctx, U.ctypes.data_as(torch_b200.C.c_void_p), None, None, None, None)
    if rc:
        raise RuntimeError(f"trg_get_state failed: {rc}")
    return U


def form_error(sim_a, sim_b, gamma, nd):
    """Relative L1 (sum |a-b| / sum |b|) of density and pressure between two forms."""
    Ua, Ub = _conserved(sim_a), _conserved(sim_b)

    def pressure(U):
        ke = sum(U[4 + i] ** 2 for i in range(nd)) / (2.0 * U[0])
        return (U[1] - ke) * (gamma - 1.0)

    def rel(a, b):
        return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))
    return {"den_rel_l1": rel(Ua[0], Ub[0]), "pre_rel_l1": rel(pressure(Ua), pressure(Ub))}


def run_batch(args, world, rank, local, pg):
    """Independent 2-D cylindrical HII-region grids of uneven sizes, in the
    FP32 form (FP32 hydro, FP64 radiation and cooling; --precision fp64 for
    the FP64 form), advanced one launch per stage for all grids, each
    timestep replayed from a captured CUDA graph; beside it the same grids
    stepped one by one (`unbatched`, on a bounded sample of grids)."""
    import torch
    import torch_b200
    from torch_b200 import workloads

    cases = workloads.blister_batch(G=args.grids, seed=2024 + rank)
    prec = torch_b200.PRECISION_FP64 if args.precision == "fp64" else torch_b200.PRECISION_FP32
    form = "fp64" if prec == torch_b200.PRECISION_FP64 else "fp32"
    grids = [torch_b200.Torch(tp, ic, precision=prec) for tp, ic in cases]
    cells = sum(g.N for g in grids)
    dt_next = min(g.dt_max for g in grids)
    b = torch_b200.Batch(grids)
    stream = torch.cuda.ExternalStream(b.stream_handle(), device=f"cuda:{local}")
    b.run_steps(args.warmup, dt_next)
    launches0 = b.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    torch.cuda.synchronize(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    b.enqueue_steps(args.steps, dt_next)
    ev1.record(stream)
    b.synchronize()
    torch.cuda.synchronize(local)
    barrier(pg)
    clk = clocks.stop()
    ms = max_over_ranks(pg, ev0.elapsed_time(ev1), local)
    launches = b.kernel_launches() - launches0
    learned = time_batch_learned(args, b, cases, prec, cells, world, local, pg, dt_next) if args.learned else None
    # per-kernel times from an event-bracketed pass of the same number of
    # steps after the timed region (per-launch events would keep the timed
    # steps from being replayed as graphs)
    b.profile(True)
    b.enqueue_steps(args.steps, dt_next)
    b.synchronize()
    prof = {}
    for name in PROFILE_NAMES:
        tt, cc = b.profile_read(name)
        if cc:
            prof[name] = {"ms": tt, "launches": cc}
    b.profile(False)
    # end to end through the batch's public API: per step every grid's
    # conserved state in from pinned host memory, the step, and out again
    hbuf = [torch.empty((7, g.N), dtype=torch.float64).pin_memory() for g in grids]
    for i, g in enumerate(grids):
        b.get_conserved(i, hbuf[i].data_ptr())
    b.synchronize()
    e2e_steps = max(1, args.e2e_steps)
    torch.cuda.synchronize(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        for i in range(len(grids)):
            b.set_conserved(i, hbuf[i].data_ptr())
        b.enqueue_steps(1, dt_next)
        for i in range(len(grids)):
            b.get_conserved(i, hbuf[i].data_ptr())
    e1.record(stream)
    b.synchronize()
    e2e_ms = max_over_ranks(pg, e0.elapsed_time(e1), local)
    ubytes = sum(7 * 8 * g.N for g in grids)
    e2e = {"value": cells * e2e_steps * world / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": ubytes,
           "d2h_bytes_per_step": ubytes, "steps": e2e_steps,
           "note": "per step through the batch API: pinned H2D of every grid's U, one batch step, D2H of U"}
    b.close()
    for g in grids:
        g.close()
    # roofline of the HBM-bound kernel with the largest share among those with a
    # stated algorithmic byte count per cell (FP64 form)
    # (the FP32 form's batch hydro pass: read U, write U1 and Q, then U1 back to U)
    per_cell = {"k_hydro_update_fp64": 280.0, "k_faces_fp64": 112.0, "k_q_from_u": 112.0,
                "k_hydro_stage_fp32": 280.0}
    roofline = None
    cand = [(v["ms"], k) for k, v in prof.items() if k in per_cell]
    if cand:
        _, kname = max(cand)
        launches_k = prof[kname]["launches"]
        bytes_launch = per_cell[kname] * cells
        avg_ms = prof[kname]["ms"] / launches_k
        peak, src = hbm_peak()
        achieved = bytes_launch / (avg_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "kernel": kname, "peak_source": src, "avg_launch_ms": avg_ms,
                    "launches": launches_k, "algorithmic_bytes_per_launch": bytes_launch,
                    "note": "batch-wide launch (all grids); per-kernel times from an event-bracketed pass"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_sample_batch(cases[:16], args.cpu_steps)
        except Exception as e:  # a missing CPU baseline must not hide the GPU number
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(e)[:200]}
    # the same kind of grids stepped one context at a time (first 16 grids)
    sample = cases[:min(16, len(cases))]
    singles = [torch_b200.Torch(tp, ic, precision=prec) for tp, ic in sample]
    for s in singles:
        s.run_steps(args.warmup, dt_next)
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for s in singles:
        s.run_steps(args.steps, dt_next)
    torch.cuda.synchronize(local)
    wall = time.perf_counter() - t0
    ucells = sum(s.N for s in singles)
    for s in singles:
        s.close()
    value = cells * args.steps * world / (ms / 1e3)
    if rank == 0:
        line = {
            "metric": "cell-updates/s batched grids", "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if form == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": f"batch of {args.grids} 2-D cylindrical HII-region grids", "cells": cells,
                       "precision": form, "parallelism": f"replicas x{world}",
                       "sizes": "nx U[64,256], ny U[64,320], Q log-U[1e47,1e49], alpha U[0,2], rc U[0.005,0.05] pc",
                       "l2": "inputs larger than L2 (no flush)"},
            "gpu_launches": int(launches), "launches_per_step": launches / max(1, args.steps), "clocks": clk,
            "kernels": prof,
            "unbatched": {"value": ucells * args.steps / wall, "grids": len(sample),
                          "note": "the first grids stepped one context after another, host wall clock"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "learned": learned,
        }
        print(json.dumps(line), flush=True)
    return 0


def time_batch_learned(args, b, cases, prec, cells, world, local, pg, dt_next):
    """The batch with the learned starting iterate: a network trained on the
    front-cell solves of the first four grids, each stepped alone for 40
    steps, then K batch steps timed with it and K more without it (the plain
    batch from nearly the same state)."""
    import torch
    import torch_b200
    recs = []
    for tp, ic in cases[:4]:
        t = torch_b200.Torch(tp, ic, precision=prec, device=local)
        t.harvest(1 << 20)
        t.run_steps(40, dt_next)
        r, _ = t.harvest_read()
        recs.append(r)
        t.close()
    recs = np.concatenate(recs)
    t0 = time.perf_counter()
    net = torch_b200.Mlp(device=local, seed=11)
    net.train(recs, epochs=30, batch=4096, lr=2e-3, seed=12)
    torch.cuda.synchronize(local)
    train_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.stream_handle(), device=f"cuda:{local}")

    def timed():
        b.run_steps(1, dt_next)  # captures this form's step graphs
        barrier(pg)
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.enqueue_steps(args.steps, dt_next)
        e1.record(stream)
        b.synchronize()
        torch.cuda.synchronize(local)
        barrier(pg)
        return max_over_ranks(pg, e0.elapsed_time(e1), local)

    b.learned_start(net)
    ms = timed()
    b.learned_start(None)
    ms_plain = timed()
    net.close()
    return {"value": cells * args.steps * world / (ms / 1e3), "ms_per_step": ms / args.steps,
            "plain_same_state": {"value": cells * args.steps * world / (ms_plain / 1e3),
                                 "ms_per_step": ms_plain / args.steps},
            "training": {"records": int(len(recs)), "grids": 4, "steps_each": 40, "epochs": 30,
                         "seconds": train_s}}


def timed_form(sim, args, local, pg, dt_next):
    """K steps of a context on its own stream, timed with CUDA events on that
    stream after one untimed step (which captures the sweep graphs), max over
    ranks (ms)."""
    import torch
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=f"cuda:{local}")
    sim.run_steps(1)
    barrier(pg)
    torch.cuda.synchronize(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sim.enqueue_steps(args.steps, dt_next)
    ev1.record(stream)
    sim.synchronize()
    torch.cuda.synchronize(local)
    barrier(pg)
    return max_over_ranks(pg, ev0.elapsed_time(ev1), local)


def time_learned(args, sim32, N, world, local, pg, sim64=None):
    """FP32 form with the learned starting iterate, after the plain FP32 timing:
    further FP32 steps record the plain solve's front cells until
    --learned-records records (or 400 steps), a network is trained on them on
    the GPU, then K steps are timed with it and K more without it (the plain
    form from nearly the same state: the harvest steps moved the front).
    With sim64 (the FP64 form's context), the state the learned timing starts
    from is also restored into the FP64 form and K of its steps are timed, so
    that the learned FP32 form and the plain FP64 form are compared on the
    same state.  Solver counters of two further steps with and without the
    network follow."""
    import torch
    import torch_b200
    sim32.harvest(int(args.learned_records))
    harvest_steps = 0
    while harvest_steps < 400:
        sim32.run_steps(10)
        harvest_steps += 10
        if sim32.harvest_read(count_only=True) >= args.learned_records:
            break
    recs, _ = sim32.harvest_read()
    sim32.harvest(0)
    t0 = time.perf_counter()
    net = torch_b200.Mlp(device=local, seed=11)
    hist = net.train(recs, epochs=30, batch=8192, lr=2e-3, seed=12)
    torch.cuda.synchronize(local)
    train_s = time.perf_counter() - t0
    dt_next = sim32.dt_max

    def timed():
        return timed_form(sim32, args, local, pg, dt_next)

    blob = sim32.checkpoint() if sim64 is not None else None
    sim32.learned_start(net)
    ms = timed()
    sim32.learned_start(None)
    ms_plain = timed()
    fp64_same = None
    if sim64 is not None:
        sim64.restore(blob)
        del blob
        ms64 = timed_form(sim64, args, local, pg, dt_next)
        fp64_same = {"value": N * args.steps * world / (ms64 / 1e3), "ms_per_step": ms64 / args.steps}
    # where the difference goes: event-bracketed passes of K steps with and without it
    breakdown = {}
    for name, n_ in (("learned", net), ("plain", None)):
        sim32.learned_start(n_)
        sim32.run_steps(1)
        sim32.profile(True)
        sim32.enqueue_steps(args.steps, dt_next)
        sim32.synchronize()
        breakdown[name] = {k: round(sim32.profile_read(k)[0] / args.steps, 4)
                           for k in ("graph_rad_sweep", "k_learned_infer", "k_hydro_stage_fp32", "k_rad_update",
                                     "k_thermo", "graph_colden_sweep")}
        sim32.profile(False)
    sim32.stats_enable(True)
    sim32.learned_start(net)
    sim32.run_steps(2)
    st = sim32.stats(reset=True)
    sim32.learned_start(None)
    sim32.run_steps(2)
    st_plain = sim32.stats(reset=True)
    sim32.stats_enable(False)
    net.close()
    return {"value": N * args.steps * world / (ms / 1e3), "ms_per_step": ms / args.steps,
            "plain_fp32_same_state": {"value": N * args.steps * world / (ms_plain / 1e3),
                                      "ms_per_step": ms_plain / args.steps},
            "plain_fp64_same_state": fp64_same,
            "training": {"records": int(len(recs)), "harvest_steps": harvest_steps, "epochs": 30,
                         "seconds": train_s, "loss_first_last": [float(hist[0]), float(hist[-1])]},
            "front_cells": st["front_cells"], "learned_cells": st["learned_cells"],
            "accepted": st["learned_accepted"] / max(1, st["learned_cells"]),
            "front_iters_per_cell": st["front_iters"] / max(1, st["front_cells"]),
            "front_iters_per_cell_plain": st_plain["front_iters"] / max(1, st_plain["front_cells"]),
            "picard_max": st["picard_max"], "picard_max_plain": st_plain["picard_max"],
            "ms_per_step_by_phase": breakdown,
            "note": "counters from two steps after the timed regions with the network, then two without it"}


def ifront_cells(hii, n):
    """I-front distance (cells) from the central star along +x: the first cell
    with HII < 0.5, linearly interpolated (the rule of the reference's
    scripts/misc/calc_if.py:43-56)."""
    x = hii.reshape(n, n, n)[n // 2, n // 2, n // 2:]
    for i in range(1, len(x)):
        if x[i] < 0.5:
            return (i - 1) + (x[i - 1] - 0.5) / (x[i - 1] - x[i])
    return float(len(x))


def run_validate(args, rank, local):
    """Accuracy of the FP32 form (and of the FP32 form with the learned start)
    against the FP64 form after --validate steps of the workload: density and
    pressure relative L1 and the I-front radius along +x."""
    import torch_b200
    if rank != 0:
        return 0
    tp, ic = build_workload(args.workload, args.n)
    n, steps = args.n, args.validate
    g, nd = tp.heatCapacityRatio, int(ic.nd)

    def pressure(U):
        return (U[1] - sum(U[4 + i] ** 2 for i in range(nd)) / (2.0 * U[0])) * (g - 1.0)

    def rel(a, b):
        return float(np.abs(a - b).sum() / np.abs(b).sum())

    t0 = time.perf_counter()
    ref = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP64, device=local)
    ref.run_steps(steps)
    s_ref = ref.state()
    ref.close()
    out = {"metric": "FP32-form error against the FP64 form", "workload": f"{args.workload} {n}^3", "steps": steps,
           "fp64_time_code": s_ref.time}
    if tp.radiation_on:
        out["ifront_fp64_cells"] = ifront_cells(s_ref.Q[2], n)
    forms = [("fp64_perturbed", "perturbed"), ("fp32", None)]
    if tp.radiation_on and args.learned:
        forms.append(("fp32_learned", "learned"))
    for name, extra in forms:
        if extra == "perturbed":
            # the problem's own sensitivity: the FP64 form from a density perturbed by 1e-7 (random, seeded)
            rng = np.random.default_rng(7)
            ic_p = dataclasses.replace(ic, den=ic.den * (1.0 + 1e-7 * rng.standard_normal(ic.den.shape)))
            sim = torch_b200.Torch(tp, ic_p, precision=torch_b200.PRECISION_FP64, device=local)
        else:
            sim = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32, device=local)
            if args.fp32_contrast is not None:
                sim.fp32_contrast(args.fp32_contrast)
        net = None
        if extra == "learned":
            # training set: the plain solve's front cells over the first 20 steps of a separate run
            h = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32, device=local)
            h.harvest(1 << 23)
            h.run_steps(20)
            recs, _ = h.harvest_read()
            h.close()
            net = torch_b200.Mlp(device=local, seed=11)
            net.train(recs, epochs=30, batch=4096, lr=2e-3, seed=12)
            sim.learned_start(net)
        sim.run_steps(steps)
        s = sim.state()
        sim.close()
        if net is not None:
            net.close()
        res = {"den_rel_l1": rel(s.U[0], s_ref.U[0]), "pre_rel_l1": rel(pressure(s.U), pressure(s_ref.U))}
        if tp.radiation_on:
            res["ifront_cells"] = ifront_cells(s.Q[2], n)
            res["ifront_diff_cells"] = abs(res["ifront_cells"] - out["ifront_fp64_cells"])
        out[name] = res
    out["wall_s"] = time.perf_counter() - t0
    print(json.dumps(out), flush=True)
    return 0


def run_ours(args, world, rank, local, pg):
    import torch
    import torch_b200

    tp, ic = build_workload(args.workload, args.n)
    N = int(np.prod(ic.ncells))
    forms = ["fp32", "fp64"] if args.precision == "both" else [args.precision]
    results = {}
    clocks = ClockSampler(local)
    clocks.start()
    sims = {}
    for form in forms:
        prec = torch_b200.PRECISION_FP32 if form == "fp32" else torch_b200.PRECISION_FP64
        ms, launches, prof, sim = time_form(args, prec, tp, ic, local, pg, PROFILE_NAMES)
        ms = max_over_ranks(pg, ms, local)
        results[form] = (ms, launches, prof)
        sims[form] = sim
    clk = clocks.stop()
    head = forms[0]
    ms_max, launches, prof = results[head]
    value = N * args.steps * world / (ms_max / 1e3)
    sim = sims[head]
    sim_tile = getattr(sim, "tile", None)
    error = None
    if "fp64" in sims and head != "fp64":
        # both forms advanced W + K steps from the same initial state
        error = form_error(sims[head], sims["fp64"], tp.heatCapacityRatio, int(ic.nd))
        error["steps"] = args.warmup + args.steps
        error["against"] = "plain FP64 form on the GPU (bit-exact twin of the FP64 oracle)"
    learned = None
    if args.learned and head == "fp32" and tp.radiation_on:
        learned = time_learned(args, sims["fp32"], N, world, local, pg, sims.get("fp64"))
    for form, s in sims.items():
        if form != head:
            s.close()

    # roofline of the dominant hydro kernel
    peak, peak_kind = hbm_peak()
    if head == "fp32" and args.workload == "sedov":
        kname = "k_hydro_stage_fp32"
        # algorithmic bytes per cell per RK2 step in FP32: stage 1 reads U0 (28 B) and
        # writes U* (28 B); stage 2 reads U* and U0 and writes U1 (84 B): 140 B per two launches
        alg_per_launch = 140.0 * N / 2.0
    elif head == "fp32":
        kname = "k_hydro_stage_fp32"
        # FP32 form of a radiation-hydro run: one launch per hydro sub-step on the
        # FP64 state, reading U (7 x 8 B) and writing the new U and its Q (2 x 7 x 8 B)
        alg_per_launch = 168.0 * N
    else:
        kname = "k_faces_fp64"
        # FP64 plain form, per face-flux launch (one per dimension, 2 stages):
        # reads the 7 primitive fields (8 B each) and writes 7 flux fields
        alg_per_launch = (7 * 8 + 7 * 8) * N
    tot_ms, count = prof.get(kname, (0.0, 0))
    avg_ms = tot_ms / count if count else float("nan")
    achieved = alg_per_launch / (avg_ms / 1e3) / 1e9 if count else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                traffic = json.load(f).get(f"{kname}:{args.workload}:{args.n}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": kname, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "avg_launch_ms": avg_ms, "launches": count, "algorithmic_bytes_per_launch": alg_per_launch}
    total_prof = sum(x[0] for x in prof.values())
    kernel_share = {k: {"ms": v[0], "launches": v[1], "share": v[0] / max(1e-9, total_prof)} for k, v in prof.items()}
    other = {}
    for form in forms[1:]:
        ms_o, l_o, p_o = results[form]
        other[f"plain_{form}"] = {"value": N * args.steps * world / (ms_o / 1e3), "ms_per_step": ms_o / args.steps,
                                  "gpu_launches": int(l_o)}

    # end to end: host buffers through the C ABI, copies inside the timed region
    e2e = None
    if args.e2e_steps > 0:
        dt_next = sim.dt_max
        st = sim.state()
        U_host = torch.from_numpy(st.U).pin_memory()
        U_out = torch.empty_like(U_host).pin_memory()
        Un = U_host.numpy()
        Uo = U_out.numpy()
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            sim.set_conserved(Un)
            sim.full_step(dt_next)
            sim.lib.trg_get_state(sim.ctx, Uo.ctypes.data_as(torch_b200.C.c_void_p), None, None, None, None)
        wall = time.perf_counter() - t0
        wall = max_over_ranks(pg, wall, local)
        e2e = {"value": N * args.e2e_steps * world / wall, "unit": UNIT,
               "h2d_bytes_per_step": int(Un.nbytes), "d2h_bytes_per_step": int(Uo.nbytes),
               "steps": args.e2e_steps,
               "note": "per step through the C ABI: pinned H2D of U (FP64), trg_full_step, D2H of U (FP64)"}
    sim.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, kind, cores, desc = cpu_sample(args.workload, 48 if args.workload == "sedov" else 32,
                                                 args.cpu_steps, max(1, min(os.cpu_count() or 1, 16)))
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": desc}
        except Exception as e:  # a missing CPU baseline must not hide the GPU number
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(e)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if head == "fp32" else "f64",
            "data": "synthetic",
            "config": dict(workload_config(args.workload, args.n, head, world),
                           autotuned_tile_z=getattr(sim_tile, "__getitem__", lambda i: None)(0)),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk, "kernels": kernel_share, "error_vs_fp64": error, "learned_fp32": learned,
        }
        line.update(other)
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["hii", "sedov", "batch", "blister"], default="hii")
    ap.add_argument("--thermo-queue", type=int, default=0,
                    help="thermal sub-cycles of cells with at least this many run through the work queue (0: off)")
    ap.add_argument("--grids", type=int, default=256, help="grids of the batch workload")
    ap.add_argument("--fp32-contrast", type=float, default=None,
                    help="pressure ratio above which the FP32 form updates a hydro cell in FP64 (library default 1e3)")
    ap.add_argument("--validate", type=int, default=0,
                    help="instead of timing: error of the FP32 form against the FP64 form after this many steps")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--tile-z", type=int, default=0,
                    help="FP32 hydro kernel tile depth (z planes per CTA) in place of the autotuner's choice")
    ap.add_argument("--precision", choices=["both", "fp32", "fp64"], default="both")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the FP32 + learned-start measurement")
    ap.add_argument("--learned-records", type=float, default=1e7,
                    help="front-cell solves harvested for the learned start's training set")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            return run_reference_arm(args, rank)
        if args.validate:
            return run_validate(args, rank, local)
        if args.workload == "batch":
            return run_batch(args, world, rank, local, pg)
        return run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
