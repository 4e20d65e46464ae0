#!/usr/bin/env python
"""Benchmark of the B200-native force-and-constraint path.

Workload (default): 65,536-molecule SPC water (196,608 atoms) -- rigid SPC,
SETTLE, LJ O-O + erfc real space at 9 A, SPME order 4 on a 128^3 grid
(~1 A), Langevin at 300 K, dt = 2 fs; seeded synthetic lattice start.
One "step" is one full MD step (integrator + constraints + neighbour
pre-step + pair forces + SPME) on device-resident state.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line.  `value` is aggregate atom-steps/s over all
ranks (each rank runs an independent replica: the path does not shard, so
N > 1 is replicas only and scaling is weak).  Device time comes from CUDA
events recorded by the library on its own stream around each step; between
timed steps the L2 cache is flushed by writing a 256 MiB buffer (outside the
timed region).  `e2e` repeats the measurement through the public C ABI with
host buffers: every step uploads positions and velocities and downloads
them again, wall-clock timed.  `--impl reference` times the CPU restatement
of the same path (oracle/, FP64, all host cores) -- the reference itself is
Rust + CUDA and cannot be built here.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ns/day and atom-steps/s on 1 B200, chosen vs plain form at matched force error"
UNIT = "atom-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--molecules", type=int, default=65536)
    p.add_argument("--skin", type=float, default=1.0, help="neighbour-list skin in angstrom")
    p.add_argument("--e2e-steps", type=int, default=20)
    p.add_argument("--equilibrate", type=int, default=300,
                   help="untimed Langevin steps (friction 50/ps) that relax the lattice start")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="water65536",
                   choices=["water65536", "batch64", "learned_shake", "argon10000"],
                   help="water65536: the NPT water box (headline); batch64: the 64-box uneven "
                        "replica batch, batched graph vs 64 sequential plain runs; learned_shake: the "
                        "solvated chain with the learned SHAKE warm start; argon10000: LJ argon NVE "
                        "(water65536 with --molecules 8192 --barostat 0 is the 8,192-water NVT box)")
    p.add_argument("--barostat", type=int, default=1,
                   help="1: NPT with the Monte-Carlo barostat at 1 bar (move every 25 steps); 0: NVT")
    p.add_argument("--tune", type=int, default=1, help="autotune the neighbour-list skin (1/0)")
    p.add_argument("--reference-cuda", type=int, default=1,
                   help="1: also time the reference's own CUDA path (oracle/_ref) on the relaxed "
                        "state, outside the timed region")
    p.add_argument("--graphs", type=int, default=1,
                   help="1: CUDA-graph steps (headline); 0: eager launches (for profilers, which "
                        "cannot see kernels inside graphs with conditional nodes)")
    return p.parse_args()


def workload_config(args, spec, world):
    return {
        "workload": f"spc-water-{args.molecules} (N={spec.n} atoms), SETTLE, LJ+erfc r_cut 9 A, "
                    f"SPME p={spec.order} grid {spec.grid[0]}^3, Langevin 300 K, dt {spec.dt_fs} fs",
        "atoms": spec.n,
        "grid": list(spec.grid),
        "barostat": ("Monte-Carlo, 1 bar, a volume move after every 25th step (device-side, "
                     "inside the step graphs); the step counter is phased so that the timed "
                     "window holds at least one move" if args.barostat else "none (NVT)"),
        "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
        "l2": "flushed between timed steps (256 MiB write, outside the timed region)",
        "start": f"lattice, relaxed by {args.equilibrate} untimed Langevin steps (50/ps)",
    }


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def force_error(F, Fo):
    """RMS and max force error relative to the reference forces Fo."""
    rms = float(np.sqrt(((F - Fo) ** 2).sum() / (Fo ** 2).sum()))
    mx = float(np.abs(F - Fo).max() / np.sqrt((Fo ** 2).sum(axis=1).mean()))
    return rms, mx


def cpu_baseline(spec, state=None, forces_gpu=None, budget_s=25.0):
    """The FP64 CPU restatement (oracle/) timed on the host cores on a bounded
    sample of the same workload: whole MD steps until ~budget_s, from the
    GPU arm's relaxed state when given.  As the checker it also evaluates
    the FP64 forces at that state, which gives the GPU forces' error."""
    import oracle as O

    cores = os.cpu_count() or 1
    err = None
    pos0 = vel0 = None
    if state is not None:
        import copy

        pos0, vel0, box = state
        spec = copy.copy(spec)
        spec.box = np.asarray(box, dtype=np.float64)  # the barostat has moved the cell
        if forces_gpu is not None:
            Fo, _, _, _ = O.forces(spec, pos0, n_threads=cores)
            rms, mx = force_error(forces_gpu, Fo)
            err = {"rms_rel": rms, "max_rel": mx,
                   "vs": "FP64 CPU oracle (exact erfc) at the state the timed steps ended in"}
    t0 = time.perf_counter()
    pos, vel, _ = O.md_run(spec, 1, "langevin", positions=pos0, velocities=vel0, n_threads=cores)
    first = time.perf_counter() - t0  # one step + initial force evaluation
    per_step_guess = first / 2.0
    k = max(1, min(20, int(budget_s / max(per_step_guess, 1e-3))))
    t0 = time.perf_counter()
    O.md_run(spec, k, "langevin", positions=pos, velocities=vel, n_threads=cores)
    dt = time.perf_counter() - t0
    # md_run evaluates the starting forces once before its k steps
    steps_equiv = k + 1
    start = "the GPU arm's relaxed state" if state is not None else "the lattice start"
    base = {"value": spec.n * steps_equiv / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{k} Langevin+SETTLE MD steps (+1 initial force evaluation) of the full "
                      f"{spec.n}-atom system from {start}, FP64 oracle (no barostat), {dt:.1f} s"}
    return base, err


def reference_cuda(spec, pos, box, skins_A, rebuilds_per_step):
    """The reference's own CUDA force path (oracle/_ref: its kernels built
    for sm_100a, its composed pair kernel regenerated from its templates,
    cuFFT) timed on the same B200 and the same relaxed positions, outside
    the timed region.  Per skin: mean device ms of one forces-only
    evaluation and of each of its stages, of one neighbour rebuild, and the
    force error against the product's forces is the tests' business."""
    import copy

    from heddle_b200 import units as U
    from oracle import refpath as R

    if not R.available():
        return {"unavailable": "oracle/_ref not built (the reference tree was absent at build time)"}
    out = {"what": "HeddleMD kernels/*.cu + composed LJ+erfc pair kernel + cuFFT, replayed by "
                   "oracle/ref_harness.cpp with the reference's launch shapes; f32, forces only"}
    for skin in skins_A:
        s = copy.copy(spec)
        s.r_skin = U.angstrom_au(skin)
        ref = R.RefForceField(s, positions=pos, box=box)
        try:
            ref.rebuild()
            t = ref.time(reps=10, energies=False)
            st = ref.stats()
        finally:
            ref.close()
        row = {"eval_ms": t["eval"], "rebuild_ms": t["rebuild"],
               "stage_us": {k: 1e3 * v for k, v in t.items() if k not in ("eval", "rebuild")},
               "entries": st["entries"], "single_pairs": st["single_pairs"], "cells": st["cells"]}
        if skin in rebuilds_per_step:
            row["ms_per_step_estimate"] = t["eval"] + t["rebuild"] * rebuilds_per_step[skin]
            row["estimate"] = ("evaluation + rebuild x the rebuild rate the product measured at this "
                               "skin; the integrator and SETTLE kernels are not included")
        out[f"skin_{skin:g}A"] = row
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from heddle_b200 import systems as S
    import oracle as O

    spec = S.spc_water(args.molecules, skin_A=2.0)
    cores = os.cpu_count() or 1
    # warm-up: one step (capped so the whole run stays within minutes)
    t0 = time.perf_counter()
    pos, vel, _ = O.md_run(spec, max(1, min(args.warmup, 1)), "langevin", n_threads=cores)
    t_step = (time.perf_counter() - t0) / 2.0
    k = max(1, min(args.steps, int(120.0 / max(t_step, 1e-3))))
    t0 = time.perf_counter()
    O.md_run(spec, k, "langevin", positions=pos, velocities=vel, n_threads=cores)
    dt = time.perf_counter() - t0
    value = spec.n * (k + 1) / dt
    sample = (f"{k} of {args.steps} requested Langevin+SETTLE MD steps (+1 force evaluation) of the "
              f"full {spec.n}-atom system, FP64 CPU restatement, {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / (k + 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        # the GPU arm's system, integrator and cut-offs; this arm's own
        # start, barostat and arithmetic
        "config": dict(workload_config(args, spec, int(os.environ.get("WORLD_SIZE", "1"))),
                       barostat="none (the CPU restatement makes no volume moves; on the GPU a "
                                "move costs one energy evaluation every 25 steps, about +4 %)",
                       start="lattice start, no relaxation",
                       arithmetic="FP64 throughout (the GPU arm: FP32 with fixed-point sums)"),
        "ns_per_day": spec.dt_fs * ((k + 1) / dt) * 0.0864,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def dist_setup(backend: str, local: int = 0):
    """(world size, rank, torch.distributed or None) from the launcher's
    environment: one process per GPU, replicas only (no exchange step); the
    group carries only barriers and the max-over-ranks timing.  A short
    timeout ends a rank that waits for a dead peer with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world <= 1:
        return world, rank, None
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
    dist.init_process_group(backend, timeout=timedelta(seconds=300), **kw)
    return world, rank, dist


def max_over_ranks(x: float, dist, device) -> float:
    """The largest value over all ranks (every rank gets it)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args):
    import torch

    import heddle_b200 as hb
    from heddle_b200 import systems as S
    from heddle_b200 import units as U

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    world, rank, dist = dist_setup("nccl", local)

    spec = S.spc_water(args.molecules, skin_A=args.skin, seed=11 + rank, velocity_seed=5 + rank)
    ctx = hb.Context(local)
    sys_ = hb.System.from_spec(ctx, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    cons.after_kick(0.0)  # initial velocity projection onto the constraint manifold
    lang = dict(kind="langevin-baoab", dt=spec.dt, friction=spec.friction,
                temperature=spec.temperature, seed=1234 + rank)
    # relax the lattice start (untimed): stiff thermostat
    ff0 = hb.ForceField.from_spec(sys_, spec)
    eq = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=50.0 / (1.0e-12 / U.AUT_S),
                       temperature=spec.temperature, seed=99 + rank)
    (eq.step_graph if args.graphs else eq.step)(ff0, cons, n_steps=args.equilibrate)
    eq.close()
    ff0.close()
    # skin autotuning on the relaxed system (untimed)
    tune = None
    if args.tune and args.graphs:
        from heddle_b200.autotune import tune_skin

        tune = tune_skin(ctx, sys_, spec, cons, lang)
        args.skin = float(tune["best_A"])
    spec.r_skin = U.angstrom_au(args.skin)
    ff = hb.ForceField.from_spec(sys_, spec)
    if tune:
        from heddle_b200.autotune import apply

        apply(ff, tune)
    # phase the step counter so that a barostat move falls in the middle of
    # the timed window: before it run max(3, W) warm-up steps and the stage
    # breakdown's min(K, 20) steps; a move follows every 25th step
    done_before = max(3, args.warmup) + min(args.steps, 20)
    step0 = (-(done_before + (args.steps + 1) // 2)) % 25 if args.barostat else 0
    it = hb.Integrator(sys_, **lang, step0=step0)
    baro = None
    if args.barostat:
        baro = hb.Barostat(sys_, U.pressure_au_bar(1.0), spec.temperature, seed=4321 + rank,
                           frequency=25, molecules=(spec.mol_offsets, spec.mol_atoms))
        it.set_barostat(baro)
    per_step_kernels, rebuild_kernels, move_kernels = it.count_launches(ff, cons)
    run = it.step_graph if args.graphs else it.step
    run(ff, cons, n_steps=max(3, args.warmup))
    ctx.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    # stage breakdown (eager launches with per-stage events; not the headline)
    ctx.timing(True)
    stage = np.zeros(8)
    for _ in range(min(args.steps, 20)):
        it.step(ff, cons, n_steps=1)
        stage += ctx.timings()
    stage /= min(args.steps, 20)

    # headline: CUDA-graph steps, one step per launch, L2 flushed in between
    rebuilds0 = ff.stats()["rebuilds"]
    moves0 = baro.stats()["attempted"] if baro else 0
    t_ms = 0.0
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            run(ff, cons, n_steps=1)
            t_ms += float(ctx.timings()[0])
    ctx.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ctx.timing(False)
    # the state the timed steps ended in and its forces (outside the timed
    # region), for the force error against the FP64 oracle
    final_state = final_forces = ref_state = None
    if rank == 0:
        ref_state = (sys_.positions(), sys_.box())
    if rank == 0 and not args.no_cpu_baseline:
        ff.step(scalars=False)
        st = sys_.state()
        final_state, final_forces = (st[0], st[1], sys_.box()), sys_.forces()
    rebuilds = ff.stats()["rebuilds"] - rebuilds0
    baro_stats = baro.stats() if baro else None
    moves = int(baro_stats["attempted"] - moves0) if baro else 0
    t_ms = max_over_ranks(t_ms, dist, f"cuda:{local}")
    steps_s = args.steps / (t_ms / 1e3)
    value = world * spec.n * steps_s
    clocks = clk.summary()

    # end to end through the C ABI with page-locked host buffers: every step
    # uploads positions and velocities and reads the whole state back, in
    # single precision (the reference's own buffer precision) and, for
    # comparison, in FP64
    k2 = max(1, min(args.e2e_steps, args.steps))

    def e2e(dtype, fused):
        host = tuple(torch.empty((spec.n, 3), dtype=dt, pin_memory=True).numpy()
                     for dt in (dtype, dtype, torch.int32, dtype))
        get = sys_.state_f32 if dtype == torch.float32 else (lambda out: sys_.state(out=out))
        put = sys_.set_state_f32 if dtype == torch.float32 else sys_.set_state
        get(host)
        if fused:  # one call per step: upload, step, read-out (captures its graph here)
            it.step_exchange(ff, cons, 1, host[0], host[1], host)
        else:
            run(ff, cons, n_steps=1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k2):
            if fused:
                # the inputs alias the outputs: the upload completes before the step
                it.step_exchange(ff, cons, 1, host[0], host[1], host)
            else:
                put(host[0], host[1])
                run(ff, cons, n_steps=1)
                get(host)
        return max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")

    fused = bool(args.graphs)
    t_e2e = e2e(torch.float32, fused)
    t_e2e_sep = e2e(torch.float32, False) if fused else t_e2e
    t_e2e64 = e2e(torch.float64, False)
    e2e_value = world * spec.n * k2 / t_e2e

    peak, peak_kind = measured_peaks()
    pair_ms = float(stage[1])
    m_grid = int(np.prod(spec.grid))
    pair_bytes = 28.0 * spec.n  # algorithmic: read posq 16 B + write force 12 B per atom
    achieved = pair_bytes / (pair_ms * 1e-3) / 1e9 if pair_ms > 0 else 0.0
    step_bytes = 100.0 * spec.n + 24.0 * m_grid
    stats = ff.stats()

    line = None
    if rank == 0:
        traffic = None
        tf = ROOT / "profiles" / "pair_kernel_traffic.json"
        if tf.exists():
            try:
                traffic = json.loads(tf.read_text()).get("dram_bytes_per_launch_full_size")
            except Exception:
                traffic = None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup) + args.equilibrate, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, spec, world),
            "ns_per_day": spec.dt_fs * steps_s * 0.0864,
            "stage_ms_per_step_eager": {"total": float(stage[0]), "pair": pair_ms,
                                        "spme_concurrent": float(stage[2]),
                                        "neighbour": float(stage[3]),
                                        "integrate_constrain": float(stage[4])},
            "neighbour": {"tiles": stats["tiles"], "entries": stats["entries"],
                          "rebuilds_in_timed_steps": rebuilds, "skin_A": args.skin,
                          "skin_autotune": tune},
            "launch_mode": ("CUDA graph per step; neighbour rebuild = device-side conditional node"
                            if args.graphs else "eager launches"),
            "roofline": {"bound": "hbm", "kernel": "k_pair4 (LJ + erfc pair kernel)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "note": "algorithmic bytes 28 B/atom per launch; the kernel is latency- and "
                                 "issue-limited (no pipe saturated), not HBM-bound; traffic is the "
                                 "packed neighbour entries read once per launch"},
            "step_roofline": {"bytes_per_step": step_bytes,
                              "achieved_gbs": step_bytes / (t_ms / args.steps * 1e-3) / 1e9,
                              "frac": step_bytes / (t_ms / args.steps * 1e-3) / 1e9 / peak},
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 3 * 4 * spec.n,
                    "d2h_bytes_per_step": (3 * 3 * 4 + 3 * 4) * spec.n,
                    "note": "per step, page-locked host buffers: positions + velocities (f32) "
                            "in; positions, velocities, forces (f32) and images (i32) out; wall "
                            "clock, over the C ABI: " + (
                                "one hb_integrator_step_exchange_f32 call per step (positions "
                                "and images copied out during the force evaluation)" if fused else
                                "hb_system_set_state_f32 / hb_integrator_step / "
                                "hb_system_get_state_f32"),
                    "separate_calls": {"value": world * spec.n * k2 / t_e2e_sep,
                                       "calls": "hb_system_set_state_f32 / hb_integrator "
                                                "step / hb_system_get_state_f32"},
                    "f64_exchange": {"value": world * spec.n * k2 / t_e2e64,
                                     "h2d_bytes_per_step": 2 * 3 * 8 * spec.n,
                                     "d2h_bytes_per_step": (3 * 3 * 8 + 3 * 4) * spec.n}},
            "gpu_launches": (per_step_kernels * args.steps + rebuild_kernels * rebuilds +
                             move_kernels * moves),
            "barostat": ({"moves_in_timed_steps": moves, "volume_A3": baro_stats["volume"] *
                          (U.BOHR_M / U.ANGSTROM_M) ** 3, "acceptance": baro_stats["acceptance"]}
                         if baro else None),
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"], line["force_error"] = cpu_baseline(spec, final_state, final_forces)
        if ref_state is not None and args.reference_cuda:
            try:
                line["reference_cuda"] = reference_cuda(
                    spec, ref_state[0], ref_state[1], [args.skin, 2.7],
                    {args.skin: rebuilds / args.steps})
            except Exception as exc:  # the comparison never costs the headline
                line["reference_cuda"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(line), flush=True)
    it.close()
    if baro:
        baro.close()
    cons.close()
    ff.close()
    sys_.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """The 64-box uneven replica batch: every box's step in one CUDA graph
    (one launch per step) against the same boxes advanced one after another,
    each with its own CUDA-graph steps (64 sequential plain runs)."""
    import torch

    import heddle_b200 as hb
    from heddle_b200 import systems as S
    from heddle_b200 import units as U

    torch.cuda.set_device(0)
    specs = S.replica_batch()
    n_atoms = sum(sp.n for sp in specs)
    master = hb.Context(0)
    objs = []
    for k, sp in enumerate(specs):
        c = hb.Context(0)
        sys_ = hb.System.from_spec(c, sp)
        cons = hb.Constraints.from_spec(sys_, sp)
        cons.after_kick(0.0)
        ff = hb.ForceField.from_spec(sys_, sp)
        eq = hb.Integrator(sys_, "langevin-baoab", sp.dt, friction=50.0 / (1.0e-12 / U.AUT_S),
                           temperature=sp.temperature, seed=99 + k)
        eq.step_graph(ff, cons, n_steps=args.equilibrate)
        eq.close()
        it = hb.Integrator(sys_, "langevin-baoab", sp.dt, friction=sp.friction,
                           temperature=sp.temperature, seed=1234 + k)
        objs.append((c, sys_, ff, cons, it))
    batch = hb.Batch(master, [(o[4], o[2], o[3]) for o in objs])
    per_step_kernels, rebuild_kernels = batch.count_launches()
    batch.step(max(3, args.warmup))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    rebuilds0 = sum(o[2].stats()["rebuilds"] for o in objs)
    master.timing(True)
    t_ms = 0.0
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            batch.step(1)
            t_ms += float(master.timings()[0])
    master.timing(False)
    rebuilds = sum(o[2].stats()["rebuilds"] for o in objs) - rebuilds0
    one_launch = batch.pair_form()
    # the same batch with one multi-system pair launch for all members, for
    # comparison with the default (a pair kernel per member)
    batch.set_pair_form(True)
    batch.step(2)
    master.timing(True)
    t_per = 0.0
    k_per = max(3, args.steps // 2)
    for _ in range(k_per):
        flush.zero_()
        torch.cuda.synchronize()
        batch.step(1)
        t_per += float(master.timings()[0])
    master.timing(False)
    batch.set_pair_form(False)
    batch.step(1)
    # 64 sequential plain runs (each box's own CUDA-graph steps, one box
    # after another), wall clock
    k_seq = max(1, args.steps // 4)
    for o in objs:
        o[4].step_graph(o[2], o[3], n_steps=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for o in objs:
        o[4].step_graph(o[2], o[3], n_steps=k_seq)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    # batched, wall clock over the same number of steps (no flush); one
    # untimed call first re-captures the graph if the eager steps grew a list
    batch.step(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.step(k_seq)
    torch.cuda.synchronize()
    t_batch_wall = time.perf_counter() - t0
    value = n_atoms * args.steps / (t_ms * 1e-3)
    # force error against the FP64 oracle for the smallest, a middle and the
    # largest box at the state the timed steps ended in (outside the timed
    # region)
    import copy

    import oracle as O

    order = sorted(range(len(specs)), key=lambda k: specs[k].n)
    ferr = {}
    for k in (order[0], order[len(order) // 2], order[-1]):
        c, sys_k, ff_k, _, _ = objs[k]
        ff_k.step(scalars=False)
        sp = copy.copy(specs[k])
        sp.box = sys_k.box()
        Fo, _, _, _ = O.forces(sp, sys_k.positions(), n_threads=os.cpu_count() or 1)
        rms, mx = force_error(sys_k.forces(), Fo)
        ferr[f"box{k}_{sp.n // 3}mol"] = {"rms_rel": rms, "max_rel": mx}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": max(3, args.warmup) + args.equilibrate, "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"replica batch: {len(specs)} SPC water boxes, N_mol log-uniform "
                               f"[256, 8192] (seed 2025), {n_atoms} atoms, Langevin 300 K + SETTLE, "
                               "SPME ~1 A grids, r_cut 9 A",
                   "atoms": n_atoms, "boxes": len(specs),
                   "l2": "flushed between timed steps (256 MiB write, outside the timed region)"},
        "batched_graph": {"atom_steps_per_s_device": value,
                          "atom_steps_per_s_wall": n_atoms * k_seq / t_batch_wall,
                          "pair_form": ("one persistent pair kernel over all members' work items"
                                        if one_launch else "a pair kernel per member")},
        "batched_graph_one_pair_launch": {"atom_steps_per_s_device": n_atoms * k_per / (t_per * 1e-3),
                                          "ms_per_step": t_per / k_per,
                                          "pair_form": "one persistent pair kernel over all members' "
                                                       "work items"},
        "sequential_plain": {"atom_steps_per_s_wall": n_atoms * k_seq / t_seq, "steps": k_seq},
        "speedup_wall": t_seq / t_batch_wall,
        "force_error": dict(ferr, vs="FP64 CPU oracle at the final state"),
        "rebuilds_in_timed_steps": rebuilds,
        "clocks": clk.summary(),
        "gpu_launches": per_step_kernels * args.steps + (rebuild_kernels // len(specs)) * rebuilds,
    }
    print(json.dumps(line), flush=True)
    batch.close()
    for o in objs:
        for x in (o[4], o[3], o[2], o[1], o[0]):
            x.close()
    master.close()
    return 0


def run_learned_shake(args):
    """The solvated 166-atom chain: plain SHAKE (relative tolerance 1e-8)
    against SHAKE warm-started by the tensor-core MLP trained on 1e5
    multiplier samples recorded from plain runs."""
    import torch

    import heddle_b200 as hb
    from heddle_b200 import systems as S
    from heddle_b200 import units as U
    import oracle as O
    from oracle import mlp as M

    torch.cuda.set_device(0)
    ctx = hb.Context(0)
    spec = S.peptide_in_water()
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    cons.after_kick(0.0)
    for dt_fs, fric, n in ((0.25, 100.0, 400), (1.0, 20.0, 200), (2.0, 5.0, 200)):
        eq = hb.Integrator(sys_, "langevin-baoab", U.time_au_fs(dt_fs),
                           friction=fric / (1.0e-12 / U.AUT_S), temperature=spec.temperature, seed=5)
        eq.step(ff, cons, n_steps=n)
        eq.close()
    pos0, vel0, _, _ = sys_.state()
    it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                       temperature=spec.temperature, seed=17)
    # 1) training data: multipliers of plain SHAKE, 1e5 samples
    cons.record(True)
    rows, t0 = [], time.perf_counter()
    while sum(len(r["lam"]) for r in rows) < 100_000:
        it.step(ff, cons, n_steps=1)
        rows.append(cons.get_record())
    t_collect = time.perf_counter() - t0
    cons.record(False)
    feats = np.concatenate([r["features"] for r in rows])[:100_000]
    targ = np.concatenate([(r["lam"] - r["lam1"]) * r["lscale"] for r in rows]).astype(np.float32)[:100_000]
    # 2) training on the device
    net = hb.ShakeMLP(ctx, seed=2)
    mean, std = feats.mean(0), feats.std(0) + 1e-6
    net.set_normalization(mean, 1.0 / std, float(targ.std() + 1e-12))
    g_dev, _ = net.gradients(feats[:1024], targ[:1024])
    g_orc, _ = M.gradients(net.params(), feats[:1024], targ[:1024], mean, 1.0 / std,
                           float(targ.std() + 1e-12))
    grad_err = float(np.linalg.norm(g_dev - g_orc) / np.linalg.norm(g_orc))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = net.train(feats, targ, epochs=40, batch=512, lr=2e-3, seed=3)
    t_train = time.perf_counter() - t0

    def measure(warm):
        sys_.set_state(pos0, vel0)
        cons.set_warm_start(net if warm else None)
        it2 = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                            temperature=spec.temperature, seed=99)
        it2.step_graph(ff, cons, n_steps=max(3, args.warmup))
        cons.shake_stats(reset=True)
        ctx.timing(True)
        it2.step_graph(ff, cons, n_steps=args.steps)
        ms = float(ctx.timings()[0])
        ctx.timing(False)
        st = cons.shake_stats()
        pos = sys_.positions()
        it2.close()
        res = []
        off, ga = spec.group_offsets, spec.group_atoms
        for g in range(len(spec.con_offsets) - 1):
            for k in range(spec.con_offsets[g], spec.con_offsets[g + 1]):
                a, b = ga[off[g] + spec.con_i[k]], ga[off[g] + spec.con_j[k]]
                d = np.linalg.norm(pos[a] - pos[b])
                res.append(abs(d * d / spec.con_dist[k] ** 2 - 1.0))
        return {"ms_per_step": ms / args.steps, "atom_steps_per_s": spec.n * args.steps / (ms * 1e-3),
                "mean_sweeps_per_group": st["mean_sweeps"], "max_rel_residual_f32": float(max(res))}

    plain = measure(False)
    warm = measure(True)
    ff.step(scalars=False)
    Fo, _, _, _ = O.forces(spec, sys_.positions(), n_threads=os.cpu_count() or 1)
    f_rms, f_max = force_error(sys_.forces(), Fo)
    # the product's cost gate: the warm start is attached only when its
    # step is faster than plain SHAKE's
    sys_.set_state(pos0, vel0)
    gate = cons.choose_warm_start(net, ff, "langevin-baoab", spec.dt, steps=args.steps,
                                  friction=spec.friction, temperature=spec.temperature, seed=99)
    chosen = warm if gate["chosen"] == "learned" else plain
    line = {
        "metric": METRIC, "value": chosen["atom_steps_per_s"], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": chosen["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"166-atom bonded chain (110 C-H SHAKE constraints, relative tol 1e-8) "
                               f"in 1900 SPC waters, {spec.n} atoms, grid {spec.grid[0]}^3, Langevin "
                               "300 K, dt 2 fs; learned SHAKE warm start",
                   "atoms": spec.n},
        "plain_shake": plain, "learned_warm_start": warm,
        "cost_gate": gate, "chosen_form": gate["chosen"],
        "force_error": {"rms_rel": f_rms, "max_rel": f_max, "vs": "FP64 CPU oracle (bonded + LJ + "
                        "SPME) at the state the warm-started run ended in"},
        "chosen_vs_plain": plain["ms_per_step"] / chosen["ms_per_step"],
        "sweeps_saved_fraction": 1.0 - warm["mean_sweeps_per_group"] / max(plain["mean_sweeps_per_group"], 1e-12),
        "training": {"samples": int(len(targ)), "epochs": 40, "batch": 512,
                     "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
                     "seconds": t_train, "collect_seconds": t_collect,
                     "gradient_rel_error_vs_oracle": grad_err},
    }
    print(json.dumps(line), flush=True)
    for o in (net, it, cons, ff, sys_, ctx):
        o.close()
    return 0


def run_argon(args):
    """Config 1: 10,000 LJ argon atoms, velocity Verlet NVE, dt 5 fs, f32,
    CUDA-graph steps; the force error against the FP64 oracle at the final
    state."""
    import torch

    import heddle_b200 as hb
    import oracle as O
    from heddle_b200 import systems as S

    torch.cuda.set_device(0)
    spec = S.lj_argon()
    ctx = hb.Context(0)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    it = hb.Integrator(sys_, "velocity-verlet", spec.dt)
    it.step_graph(ff, None, n_steps=max(3, args.warmup))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    ctx.timing(True)
    t_ms = 0.0
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            it.step_graph(ff, None, n_steps=1)
            t_ms += float(ctx.timings()[0])
    ctx.timing(False)
    ff.step(scalars=False)
    pos, F = sys_.positions(), sys_.forces()
    Fo, _, _, _ = O.forces(spec, pos)
    rms, mx = force_error(F, Fo)
    steps_s = args.steps / (t_ms * 1e-3)
    line = {
        "metric": METRIC, "value": spec.n * steps_s, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "lj-argon-10000: LJ argon NVE, f32, 10,000 atoms on a 22^3 grid with "
                               "jitter, r_c 2.5 sigma, velocity Verlet, dt 5 fs, CUDA graph per step",
                   "atoms": spec.n, "l2": "flushed between timed steps"},
        "ns_per_day": spec.dt_fs * steps_s * 0.0864, "clocks": clk.summary(),
        "force_error": {"rms_rel": rms, "max_rel": mx, "vs": "FP64 CPU oracle at the final state"},
    }
    print(json.dumps(line), flush=True)
    for o in (it, ff, sys_, ctx):
        o.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch64":
        return run_batch(args)
    if args.workload == "learned_shake":
        return run_learned_shake(args)
    if args.workload == "argon10000":
        return run_argon(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
