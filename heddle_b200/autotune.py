"""Autotuner for the neighbour-list skin and the force path's launch shapes.

The skin trades pair-kernel work (entries grow roughly as (r_cut + skin)^3)
against rebuild frequency (a rebuild runs when any atom moved more than
skin / 2).  The residency of the persistent pair kernel (blocks per SM)
trades its own throughput against room for the reciprocal-space chain that
runs concurrently on the second stream.  Both depend on the system, so they
are measured: each candidate skin gets its own force field on the same
device-resident system, a short run of CUDA-graph steps is timed with CUDA
events and the fastest wins; then, at that skin, one launch-shape knob at a
time (each kept at its best before the next is swept): the pair kernel's
residency, its entries per work item (shorter items balance better, longer
ones reload the i-tile less often), the reciprocal transform form (the
whole-plane pass or line passes, where both exist) and the gather form
(one thread per (atom, c offset) or per atom, spline orders 4 and 8).
Results are keyed by a size class (atoms, grid) and can be kept in a JSON
cache file.
"""

from __future__ import annotations

import json
from pathlib import Path

from . import units as U
from . import _native as N
from .api import Constraints, ForceField, Integrator, System


def size_class(spec) -> str:
    grid = "x".join(str(g) for g in spec.grid) if spec.grid else "none"
    return f"n{spec.n}-grid{grid}-rc{spec.r_cut_coul or 0:.3f}"


def _time_steps(ctx, sys_, ff, cons, integrator_kwargs, steps, warm) -> float:
    it = Integrator(sys_, **integrator_kwargs)
    it.step_graph(ff, cons, n_steps=warm)
    ctx.timing(True)
    it.step_graph(ff, cons, n_steps=steps)
    ms = float(ctx.timings()[0]) / steps
    ctx.timing(False)
    it.close()
    return ms


def tune_skin(ctx, sys_: System, spec, cons: Constraints | None, integrator_kwargs: dict,
              candidates_A=(1.2, 1.6, 2.0, 2.5, 3.0), residencies=(4, 5, 6, 7, 8),
              chunks=(2, 4, 8, 16), steps: int = 150, warm: int = 20,
              cache: Path | None = None) -> dict:
    """Time `steps` graph-mode MD steps per candidate skin (angstrom), then
    per launch-shape knob at the best skin; return {"best_A": skin,
    "pair_blocks_per_sm": r, "pair_chunk": c, "fft_plane": 0/1,
    "gather_form": 0/1, "ms_per_step": {skin: ms}, "residency_ms": {r: ms},
    "chunk_ms": {c: ms}, "fft_plane_ms": {...}, "gather_form_ms": {...}}.
    Skins the box cannot hold are skipped.  The system state advances
    during tuning (the runs are real MD steps)."""
    from ._native import HeddleError

    key = size_class(spec)
    if cache is not None and cache.exists():
        data = json.loads(cache.read_text())
        if key in data:
            return data[key]
    times = {}
    for skin in candidates_A:
        try:
            ff = ForceField.from_spec(sys_, spec, r_skin=U.angstrom_au(skin))
        except HeddleError:
            continue  # 2 (r_cut + skin) does not fit the box
        times[skin] = _time_steps(ctx, sys_, ff, cons, integrator_kwargs, steps, warm)
        ff.close()
    best = min(times, key=times.get)
    ff = ForceField.from_spec(sys_, spec, r_skin=U.angstrom_au(best))

    def sweep(param, values):
        t = {}
        for v in values:
            N.check(ff.lib.hb_forcefield_set_launch(ff.h, param, int(v)))
            t[v] = _time_steps(ctx, sys_, ff, cons, integrator_kwargs, steps, warm)
        b = min(t, key=t.get)
        N.check(ff.lib.hb_forcefield_set_launch(ff.h, param, int(b)))
        return b, {str(k): v for k, v in t.items()}

    best_r, res_times = sweep(N.HB_LAUNCH_PAIR_BLOCKS_PER_SM, residencies)
    best_c, chunk_times = sweep(N.HB_LAUNCH_PAIR_CHUNK, chunks)
    result = {"best_A": best, "pair_blocks_per_sm": best_r, "pair_chunk": best_c,
              "ms_per_step": {str(k): v for k, v in times.items()},
              "residency_ms": res_times, "chunk_ms": chunk_times}
    grid = spec.grid if spec.alpha is not None else None
    if grid is not None:
        if grid[0] == grid[1] and grid[0] in (64, 128):
            result["fft_plane"], result["fft_plane_ms"] = sweep(N.HB_LAUNCH_FFT_PLANE, (1, 0))
        if spec.order in (4, 8):
            result["gather_form"], result["gather_form_ms"] = sweep(N.HB_LAUNCH_GATHER_FORM, (1, 0))
    ff.close()
    if cache is not None:
        data = json.loads(cache.read_text()) if cache.exists() else {}
        data[key] = result
        cache.write_text(json.dumps(data, indent=1))
    return result


def apply(ff: ForceField, tuned: dict) -> None:
    """Set a force field's launch shapes to an autotuner result."""
    for key, param in (("pair_blocks_per_sm", N.HB_LAUNCH_PAIR_BLOCKS_PER_SM),
                       ("pair_chunk", N.HB_LAUNCH_PAIR_CHUNK),
                       ("fft_plane", N.HB_LAUNCH_FFT_PLANE),
                       ("gather_form", N.HB_LAUNCH_GATHER_FORM)):
        if key in tuned:
            N.check(ff.lib.hb_forcefield_set_launch(ff.h, param, int(tuned[key])))
