"""Autotuner for the neighbour-list skin and the pair kernel's launch shape.

The skin trades pair-kernel work (entries grow roughly as (r_cut + skin)^3)
against rebuild frequency (a rebuild runs when any atom moved more than
skin / 2).  The residency of the persistent pair kernel (blocks per SM)
trades its own throughput against room for the reciprocal-space chain that
runs concurrently on the second stream.  Both depend on the system, so they
are measured: each candidate skin gets its own force field on the same
device-resident system, a short run of CUDA-graph steps is timed with CUDA
events and the fastest wins; then the residency is swept at that skin.
Results are keyed by a size class (atoms, grid) and can be kept in a JSON
cache file.
"""

from __future__ import annotations

import json
from pathlib import Path

from . import units as U
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
              steps: int = 150, warm: int = 20, cache: Path | None = None) -> dict:
    """Time `steps` graph-mode MD steps per candidate skin (angstrom), then
    per pair-kernel residency at the best skin; return {"best_A": skin,
    "pair_blocks_per_sm": r, "ms_per_step": {skin: ms}, "residency_ms":
    {r: ms}}.  Skins the box cannot hold are skipped.  The system state
    advances during tuning (the runs are real MD steps)."""
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
    res_times = {}
    ff = ForceField.from_spec(sys_, spec, r_skin=U.angstrom_au(best))
    for r in residencies:
        ff.set_launch(pair_blocks_per_sm=r)
        res_times[r] = _time_steps(ctx, sys_, ff, cons, integrator_kwargs, steps, warm)
    ff.close()
    best_r = min(res_times, key=res_times.get)
    result = {"best_A": best, "pair_blocks_per_sm": best_r,
              "ms_per_step": {str(k): v for k, v in times.items()},
              "residency_ms": {str(k): v for k, v in res_times.items()}}
    if cache is not None:
        data = json.loads(cache.read_text()) if cache.exists() else {}
        data[key] = result
        cache.write_text(json.dumps(data, indent=1))
    return result
