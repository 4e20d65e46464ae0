"""Autotuner for the neighbour-list skin.

The skin trades pair-kernel work (entries grow roughly as (r_cut + skin)^3)
against rebuild frequency (a rebuild runs when any atom moved more than
skin / 2).  The best value depends on the system and its temperature, so it
is measured: each candidate skin gets its own force field on the same
device-resident system, a short run of CUDA-graph steps is timed with CUDA
events, and the fastest candidate wins.  Results are keyed by a size class
(atoms, grid) and can be kept in a JSON cache file.
"""

from __future__ import annotations

import json
from pathlib import Path

from . import units as U
from .api import Constraints, ForceField, Integrator, System


def size_class(spec) -> str:
    grid = "x".join(str(g) for g in spec.grid) if spec.grid else "none"
    return f"n{spec.n}-grid{grid}-rc{spec.r_cut_coul or 0:.3f}"


def tune_skin(ctx, sys_: System, spec, cons: Constraints | None, integrator_kwargs: dict,
              candidates_A=(0.8, 1.2, 1.6, 2.0, 2.5), steps: int = 40, warm: int = 10,
              cache: Path | None = None) -> dict:
    """Time `steps` graph-mode MD steps per candidate skin (angstrom) and
    return {"best_A": skin, "ms_per_step": {skin: ms}}.  The system state
    advances during tuning (the runs are real MD steps)."""
    key = size_class(spec)
    if cache is not None and cache.exists():
        data = json.loads(cache.read_text())
        if key in data:
            return data[key]
    times = {}
    for skin in candidates_A:
        ff = ForceField.from_spec(sys_, spec, r_skin=U.angstrom_au(skin))
        it = Integrator(sys_, **integrator_kwargs)
        it.step_graph(ff, cons, n_steps=warm)
        ctx.timing(True)
        it.step_graph(ff, cons, n_steps=steps)
        ms = float(ctx.timings()[0]) / steps
        ctx.timing(False)
        times[skin] = ms
        it.close()
        ff.close()
    best = min(times, key=times.get)
    result = {"best_A": best, "ms_per_step": {str(k): v for k, v in times.items()}}
    if cache is not None:
        data = json.loads(cache.read_text()) if cache.exists() else {}
        data[key] = result
        cache.write_text(json.dumps(data, indent=1))
    return result
