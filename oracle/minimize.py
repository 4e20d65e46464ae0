"""CPU restatement of the steepest-descent minimiser (test infrastructure
only: the checker of heddle_b200's hb_min.cu).

Follows SteepestDescentMinimizer::step / check_convergence
(src/minimizer/steepest_descent.rs:123-283) and the runner's pre-loop check
(src/runner.rs:1896-1965) in FP64: F_max = max_i |F_i|, trial x + s F / F_max,
position-only constraint projection (Gauss-Seidel with gradients at the
current positions, settle_positions_no_velocity / shake_positions_no_velocity,
kernels/settle.cu:519-584 and kernels/shake.cu:558-697), accept on an energy
drop (s = min(1.2 s, s_max)), else restore (s = 0.2 s).  Energies are the
oracle's potential energy (LJ + real-space Coulomb + reciprocal - self +
bonded)."""

from __future__ import annotations

import numpy as np

import oracle as O


def potential(spec, pos) -> tuple:
    F, _, _, T = O.forces(spec, pos)
    e = T["lj"] + T["coulomb_real"] + T["recip"] - T["self"] + T["bonded"]
    return F, e


def project(spec, pos, tol: float = 3.57e-6, max_iter: int = 32, rel_tol: float = 0.0):
    """Position-only projection of every constraint group of spec (SHAKE
    groups relative to d^2 when rel_tol > 0)."""
    if spec.group_offsets is None:
        return pos
    pos = pos.copy()
    L = np.asarray(spec.box[:3], dtype=np.float64)
    inv_m = 1.0 / np.asarray(spec.masses, dtype=np.float64)
    go, ga = spec.group_offsets, spec.group_atoms
    kinds = spec.group_kind if spec.group_kind is not None else np.zeros(len(go) - 1, dtype=int)
    for g in range(len(go) - 1):
        ids = ga[go[g]:go[g + 1]]
        x = pos[ids] - pos[ids[0]]
        x -= L * np.round(x / L)
        xu = x.copy()
        if kinds[g] == 0:
            # SETTLE triangle: O-H, O-H, H-H from the canonical distances
            ra, rb, rc = spec.settle_ra[g], spec.settle_rb[g], spec.settle_rc[g]
            d_oh = float(np.hypot(ra + rb, rc))
            cons = [(0, 1, d_oh), (0, 2, d_oh), (1, 2, 2.0 * rc)]
        else:
            co = spec.con_offsets
            cons = [(spec.con_i[k], spec.con_j[k], spec.con_dist[k]) for k in range(co[g], co[g + 1])]
        grad = [x[i] - x[j] for i, j, _ in cons]
        for _ in range(max_iter):
            conv = True
            for k, (i, j, dist) in enumerate(cons):
                d = x[i] - x[j]
                sigma = d @ d - dist ** 2
                if abs(sigma) > (rel_tol * dist ** 2 if kinds[g] != 0 and rel_tol else tol):
                    conv = False
                    den = 2.0 * (d @ grad[k]) * (inv_m[ids[i]] + inv_m[ids[j]])
                    if den == 0.0:
                        continue
                    lam = sigma / den
                    x[i] -= lam * inv_m[ids[i]] * grad[k]
                    x[j] += lam * inv_m[ids[j]] * grad[k]
            if conv:
                break
        pos[ids] += x - xu
    return pos


def steepest_descent(spec, pos=None, initial_step=1e-12 / 5.29177210903e-11,
                     max_step=1e-10 / 5.29177210903e-11, inc=1.2, dec=0.2, ftol=0.0, etol=0.0,
                     max_iter=100):
    """Reports [(iteration, energy, max_force, step, accepted, reason)] and
    the final positions; reason as the device's HB_MIN_* codes."""
    pos = np.array(spec.positions if pos is None else pos, dtype=np.float64)
    F, e = potential(spec, pos)
    fmax = float(np.sqrt((F * F).sum(1).max()))
    reason = 3 if fmax == 0.0 else (1 if ftol > 0 and fmax <= ftol else 0)
    rows = [(0, e, fmax, 0.0, True, reason)]
    step = initial_step
    it = 0
    while reason == 0 and it < max_iter:
        it += 1
        prev = e
        trial = project(spec, pos + F * (step / fmax))
        Ft, et = potential(spec, trial)
        used = step
        if et < e:
            pos, F, e = trial, Ft, et
            step = min(step * inc, max_step)
            acc = True
        else:
            step *= dec
            acc = False
        fmax = float(np.sqrt((F * F).sum(1).max()))
        reason = 3 if fmax == 0.0 else (1 if ftol > 0 and fmax <= ftol else 0)
        if not reason and acc and etol > 0 and abs(e - prev) <= etol * max(abs(e), abs(prev), 1e-30):
            reason = 2
        rows.append((it, e, fmax, used, acc, reason))
    return rows, pos
