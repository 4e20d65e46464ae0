"""Run a simulation from a TOML configuration: the runner's setup path
(src/runner.rs:785-1180) over this engine.

    python -m heddle_b200.run path/to/name.in.toml

reads the configuration, the initial extended-XYZ frame and the topology,
builds the system, force field (LJ, SPME, bonded terms, exclusions by the
topology rules), constraint groups and each phase's integrator / barostat,
and writes `<root>.out.<phase>.xyz`, `<root>.out.<phase>.log` and
`<root>.out.<phase>.timings` (per-stage device and host times) beside the
configuration (`<root>` = file name without `.toml` and one `.in`), in SI
units like the reference.  Initial velocities, when the XYZ frame has none,
are Maxwell-Boltzmann at [simulation].temperature from the ChaCha8 seed.
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

from . import api as A
from . import units as U
from .io import (ConfigError, LogWriter, MinimizationConfig, MinlogWriter, StageTimes,
                 TrajectoryWriter, load_config, read_topology, read_xyz, write_timings)
from .systems import settle_geometry
from .topology import effective_exclusions, exclusion_csr
from .velocities import generate_velocities


def config_root(path: Path) -> str:
    name = path.name
    if name.endswith(".toml"):
        name = name[: -len(".toml")]
    if name.endswith(".in"):
        name = name[: -len(".in")]
    return name


def build(cfg, ctx):
    """Device objects for a loaded configuration: (system, force field,
    constraints or None, type names, extras dict)."""
    frame = read_xyz(cfg.init)
    topo = read_topology(cfg.topology) if cfg.topology else None
    names = [t["name"] for t in cfg.particle_types]
    try:
        types = np.array([names.index(s) for s in frame.species], dtype=np.uint32)
    except ValueError as e:
        raise ConfigError(f"initial frame: unknown species ({e})")
    n = len(types)
    masses = np.array([cfg.particle_types[t]["mass"] for t in types])
    charges = np.array([cfg.particle_types[t]["charge"] for t in types])
    if topo:
        for a, q in topo.charges.items():
            charges[a] = q
    # constraint groups
    g_off, g_atoms, g_kind, ra, rb, rc = [0], [], [], [], [], []
    c_off, c_i, c_j, c_d = [0], [], [], []
    groups = []
    n_cons = 0
    if topo:
        for atoms, tname in topo.constraints:
            ct = cfg.constraint_types.get(tname)
            if ct is None:
                raise ConfigError(f"topology: unknown constraint type {tname!r}")
            groups.append(atoms)
            g_atoms += atoms
            g_off.append(len(g_atoms))
            if ct["kind"] == "settle":
                d_oh, d_hh = ct["d_OH"], ct["d_HH"]
                hoh = 2.0 * np.degrees(np.arcsin(0.5 * d_hh / d_oh))
                a_, b_, c_ = settle_geometry(d_oh, hoh, masses[atoms[0]], masses[atoms[1]])
                g_kind.append(0)
                ra.append(a_), rb.append(b_), rc.append(c_)
                n_cons += 3
            else:
                if len(atoms) != ct["atoms"]:
                    raise ConfigError(f"constraint row of type {tname!r} needs {ct['atoms']} atoms")
                g_kind.append(1)
                ra.append(0.0), rb.append(0.0), rc.append(0.0)
                for i, j, d in ct["constraints"]:
                    c_i.append(i), c_j.append(j), c_d.append(d)
                n_cons += len(ct["constraints"])
            c_off.append(len(c_i))
    vel = frame.velocities
    if vel is None:
        vel = generate_velocities(masses, cfg.temperature, cfg.seed, n_cons)
    sys_ = A.System(ctx, frame.positions, masses, charges, types, frame.box, velocities=vel,
                    images=frame.images)
    # force field
    nt = len(names)
    sig, eps = np.ones((nt, nt)), np.zeros((nt, nt))
    cut_max = max([p["cutoff"] for p in cfg.pair_interactions], default=0.0)
    if cfg.spme:
        cut_max = max(cut_max, cfg.spme["r_cut_real"])
    cut, sw = np.full((nt, nt), cut_max), np.full((nt, nt), cut_max)
    for p in cfg.pair_interactions:
        for a, b in (p["between"], p["between"][::-1]):
            sig[a, b], eps[a, b], cut[a, b], sw[a, b] = p["sigma"], p["epsilon"], p["cutoff"], p["r_switch"]
    conf = {}
    if cfg.pair_interactions:
        conf["lennard_jones"] = A.LennardJonesParams(sig, eps, cut, sw)
    if cfg.spme:
        conf["spme"] = A.SpmeParams(cfg.spme["alpha"], cfg.spme["r_cut_real"], cfg.spme["grid"],
                                    cfg.spme["spline_order"])
    bonds, angles, dihedrals, dscales = [], [], [], []
    if topo:
        if topo.bonds:
            bk = [cfg.bond_types[t] for *_, t in topo.bonds]
            conf["harmonic_bond"] = A.HarmonicBondParams(
                np.array([(i, j) for i, j, _ in topo.bonds], dtype=np.uint32),
                np.array([b["k"] for b in bk]), np.array([b["r0"] for b in bk]))
            bonds = [(i, j) for i, j, _ in topo.bonds]
        if topo.angles:
            at = [cfg.angle_types[t] for *_, t in topo.angles]
            conf["harmonic_angle"] = A.HarmonicAngleParams(
                np.array([(i, j, k) for i, j, k, _ in topo.angles], dtype=np.uint32),
                np.array([a["k_theta"] for a in at]), np.array([a["theta_0"] for a in at]))
            angles = [(i, j, k) for i, j, k, _ in topo.angles]
        if topo.dihedrals:
            dt = [cfg.dihedral_types[t] for *_, t in topo.dihedrals]
            conf["periodic_dihedral"] = A.PeriodicDihedralParams(
                np.array([(i, j, k, l) for i, j, k, l, _ in topo.dihedrals], dtype=np.uint32),
                np.array([d["k_phi"] for d in dt]), np.array([d["phi_0"] for d in dt]),
                np.array([d["n"] for d in dt], dtype=np.uint32))
            dihedrals = [(i, j, k, l) for i, j, k, l, _ in topo.dihedrals]
            dscales = [(d["scale_lj_14"], d["scale_coul_14"]) for d in dt]
    eff = effective_exclusions(n, bonds, angles, dihedrals, dscales, groups,
                               topo.exclusions if topo else ())
    excl = exclusion_csr(n, eff) if eff else None
    ff = A.ForceField(sys_, conf, excl, r_skin=cfg.r_skin)
    cons = None
    if groups:
        cons = A.Constraints(sys_, g_off, g_atoms, g_kind, (ra, rb, rc) if any(k == 0 for k in g_kind) else None,
                             (c_off, c_i, c_j, c_d) if c_i else None)
        cons.after_kick(0.0)  # initial velocity projection
    mols = None
    if groups:
        mols = molecule_csr(n, groups, bonds)
    return sys_, ff, cons, names, {"n_constraints": n_cons, "molecules": mols}


def molecule_csr(n, groups, bonds):
    """Connected components of bonds and constraint groups (the molecule
    partition the barostat scales)."""
    parent = list(range(n))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for g in groups:
        for a in g[1:]:
            parent[find(a)] = find(g[0])
    for i, j in bonds:
        parent[find(i)] = find(j)
    comp = {}
    for a in range(n):
        comp.setdefault(find(a), []).append(a)
    mols = sorted(comp.values(), key=lambda m: m[0])
    off = np.cumsum([0] + [len(m) for m in mols]).astype(np.uint32)
    return off, np.concatenate(mols).astype(np.uint32)


def log_columns(ph) -> list:
    """Extra log columns after step,time,kinetic_energy,temperature: the
    thermostat's, then the barostat's (src/runner.rs:1437-1443), with the
    names and dimensions of their log_column_names (box volumes are written
    in bohr^3, unconverted, like the reference's Dimensionless columns)."""
    cols = []
    t = ph.thermostat["kind"] if ph.thermostat else None
    if t in ("csvr", "andersen", "berendsen"):
        cols.append((f"{t}_conserved", "energy"))
    b = ph.barostat["kind"] if ph.barostat else None
    if b == "monte-carlo":
        cols += [("box_volume", "dimensionless"), ("mc_acceptance", "dimensionless"),
                 ("mc_volume_step", "dimensionless"), ("mc_conserved", "energy")]
    elif b == "c-rescale":
        cols += [("pressure", "pressure"), ("box_volume", "dimensionless"),
                 ("c_rescale_conserved", "energy")]
    elif b == "berendsen":
        cols += [("pressure", "pressure"), ("box_volume", "dimensionless")]
    return cols


def log_values(ph, ke: float, pe: float, thermo, baro) -> list:
    """Values of log_columns(ph) (csvr.rs:247-253, andersen.rs:180-187,
    berendsen.rs:191-197, mc_barostat.rs:374-385,
    c_rescale_barostat.rs:287-300, berendsen_barostat.rs:219-225)."""
    vals = []
    if thermo is not None:
        st = thermo.stats()
        vals.append(ke + pe if thermo.kind == "andersen" else ke + pe - st["injection"])
    if baro is not None:
        st = baro.stats()
        if ph.barostat["kind"] == "monte-carlo":
            vals += [st["volume"], st["acceptance"], st["max_volume_step"],
                     ke + pe + st["conserved_term"]]
        else:
            vals += [st["pressure"], st["volume"]]
            if ph.barostat["kind"] == "c-rescale":
                vals.append(ke + pe + ph.barostat["pressure"] * st["volume"] - st["injection"])
    return vals


class MinimizationError(RuntimeError):
    """A minimisation phase ended without converging (the reference's
    RunnerError::MinimizerNonConvergence)."""


def minimize(ph, sys_, ff, cons, names, base: Path, root: str) -> list:
    """One [[minimization]] phase (src/runner.rs:1804-2140): the iteration-0
    row and frame, a minlog row every minlog_every iterations (and the final
    one), a frame every trajectory_every accepted iterations (positions
    only, time 0); non-convergence is an error."""
    out = ph.output
    written = []
    log = traj = None
    if out["minlog_every"] > 0:
        lp = out.get("minlog_path") or base / f"{root}.out.{ph.name}.minlog"
        log = MinlogWriter(lp)
        written.append(lp)
    if out["trajectory_every"] > 0:
        tp = out.get("trajectory_path") or base / f"{root}.out.{ph.name}.xyz"
        traj = TrajectoryWriter(tp, names, False, out["include_images"])
        written.append(tp)
    a = ph.algorithm
    m = A.Minimizer(ff, cons, a["initial_step"], a["max_step"], a["step_increase"],
                    a["step_decrease"], a["force_tolerance"], a["energy_tolerance"],
                    a["max_iterations"])
    types = np.asarray(sys_._t)

    def frame(it):
        pos, _, img, _ = sys_.state()
        traj.write(it, 0.0, sys_.box(), types, pos, None, img)

    try:
        r = m.begin()
        last_logged = None
        if log:
            log.write(r)
            last_logged = 0
        if traj:
            frame(0)
        while r["converged"] is None and r["iteration"] < a["max_iterations"]:
            # chunks end on the trajectory cadence so frames see their state
            k = a["max_iterations"] - r["iteration"]
            if traj:
                k = min(k, out["trajectory_every"] - r["iteration"] % out["trajectory_every"])
            rows = m.iterate(min(k, 256))
            if not rows:
                break
            for r in rows:
                if log and r["iteration"] % out["minlog_every"] == 0:
                    log.write(r)
                    last_logged = r["iteration"]
            if traj and r["accepted"] and r["iteration"] % out["trajectory_every"] == 0:
                frame(r["iteration"])
        if r["converged"] is None:
            raise MinimizationError(
                f"minimization phase `{ph.name}` failed to converge after {r['iteration']} "
                f"iterations (max_force = {r['max_force'] * U.FORCE_N:.3e} N, "
                f"step = {r['step'] * U.BOHR_M:.3e} m)")
        if log and last_logged != r["iteration"]:
            log.write(r)
    finally:
        m.close()
        for w in (log, traj):
            if w:
                w.close()
    return written


# device stages reported by the library per call (hb_timing_get)
DEVICE_STAGES = [(1, "pair_force"), (2, "spme_reciprocal"), (3, "neighbor_list"),
                 (4, "integrate_constrain"), (0, "step_total")]


def run(config_path, ctx=None) -> list:
    """Run every phase; returns the written output paths."""
    t_run = time.perf_counter()
    t0 = time.perf_counter()
    cfg = load_config(config_path)
    pre = StageTimes()  # the setup stages, replayed into the first phase's timings
    pre.record("config_load", time.perf_counter() - t0)
    own = ctx is None
    t0 = time.perf_counter()
    ctx = ctx or A.Context(0)
    pre.record("gpu_init", time.perf_counter() - t0)
    t0 = time.perf_counter()
    sys_, ff, cons, names, extra = build(cfg, ctx)
    pre.record("init_load", time.perf_counter() - t0)
    root = config_root(Path(cfg.path))
    base = Path(cfg.path).parent
    written = []
    n = sys_.n
    dof = max(3 * n - extra["n_constraints"] - 3, 1)
    step = 0
    for k_ph, ph in enumerate(cfg.phases):
        times = pre if k_ph == 0 else StageTimes()
        t_phase = time.perf_counter()
        tpath = ph.output.get("timings_path") or base / f"{root}.out.{ph.name}.timings"
        if isinstance(ph, MinimizationConfig):
            written += minimize(ph, sys_, ff, cons, names, base, root)
            times.record("total_runtime", time.perf_counter() - (t_run if k_ph == 0 else t_phase))
            write_timings(tpath, times)
            written.append(tpath)
            continue
        kw = dict(ph.integrator)
        kind = kw.pop("kind")
        it = A.Integrator(sys_, kind, ph.dt, step0=step, **kw)
        thermo = baro = None
        if ph.thermostat:
            t = ph.thermostat
            thermo = A.Thermostat(sys_, t["kind"], t["temperature"], seed=t.get("seed", 0),
                                  tau=t.get("tau", 0.0), collision_rate=t.get("collision_rate", 0.0),
                                  n_constraints=extra["n_constraints"])
            it.set_thermostat(thermo)
        if ph.barostat:
            b = ph.barostat
            if b["kind"] == "monte-carlo":
                baro = A.Barostat(sys_, b["pressure"], b["temperature"], b["seed"], b["frequency"],
                                  b["volume_step"], molecules=extra["molecules"])
            else:
                baro = A.PressureCoupling(sys_, b["kind"].replace("-", "_"), b["pressure"], b["tau"],
                                          b["compressibility"], temperature=b.get("temperature", 0.0),
                                          seed=b.get("seed", 0))
            it.set_barostat(baro)
        out = ph.output
        traj = log = None
        if out["trajectory_every"] > 0:
            tp = out.get("trajectory_path") or base / f"{root}.out.{ph.name}.xyz"
            traj = TrajectoryWriter(tp, names, out["include_velocities"], out["include_images"])
            written.append(tp)
        if out["log_every"] > 0:
            lp = out.get("log_path") or base / f"{root}.out.{ph.name}.log"
            log = LogWriter(lp, log_columns(ph))
            written.append(lp)
        types = None
        done = 0
        cadence = [c for c in (out["trajectory_every"], out["log_every"]) if c > 0]
        ctx.timing(True)
        while done < ph.n_steps:
            k = ph.n_steps - done
            for c in cadence:
                k = min(k, c - (done % c))
            it.step(ff, cons, n_steps=k, scalar_every=k if (log and (done + k) % out["log_every"] == 0) else 0)
            t_dev = ctx.timings()
            for idx, name in DEVICE_STAGES:
                times.record(name, t_dev[idx] * 1e-3, k)
            done += k
            t_au = (step + done) * ph.dt
            if traj and done % out["trajectory_every"] == 0:
                t0 = time.perf_counter()
                pos, vel, img, _ = sys_.state()
                times.record("device_to_host_download", time.perf_counter() - t0)
                if types is None:
                    types = np.asarray(sys_._t)
                t0 = time.perf_counter()
                traj.write(step + done, t_au, sys_.box(), types, pos, vel, img)
                times.record("trajectory_write", time.perf_counter() - t0)
            if log and done % out["log_every"] == 0:
                t0 = time.perf_counter()
                ke = sys_.kinetic()[0]
                log.write(step + done, t_au, ke, 2.0 * ke / dof,
                          log_values(ph, ke, ff.scalars()["potential"], thermo, baro))
                times.record("log_write", time.perf_counter() - t0)
        ctx.timing(False)
        step += ph.n_steps
        times.record("total_runtime", time.perf_counter() - (t_run if k_ph == 0 else t_phase))
        write_timings(tpath, times)
        written.append(tpath)
        for w in (traj, log):
            if w:
                w.close()
        it.close()
        for c in (thermo, baro):
            if c:
                c.close()
    for o in (cons, ff, sys_):
        if o is not None:
            o.close()
    if own:
        ctx.close()
    return written


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print("usage: python -m heddle_b200.run <config.toml>", file=sys.stderr)
        return 2
    try:
        for p in run(argv[0]):
            print(p)
    except ConfigError as e:
        print(f"configuration error: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
