"""TOML configuration, extended-XYZ and topology files: the reference's input
and output formats for the force path.

Follows src/io/config.rs (schema version 1, SI units in the file, converted
to Hartree atomic units on load), src/io/init_state.rs / trajectory.rs
(extended XYZ: a count line, a header with `Lattice="..."` -- the nine
lattice components row-major, rows a = (lx, 0, 0), b = (xy, ly, 0),
c = (xz, yz, lz) -- and `Properties=species:S:1:pos:R:3[:velo:R:3]
[:image:I:3]`, reals written as `{:.9e}`), src/io/log_output.rs (CSV log
`step,time,kinetic_energy,temperature,...`) and the topology file's
`[bonds]`, `[angles]`, `[dihedrals]`, `[exclusions]`, `[constraints]` and
`[charges]` sections.

Supported slot kinds: integrators "velocity-verlet" (with `lossless`) and
"langevin-baoab", thermostats "csvr", "andersen" and "berendsen", barostats
"monte-carlo", "c-rescale" and "berendsen", constraint types "settle" and
"shake", bond/angle types "harmonic", dihedral types "periodic", pair
potential "lennard-jones", neighbour list "cell-list".  Other kinds the
reference registers (thermostat nose-hoover-chain, barostat mtk-npt, Morse
bonds, all-pairs lists) are rejected with a ConfigError that names them.
[[minimization]] phases (steepest descent) run in document order with the
[[phase]] entries.
"""

from __future__ import annotations

import math
import re
import tomllib
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import units as U


class ConfigError(ValueError):
    """An invalid or unsupported configuration (ConfigError of src/io/config.rs)."""


# ---------------------------------------------------------------------------
# number formatting: Rust's `{:.9e}` (no exponent padding, no '+')
# ---------------------------------------------------------------------------
def fmt_e(x: float, digits: int = 9) -> str:
    s = f"{float(x):.{digits}e}"
    mant, exp = s.split("e")
    return f"{mant}e{int(exp)}"


# ---------------------------------------------------------------------------
# configuration
# ---------------------------------------------------------------------------
@dataclass
class PhaseConfig:
    name: str
    n_steps: int
    dt: float                      # aut
    integrator: dict
    thermostat: dict | None = None
    barostat: dict | None = None
    output: dict = field(default_factory=dict)


@dataclass
class Config:
    path: Path
    schema_version: int
    init: Path
    topology: Path | None
    seed: int
    temperature: float             # k_B T in hartree
    phases: list
    particle_types: list           # [{name, mass (m_e), charge (e)}]
    pair_interactions: list        # [{between (i, j), sigma, epsilon, cutoff, r_switch}] (a.u.)
    bond_types: dict               # name -> {k, r0}
    angle_types: dict              # name -> {k_theta, theta_0}
    dihedral_types: dict           # name -> {k_phi, n, phi_0, scale_lj_14, scale_coul_14}
    constraint_types: dict         # name -> {kind, ...} (a.u.)
    spme: dict | None
    r_skin: float                  # bohr


_UNSUPPORTED = {
    "thermostat": ("nose-hoover-chain",),
    "barostat": ("mtk-npt",),
}

KB_J = 1.380649e-23  # J/K


def _req(table: dict, key: str, where: str):
    if key not in table:
        raise ConfigError(f"[{where}] is missing `{key}`")
    return table[key]


def _finite(v, where):
    v = float(v)
    if not math.isfinite(v):
        raise ConfigError(f"{where}: value must be finite, got {v}")
    return v


def _positive(v, where):
    v = _finite(v, where)
    if v <= 0.0:
        raise ConfigError(f"{where}: value must be finite and strictly positive, got {v}")
    return v


def _temperature(table, where):
    return U.temperature_au_k(_positive(_req(table, "temperature", where), f"{where}.temperature"))


def _thermostat(t: dict) -> dict:
    """[phase.thermostat]: csvr (temperature, tau, seed), andersen
    (temperature, collision_rate, seed), berendsen (temperature, tau);
    src/integrator/csvr.rs:18-40, andersen.rs:18-50, berendsen.rs:20-60."""
    kind = t.get("kind")
    if kind == "csvr":
        return {"kind": kind, "temperature": _temperature(t, "thermostat"),
                "tau": _positive(_req(t, "tau", "thermostat"), "thermostat.tau") / U.AUT_S,
                "seed": int(_req(t, "seed", "thermostat"))}
    if kind == "andersen":
        rate = _finite(_req(t, "collision_rate", "thermostat"), "thermostat.collision_rate")
        if rate < 0.0:
            raise ConfigError(f"thermostat.collision_rate: value must be finite and non-negative, "
                              f"got {rate}")
        return {"kind": kind, "temperature": _temperature(t, "thermostat"),
                "collision_rate": rate * U.AUT_S, "seed": int(_req(t, "seed", "thermostat"))}
    if kind == "berendsen":
        return {"kind": kind, "temperature": _temperature(t, "thermostat"),
                "tau": _positive(_req(t, "tau", "thermostat"), "thermostat.tau") / U.AUT_S}
    raise ConfigError(f"thermostat kind {kind!r} is not supported by this engine "
                      f"(known to the reference: {', '.join(_UNSUPPORTED['thermostat'])})")


def _barostat(b: dict) -> dict:
    """[phase.barostat]: monte-carlo (pressure, temperature, frequency,
    volume_step, seed), c-rescale (pressure, temperature, tau,
    compressibility, seed), berendsen (pressure, tau, compressibility);
    src/integrator/mc_barostat.rs, c_rescale_barostat.rs:14-45,
    berendsen_barostat.rs:20-60."""
    kind = b.get("kind")
    pressure = _finite(_req(b, "pressure", "barostat"), "barostat.pressure") / U.PRESSURE_PA
    if kind == "monte-carlo":
        vs = b.get("volume_step")
        out = {"kind": kind, "pressure": pressure, "temperature": _temperature(b, "barostat"),
               "frequency": int(b.get("frequency", 25)),
               "volume_step": None if vs is None else
               _positive(vs, "barostat.volume_step") / U.BOHR_M ** 3,
               "seed": int(_req(b, "seed", "barostat"))}
        if out["frequency"] < 1:
            raise ConfigError("barostat.frequency: value must be >= 1, got 0")
        return out
    if kind in ("c-rescale", "berendsen"):
        out = {"kind": kind, "pressure": pressure,
               "tau": _positive(_req(b, "tau", "barostat"), "barostat.tau") / U.AUT_S,
               "compressibility": _positive(_req(b, "compressibility", "barostat"),
                                            "barostat.compressibility") * U.PRESSURE_PA}
        if kind == "c-rescale":
            out["temperature"] = _temperature(b, "barostat")
            out["seed"] = int(_req(b, "seed", "barostat"))
        return out
    raise ConfigError(f"barostat kind {kind!r} is not supported by this engine "
                      f"(known to the reference: {', '.join(_UNSUPPORTED['barostat'])})")


def _out_path(base: Path, p):
    return None if p is None else (Path(p) if Path(p).is_absolute() else base / p)


@dataclass
class MinimizationConfig:
    name: str
    algorithm: dict                # steepest-descent parameters (a.u.)
    output: dict = field(default_factory=dict)


def _minimization(m: dict, base: Path) -> MinimizationConfig:
    """[[minimization]]: name, [minimization.algorithm] kind
    "steepest-descent" (SteepestDescentParams with the reference's defaults
    and checks, src/minimizer/steepest_descent.rs:20-62, 300-380) and
    [minimization.output] (src/io/config.rs:680-710)."""
    name = str(_req(m, "name", "minimization"))
    alg = dict(_req(m, "algorithm", f"minimization {name}"))
    if alg.get("kind") != "steepest-descent":
        raise ConfigError(f"minimizer kind {alg.get('kind')!r} does not match any registered builder")
    w = "minimization.algorithm"
    a = {"initial_step": _positive(alg.get("initial_step", 1.0e-12), f"{w}.initial_step") / U.BOHR_M,
         "max_step": _positive(alg.get("max_step", 1.0e-10), f"{w}.max_step") / U.BOHR_M,
         "step_increase": _finite(alg.get("step_increase", 1.2), f"{w}.step_increase"),
         "step_decrease": _finite(alg.get("step_decrease", 0.2), f"{w}.step_decrease"),
         "force_tolerance": _finite(alg.get("force_tolerance", 1.0e-10), f"{w}.force_tolerance")
         / U.FORCE_N,
         "energy_tolerance": _finite(alg.get("energy_tolerance", 1.0e-7), f"{w}.energy_tolerance"),
         "max_iterations": int(alg.get("max_iterations", 1000))}
    if a["max_step"] < a["initial_step"]:
        raise ConfigError(f"{w}.max_step must be >= initial_step")
    if a["step_increase"] < 1.0:
        raise ConfigError(f"{w}.step_increase must be finite and >= 1.0, got {a['step_increase']}")
    if not 0.0 < a["step_decrease"] < 1.0:
        raise ConfigError(f"{w}.step_decrease must be finite and in (0.0, 1.0), got {a['step_decrease']}")
    if a["force_tolerance"] < 0.0 or a["energy_tolerance"] < 0.0:
        raise ConfigError(f"{w}: tolerances must be finite and >= 0.0")
    if a["max_iterations"] <= 0:
        raise ConfigError(f"{w}.max_iterations must be strictly positive")
    out = dict(m.get("output", {}))
    output = {"minlog_every": int(out.get("minlog_every", 1)),
              "trajectory_every": int(out.get("trajectory_every", 0)),
              "include_images": bool(out.get("include_images", True)),
              "minlog_path": _out_path(base, out.get("minlog_path")),
              "trajectory_path": _out_path(base, out.get("trajectory_path")),
              "timings_path": _out_path(base, out.get("timings_path"))}
    return MinimizationConfig(name, a, output)


def load_config(path) -> Config:
    """Parse and validate a schema-1 TOML configuration (SI units)."""
    path = Path(path)
    with open(path, "rb") as f:
        doc = tomllib.load(f)
    if doc.get("schema_version") != 1:
        raise ConfigError(f"unsupported schema_version {doc.get('schema_version')!r} (expected 1)")
    units = doc.get("units", "si")
    if units != "si":
        raise ConfigError(f"units = {units!r}: only \"si\" files are read")
    base = path.parent
    init = base / _req(doc, "init", "top level")
    topo = base / doc["topology"] if "topology" in doc else None
    sim = _req(doc, "simulation", "top level")
    seed = int(_req(sim, "seed", "simulation"))
    temp_k = _finite(_req(sim, "temperature", "simulation"), "simulation.temperature")
    md_phases = []
    for p in doc.get("phase", []):
        name = str(_req(p, "name", "phase"))
        n_steps = int(_req(p, "n_steps", f"phase {name}"))
        dt = U.time_au_fs(_positive(_req(p, "dt", f"phase {name}"), f"phase.{name}.dt") * 1e15)
        integ = dict(_req(p, "integrator", f"phase {name}"))
        kind = integ.get("kind")
        if kind == "velocity-verlet":
            integ = {"kind": "velocity-verlet-lossless" if integ.get("lossless") else "velocity-verlet"}
        elif kind == "langevin-baoab":
            integ = {"kind": "langevin-baoab",
                     "friction": _positive(_req(integ, "friction", "phase.integrator"),
                                           "phase.integrator.friction") * U.AUT_S,
                     "temperature": U.temperature_au_k(_positive(
                         _req(integ, "temperature", "phase.integrator"), "phase.integrator.temperature")),
                     "seed": int(_req(integ, "seed", "phase.integrator"))}
        else:
            raise ConfigError(f"[integrator] section's `kind = \"{kind}\"` does not match any "
                              "registered builder")
        thermo = p.get("thermostat")
        if thermo is not None:
            thermo = _thermostat(thermo)
        baro = p.get("barostat")
        if baro is not None:
            baro = _barostat(baro)
        if (thermo or (baro and baro["kind"] != "monte-carlo")) and integ["kind"] != "velocity-verlet":
            raise ConfigError("a thermostat or a per-step barostat needs the (non-lossless) "
                              "velocity-verlet integrator")
        out = dict(p.get("output", {}))
        # defaults of RawOutputConfig (src/io/config.rs:595-604, 860-875)
        output = {"trajectory_every": int(out.get("trajectory_every", 100)),
                  "include_velocities": bool(out.get("include_velocities", True)),
                  "include_images": bool(out.get("include_images", True)),
                  "log_every": int(out.get("log_every", 100)),
                  "trajectory_path": _out_path(base, out.get("trajectory_path")),
                  "log_path": _out_path(base, out.get("log_path")),
                  "timings_path": _out_path(base, out.get("timings_path"))}
        md_phases.append(PhaseConfig(name, n_steps, dt, integ, thermo, baro, output))
    min_phases = [_minimization(m, base) for m in doc.get("minimization", [])]
    # [[phase]] and [[minimization]] run in document order
    # (src/io/config.rs:1255-1290)
    order = re.findall(r"^\s*\[\[\s*(phase|minimization)\s*\]\]", path.read_text(), flags=re.M)
    if sorted(order) != sorted(["phase"] * len(md_phases) + ["minimization"] * len(min_phases)):
        raise ConfigError("could not order the [[phase]] / [[minimization]] entries")
    it_md, it_min = iter(md_phases), iter(min_phases)
    phases = [next(it_md) if k == "phase" else next(it_min) for k in order]
    if not phases:
        raise ConfigError("no [[phase]] or [[minimization]] entries")
    ptypes = []
    for t in _req(doc, "particle_types", "top level"):
        ptypes.append({"name": str(_req(t, "name", "particle_types")),
                       "mass": U.mass_au_kg(_positive(_req(t, "mass", "particle_types"),
                                                      "particle_types.mass")),
                       "charge": _finite(t.get("charge", 0.0), "particle_types.charge") / U.E_C})
    names = [t["name"] for t in ptypes]
    if len(set(names)) != len(names):
        raise ConfigError("particle type names must be unique")
    pairs = []
    for pi in doc.get("pair_interactions", []):
        a, b = _req(pi, "between", "pair_interactions")
        for x in (a, b):
            if x not in names:
                raise ConfigError(f"pair_interactions: unknown particle type {x!r}")
        if pi.get("potential") != "lennard-jones":
            raise ConfigError(f"pair potential {pi.get('potential')!r} is not supported")
        cut = U.length_au(_positive(_req(pi, "cutoff", "pair_interactions"), "cutoff"))
        rsw = U.length_au(_positive(pi.get("r_switch", 0.9 * pi["cutoff"]), "r_switch"))
        if rsw > cut:
            raise ConfigError("pair_interactions: r_switch must not exceed the cutoff")
        pairs.append({"between": (names.index(a), names.index(b)),
                      "sigma": U.length_au(_positive(_req(pi, "sigma", "pair_interactions"), "sigma")),
                      "epsilon": U.energy_au_j(_positive(_req(pi, "epsilon", "pair_interactions"),
                                                         "epsilon")),
                      "cutoff": cut, "r_switch": rsw})
    bonds = {}
    for bt in doc.get("bond_types", []):
        if bt.get("potential") != "harmonic":
            raise ConfigError(f"bond potential {bt.get('potential')!r} is not supported")
        bonds[bt["name"]] = {"k": U.energy_au_j(_positive(bt["k"], "bond_types.k")) * U.BOHR_M ** 2,
                             "r0": U.length_au(_positive(bt["r0"], "bond_types.r0"))}
    angles = {}
    for at in doc.get("angle_types", []):
        if at.get("potential") != "harmonic":
            raise ConfigError(f"angle potential {at.get('potential')!r} is not supported")
        angles[at["name"]] = {"k_theta": U.energy_au_j(_positive(at["k_theta"], "angle_types.k_theta")),
                              "theta_0": _finite(at["theta_0"], "angle_types.theta_0")}
    dihedrals = {}
    for dt_ in doc.get("dihedral_types", []):
        if dt_.get("potential") != "periodic":
            raise ConfigError(f"dihedral potential {dt_.get('potential')!r} is not supported")
        n = int(dt_["n"])
        if not 1 <= n <= 6:
            raise ConfigError("dihedral_types.n must be an integer in [1, 6]")
        dihedrals[dt_["name"]] = {"k_phi": U.energy_au_j(_finite(dt_["k_phi"], "k_phi")), "n": n,
                                  "phi_0": _finite(dt_["phi_0"], "phi_0"),
                                  "scale_lj_14": float(dt_.get("scale_lj_14", 0.5)),
                                  "scale_coul_14": float(dt_.get("scale_coul_14", 1.0 / 1.2))}
    cons = {}
    for ct in doc.get("constraint_types", []):
        kind = ct.get("kind")
        if kind == "settle":
            cons[ct["name"]] = {"kind": "settle",
                                "d_OH": U.length_au(_positive(ct["d_OH"], "d_OH")),
                                "d_HH": U.length_au(_positive(ct["d_HH"], "d_HH"))}
        elif kind == "shake":
            na = int(ct["atoms"])
            rows = [(int(c["i"]), int(c["j"]), U.length_au(_positive(c["d"], "constraints.d")))
                    for c in ct["constraints"]]
            for i, j, _ in rows:
                if not (0 <= i < na and 0 <= j < na and i != j):
                    raise ConfigError("shake constraint indices out of range")
            cons[ct["name"]] = {"kind": "shake", "atoms": na, "constraints": rows}
        else:
            raise ConfigError(f"constraint kind {kind!r} is not supported")
    spme = None
    if "spme" in doc:
        s = doc["spme"]
        spme = {"alpha": _positive(s["alpha"], "spme.alpha") * U.BOHR_M,
                "r_cut_real": U.length_au(_positive(s["r_cut_real"], "spme.r_cut_real")),
                "grid": tuple(int(g) for g in s["grid"]),
                "spline_order": int(s.get("spline_order", 4))}
    nl = doc.get("neighbor_list", {"mode": "cell-list", "r_skin": 0.0})
    if nl.get("mode", "cell-list") != "cell-list":
        if spme is not None:
            raise ConfigError("all-pairs neighbour search cannot be combined with SPME")
        raise ConfigError(f"neighbour list mode {nl.get('mode')!r} is not supported")
    r_skin = U.length_au(float(nl.get("r_skin", 0.0)))
    return Config(path, 1, init, topo, seed, U.temperature_au_k(temp_k), phases, ptypes, pairs,
                  bonds, angles, dihedrals, cons, spme, r_skin)


# ---------------------------------------------------------------------------
# extended XYZ
# ---------------------------------------------------------------------------
@dataclass
class Frame:
    species: list
    positions: np.ndarray           # (n, 3) bohr
    box: np.ndarray                 # lx, ly, lz, xy, xz, yz (bohr)
    velocities: np.ndarray | None = None   # bohr / aut
    images: np.ndarray | None = None
    step: int | None = None
    time: float | None = None       # aut


def _parse_header(line: str) -> dict:
    out, i = {}, 0
    while i < len(line):
        while i < len(line) and line[i] == " ":
            i += 1
        if i >= len(line):
            break
        j = line.index("=", i)
        key = line[i:j]
        if line[j + 1] == '"':
            k = line.index('"', j + 2)
            out[key] = line[j + 2:k]
            i = k + 1
        else:
            k = line.find(" ", j + 1)
            k = len(line) if k < 0 else k
            out[key] = line[j + 1:k]
            i = k
    return out


def read_xyz(path, index: int = 0) -> Frame:
    """Frame `index` (0 = first, -1 = last) of an extended-XYZ file (SI)."""
    frames = []
    with open(path) as f:
        lines = f.read().splitlines()
    p = 0
    while p < len(lines):
        if not lines[p].strip():
            p += 1
            continue
        try:
            n = int(lines[p])
        except ValueError:
            raise ConfigError(f"particle-count line is not a non-negative integer: {lines[p]!r}")
        frames.append((p, n))
        p += n + 2
    if not frames:
        raise ConfigError("empty XYZ file")
    p, n = frames[index]
    hdr = _parse_header(lines[p + 1])
    lat = [float(x) for x in hdr.get("Lattice", "").split()]
    if len(lat) != 9:
        raise ConfigError("`Lattice` needs 9 components")
    if lat[1] != 0.0 or lat[2] != 0.0 or lat[5] != 0.0:
        raise ConfigError("`Lattice` must be lower-triangular (a along x, b in the xy plane)")
    box = np.array([lat[0], lat[4], lat[8], lat[3], lat[6], lat[7]]) / U.BOHR_M
    props = hdr.get("Properties", "species:S:1:pos:R:3").split(":")
    cols, c = {}, 0
    for q in range(0, len(props), 3):
        name, width = props[q], int(props[q + 2])
        cols[name] = (c, width)
        c += width
    species, pos, vel, img = [], np.zeros((n, 3)), None, None
    if "velo" in cols:
        vel = np.zeros((n, 3))
    if "image" in cols:
        img = np.zeros((n, 3), dtype=np.int32)
    for a in range(n):
        tok = lines[p + 2 + a].split()
        species.append(tok[cols["species"][0]])
        c0 = cols["pos"][0]
        pos[a] = [float(x) for x in tok[c0:c0 + 3]]
        if vel is not None:
            c0 = cols["velo"][0]
            vel[a] = [float(x) for x in tok[c0:c0 + 3]]
        if img is not None:
            c0 = cols["image"][0]
            img[a] = [int(x) for x in tok[c0:c0 + 3]]
    step = int(hdr["Step"]) if "Step" in hdr else None
    time = float(hdr["Time"]) / U.AUT_S if "Time" in hdr else None
    return Frame(species, pos / U.BOHR_M, box, None if vel is None else vel / U.VELOCITY_MS,
                 img, step, time)


class TrajectoryWriter:
    """Extended-XYZ frames in SI with `{:.9e}` reals (src/io/trajectory.rs:108-175);
    refuses to overwrite an existing file."""

    def __init__(self, path, type_names, include_velocities=False, include_images=False):
        self.f = open(path, "x")
        self.names = list(type_names)
        self.vel = include_velocities
        self.img = include_images

    def write(self, step: int, time_au: float, box, types, positions, velocities=None,
              images=None) -> None:
        n = len(types)
        b = np.asarray(box, dtype=np.float64) * U.BOHR_M
        props = "species:S:1:pos:R:3" + (":velo:R:3" if self.vel else "") + (
            ":image:I:3" if self.img else "")
        z = fmt_e(0.0)
        lat = " ".join([fmt_e(b[0]), z, z, fmt_e(b[3]), fmt_e(b[1]), z, fmt_e(b[4]), fmt_e(b[5]),
                        fmt_e(b[2])])
        out = [f"{n}", f'Lattice="{lat}" Properties={props} Step={step} Time={fmt_e(time_au * U.AUT_S)}']
        P = np.asarray(positions, dtype=np.float64) * U.BOHR_M
        V = None if velocities is None else np.asarray(velocities, dtype=np.float64) * U.VELOCITY_MS
        for i in range(n):
            t = int(types[i])
            row = [self.names[t] if t < len(self.names) else "?", fmt_e(P[i, 0]), fmt_e(P[i, 1]),
                   fmt_e(P[i, 2])]
            if self.vel:
                row += [fmt_e(V[i, 0]), fmt_e(V[i, 1]), fmt_e(V[i, 2])]
            if self.img:
                row += [str(int(x)) for x in images[i]]
            out.append(" ".join(row))
        self.f.write("\n".join(out) + "\n")

    def close(self) -> None:
        self.f.close()


# SI factor of each extra-column dimension (atomic value x factor)
DIMENSION_SI = {"energy": U.HARTREE_J, "volume": U.BOHR_M ** 3, "pressure": U.PRESSURE_PA,
                "dimensionless": 1.0}


class LogWriter:
    """CSV log `step,time,kinetic_energy,temperature[,extras]` in SI
    (src/io/log_output.rs); extra columns are (name, dimension) pairs."""

    def __init__(self, path, extra_columns=()):
        self.f = open(path, "x")
        self.extra = [(c, "dimensionless") if isinstance(c, str) else c for c in extra_columns]
        names = [c for c, _ in self.extra]
        self.f.write(",".join(["step", "time", "kinetic_energy", "temperature"] + names) + "\n")

    def write(self, step: int, time_au: float, ke_au: float, temp_au: float, extras=()) -> None:
        vals = [str(step), fmt_e(time_au * U.AUT_S), fmt_e(ke_au * U.HARTREE_J),
                fmt_e(temp_au * U.HARTREE_K)] + [
                    fmt_e(v * DIMENSION_SI[d]) for v, (_, d) in zip(extras, self.extra)]
        self.f.write(",".join(vals) + "\n")

    def close(self) -> None:
        self.f.close()


class MinlogWriter:
    """Minimisation log `iter,energy,max_force,step,accepted` in SI
    (src/io/minlog_output.rs:30-70); rows are Minimizer reports."""

    def __init__(self, path):
        self.f = open(path, "x")
        self.f.write("iter,energy,max_force,step,accepted\n")

    def write(self, r: dict) -> None:
        self.f.write(f"{r['iteration']},{fmt_e(r['energy'] * U.HARTREE_J)},"
                     f"{fmt_e(r['max_force'] * U.FORCE_N)},{fmt_e(r['step'] * U.BOHR_M)},"
                     f"{1 if r['accepted'] else 0}\n")

    def close(self) -> None:
        self.f.close()


# ---------------------------------------------------------------------------
# topology file
# ---------------------------------------------------------------------------
@dataclass
class Topology:
    bonds: list = field(default_factory=list)        # (i, j, type)
    angles: list = field(default_factory=list)       # (i, j, k, type)
    dihedrals: list = field(default_factory=list)    # (i, j, k, l, type)
    exclusions: list = field(default_factory=list)   # (i, j, s_lj, s_coul)
    constraints: list = field(default_factory=list)  # ([atoms], type)
    charges: dict = field(default_factory=dict)      # atom -> charge (e)


def read_topology(path) -> Topology:
    t = Topology()
    section = None
    with open(path) as f:
        for raw in f:
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            if line.startswith("[") and line.endswith("]"):
                section = line[1:-1].strip()
                continue
            tok = line.split()
            if section == "bonds":
                t.bonds.append((int(tok[0]), int(tok[1]), tok[2]))
            elif section == "angles":
                t.angles.append((int(tok[0]), int(tok[1]), int(tok[2]), tok[3]))
            elif section == "dihedrals":
                t.dihedrals.append((int(tok[0]), int(tok[1]), int(tok[2]), int(tok[3]), tok[4]))
            elif section == "exclusions":
                t.exclusions.append((int(tok[0]), int(tok[1]), float(tok[2]), float(tok[3])))
            elif section == "constraints":
                t.constraints.append(([int(x) for x in tok[:-1]], tok[-1]))
            elif section == "charges":
                t.charges[int(tok[0])] = float(tok[1]) / U.E_C
            else:
                raise ConfigError(f"topology: unknown section [{section}]")
    return t


class StageTimes:
    """Per-stage count, total, min and max time of one phase -- the
    reference's timings accumulator (src/timings.rs:120-150, 440-505).
    Device stages arrive per call of several steps (the library times the
    stages of a whole call), so a call of k steps adds k samples whose
    min / max are the call's mean per step; host stages add one sample per
    measurement."""

    def __init__(self):
        self.acc = {}

    def record(self, name: str, seconds: float, count: int = 1) -> None:
        if count <= 0:
            return
        ns = seconds * 1e9
        per = ns / count
        a = self.acc.get(name)
        if a is None:
            self.acc[name] = [count, ns, per, per]
        else:
            a[0] += count
            a[1] += ns
            a[2] = min(a[2], per)
            a[3] = max(a[3], per)

    def rows(self):
        return [(k, int(v[0]), v[1], v[2], v[3]) for k, v in self.acc.items() if v[0] > 0]


def write_timings(path, times: StageTimes) -> None:
    """The `.timings` table of src/timings.rs:513-548: one row per stage
    with count, total ms, mean / min / max us; an existing file is an error
    (the reference's OutputExists)."""
    with open(path, "x") as f:
        f.write(f"{'stage':<28} {'count':>10} {'total_ms':>14} {'mean_us':>13} {'min_us':>11} {'max_us':>11}\n")
        for name, count, total_ns, min_ns, max_ns in times.rows():
            f.write(f"{name:<28} {count:>10} {total_ns / 1e6:>14.3f} {total_ns / 1e3 / count:>13.1f} "
                    f"{min_ns / 1e3:>11.1f} {max_ns / 1e3:>11.1f}\n")
