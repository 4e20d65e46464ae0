"""Configuration / extended-XYZ / topology I/O (src/io/config.rs,
src/io/trajectory.rs, src/io/log_output.rs semantics) on CPU."""

from pathlib import Path

import numpy as np
import pytest

from heddle_b200 import units as U
from heddle_b200.io import (ConfigError, LogWriter, TrajectoryWriter, fmt_e, load_config,
                            read_topology, read_xyz)
from heddle_b200.run import config_root, molecule_csr

CFG = Path(__file__).resolve().parent / "golden" / "configs"


def test_real_format_matches_rust_exponent_style():
    # `{:.9e}`: no exponent padding, no '+'
    assert fmt_e(2.0e-9) == "2.000000000e-9"
    assert fmt_e(0.0) == "0.000000000e0"
    assert fmt_e(-7.5e-10) == "-7.500000000e-10"
    assert fmt_e(1234.5) == "1.234500000e3"
    assert fmt_e(1.0) == "1.000000000e0"


def test_config_units_are_converted_to_atomic():
    c = load_config(CFG / "argon.in.toml")
    assert c.schema_version == 1 and len(c.phases) == 1
    ph = c.phases[0]
    assert ph.n_steps == 100 and ph.dt == pytest.approx(U.time_au_fs(5.0))
    assert ph.integrator == {"kind": "velocity-verlet"}
    assert c.particle_types[0]["mass"] == pytest.approx(U.mass_au_kg(6.6335e-26))
    p = c.pair_interactions[0]
    assert p["sigma"] == pytest.approx(U.length_au(3.405e-10))
    assert p["epsilon"] == pytest.approx(U.energy_au_j(1.654e-21))
    assert c.r_skin == pytest.approx(U.length_au(1.0e-10))
    w = load_config(CFG / "water.in.toml")
    assert w.phases[0].barostat["kind"] == "monte-carlo"
    assert w.phases[0].barostat["pressure"] == pytest.approx(1.0e5 / U.PRESSURE_PA)
    assert w.spme["alpha"] == pytest.approx(4.4620e9 * U.BOHR_M)
    assert w.constraint_types["SPC"]["kind"] == "settle"
    cr = load_config(CFG / "water_cr.in.toml").phases[0]
    assert cr.thermostat == {"kind": "csvr", "temperature": pytest.approx(U.temperature_au_k(300.0)),
                             "tau": pytest.approx(1.0e-13 / U.AUT_S), "seed": 11}
    assert cr.barostat["kind"] == "c-rescale" and cr.barostat["seed"] == 13
    assert cr.barostat["tau"] == pytest.approx(1.0e-12 / U.AUT_S)
    # inverse pressure: 4.5e-10 / Pa in bohr^3 / hartree
    assert cr.barostat["compressibility"] == pytest.approx(4.5e-10 * U.PRESSURE_PA)
    ch = load_config(CFG / "chain.in.toml")
    assert ch.bond_types["CC"]["k"] == pytest.approx(U.energy_au_j(4.3e2) * U.BOHR_M ** 2)
    assert ch.dihedral_types["X"]["n"] == 3
    assert ch.constraint_types["CH3"]["atoms"] == 4


@pytest.mark.parametrize("patch,message", [
    ("[phase.thermostat]\nkind = \"nose-hoover-chain\"\n", "thermostat kind 'nose-hoover-chain'"),
    ("[phase.barostat]\nkind = \"mtk-npt\"\npressure = 1.0e5\n", "barostat kind 'mtk-npt'"),
    ("[phase.thermostat]\nkind = \"csvr\"\ntemperature = 300.0\nseed = 1\n", "missing `tau`"),
    ("[phase.thermostat]\nkind = \"andersen\"\ntemperature = 300.0\ncollision_rate = -1.0\nseed = 1\n",
     "collision_rate"),
    ("[phase.barostat]\nkind = \"c-rescale\"\npressure = 1.0e5\ntau = 1e-12\ncompressibility = 0.0\n"
     "temperature = 300.0\nseed = 1\n", "compressibility"),
])
def test_unsupported_slots_are_rejected(tmp_path, patch, message):
    text = (CFG / "argon.in.toml").read_text().replace("[phase.output]", patch + "\n[phase.output]")
    (tmp_path / "argon.in.xyz").write_text((CFG / "argon.in.xyz").read_text())
    p = tmp_path / "x.in.toml"
    p.write_text(text)
    with pytest.raises(ConfigError, match=message):
        load_config(p)


def test_thermostat_needs_velocity_verlet(tmp_path):
    (tmp_path / "water.in.xyz").write_text((CFG / "water.in.xyz").read_text())
    (tmp_path / "water.in.topology").write_text((CFG / "water.in.topology").read_text())
    text = (CFG / "water.in.toml").read_text().replace(
        "[phase.barostat]", "[phase.thermostat]\nkind = \"berendsen\"\ntemperature = 300.0\n"
        "tau = 1.0e-13\n\n[phase.barostat]")
    p = tmp_path / "w.in.toml"
    p.write_text(text)
    with pytest.raises(ConfigError, match="velocity-verlet"):
        load_config(p)


def test_log_columns_follow_the_reference_slots():
    from heddle_b200.run import log_columns
    w = load_config(CFG / "water.in.toml").phases[0]
    assert [c for c, _ in log_columns(w)] == ["box_volume", "mc_acceptance", "mc_volume_step",
                                              "mc_conserved"]
    cr = load_config(CFG / "water_cr.in.toml").phases[0]
    assert log_columns(cr) == [("csvr_conserved", "energy"), ("pressure", "pressure"),
                               ("box_volume", "dimensionless"), ("c_rescale_conserved", "energy")]
    assert log_columns(load_config(CFG / "argon.in.toml").phases[0]) == []


def test_minimization_phase_order_and_defaults(tmp_path):
    from heddle_b200.io import MinimizationConfig, PhaseConfig
    c = load_config(CFG / "argon_min.in.toml")
    assert [type(p) for p in c.phases] == [MinimizationConfig, PhaseConfig]
    m = c.phases[0]
    assert m.name == "relax"
    a = m.algorithm
    # reference defaults (src/minimizer/steepest_descent.rs:43-62) in a.u.
    assert a["initial_step"] == pytest.approx(1.0e-12 / U.BOHR_M)
    assert a["max_step"] == pytest.approx(1.0e-10 / U.BOHR_M)
    assert (a["step_increase"], a["step_decrease"]) == (1.2, 0.2)
    assert a["force_tolerance"] == pytest.approx(1.0e-13 / U.FORCE_N)
    assert a["energy_tolerance"] == 1.0e-7 and a["max_iterations"] == 2000
    assert m.output["minlog_every"] == 5 and m.output["trajectory_every"] == 10
    assert m.output["include_images"] is True
    # a [[phase]] before a [[minimization]] keeps its place
    text = (CFG / "argon_min.in.toml").read_text()
    i, j = text.index("[[minimization]]"), text.index("[[phase]]")
    k = text.index("[[particle_types]]")
    swapped = text[:i] + text[j:k] + text[i:j] + text[k:]
    (tmp_path / "argon.in.xyz").write_text((CFG / "argon.in.xyz").read_text())
    p = tmp_path / "s.in.toml"
    p.write_text(swapped)
    assert [type(q) for q in load_config(p).phases] == [PhaseConfig, MinimizationConfig]
    for old, new, msg in (('kind = "steepest-descent"', 'kind = "lbfgs"', "lbfgs"),
                          ("max_iterations = 2000", "max_iterations = 0", "max_iterations"),
                          ("max_iterations = 2000", "step_decrease = 1.5", "step_decrease")):
        p.write_text(text.replace(old, new))
        with pytest.raises(ConfigError, match=msg):
            load_config(p)


def test_output_defaults_follow_the_reference():
    ph = load_config(CFG / "water.in.toml").phases[0]
    # include_velocities defaults to true (src/io/config.rs:865-868)
    assert ph.output["include_velocities"] is True and ph.output["include_images"] is True


def test_minlog_rows_are_si(tmp_path):
    from heddle_b200.io import MinlogWriter
    w = MinlogWriter(tmp_path / "m.minlog")
    w.write({"iteration": 0, "energy": 1.0, "max_force": 2.0, "step": 0.0, "accepted": True})
    w.write({"iteration": 10, "energy": -1.0, "max_force": 0.5, "step": 1.0, "accepted": False})
    w.close()
    lines = (tmp_path / "m.minlog").read_text().splitlines()
    assert lines[0] == "iter,energy,max_force,step,accepted"
    assert lines[1] == f"0,{fmt_e(U.HARTREE_J)},{fmt_e(2.0 * U.FORCE_N)},0.000000000e0,1"
    assert lines[2] == f"10,{fmt_e(-U.HARTREE_J)},{fmt_e(0.5 * U.FORCE_N)},{fmt_e(U.BOHR_M)},0"


def test_bad_values_are_rejected(tmp_path):
    (tmp_path / "argon.in.xyz").write_text((CFG / "argon.in.xyz").read_text())
    for old, new, msg in (("schema_version = 1", "schema_version = 2", "schema_version"),
                          ("dt = 5.0e-15", "dt = -1.0", "strictly positive"),
                          ("r_switch = 8.5125e-10", "r_switch = 9.0e-10", "r_switch")):
        p = tmp_path / "y.in.toml"
        p.write_text((CFG / "argon.in.toml").read_text().replace(old, new))
        with pytest.raises(ConfigError, match=msg):
            load_config(p)


def test_xyz_round_trip(tmp_path):
    f = read_xyz(CFG / "water.in.xyz")
    assert len(f.species) == 648 and f.species[:3] == ["O", "H", "H"]
    rng = np.random.default_rng(1)
    vel = rng.normal(scale=1e-4, size=f.positions.shape)
    img = rng.integers(-2, 3, size=f.positions.shape)
    w = TrajectoryWriter(tmp_path / "t.xyz", ["O", "H"], True, True)
    types = np.array([0, 1, 1] * 216)
    w.write(7, 123.0, f.box, types, f.positions, vel, img)
    w.write(8, 124.0, f.box, types, f.positions + 0.5, vel, img)
    w.close()
    g = read_xyz(tmp_path / "t.xyz", index=-1)
    assert g.step == 8 and g.time == pytest.approx(124.0, rel=1e-9)
    assert np.allclose(g.positions, f.positions + 0.5, rtol=1e-9, atol=0)
    assert np.allclose(g.velocities, vel, rtol=1e-9, atol=0)
    assert np.array_equal(g.images, img)
    assert np.allclose(g.box, f.box, rtol=1e-9)
    with pytest.raises(FileExistsError):
        TrajectoryWriter(tmp_path / "t.xyz", ["O"])


def test_log_format(tmp_path):
    w = LogWriter(tmp_path / "l.log", [("potential_energy", "energy")])
    w.write(5, 10.0, 0.001, 0.00095, [-0.5])
    w.close()
    lines = (tmp_path / "l.log").read_text().splitlines()
    assert lines[0] == "step,time,kinetic_energy,temperature,potential_energy"
    cols = lines[1].split(",")
    assert cols[0] == "5" and float(cols[3]) == pytest.approx(0.00095 * U.HARTREE_K)
    assert float(cols[4]) == pytest.approx(-0.5 * U.HARTREE_J)


def test_topology_sections_and_molecules():
    t = read_topology(CFG / "chain.in.topology")
    assert len(t.bonds) == 3 and len(t.angles) == 6 and len(t.dihedrals) == 1
    assert t.constraints[0][1] == "CH3" and len(t.constraints[0][0]) == 4
    assert len(t.charges) == 14
    groups = [a for a, _ in t.constraints]
    off, atoms = molecule_csr(638, groups, [(i, j) for i, j, _ in t.bonds])
    # the 14-atom chain is one molecule, every water another
    assert off[1] == 14 and len(off) - 1 == 1 + (638 - 14) // 3
    assert config_root(Path("a/b/chain.in.toml")) == "chain"


def test_timings_table_format_and_no_overwrite(tmp_path):
    """The `.timings` writer follows src/timings.rs:513-548: a header row and
    one row per stage (count, total ms, mean / min / max us), and it never
    overwrites an existing file (the reference's OutputExists)."""
    from heddle_b200.io import StageTimes, write_timings

    t = StageTimes()
    t.record("pair_force", 3e-3, 10)    # one call of 10 steps: mean 300 us
    t.record("pair_force", 1e-3, 5)     # 5 steps: mean 200 us
    t.record("log_write", 2e-4)
    path = tmp_path / "x.out.run.timings"
    write_timings(path, t)
    rows = path.read_text().splitlines()
    assert rows[0] == (f"{'stage':<28} {'count':>10} {'total_ms':>14} {'mean_us':>13} "
                       f"{'min_us':>11} {'max_us':>11}")
    f = rows[1].split()
    assert f[0] == "pair_force" and f[1] == "15" and f[2] == "4.000"
    assert f[3] == "266.7" and f[4] == "200.0" and f[5] == "300.0"
    assert rows[2].split()[:2] == ["log_write", "1"]
    with pytest.raises(FileExistsError):
        write_timings(path, t)
