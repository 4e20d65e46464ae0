"""End-to-end runs from schema-1 configurations (TOML + extended XYZ +
topology) through the runner: outputs in the reference's formats, repeat
runs byte-identical at file level (tests/determinism.rs:93-121), energy
conservation of the NVE argon run, the NPT water run's barostat and the
bonded chain's constraints."""

import re
import shutil
from pathlib import Path

import numpy as np
import pytest

from heddle_b200 import run as R
from heddle_b200.io import load_config, read_xyz

pytestmark = pytest.mark.gpu

CFG = Path(__file__).resolve().parent / "golden" / "configs"


def staged(tmp_path, name):
    for f in CFG.glob(f"{name}.in.*"):
        shutil.copy(f, tmp_path / f.name)
    return tmp_path / f"{name}.in.toml"


def test_argon_run_is_byte_identical_and_conserves_energy(ctx, tmp_path):
    outs = []
    for k in range(2):
        d = tmp_path / f"r{k}"
        d.mkdir()
        paths = R.run(staged(d, "argon"), ctx=ctx)
        assert [p.name for p in paths] == ["argon.out.run.xyz", "argon.out.run.log", "argon.out.run.timings"]
        # trajectories and logs are byte-identical run to run; the timings are times
        outs.append([p.read_bytes() for p in paths[:2]])
    assert outs[0] == outs[1]
    # the .timings table (src/timings.rs:513-548): header, device stages
    # counted per step, host stages, the whole run
    rows = (tmp_path / "r0" / "argon.out.run.timings").read_text().splitlines()
    assert rows[0].split() == ["stage", "count", "total_ms", "mean_us", "min_us", "max_us"]
    table = {r.split()[0]: r.split()[1:] for r in rows[1:]}
    for stage in ("pair_force", "neighbor_list", "integrate_constrain", "step_total"):
        assert int(table[stage][0]) == 100
    for stage in ("config_load", "gpu_init", "init_load", "trajectory_write", "log_write", "total_runtime"):
        assert stage in table
    assert float(table["total_runtime"][1]) >= float(table["step_total"][1])
    logf = tmp_path / "r0" / "argon.out.run.log"
    # an NVE phase logs only the base columns (src/io/log_output.rs:40-60)
    assert logf.read_text().splitlines()[0] == "step,time,kinetic_energy,temperature"
    log = np.loadtxt(logf, delimiter=",", skiprows=1)
    last = read_xyz(tmp_path / "r0" / "argon.out.run.xyz", index=-1)
    assert last.step == 100 and last.velocities is not None
    # the logged kinetic energy (J) is that of the written velocities
    m = 6.6335e-26
    ke = 0.5 * m * float((last.velocities ** 2).sum()) * (5.29177210903e-11 / 2.4188843265857195e-17) ** 2
    assert log[-1, 0] == 100 and log[-1, 2] == pytest.approx(ke, rel=1e-6)


def test_water_npt_run(ctx, tmp_path):
    cfg = staged(tmp_path, "water")
    paths = R.run(cfg, ctx=ctx)
    first = read_xyz(load_config(cfg).init)
    last = read_xyz(tmp_path / "water.out.npt.xyz", index=-1)
    assert last.step == 60 and last.images is not None
    # the Monte-Carlo barostat ran (6 moves): the volume moved
    assert not np.allclose(last.box, first.box)
    # rigid waters (minimum image)
    p = last.positions.reshape(-1, 3, 3)
    d = p[:, 1] - p[:, 0]
    d -= last.box[:3] * np.round(d / last.box[:3])
    assert np.abs(np.linalg.norm(d, axis=1) - 1.8897261246).max() < 1e-4


def test_water_csvr_c_rescale_run(ctx, tmp_path):
    for f in CFG.glob("water.in.*"):
        shutil.copy(f, tmp_path / f.name)
    cfg = staged(tmp_path, "water_cr")
    paths = R.run(cfg, ctx=ctx)
    assert [p.name for p in paths] == ["water_cr.out.npt.xyz", "water_cr.out.npt.log",
                                       "water_cr.out.npt.timings"]
    lines = (tmp_path / "water_cr.out.npt.log").read_text().splitlines()
    assert lines[0] == ("step,time,kinetic_energy,temperature,csvr_conserved,pressure,box_volume,"
                        "c_rescale_conserved")
    log = np.loadtxt(tmp_path / "water_cr.out.npt.log", delimiter=",", skiprows=1)
    assert list(log[:, 0]) == [10, 20, 30, 40, 50, 60]
    first = read_xyz(load_config(cfg).init)
    last = read_xyz(tmp_path / "water_cr.out.npt.xyz", index=-1)
    # box_volume is written in bohr^3, like the reference's Dimensionless column
    v_last = float(np.prod(last.box[:3]))
    assert log[-1, 6] == pytest.approx(v_last, rel=1e-8)
    assert not np.allclose(last.box, first.box)
    p = last.positions.reshape(-1, 3, 3)
    d = p[:, 1] - p[:, 0]
    d -= last.box[:3] * np.round(d / last.box[:3])
    # positions are scaled atom by atom after the constraint step (the
    # reference's c-rescale fragment), so bonds carry the last mu
    assert np.abs(np.linalg.norm(d, axis=1) / 1.8897261246 - 1.0).max() < 2e-3


def test_argon_minimization_then_md(ctx, tmp_path):
    shutil.copy(CFG / "argon.in.xyz", tmp_path / "argon.in.xyz")
    cfg = staged(tmp_path, "argon_min")
    paths = R.run(cfg, ctx=ctx)
    assert [p.name for p in paths] == ["argon_min.out.relax.minlog", "argon_min.out.relax.xyz",
                                       "argon_min.out.relax.timings", "argon_min.out.run.xyz",
                                       "argon_min.out.run.log", "argon_min.out.run.timings"]
    lines = (tmp_path / "argon_min.out.relax.minlog").read_text().splitlines()
    assert lines[0] == "iter,energy,max_force,step,accepted"
    rows = np.loadtxt(tmp_path / "argon_min.out.relax.minlog", delimiter=",", skiprows=1)
    assert rows[0, 0] == 0 and rows[0, 3] == 0.0 and rows[0, 4] == 1
    assert all(int(i) % 5 == 0 for i in rows[:-1, 0])
    acc = rows[rows[:, 4] == 1, 1]
    assert np.all(np.diff(acc) < 0)  # accepted energies fall
    first = read_xyz(tmp_path / "argon_min.out.relax.xyz", index=0)
    assert first.step == 0 and first.velocities is None and first.images is not None
    # frames: iteration 0, then accepted iterations that are multiples of 10
    text = (tmp_path / "argon_min.out.relax.xyz").read_text()
    steps = [int(x) for x in re.findall(r"Step=(\d+)", text)]
    want = [0] + [int(i) for i, a in zip(rows[1:, 0], rows[1:, 4]) if a == 1 and int(i) % 10 == 0]
    assert steps == want and len(steps) > 1
    md = read_xyz(tmp_path / "argon_min.out.run.xyz", index=-1)
    assert md.step == 20


def test_bonded_chain_run(ctx, tmp_path):
    cfg = staged(tmp_path, "chain")
    R.run(cfg, ctx=ctx)
    last = read_xyz(tmp_path / "chain.out.run.xyz", index=-1)
    assert last.step == 40
    # SHAKE groups hold their C-H lengths
    for c, hs in ((0, (1, 2, 3)), (4, (5, 6))):
        for h in hs:
            d = last.positions[h] - last.positions[c]
            assert abs(np.linalg.norm(d) - 1.09e-10 / 5.29177210903e-11) < 1e-4
