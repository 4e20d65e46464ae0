"""Bit-exact time reversal of the lossless velocity-Verlet integrator
(64-bit fixed-point state) through the whole force path, following the
reference's protocol (rqm/pipeline-reversibility.md,
tests/integration_lossless.rs:302-395): forward K steps, flip velocities,
forward K steps, flip again; positions, velocities, images and forces must
equal the start bit for bit.  Both integrators also follow the FP64 oracle's
velocity-Verlet trajectory.

The force field runs with exact pair accumulation (per-pair fixed point and
per-pair minimum image), so forces are a function of positions alone and the
round trip holds across neighbour-list rebuilds, which happen at different
configurations forward and backward.  A negative companion shows the plain
integrator does not round-trip."""

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def round_trip(ctx, spec, steps, kind="velocity-verlet-lossless", exact=True):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec, exact_pairs=exact)
    it = hb.Integrator(sys_, kind, spec.dt)
    ff.step()  # F(x0) for the first kick (the integrator's warm-up does the same)
    start = sys_.state()
    r0 = ff.stats()["rebuilds"]
    it.step_graph(ff, None, n_steps=steps)
    mid = sys_.state()
    sys_.flip_velocities()
    it.step_graph(ff, None, n_steps=steps)
    sys_.flip_velocities()
    end = sys_.state()
    rebuilds = ff.stats()["rebuilds"] - r0
    it.close(), ff.close(), sys_.close()
    return start, mid, end, rebuilds


CASES = {
    # config 1: LJ argon NVE, 10,000 atoms, dt 5 fs, skin 0.3 r_cut
    "argon-10000": (lambda: S.lj_argon(), 1000),
    # Coulomb + SPME through the lossless path, small skin so the list is
    # rebuilt often
    "ionic-32768": (lambda: S.ionic_lattice(32, skin_A=0.3), 1000),
    # the 196k-atom scale of the NPT water configuration (195,112 ions,
    # 192^3 grid)
    "ionic-195112": (lambda: S.ionic_lattice(58, skin_A=0.5), 1000),
}


@pytest.mark.parametrize("case", list(CASES))
def test_lossless_round_trip_is_bit_exact(ctx, case):
    maker, steps = CASES[case]
    spec = maker()
    start, mid, end, rebuilds = round_trip(ctx, spec, steps)
    assert not np.array_equal(start[0], mid[0])  # the system moved
    assert rebuilds >= 2, rebuilds  # and the list was rebuilt on the way
    for name, a, b in zip(("positions", "velocities", "images", "forces"), start, end):
        assert np.array_equal(a, b), (name, int((a != b).sum()))


def test_plain_integrator_does_not_round_trip(ctx):
    spec = S.lj_argon()
    start, _, end, _ = round_trip(ctx, spec, 100, kind="velocity-verlet", exact=False)
    assert not (np.array_equal(start[0], end[0]) and np.array_equal(start[1], end[1]))


def rms_rel(F, R):
    return float(np.sqrt(((F - R) ** 2).sum() / (R ** 2).sum()))


@pytest.mark.parametrize("kind", ["velocity-verlet", "velocity-verlet-lossless"])
def test_velocity_verlet_ions_follow_oracle(ctx, kind):
    spec = S.ionic_lattice(10, skin_A=1.0)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec, exact_pairs=kind.endswith("lossless"))
    it = hb.Integrator(sys_, kind, spec.dt)
    pos0, vel0, _, _ = sys_.state()
    it.step(ff, None, n_steps=10)
    pos1, vel1, _, F1 = sys_.state()
    p_o, v_o, F_o = O.md_run(spec, 10, "vv", positions=pos0, velocities=vel0)
    L = spec.box[0]
    d = pos1 - p_o
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-4
    assert rms_rel(vel1, v_o) < 1e-4
    assert rms_rel(F1, F_o) < 2e-5
    it.close(), ff.close(), sys_.close()


def test_lossless_rejects_constraints(ctx):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    it = hb.Integrator(sys_, "velocity-verlet-lossless", spec.dt)
    with pytest.raises(hb.HeddleError) as e:
        it.step(ff, cons)
    assert e.value.name == "HB_ERR_UNSUPPORTED"
    it.close(), cons.close(), ff.close(), sys_.close()
