"""GPU parity of the velocity thermostats and per-step pressure couplings
(C ABI) against oracle/coupling.py: one step of CSVR, Berendsen, Andersen
and c-rescale checked term by term against a plain velocity-Verlet step from
the same state; canonical temperatures over longer runs; the conserved
quantity of CSVR; the direction of Berendsen pressure coupling; forces that
still match the oracle after many box changes; graph replay equal to eager
launches."""

import dataclasses

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import systems as S
from heddle_b200 import units as U
from oracle import coupling as OC

pytestmark = pytest.mark.gpu

SEED = 9


def water():
    return S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3)


def build(ctx, spec, cons=True):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    c = None
    if cons and spec.group_offsets is not None:
        c = hb.Constraints.from_spec(sys_, spec)
        c.after_kick(0.0)
    it = hb.Integrator(sys_, "velocity-verlet", spec.dt)
    return sys_, ff, c, it


def close(*objs):
    for o in objs:
        if o is not None:
            o.close()


def plain_step(ctx, spec, scalars=False):
    """State after one uncoupled velocity-Verlet step from spec's state."""
    sys_, ff, c, it = build(ctx, spec)
    it.step(ff, c, n_steps=1, scalar_every=1 if scalars else 0)
    out = sys_.state(), sys_.box(), ff.scalars() if scalars else None
    v_cons = c.virial().sum() if c is not None else 0.0
    close(it, c, ff, sys_)
    return out, v_cons


def pre_kick_kinetic(spec, vel, force):
    """K of the velocities before the final half kick (v - F dt / 2m)."""
    inv_m = (1.0 / spec.masses.astype(np.float32)).astype(np.float64)
    v = vel - 0.5 * spec.dt * force * inv_m[:, None]
    return 0.5 * float((spec.masses[:, None] * v * v).sum())


def test_csvr_step_matches_oracle(ctx):
    spec = water()
    (st0, _, _), _ = plain_step(ctx, spec)
    pos_p, vel_p, img_p, F_p = st0
    sys_, ff, c, it = build(ctx, spec)
    tau = U.time_au_fs(100.0)
    th = hb.Thermostat(sys_, "csvr", spec.temperature, seed=SEED, tau=tau, n_constraints=3 * 216)
    it.set_thermostat(th)
    it.step(ff, c, n_steps=1)
    pos, vel, img, F = sys_.state()
    st = th.stats()
    assert st["draws"] == 1 and st["dof"] == 3 * 648 - 3 * 216 - 3
    o = OC.csvr(st["kinetic"], int(st["dof"]), spec.temperature, spec.dt, tau, SEED, 0)
    assert st["sum_squares"] == pytest.approx(o["s"], rel=1e-12)
    assert st["r"] == pytest.approx(o["r"], rel=1e-13, abs=1e-15)
    assert st["factor"] == pytest.approx(o["factor"], rel=1e-13)
    assert st["injection"] == pytest.approx(o["k_new"] - st["kinetic"], rel=1e-10, abs=1e-14)
    # K is the kinetic energy after the projection, before the final kick
    assert st["kinetic"] == pytest.approx(pre_kick_kinetic(spec, vel_p, F_p), rel=2e-5)
    # the rescale is the plain step's velocities times the factor (f32)
    fac = np.float32(st["factor"])
    assert np.array_equal(vel, (vel_p.astype(np.float32) * fac).astype(np.float64))
    assert np.array_equal(pos, pos_p) and np.array_equal(img, img_p)
    close(it, th, c, ff, sys_)


def test_berendsen_thermostat_step_matches_oracle(ctx):
    spec = water()
    (st0, _, _), _ = plain_step(ctx, spec)
    vel_p = st0[1]
    sys_, ff, c, it = build(ctx, spec)
    tau = U.time_au_fs(50.0)
    th = hb.Thermostat(sys_, "berendsen", 1.5 * spec.temperature, tau=tau, n_constraints=3 * 216)
    it.set_thermostat(th)
    it.step(ff, c, n_steps=1)
    vel = sys_.state()[1]
    st = th.stats()
    f, inj = OC.berendsen_thermostat(st["kinetic"], int(st["dof"]), 1.5 * spec.temperature,
                                     spec.dt, tau)
    assert st["factor"] == pytest.approx(f, rel=1e-14) and f > 1.0
    assert st["injection"] == pytest.approx(inj, rel=1e-12)
    assert np.array_equal(vel, (vel_p.astype(np.float32) * np.float32(f)).astype(np.float64))
    close(it, th, c, ff, sys_)


@pytest.mark.parametrize("p_coll", [1.0, 0.3])
def test_andersen_step_matches_oracle(ctx, p_coll):
    spec = S.lj_argon()
    (st0, _, _), _ = plain_step(ctx, spec)
    vel_p = st0[1]
    sys_, ff, c, it = build(ctx, spec)
    kt = spec.temperature
    th = hb.Thermostat(sys_, "andersen", kt, seed=SEED, collision_rate=p_coll / spec.dt)
    it.set_thermostat(th)
    it.step(ff, c, n_steps=1)
    vel = sys_.state()[1]
    assert th.stats()["draws"] == 1
    inv_m = (1.0 / spec.masses.astype(np.float32)).astype(np.float64)
    p = min(max((p_coll / spec.dt) * spec.dt, 0.0), 1.0)
    ref, hit = OC.andersen(vel_p, inv_m, kt, p, SEED, 0)
    moved = np.any(vel != vel_p, axis=1)
    assert np.array_equal(moved, hit)
    if p_coll == 1.0:
        assert hit.all()
    else:
        assert 0.25 < hit.mean() < 0.35
    assert np.allclose(vel[hit], ref[hit], rtol=2e-6, atol=1e-12)
    close(it, th, c, ff, sys_)


def test_c_rescale_step_matches_oracle(ctx):
    spec = water()
    (st0, box0_p, sc_p), vcons_p = plain_step(ctx, spec, scalars=True)
    pos_p, vel_p, img_p, F_p = st0
    sys_, ff, c, it = build(ctx, spec)
    box0 = sys_.box()
    p0 = U.pressure_au_bar(1.0)
    tau, kappa = U.time_au_fs(1000.0), 4.5e-10 * U.PRESSURE_PA
    pc = hb.PressureCoupling(sys_, "c_rescale", p0, tau, kappa, temperature=spec.temperature,
                             seed=SEED)
    it.set_barostat(pc)
    it.step(ff, c, n_steps=1)
    pos, vel, img, F = sys_.state()
    st = pc.stats()
    assert st["draws"] == 1
    # the virial is the force field's plus the constraint virial of the step
    assert st["virial"] == pytest.approx(sc_p["virial"] + vcons_p, rel=1e-6, abs=1e-9)
    assert st["kinetic"] == pytest.approx(pre_kick_kinetic(spec, vel_p, F_p), rel=2e-5)
    o = OC.pressure_coupling("c_rescale", st["kinetic"], st["virial"], box0, p0, spec.temperature,
                             spec.dt, tau, kappa, SEED, 0)
    assert st["pressure"] == pytest.approx(o["pressure"], rel=1e-14, abs=1e-20)
    assert st["mu"] == pytest.approx(o["mu"], rel=1e-15)
    assert st["volume"] == pytest.approx(o["volume"], rel=1e-14)
    assert np.allclose(sys_.box(), o["box"], rtol=1e-15, atol=0)
    mu = np.float32(st["mu"])
    assert np.array_equal(pos, (pos_p.astype(np.float32) * mu).astype(np.float64))
    assert np.array_equal(vel, vel_p) and np.array_equal(img, img_p)
    close(it, pc, c, ff, sys_)


def kinetic_temperature(sys_, dof):
    return 2.0 * sys_.kinetic()[0] / dof


@pytest.mark.parametrize("kind", ["csvr", "berendsen", "andersen"])
def test_thermostat_reaches_the_target_temperature(ctx, kind):
    spec = S.lj_argon()
    sys_, ff, c, it = build(ctx, spec)
    target = 1.5 * spec.temperature
    dof = 3 * spec.n - 3
    kw = {"collision_rate": 1.0 / U.time_au_fs(500.0)} if kind == "andersen" else \
        {"tau": U.time_au_fs(250.0)}
    th = hb.Thermostat(sys_, kind, target, seed=SEED, **kw)
    it.set_thermostat(th)
    it.step(ff, c, n_steps=1000)
    temps = []
    for _ in range(50):
        it.step(ff, c, n_steps=10)
        temps.append(kinetic_temperature(sys_, dof))
    assert np.mean(temps) == pytest.approx(target, rel=0.03), (kind, np.mean(temps) / target)
    close(it, th, c, ff, sys_)


def test_csvr_conserved_quantity(ctx):
    # a switched LJ tail (0.85 rc .. rc) so that K + U itself is conserved
    # without a thermostat; a hard cutoff would add the jumps of pairs that
    # cross it
    spec = S.lj_argon()
    spec = dataclasses.replace(spec, lj_switch=0.85 * spec.lj_cutoff)
    sys_, ff, c, it = build(ctx, spec)
    ff.step(scalars=True)
    h0 = sys_.kinetic()[0] + ff.scalars()["potential"]
    th = hb.Thermostat(sys_, "csvr", 1.3 * spec.temperature, seed=SEED, tau=U.time_au_fs(200.0))
    it.set_thermostat(th)
    it.step(ff, c, n_steps=400, scalar_every=400)
    k1 = sys_.kinetic()[0]
    u1 = ff.scalars()["potential"]
    inj = th.stats()["injection"]
    assert abs(inj) > 1e-3 * abs(u1)  # the thermostat did work
    h1 = k1 + u1 - inj
    # the reference's order measures K before the final half kick and
    # rescales after it, so K + U - injection is conserved only up to the
    # kick's share of each rescale
    assert abs(h1 - h0) < 1e-3 * abs(u1), (h0, h1, inj)
    close(it, th, c, ff, sys_)


@pytest.mark.parametrize("graphs", [False, True])
def test_berendsen_pressure_direction_and_forces_after_box_changes(ctx, graphs):
    spec = water()
    vols = {}
    for sign in (+1.0, -1.0):
        sys_, ff, c, it = build(ctx, spec)
        th = hb.Thermostat(sys_, "csvr", spec.temperature, seed=SEED, tau=U.time_au_fs(100.0),
                           n_constraints=3 * 216)
        pc = hb.PressureCoupling(sys_, "berendsen", sign * U.pressure_au_bar(2000.0),
                                 U.time_au_fs(1000.0), 4.5e-10 * U.PRESSURE_PA)
        it.set_thermostat(th)
        it.set_barostat(pc)
        if graphs:
            it.step_graph(ff, c, n_steps=150)
        else:
            it.step(ff, c, n_steps=150)
        st = pc.stats()
        box = sys_.box()
        vols[sign] = st["volume"]
        assert st["volume"] == pytest.approx(np.prod(box[:3]), rel=1e-12)
        assert st["guarded"] == 0
        # the list survives the small per-step scalings (it is rebuilt only
        # when an atom leaves its scaled skin), yet the forces stay exact
        assert ff.stats()["rebuilds"] < 75, ff.stats()
        # forces at the final configuration and box against the oracle
        ff.step(scalars=False)
        pos, _, _, F = sys_.state()
        Fo, _, _, _ = O.forces(dataclasses.replace(spec, box=box), pos)
        err = float(np.sqrt(((F - Fo) ** 2).sum() / (Fo ** 2).sum()))
        assert err < 1e-5, err
        close(it, pc, th, c, ff, sys_)
    # a higher target pressure ends in a smaller box (the lattice start's
    # own pressure sets the absolute direction)
    assert vols[+1.0] < vols[-1.0]


def test_coupled_graph_replay_equals_eager(ctx):
    spec = water()
    outs = []
    for graphs in (False, True):
        sys_, ff, c, it = build(ctx, spec)
        th = hb.Thermostat(sys_, "csvr", spec.temperature, seed=SEED, tau=U.time_au_fs(100.0),
                           n_constraints=3 * 216)
        pc = hb.PressureCoupling(sys_, "c_rescale", U.pressure_au_bar(1.0), U.time_au_fs(1000.0),
                                 4.5e-10 * U.PRESSURE_PA, temperature=spec.temperature, seed=SEED)
        it.set_thermostat(th)
        it.set_barostat(pc)
        if graphs:
            it.step_graph(ff, c, n_steps=40)
        else:
            it.step(ff, c, n_steps=40)
        outs.append((sys_.state(), sys_.box(), th.stats(), pc.stats()))
        close(it, pc, th, c, ff, sys_)
    (s0, b0, t0, p0), (s1, b1, t1, p1) = outs
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)
    assert np.array_equal(b0, b1) and t0 == t1 and p0 == p1


def test_coupling_is_rejected_where_the_reference_rejects_it(ctx):
    spec = S.lj_argon()
    sys_ = hb.System.from_spec(ctx, spec)
    lang = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=1e-3,
                         temperature=spec.temperature, seed=1)
    th = hb.Thermostat(sys_, "csvr", spec.temperature, seed=1, tau=100.0)
    with pytest.raises(hb.HeddleError, match="velocity-Verlet"):
        lang.set_thermostat(th)
    with pytest.raises(hb.HeddleError, match="tau"):
        hb.Thermostat(sys_, "csvr", spec.temperature, seed=1, tau=0.0)
    vv = hb.Integrator(sys_, "velocity-verlet", spec.dt)
    mc = hb.Barostat(sys_, 1e-9, spec.temperature, 1)
    pc = hb.PressureCoupling(sys_, "berendsen", 1e-9, 100.0, 1.0)
    vv.set_barostat(mc)
    with pytest.raises(hb.HeddleError, match="one barostat"):
        vv.set_barostat(pc)
    close(vv, lang, pc, mc, th, sys_)
