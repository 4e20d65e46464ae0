"""GPU parity of the Monte-Carlo barostat (C ABI) against the oracle and a
restatement of McBarostat::apply_move (src/integrator/mc_barostat.rs:218-360):
the Philox draw and proposal, the centre-of-mass scaling, the trial energy,
the Metropolis quantity w, revert-on-reject to the byte, the width guard,
the step-size adaptation, and graph replay equal to eager launches."""

import dataclasses
import math

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import systems as S
from heddle_b200 import units as U

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5


def rms_rel(F, R):
    return float(np.sqrt(((F - R) ** 2).sum() / (R ** 2).sum()))


def draw(seed: int, counter: int):
    """u1, u2 of move `counter` (1-based): Philox key = seed, counter = (move, 0, 0)."""
    o = O.philox(seed & 0xFFFFFFFF, seed >> 32, [counter & 0xFFFFFFFF, counter >> 32, 0, 0])
    return (float(o[0]) + 0.5) / 4294967296.0, (float(o[1]) + 0.5) / 4294967296.0


def seed_with(pred, start=1):
    s = start
    while not pred(draw(s, 1)[0]):
        s += 1
    return s


def setup(ctx, n_mol=512, r_cut_A=7.0, skin_A=1.0):
    spec = S.spc_water(n_mol, r_cut_A=r_cut_A, skin_A=skin_A, seed=5)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=True)
    return spec, sys_, ff


def molecules(spec):
    return spec.mol_offsets, spec.mol_atoms


def test_accepted_move_matches_oracle(ctx):
    spec, sys_, ff = setup(ctx)
    pos0, vel0, img0, F0 = sys_.state()
    box0 = sys_.box()
    u_old = ff.scalars()["potential"]
    kt = spec.temperature
    # a draw with a clear volume change; the pressure's sign makes P dV
    # dominate w with the sign that accepts
    seed = seed_with(lambda u1: abs(2 * u1 - 1) > 0.4)
    u1, u2 = draw(seed, 1)
    v0 = float(np.prod(box0[:3]))
    dv = (0.01 * v0) * (2.0 * u1 - 1.0)
    p = -math.copysign(1e-2, dv)
    baro = hb.Barostat(sys_, p, kt, seed, frequency=1, molecules=molecules(spec))
    baro.move(ff)
    st = baro.stats()
    # proposal: bit-exact FP64 restatement
    assert st["draws"] == 1 and st["last_trial"] == 1
    assert st["last_u2"] == u2
    assert st["last_dv"] == dv
    assert st["last_u_old"] == u_old
    assert abs(st["last_scale"] - np.cbrt((v0 + dv) / v0)) <= 2e-16
    assert st["last_accepted"] == 1 and st["accepted"] == 1
    box1 = sys_.box()
    assert np.allclose(box1, box0 * st["last_scale"], rtol=1e-15, atol=0)
    # centre-of-mass scaling against the oracle (unwrapped coordinates)
    pos1, vel1, img1, F1 = sys_.state()
    po, io = O.mc_scale_com(spec.mol_offsets, spec.mol_atoms, spec.masses, box0, box1,
                            st["last_scale"], pos0, img0)
    L1 = box1[:3]
    assert np.abs((pos1 + img1 * L1) - (po + io * L1)).max() < 1e-4
    assert np.array_equal(vel1, vel0)
    # every water stays rigid (SETTLE geometry untouched by the move)
    d = pos1.reshape(-1, 3, 3)
    oh = d[:, 1] - d[:, 0]
    oh -= L1 * np.round(oh / L1)
    assert np.abs(np.linalg.norm(oh, axis=1) - spec.meta["r_oh"]).max() < 2e-5
    # trial forces and energy: the force field evaluated at the new box
    sp1 = dataclasses.replace(spec, box=box1)
    Fo, _, _, _ = O.forces(sp1, pos1)
    assert rms_rel(F1, Fo) <= FORCE_RMS_TOL
    _, _, _, Tp = O.forces(sp1, pos1, poly_erfc=True)
    pe1 = Tp["lj"] + Tp["coulomb_real"] + Tp["recip"] - Tp["self"]
    assert abs(st["last_u_new"] - pe1) <= 1e-5 * abs(pe1)
    n_mol = spec.n // 3
    w = (st["last_u_new"] - u_old) + p * dv - n_mol * kt * math.log((v0 + dv) / v0)
    assert abs(st["last_w"] - w) <= 1e-12 * max(1.0, abs(w))
    assert st["volume"] == pytest.approx(v0 + dv, rel=1e-14)
    baro.close(), ff.close(), sys_.close()


def test_rejected_move_restores_state_bytewise(ctx):
    spec, sys_, ff = setup(ctx)
    before = sys_.state()
    box0 = sys_.box()
    sc0 = ff.scalars()
    seed = seed_with(lambda u1: abs(2 * u1 - 1) > 0.4)
    u1, _ = draw(seed, 1)
    p = math.copysign(1e-2, 2 * u1 - 1)  # P dV >> 0: always rejected
    baro = hb.Barostat(sys_, p, spec.temperature, seed, frequency=1, molecules=molecules(spec))
    baro.move(ff)
    st = baro.stats()
    assert st["last_trial"] == 1 and st["last_accepted"] == 0 and st["accepted"] == 0
    assert st["last_w"] > 1.0
    assert np.array_equal(sys_.box(), box0)
    after = sys_.state()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    assert ff.scalars() == sc0
    # the list was rebuilt against the trial box; the next evaluation
    # rebuilds against the restored one and reproduces the forces exactly
    ff.step(scalars=True)
    assert np.array_equal(sys_.forces(), before[3])
    assert ff.scalars() == sc0
    baro.close(), ff.close(), sys_.close()


def test_width_guard_rejects_before_any_work(ctx):
    # 216 waters: L = 18.6 A, r_search = 8 A; a contraction below 2 r_search
    spec, sys_, ff = setup(ctx, n_mol=216)
    before = sys_.state()
    box0 = sys_.box()
    v0 = float(np.prod(box0[:3]))
    width = box0[0]
    r_search = U.angstrom_au(8.0)
    lim = (2 * r_search / width) ** 3  # V'/V below which the guard fires
    vs = 0.8 * v0
    seed = seed_with(lambda u1: 1.0 + 0.8 * (2 * u1 - 1) < lim * 0.98)
    baro = hb.Barostat(sys_, 1e-9, spec.temperature, seed, frequency=1, volume_step=vs,
                       molecules=molecules(spec))
    baro.move(ff)
    st = baro.stats()
    assert st["last_trial"] == 0 and st["attempted"] == 1 and st["accepted"] == 0
    assert np.array_equal(sys_.box(), box0)
    for a, b in zip(before, sys_.state()):
        assert np.array_equal(a, b)
    baro.close(), ff.close(), sys_.close()


def test_move_sequence_follows_restated_bookkeeping(ctx):
    spec, sys_, ff = setup(ctx, n_mol=216)
    kt = spec.temperature
    p = U.pressure_au_bar(1.0)
    seed = 77
    baro = hb.Barostat(sys_, p, kt, seed, frequency=1, molecules=molecules(spec))
    v = float(np.prod(sys_.box()[:3]))
    max_dv = 0.01 * v
    win_att = win_acc = 0
    n_acc = 0
    injection = 0.0
    n_mol = spec.n // 3
    for k in range(1, 31):
        ff.step(scalars=True)
        baro.move(ff)
        st = baro.stats()
        u1, u2 = draw(seed, k)
        dv = max_dv * (2.0 * u1 - 1.0)
        assert st["last_dv"] == dv and st["last_u2"] == u2
        assert st["last_trial"] == 1
        w = (st["last_u_new"] - st["last_u_old"]) + p * dv - n_mol * kt * math.log((v + dv) / v)
        assert abs(st["last_w"] - w) <= 1e-12 * max(1.0, abs(w))
        acc = st["last_w"] <= 0.0 or u2 < math.exp(-st["last_w"] / kt)
        assert bool(st["last_accepted"]) == acc
        v_post = v + dv if acc else v
        if acc:
            injection += p * dv
        n_acc += acc
        win_att += 1
        win_acc += acc
        if win_att >= 10:
            if win_acc < 0.25 * win_att:
                max_dv /= 1.1
            elif win_acc > 0.75 * win_att:
                max_dv = min(max_dv * 1.1, 0.3 * v_post)
            win_att = win_acc = 0
        v = v_post
        assert st["max_volume_step"] == max_dv
        assert st["volume"] == pytest.approx(v, rel=1e-13)
    assert st["attempted"] == 30 and st["accepted"] == n_acc
    assert st["conserved_term"] == pytest.approx(p * v - injection, rel=1e-9, abs=1e-12)
    assert np.prod(sys_.box()[:3]) == pytest.approx(v, rel=1e-13)
    baro.close(), ff.close(), sys_.close()


def run_npt(ctx, spec, graph: bool, n_steps=40):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                       temperature=spec.temperature, seed=3)
    baro = hb.Barostat(sys_, U.pressure_au_bar(1.0), spec.temperature, 21, frequency=10,
                       molecules=molecules(spec))
    it.set_barostat(baro)
    counts = it.count_launches(ff, cons)
    if graph:
        it.step_graph(ff, cons, n_steps=n_steps)
    else:
        it.step(ff, cons, n_steps=n_steps)
    out = sys_.state(), sys_.box(), baro.stats(), ff.stats()["rebuilds"], counts
    for o in (it, baro, cons, ff, sys_):
        o.close()
    return out


def test_npt_graph_replay_equals_eager(ctx):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=8)
    (se, be, ste, re_, ce) = run_npt(ctx, spec, graph=False)
    (sg, bg, stg, rg, cg) = run_npt(ctx, spec, graph=True)
    assert ste["attempted"] == 4 and stg["attempted"] == 4
    assert np.array_equal(be, bg)
    for a, b in zip(se, sg):
        assert np.array_equal(a, b)
    assert ste == stg
    assert re_ == rg
    assert ce == cg and ce[2] > 0
