"""GPU parity of the constraint and integrator path (C ABI) against the FP64
oracle: SETTLE / SHAKE position resets and velocity projections, one
velocity-Verlet step with the reference's hook order, multi-step rigidity,
byte-identical repeat runs, CUDA-graph replay equal to eager launches, and
the Langevin thermostat's temperature."""

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def rms_rel(F, R):
    return float(np.sqrt(((F - R) ** 2).sum() / (R ** 2).sum()))


def make(ctx, spec, with_cons=True, kind="velocity-verlet", seed=9):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec) if with_cons else None
    it = hb.Integrator(sys_, kind, spec.dt, friction=spec.friction, temperature=spec.temperature, seed=seed)
    return sys_, ff, cons, it


def close(*objs):
    for o in objs:
        if o is not None:
            o.close()


def geometry_error(pos, spec):
    # atoms are wrapped one by one, so bond vectors take the minimum image
    p = pos.reshape(-1, 3, 3)
    L = spec.box[:3]

    def dist(a, b):
        d = p[:, a] - p[:, b]
        d -= L * np.round(d / L)
        return np.linalg.norm(d, axis=1)

    d1 = dist(0, 1) - spec.meta["r_oh"]
    d2 = dist(0, 2) - spec.meta["r_oh"]
    d3 = dist(1, 2) - spec.meta["d_hh"]
    return float(np.abs(np.concatenate([d1, d2, d3])).max())


@pytest.mark.parametrize("shake", [False, True], ids=["settle", "shake"])
def test_position_reset_matches_converged_projection(ctx, shake):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0)
    if shake:
        spec = S.water_shake_groups(spec)
    sys_ = hb.System.from_spec(ctx, spec)
    cons = hb.Constraints.from_spec(sys_, spec, shake_tol=1e-10, shake_max_iter=500)
    ref = sys_.positions()
    cons.before_drift()
    rng = np.random.default_rng(4)
    moved = ref + rng.normal(scale=0.01, size=ref.shape)
    sys_.set_state(moved, np.zeros_like(moved))
    cons.after_drift(spec.dt)
    pos, vel, _, _ = sys_.state()
    start = sys_  # positions uploaded from f64 -> f32: use the device's copy as input
    p_o, v_o, _, used = O.constrain_positions(spec, ref, moved.astype(np.float32).astype(np.float64),
                                              np.zeros_like(moved), spec.dt)
    assert used >= 0
    # the reset is the same projection: agreement to f32 resolution
    assert np.abs(pos - p_o).max() < 2e-5
    assert geometry_error(pos, spec) < 2e-5
    assert rms_rel(vel, v_o) < 1e-3
    close(cons, start)


def test_velocity_projection_zeroes_bond_velocities(ctx):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0)
    sys_ = hb.System.from_spec(ctx, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    rng = np.random.default_rng(5)
    v0 = rng.normal(scale=1e-3, size=(spec.n, 3))
    sys_.set_state(None, v0)
    cons.after_kick(spec.dt)
    pos, vel, _, _ = sys_.state()
    v_o, _ = O.constrain_velocities(spec, pos, v0.astype(np.float32).astype(np.float64), spec.dt)
    assert rms_rel(vel, v_o) < 1e-5
    p = pos.reshape(-1, 3, 3)
    u = vel.reshape(-1, 3, 3)
    for a, b in ((0, 1), (0, 2), (1, 2)):
        rel = np.einsum("mi,mi->m", p[:, a] - p[:, b], u[:, a] - u[:, b])
        assert np.abs(rel).max() < 1e-5 * np.abs(v0).max() * 2.0
    close(cons, sys_)


def test_velocity_verlet_step_matches_oracle(ctx):
    spec = S.spc_water(512, skin_A=2.0)
    sys_, ff, cons, it = make(ctx, spec)
    pos0, vel0, _, _ = sys_.state()
    it.step(ff, cons, n_steps=1)
    pos1, vel1, _, F1 = sys_.state()
    p_o, v_o, F_o = O.md_run(spec, 1, "vv", positions=pos0, velocities=vel0)
    L = spec.box[0]
    d = pos1 - p_o
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 5e-5
    assert rms_rel(vel1, v_o) < 1e-4
    assert rms_rel(F1, F_o) < 2e-5
    close(it, cons, ff, sys_)


def test_settle_dynamics_stays_rigid_and_deterministic(ctx):
    spec = S.spc_water(512, skin_A=2.0)
    runs = []
    for _ in range(2):
        sys_, ff, cons, it = make(ctx, spec)
        it.step(ff, cons, n_steps=40)
        runs.append(sys_.state())
        st = ff.stats()
        close(it, cons, ff, sys_)
    assert geometry_error(runs[0][0], spec) < 5e-5
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)


def test_graph_replay_equals_eager(ctx):
    spec = S.spc_water(512, skin_A=2.0)
    sys_a, ff_a, cons_a, it_a = make(ctx, spec)
    it_a.step(ff_a, cons_a, n_steps=12)
    sa = sys_a.state()
    sys_b, ff_b, cons_b, it_b = make(ctx, spec)
    it_b.step_graph(ff_b, cons_b, n_steps=12)
    sb = sys_b.state()
    for a, b in zip(sa, sb):
        assert np.array_equal(a, b)
    close(it_a, cons_a, ff_a, sys_a, it_b, cons_b, ff_b, sys_b)


def test_langevin_graph_replay_equals_eager(ctx):
    # the Philox draw counter lives on the device, so graph replays draw
    # the same noise as eager launches, and the rebuild condition is the
    # same device-side decision
    spec = S.spc_water(512, skin_A=0.5)
    sa, fa, ca, ia = make(ctx, spec, kind="langevin-baoab", seed=77)
    ia.step(fa, ca, n_steps=15)
    st_a = sa.state()
    rb_a = fa.stats()["rebuilds"]
    sb, fb, cb, ib = make(ctx, spec, kind="langevin-baoab", seed=77)
    ib.step_graph(fb, cb, n_steps=15)
    st_b = sb.state()
    rb_b = fb.stats()["rebuilds"]
    assert rb_a == rb_b and rb_a > 1
    for a, b in zip(st_a, st_b):
        assert np.array_equal(a, b)
    top, body, _ = ib.count_launches(fb, cb)
    # fused step head + displacement check, the reciprocal chain, the pair
    # kernel and the finalize every step; the rebuild's kernels in the IF node
    assert top >= 8 and body > 5
    close(ia, ca, fa, sa, ib, cb, fb, sb)


def test_neighbor_rebuilds_happen_on_device(ctx):
    spec = S.spc_water(512, skin_A=0.5)
    sys_, ff, cons, it = make(ctx, spec)
    before = ff.stats()["rebuilds"]
    it.step(ff, cons, n_steps=30)
    after = ff.stats()["rebuilds"]
    assert after > before
    # forces after many rebuilds still match the oracle at the current positions
    ff.step(scalars=False)
    pos = sys_.positions()
    Fo, _, _, _ = O.forces(spec, pos)
    assert rms_rel(sys_.forces(), Fo) < 1e-5
    close(it, cons, ff, sys_)


def test_langevin_thermostat_reaches_temperature(ctx):
    spec = S.spc_water(512, skin_A=2.0, friction_per_ps=50.0)
    sys_, ff, cons, it = make(ctx, spec, kind="langevin-baoab", seed=123)
    it.step(ff, cons, n_steps=300)
    ke = []
    for _ in range(10):
        it.step(ff, cons, n_steps=20)
        ke.append(sys_.kinetic()[0])
    ndof = 3 * spec.n - 3 * (spec.n // 3) - 3
    t_ratio = np.mean(ke) / (0.5 * ndof * spec.temperature)
    assert 0.85 < t_ratio < 1.15, t_ratio
    assert geometry_error(sys_.positions(), spec) < 5e-5
    close(it, cons, ff, sys_)
