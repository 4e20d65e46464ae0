"""GPU parity of the learned SHAKE warm start: the tensor-core network's
forward pass and gradients against the CPU statement (oracle/mlp.py, FP64
with the same bfloat16 operand rounding), training that lowers the loss, and
SHAKE warm-started by a network trained on multipliers from plain runs: the
same tolerance is met with fewer sweeps."""

import numpy as np
import pytest

import heddle_b200 as hb
from heddle_b200 import systems as S
from oracle import mlp as M

pytestmark = pytest.mark.gpu


def random_net(ctx, seed=3):
    rng = np.random.default_rng(seed)
    net = hb.ShakeMLP(ctx, seed=seed)
    p = rng.normal(scale=0.25, size=M.NPARAM).astype(np.float32)
    net.set_params(p)
    mean = rng.normal(scale=0.5, size=8).astype(np.float32)
    inv = rng.uniform(0.5, 2.0, size=8).astype(np.float32)
    net.set_normalization(mean, inv, 0.7)
    return net, p.astype(np.float64), mean, inv, rng


def test_forward_matches_oracle(ctx):
    net, p, mean, inv, rng = random_net(ctx)
    x = rng.normal(size=(1000, 8)).astype(np.float32)
    y = net.predict(x)
    yo, _ = M.forward(p, x, mean, inv, 0.7)
    assert np.abs(y - yo).max() < 2e-3
    assert np.abs(y - yo).mean() < 2e-5
    net.close()


@pytest.mark.parametrize("rows", [128, 300, 1024])
def test_gradients_match_oracle(ctx, rows):
    net, p, mean, inv, rng = random_net(ctx, seed=rows)
    x = rng.normal(size=(rows, 8)).astype(np.float32)
    t = rng.normal(size=rows).astype(np.float32)
    g, loss = net.gradients(x, t)
    go, lo = M.gradients(p, x, t, mean, inv, 0.7)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    for name, a, b in (("W1", M.OFF_W1, M.OFF_B1), ("b1", M.OFF_B1, M.OFF_W2),
                       ("W2", M.OFF_W2, M.OFF_B2), ("b2", M.OFF_B2, M.OFF_W3),
                       ("w3", M.OFF_W3, M.OFF_B3), ("b3", M.OFF_B3, M.NPARAM)):
        err = np.linalg.norm(g[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-12)
        assert err < 5e-3, (name, err)
    net.close()


def test_training_lowers_loss(ctx):
    rng = np.random.default_rng(11)
    x = rng.normal(size=(20000, 8)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * x[:, 3]).astype(np.float32)
    net = hb.ShakeMLP(ctx, seed=5)
    losses = net.train(x, t, epochs=15, batch=512, lr=3e-3, seed=1)
    assert losses[-1] < 0.1 * losses[0], losses
    y = net.predict(x[:2000])
    assert np.corrcoef(y, t[:2000])[0, 1] > 0.97
    # the device loss is the oracle's loss of the trained parameters
    _, lo = M.gradients(net.params(), x[:1024], t[:1024])
    g, l_dev = net.gradients(x[:1024], t[:1024])
    assert abs(l_dev - lo) <= 1e-4 * abs(lo)
    net.close()


@pytest.fixture(scope="module")
def chain(ctx):
    """The solvated chain relaxed from its lattice start: stiff short-step
    Langevin, then the production step with light friction."""
    from heddle_b200 import units as U

    spec = S.peptide_in_water()
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    cons.after_kick(0.0)
    for dt_fs, fric, n in ((0.25, 100.0, 400), (1.0, 20.0, 200), (2.0, 5.0, 200)):
        it = hb.Integrator(sys_, "langevin-baoab", U.time_au_fs(dt_fs),
                           friction=fric / (1.0e-12 / U.AUT_S), temperature=spec.temperature, seed=5)
        it.step(ff, cons, n_steps=n)
        it.close()
    pos, vel, _, _ = sys_.state()
    for o in (cons, ff, sys_):
        o.close()
    spec.positions, spec.velocities = pos, vel
    return spec


def chain_run(ctx, spec, steps, warm=None, record=False):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                       temperature=spec.temperature, seed=17)
    if warm is not None:
        cons.set_warm_start(warm)
    cons.record(record)
    rows = []
    cons.shake_stats(reset=True)
    for _ in range(steps):
        it.step(ff, cons, n_steps=1)
        if record:
            rows.append(cons.get_record())
    st = cons.shake_stats()
    pos = sys_.positions()
    for o in (it, cons, ff, sys_):
        o.close()
    return st, pos, rows


def shake_residual(pos, spec):
    n_pep = spec.meta["n_peptide"]
    off, gi, cj, ci = spec.group_offsets, spec.group_atoms, spec.con_j, spec.con_i
    res = []
    for g in range(len(spec.con_offsets) - 1):
        for k in range(spec.con_offsets[g], spec.con_offsets[g + 1]):
            a, b = gi[off[g] + ci[k]], gi[off[g] + cj[k]]
            if a < n_pep:
                d = np.linalg.norm(pos[a] - pos[b])
                res.append(abs(d * d / spec.con_dist[k] ** 2 - 1.0))
    return float(np.max(res))


def test_learned_warm_start_saves_sweeps(ctx, chain):
    spec = chain
    st0, pos0, rows = chain_run(ctx, spec, 150, record=True)
    feats = np.concatenate([r["features"] for r in rows])
    targ = np.concatenate([(r["lam"] - r["lam1"]) * r["lscale"] for r in rows]).astype(np.float32)
    net = hb.ShakeMLP(ctx, seed=2)
    mean, std = feats.mean(0), feats.std(0) + 1e-6
    net.set_normalization(mean, 1.0 / std, float(targ.std() + 1e-12))
    losses = net.train(feats, targ, epochs=40, batch=256, lr=2e-3, seed=3)
    assert losses[-1] < 0.05 * losses[0], losses
    st1, pos1, _ = chain_run(ctx, spec, 150, warm=net)
    # same tolerance, fewer sweeps
    assert st1["mean_sweeps"] < 0.75 * st0["mean_sweeps"], (st0, st1)
    tol_store = 1e-5  # f32 storage of the constrained positions
    assert shake_residual(pos0, spec) < tol_store and shake_residual(pos1, spec) < tol_store
    # the cost gate times both forms, keeps the faster one and leaves the
    # state as it found it
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    p_before = sys_.positions()
    g = cons.choose_warm_start(net, ff, "langevin-baoab", spec.dt, steps=20, friction=spec.friction,
                               temperature=spec.temperature, seed=5)
    assert np.array_equal(sys_.positions(), p_before)
    faster = "learned" if g["learned"]["ms_per_step"] < g["plain"]["ms_per_step"] else "plain"
    assert g["chosen"] == faster
    assert g["learned"]["mean_sweeps"] < g["plain"]["mean_sweeps"]
    assert (cons._mlp is net) == (faster == "learned")
    for o in (cons, ff, sys_):
        o.close()
    net.close()


def test_bounded_wait_times_out_and_the_next_call_succeeds(ctx, chain):
    # the failure path of the tensor-core network without a GPU fault: with
    # issue=False no MMA is issued, so the first bounded mbarrier wait runs
    # out (short poll limit), the kernel frees its tensor memory and the
    # call reports HB_ERR_DEVICE_TIMEOUT; the next call works normally
    net, p, mean, inv, rng = random_net(ctx, seed=21)
    x = rng.normal(size=(300, 8)).astype(np.float32)
    y0 = net.predict(x)
    net.set_wait_limit(polls=1024, issue=False)
    with pytest.raises(hb.HeddleError) as e:
        net.predict(x)
    assert e.value.name == "HB_ERR_DEVICE_TIMEOUT"
    net.set_wait_limit()
    assert np.array_equal(net.predict(x), y0)
    # inside an integrator step: the step reports the timeout, the timed-out
    # rows get no correction (plain SHAKE start), the constraints still hold
    spec = chain
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                       temperature=spec.temperature, seed=17)
    cons.set_warm_start(net)
    net.set_wait_limit(polls=1024, issue=False)
    with pytest.raises(hb.HeddleError) as e:
        it.step(ff, cons, n_steps=1)
    assert e.value.name == "HB_ERR_DEVICE_TIMEOUT"
    assert shake_residual(sys_.positions(), spec) < 1e-5
    net.set_wait_limit()
    it.step(ff, cons, n_steps=2)
    assert shake_residual(sys_.positions(), spec) < 1e-5
    for o in (it, cons, ff, sys_, net):
        o.close()
