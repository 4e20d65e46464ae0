"""Batched replicas (C ABI): every member's step captured into one CUDA graph
must advance each member exactly as that member run alone would -- byte for
byte, including device-side neighbour rebuild decisions -- for boxes of
uneven sizes and both integrators, with one multi-system pair kernel for
all members and with a pair kernel per member."""

import numpy as np
import pytest

import heddle_b200 as hb
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def member(spec, kind, seed):
    ctx = hb.Context(0)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    it = hb.Integrator(sys_, kind, spec.dt, friction=spec.friction,
                       temperature=spec.temperature, seed=seed)
    return ctx, sys_, ff, cons, it


def close_all(objs):
    for o in reversed(objs):
        o.close()


@pytest.mark.parametrize("one_launch", [True, False], ids=["one-pair-launch", "pair-per-member"])
@pytest.mark.parametrize("kind", ["velocity-verlet", "langevin-baoab"])
def test_batch_matches_members_run_alone(ctx, kind, one_launch):
    specs = [S.spc_water(n, r_cut_A=7.0, skin_A=0.8, seed=20 + n) for n in (216, 300, 512, 343)]
    steps = 30
    # alone: each member's own graph steps
    alone = []
    for k, spec in enumerate(specs):
        c, sys_, ff, cons, it = member(spec, kind, 100 + k)
        it.step_graph(ff, cons, n_steps=steps)
        alone.append((sys_.state(), ff.stats()["rebuilds"]))
        close_all([c, sys_, ff, cons, it])
    # together: one graph launch per step
    members, objs = [], []
    for k, spec in enumerate(specs):
        c, sys_, ff, cons, it = member(spec, kind, 100 + k)
        members.append((it, ff, cons))
        objs.append((c, sys_, ff, cons, it))
    batch = hb.Batch(ctx, members)
    batch.set_pair_form(one_launch)
    # the members share the pair physics: one multi-system pair kernel
    # replaces their pair launches when asked to
    assert batch.pair_form() == one_launch
    top, body = batch.count_launches()
    assert top > 0 and body == 10 * len(specs)
    batch.step(steps)
    for k, (c, sys_, ff, cons, it) in enumerate(objs):
        state, rebuilds = alone[k]
        for a, b in zip(state, sys_.state()):
            assert np.array_equal(a, b)
        assert ff.stats()["rebuilds"] == rebuilds
    batch.close()
    for o in objs:
        close_all(list(o))


def test_batch_rejects_shared_context(ctx):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=0.8)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    it = hb.Integrator(sys_, "velocity-verlet", spec.dt)
    with pytest.raises(hb.HeddleError):
        hb.Batch(ctx, [(it, ff, None)])
    it.close(), ff.close(), sys_.close()
