"""GPU check of the fused Langevin + SETTLE step head (C ABI
hb_constraints_fuse_head): on a system whose every atom is in a SETTLE water,
the one-kernel head (kick, velocity projection, drift / O / drift, position
reset, one thread per water) gives byte for byte the trajectory of the four
separate kernels, in eager steps and in graph steps, and launches four
kernels fewer per step."""

import numpy as np
import pytest

import heddle_b200 as hb
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def build(ctx, spec, fused):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    cons.fuse_head(fused)
    it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                       temperature=spec.temperature, seed=17)
    return [it, cons, ff, sys_]


def test_fused_head_matches_the_separate_kernels(ctx):
    spec = S.spc_water(512, skin_A=2.0)
    a = build(ctx, spec, True)
    b = build(ctx, spec, False)
    ka, kb = a[0].count_launches(a[2], a[1]), b[0].count_launches(b[2], b[1])
    assert ka[0] == kb[0] - 4
    for it, cons, ff, sys_ in (a, b):
        it.step(ff, cons, n_steps=5)
        it.step_graph(ff, cons, n_steps=40)
    sa, sb = a[3].state(), b[3].state()
    for x, y, name in zip(sa, sb, ("positions", "velocities", "images", "forces")):
        assert np.array_equal(x, y), name
    # the draw counter advanced once per step in both forms
    for it, cons, ff, sys_ in (a, b):
        it.step_graph(ff, cons, n_steps=1)
    assert np.array_equal(a[3].state()[1], b[3].state()[1])
    # switching the form recaptures the graphs and keeps the trajectory
    a[1].fuse_head(False)
    b[1].fuse_head(True)
    for it, cons, ff, sys_ in (a, b):
        it.step_graph(ff, cons, n_steps=3)
    for x, y in zip(a[3].state(), b[3].state()):
        assert np.array_equal(x, y)
    for obj in a + b:
        obj.close()
