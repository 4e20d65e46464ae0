"""GPU checks of the exchange step (C ABI hb_integrator_step_exchange_f32):
upload, steps and read-out in one call give byte for byte the state that the
separate calls give (hb_system_set_state_f32, hb_integrator_step_graph,
hb_system_get_state_f32): with page-locked host arrays (positions and image
counts copied out while the last step's force evaluation runs) and pageable
ones, for Langevin with Monte-Carlo barostat moves (a move at the end of a
call reads everything after it) and for velocity Verlet with per-step
c-rescale coupling (positions scaled in the step's tail)."""

import numpy as np
import pytest
import torch

import heddle_b200 as hb
from heddle_b200 import systems as S
from heddle_b200 import units as U

pytestmark = pytest.mark.gpu

TYPES = (np.float32, np.float32, np.int32, np.float32)


def host(n, pinned):
    if pinned:
        return tuple(torch.empty((n, 3), dtype=getattr(torch, np.dtype(t).name), pin_memory=True)
                     .numpy() for t in TYPES)
    return tuple(np.zeros((n, 3), dtype=t) for t in TYPES)


def build(ctx, spec, kind):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    if kind == "langevin":
        it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=spec.friction,
                           temperature=spec.temperature, seed=5)
        coupling = hb.Barostat(sys_, U.pressure_au_bar(1.0), spec.temperature, 21, frequency=3,
                               molecules=(spec.mol_offsets, spec.mol_atoms))
    else:
        it = hb.Integrator(sys_, "velocity-verlet", spec.dt)
        coupling = hb.PressureCoupling(sys_, "c_rescale", U.pressure_au_bar(1.0),
                                       U.time_au_fs(1000.0), 4.5e-10 * U.PRESSURE_PA,
                                       temperature=spec.temperature, seed=3)
    it.set_barostat(coupling)
    return [it, coupling, cons, ff, sys_]


@pytest.mark.parametrize("kind", ["langevin", "vv-c-rescale"])
@pytest.mark.parametrize("pinned", [True, False])
def test_exchange_step_matches_separate_calls(ctx, kind, pinned):
    spec = S.spc_water(512, skin_A=2.0)
    a = build(ctx, spec, kind)
    b = build(ctx, spec, kind)
    n = spec.n
    outs = (host(n, pinned), host(n, pinned))  # alternating host arrays: new pointers
    ref = host(n, False)
    a[4].state_f32(outs[1])
    start = outs[1][0].copy()
    # calls of 1 step put barostat moves (every 3rd step) at a call's end and
    # elsewhere; the calls of 2 and 4 steps run plain graphs before the last
    for k, n_steps in enumerate((1, 1, 1, 1, 1, 1, 2, 4, 1)):
        out, prev = outs[k % 2], outs[(k + 1) % 2]
        p_in, v_in = prev[0].copy(), prev[1].copy()
        if k == 4:
            p_in, v_in = None, None  # nothing uploaded: the device state continues
        a[0].step_exchange(a[3], a[2], n_steps, p_in, v_in, out)
        if p_in is not None:
            b[4].set_state_f32(p_in, v_in)
        b[0].step_graph(b[3], b[2], n_steps)
        b[4].state_f32(ref)
        for x, y, name in zip(out, ref, ("positions", "velocities", "images", "forces")):
            assert np.array_equal(x, y), (k, name)
    assert not np.array_equal(outs[0][0], start)
    if kind == "langevin":
        assert a[1].stats()["attempted"] == b[1].stats()["attempted"] == 13 // 3
    # a partial read-out: only forces
    frc = host(n, pinned)[3]
    a[0].step_exchange(a[3], a[2], 1, out=(None, None, None, frc))
    b[0].step_graph(b[3], b[2], 1)
    b[4].state_f32(ref)
    assert np.array_equal(frc, ref[3])
    for obj in a + b:
        obj.close()


def test_exchange_step_rejects_bad_input(ctx):
    """A non-finite uploaded position fails the call before any step runs."""
    spec = S.spc_water(512, skin_A=2.0)
    it, coupling, cons, ff, sys_ = build(ctx, spec, "langevin")
    out = host(spec.n, True)
    sys_.state_f32(out)
    p_bad = out[0].copy()
    p_bad[3, 1] = np.nan
    with pytest.raises(hb.HeddleError, match="non-finite position for atom 3"):
        it.step_exchange(ff, cons, 1, p_bad, None, out)
    with pytest.raises(hb.HeddleError):
        it.step_exchange(ff, cons, 0, None, None, out)
    for obj in (it, coupling, cons, ff, sys_):
        obj.close()
