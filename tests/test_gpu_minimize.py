"""GPU parity of the steepest-descent minimiser (C ABI) against
oracle/minimize.py: the first iterations' energies, forces, steps and
accept / reject decisions; convergence with monotone accepted energies and
the final energy equal to the oracle's at the final positions; SETTLE
geometry kept by the position-only projection; chunked calls equal to one
call; the reference's parameter checks."""

import numpy as np
import pytest

import heddle_b200 as hb
from heddle_b200 import systems as S
from oracle import minimize as OM

pytestmark = pytest.mark.gpu


def build(ctx, spec, cons=False):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    c = hb.Constraints.from_spec(sys_, spec) if cons else None
    return sys_, ff, c


def close(*objs):
    for o in objs:
        if o is not None:
            o.close()


def test_first_iterations_match_oracle(ctx):
    spec = S.lj_argon()
    sys_, ff, _ = build(ctx, spec)
    m = hb.Minimizer(ff, energy_tolerance=0.0, force_tolerance=0.0, max_iterations=20)
    rows = [m.begin()] + m.iterate(20)
    pos0 = spec.positions.astype(np.float32).astype(np.float64)
    ref, _ = OM.steepest_descent(spec, pos0, max_iter=20)
    assert len(rows) == len(ref) == 21
    for r, (it, e, fm, step, acc, _) in zip(rows, ref):
        assert r["iteration"] == it and r["accepted"] == acc, (r, it)
        assert r["energy"] == pytest.approx(e, rel=2e-5)
        assert r["max_force"] == pytest.approx(fm, rel=2e-4)
        assert r["step"] == pytest.approx(step, rel=1e-6)
    close(m, ff, sys_)


def test_converges_with_monotone_energy(ctx):
    spec = S.lj_argon()
    sys_, ff, _ = build(ctx, spec)
    m = hb.Minimizer(ff, max_iterations=2000)
    rows = m.run(chunk=100)
    assert rows[-1]["converged"] in ("energy_tolerance", "force_tolerance"), rows[-1]
    acc = [r["energy"] for r in rows if r["accepted"]]
    assert all(b < a for a, b in zip(acc, acc[1:]))
    # the last accepted energy is the oracle's energy at the final positions
    pos = sys_.positions()
    _, e = OM.potential(spec, pos)
    assert rows[-1]["energy"] == pytest.approx(e, rel=1e-5)
    assert rows[-1]["energy"] < rows[0]["energy"]
    close(m, ff, sys_)


def test_settle_water_stays_rigid(ctx):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3)
    sys_, ff, c = build(ctx, spec, cons=True)
    m = hb.Minimizer(ff, c, energy_tolerance=0.0, max_iterations=150)
    rows = m.run(chunk=50)
    assert len(rows) == 151
    acc = [r["energy"] for r in rows if r["accepted"]]
    assert len(acc) > 50 and all(b < a for a, b in zip(acc, acc[1:]))
    pos = sys_.positions()
    d = pos.reshape(-1, 3, 3)
    L = spec.box[:3]
    for a, b, ref in ((0, 1, spec.meta["r_oh"]), (0, 2, spec.meta["r_oh"])):
        v = d[:, b] - d[:, a]
        v -= L * np.round(v / L)
        assert np.abs(np.linalg.norm(v, axis=1) - ref).max() < 2e-5
    _, e = OM.potential(spec, pos)
    assert rows[-1]["energy"] == pytest.approx(e, rel=1e-5)
    close(m, c, ff, sys_)


def test_chunked_calls_equal_one_call(ctx):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3)
    outs = []
    for chunks in ([40], [7, 13, 20]):
        sys_, ff, c = build(ctx, spec, cons=True)
        m = hb.Minimizer(ff, c, energy_tolerance=0.0, max_iterations=40)
        rows = [m.begin()]
        for k in chunks:
            rows += m.iterate(k)
        outs.append((rows, sys_.state()))
        close(m, c, ff, sys_)
    (r0, s0), (r1, s1) = outs
    assert r0 == r1
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)


def test_parameters_are_checked(ctx):
    spec = S.lj_argon()
    sys_, ff, _ = build(ctx, spec)
    for kw, msg in (({"max_step": 1e-3, "initial_step": 1e-2}, "max_step"),
                    ({"step_decrease": 1.0}, "step_decrease"),
                    ({"step_increase": 0.9}, "step_increase"),
                    ({"max_iterations": 0}, "max_iterations")):
        with pytest.raises(hb.HeddleError, match=msg):
            hb.Minimizer(ff, **kw)
    close(ff, sys_)
