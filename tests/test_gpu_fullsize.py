"""Parity at the full sizes of the benchmark configurations.

Each water box is relaxed on the GPU from its lattice start (stiff Langevin
with SETTLE, CUDA-graph steps), so the forces compared are those of a hot
liquid, including the few large pair forces that bypass the pair kernel's
int32 shared sums.  At the relaxed state:

* the neighbour set held by the packed list equals the oracle's f32
  minimum-image enumeration within r_cut + r_skin, bit for bit;
* the forces are within 1e-5 relative RMS of the FP64 oracle (exact erfc),
  the tolerance of the configuration contract;
* the potential-energy terms are within 1e-5 of the potential energy of the
  oracle evaluated with the device's erfc polynomial.

Sizes: 8,192 waters (24,576 atoms, SPME 64^3, r_cut 9 A), 65,536 waters
(196,608 atoms, SPME 128^3), and the smallest, median and largest boxes of
the 64-box uneven replica batch.  The measured errors are printed (pytest
-s shows them).
"""

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


def max_rel(F, R):
    return float(np.abs(F - R).max() / np.sqrt((R ** 2).sum(axis=1).mean()))


def relaxed(ctx, spec, steps=300):
    """Relax the lattice start on the GPU and return the spec at that state."""
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cons = hb.Constraints.from_spec(sys_, spec)
    cons.after_kick(0.0)
    it = hb.Integrator(sys_, "langevin-baoab", spec.dt, friction=50.0 / (1.0e-12 / U.AUT_S),
                       temperature=spec.temperature, seed=99)
    it.step_graph(ff, cons, n_steps=steps)
    pos, vel, _, _ = sys_.state()
    for o in (it, cons, ff, sys_):
        o.close()
    spec.positions, spec.velocities = pos, vel
    return spec


def check_parity(ctx, spec, label, pairs=True):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=False)
    pos, F = sys_.positions(), sys_.forces()
    ff.step(scalars=True)
    F_ev, sc = sys_.forces(), ff.scalars()
    if pairs:
        got, dups = ff.neighbor_pairs()
    ff.close(), sys_.close()
    Fo, _, _, To = O.forces(spec, pos)
    _, _, _, Tp = O.forces(spec, pos, poly_erfc=True)
    r, m = rms_rel(F, Fo), max_rel(F, Fo)
    print(f"\n{label}: N={spec.n} force rms_rel {r:.3e} max_rel {m:.3e} "
          f"(with energies: rms_rel {rms_rel(F_ev, Fo):.3e})")
    assert r <= FORCE_RMS_TOL, (r, m)
    assert rms_rel(F_ev, Fo) <= FORCE_RMS_TOL
    assert m < 2e-4
    pe = Tp["lj"] + Tp["coulomb_real"] + Tp["recip"] - Tp["self"]
    for key in ("lj", "coulomb_real", "recip", "self"):
        assert abs(sc[key] - Tp[key]) <= 1e-5 * abs(pe), (key, sc[key], Tp[key])
    assert abs(sc["potential"] - pe) <= 1e-5 * abs(pe)
    if pairs:
        ref = O.neighbor_pairs_f32(pos.astype(np.float32), spec.box.astype(np.float32),
                                   np.float32(spec.r_cut_coul + spec.r_skin))
        assert dups == 0
        assert got.shape == ref.shape and np.array_equal(got, ref)
    return r, m


def test_water_8192_config2_full_size(ctx):
    spec = relaxed(ctx, S.spc_water(8192, skin_A=2.0))
    assert tuple(spec.grid) == (64, 64, 64) and spec.n == 24576
    check_parity(ctx, spec, "spc-water-8192")


def test_water_65536_config3_full_size(ctx):
    spec = relaxed(ctx, S.spc_water(65536, skin_A=2.0))
    assert tuple(spec.grid) == (128, 128, 128) and spec.n == 196608
    check_parity(ctx, spec, "spc-water-65536")


def test_replica_batch_boxes_full_size(ctx):
    specs = S.replica_batch()
    order = np.argsort([sp.n for sp in specs])
    for k in (order[0], order[len(order) // 2], order[-1]):
        spec = relaxed(ctx, specs[k], steps=200)
        check_parity(ctx, spec, f"replica box {k}")
