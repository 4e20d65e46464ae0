"""GPU parity of the force path (C ABI) against the FP64 oracle.

Bars: neighbour sets bit-exact under the stated f32 rule; forces within
1e-5 relative RMS of the FP64 oracle (the tolerance of the configuration
contract); energy terms within 1e-5 relative; repeat runs byte-identical.
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


def gpu_forces(ctx, spec, scalars=True):
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=scalars)
    pos = sys_.positions()
    F = sys_.forces()
    out = (pos, F, ff.scalars() if scalars else None, ff.per_atom() if scalars else None, ff.stats())
    ff.close()
    sys_.close()
    return out


@pytest.fixture(scope="module")
def water512():
    return S.spc_water(512, skin_A=2.0)


def test_water_forces_energies_match_oracle(ctx, water512):
    spec = water512
    pos, F, sc, (E, W), st = gpu_forces(ctx, spec)
    Fo, Eo, Wo, To = O.forces(spec, pos)
    # pairs within 1e-6 of a cutoff are harmless here: LJ is switched to
    # zero at r_cut and erfc(beta r_cut) = 1e-5
    r = rms_rel(F, Fo)
    assert r <= FORCE_RMS_TOL, (r, max_rel(F, Fo))
    assert max_rel(F, Fo) < 1e-4
    # energies against the oracle evaluated with the same erfc form the
    # device uses (Abramowitz-Stegun 7.1.26 in f32, as the reference's f32
    # build): the net real-space Coulomb energy is a small residue of large
    # cancelling pair terms, so the polynomial's 1.5e-7 error shows there
    _, Ep, _, Tp = O.forces(spec, pos, poly_erfc=True)
    pe_ref = Tp["lj"] + Tp["coulomb_real"] + Tp["recip"] - Tp["self"]
    # each term to 1e-5 of the potential energy: the real-space Coulomb
    # term is a residue of pair energies ~6000x larger in magnitude, so its
    # own relative error reflects f32 rounding of those pair terms
    for key, ref in (("lj", Tp["lj"]), ("coulomb_real", Tp["coulomb_real"]), ("recip", Tp["recip"]),
                     ("self", Tp["self"])):
        assert abs(sc[key] - ref) <= 1e-5 * abs(pe_ref), (key, sc[key], ref)
    Eo = Ep
    assert abs(sc["potential"] - pe_ref) <= 1e-5 * abs(pe_ref)
    assert abs(sc["virial_pair"] - To["virial_pair"]) <= 1e-5 * abs(To["virial_pair"])
    assert abs(sc["virial_recip"] - To["virial_recip"]) <= 1e-5 * abs(To["virial_recip"])
    # per-atom shares sum to the totals and track the oracle
    assert abs(E.sum() - pe_ref) <= 1e-4 * abs(pe_ref)
    assert float(np.sqrt(((E - Eo) ** 2).mean()) / np.sqrt((Eo ** 2).mean())) < 1e-4


def test_argon_lj_forces_match_oracle(ctx):
    spec = S.lj_argon()
    pos, F, sc, _, _ = gpu_forces(ctx, spec)
    Fo, _, _, To = O.forces(spec, pos)
    assert rms_rel(F, Fo) <= FORCE_RMS_TOL
    assert abs(sc["lj"] - To["lj"]) <= 1e-5 * abs(To["lj"])


@pytest.mark.parametrize("maker", [
    lambda: S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3),
    lambda: S.spc_water(512, skin_A=2.0),
    lambda: S.lj_argon(n_atoms=1000, n_side=10, box_m=7.84e-9 * 10 / 22),
], ids=["water216", "water512", "argon1000"])
def test_neighbor_set_bit_exact(ctx, maker):
    spec = maker()
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    pairs, dups = ff.neighbor_pairs()
    pos = sys_.positions().astype(np.float32)
    rc_max = max(float(np.max(spec.lj_cutoff[spec.lj_epsilon != 0])) if spec.lj_sigma is not None else 0.0,
                 spec.r_cut_coul or 0.0)
    ref = O.neighbor_pairs_f32(pos, spec.box.astype(np.float32), np.float32(rc_max + spec.r_skin))
    ff.close()
    sys_.close()
    assert dups == 0
    assert pairs.shape == ref.shape
    assert np.array_equal(pairs, ref)


def test_repeat_runs_byte_identical(ctx, water512):
    a = gpu_forces(ctx, water512)
    b = gpu_forces(ctx, water512)
    assert np.array_equal(a[1], b[1])
    assert a[2] == b[2]
    assert np.array_equal(a[3][0], b[3][0])


def test_golden_water_216(ctx):
    from pathlib import Path
    gold = np.load(Path(__file__).resolve().parent / "golden" / "water_216.npz")
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3, velocity_seed=4)
    pos, F, sc, _, _ = gpu_forces(ctx, spec)
    # the golden forces are at the f64 positions; the device holds f32
    # positions, so compare with the looser bar of the input rounding
    assert rms_rel(F, gold["forces"]) < 2e-5
    Fo, _, _, _ = O.forces(spec, pos)
    assert rms_rel(F, Fo) <= FORCE_RMS_TOL


@pytest.mark.parametrize("order", [4, 5, 6, 8])
def test_spme_ewald_known_answer_on_device(ctx, order):
    # tests/spme_pipeline.rs:101-190 on the device: 4 charges, 1 nm box,
    # alpha 4e9 1/m, grid 16^3; E_recip within 5e-3 of the explicit Ewald sum
    L = U.length_au(1e-9)
    pos = np.array([[0.1e-9, 0.0, 0.0], [-0.1e-9, 0.2e-9, 0.0], [0.0, -0.2e-9, 0.15e-9],
                    [-0.15e-9, 0.1e-9, -0.1e-9]]) / U.BOHR_M
    q = np.array([1.0, -1.0, 2.0, -2.0])
    alpha = 4.0e9 * U.BOHR_M
    sys_ = hb.System(ctx, pos, np.ones(4), q, np.zeros(4, dtype=np.uint32), [L, L, L, 0, 0, 0])
    ff = hb.ForceField(sys_, {"spme": hb.SpmeParams(alpha, 0.3 * L, (16, 16, 16), order)}, r_skin=0.0)
    ff.step(scalars=True)
    e = ff.scalars()["recip"]
    ref = O.ewald_recip_energy(pos, q, [L, L, L, 0, 0, 0], alpha, 8)
    ff.close()
    sys_.close()
    assert abs(e - ref) / abs(ref) < 5e-3


def test_error_paths(ctx):
    spec = S.spc_water(64, r_cut_A=5.0, skin_A=0.5)
    sys_ = hb.System.from_spec(ctx, spec)
    with pytest.raises(hb.HeddleError) as e:
        hb.ForceField.from_spec(sys_, spec, r_skin=U.angstrom_au(3.0))
    assert e.value.name == "HB_ERR_BOX_TOO_SMALL"
    bad = hb.SpmeParams(spec.alpha, spec.r_cut_coul, (6, 16, 16), 4)
    with pytest.raises(hb.HeddleError) as e:
        hb.ForceField(sys_, {"spme": bad}, r_skin=spec.r_skin)
    assert e.value.name == "HB_ERR_INVALID_GRID"
    with pytest.raises(hb.HeddleError) as e:
        hb.Constraints(sys_, [0, 2], [0, 1], [0], settle_geometry=([1.0], [1.0], [1.0]))
    assert e.value.name == "HB_ERR_CONSTRAINT_SHAPE"
    with pytest.raises(hb.HeddleError) as e:
        hb.System(ctx, np.array([[np.nan, 0, 0]]), [1.0], [0.0], [0], [10, 10, 10, 0, 0, 0])
    assert e.value.name == "HB_ERR_NOT_FINITE"
    sys_.close()


def test_tiny_systems(ctx):
    # two atoms, one partial tile; and an empty system
    L = 40.0
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.5, -0.2]])
    sys_ = hb.System(ctx, pos, [1.0, 1.0], [0.5, -0.5], [0, 0], [L, L, L, 0, 0, 0])
    p = hb.LennardJonesParams(np.array([[2.5]]), np.array([[0.01]]), np.array([[8.0]]), np.array([[8.0]]))
    ff = hb.ForceField(sys_, {"lennard_jones": p, "spme": hb.SpmeParams(0.3, 8.0, (16, 16, 16), 4)}, r_skin=1.0)
    ff.step(scalars=True)
    F = sys_.forces()

    class Sp:
        pass
    sp = Sp()
    sp.positions, sp.charges, sp.types, sp.box = pos, np.array([0.5, -0.5]), np.zeros(2, dtype=np.int32), [L, L, L, 0, 0, 0]
    sp.lj_sigma, sp.lj_epsilon, sp.lj_cutoff, sp.lj_switch = [[2.5]], [[0.01]], [[8.0]], [[8.0]]
    sp.alpha, sp.r_cut_coul, sp.grid, sp.order, sp.excl_offsets = 0.3, 8.0, (16, 16, 16), 4, None
    Fo, _, _, _ = O.forces(sp, sys_.positions())
    assert rms_rel(F, Fo) < 1e-5
    ff.close()
    sys_.close()
    empty = hb.System(ctx, np.zeros((0, 3)), [], [], [], [L, L, L, 0, 0, 0])
    ff0 = hb.ForceField(empty, {"lennard_jones": p}, r_skin=1.0)
    ff0.step(scalars=True)
    assert ff0.scalars()["potential"] == 0.0
    ff0.close()
    empty.close()


@pytest.mark.parametrize("grid", [(27, 27, 27), (30, 36, 45), (50, 54, 60), (20, 24, 25),
                                  (64, 64, 64), (128, 128, 40), (128, 128, 27)],
                         ids=lambda g: "x".join(map(str, g)))
def test_compiled_fft_sizes_match_oracle(ctx, grid):
    # every compile-time specialised FFT length (radix 2/3/4/5 stage plans),
    # also anisotropic grids: reciprocal energy and total forces vs FP64.
    # 64 x 64 and 128 x 128 (a, b) planes take the whole-plane pass (kc-major
    # half spectrum, in-place transforms of each plane in shared memory),
    # with even and odd c lengths
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=4)
    spec.grid = grid
    pos, F, sc, _, _ = gpu_forces(ctx, spec)
    Fo, _, _, To = O.forces(spec, pos)
    assert rms_rel(F, Fo) <= FORCE_RMS_TOL
    _, _, _, Tp = O.forces(spec, pos, poly_erfc=True)
    assert abs(sc["recip"] - Tp["recip"]) <= 1e-5 * abs(Tp["recip"])


@pytest.mark.parametrize("maker", [
    lambda: S.spc_water(512, skin_A=2.0),
    lambda: S.lj_argon(),
    lambda: S.peptide_in_water(),
], ids=["water512", "argon10000", "chain"])
def test_force_only_kernel_matches_oracle(ctx, maker):
    # steps without and with energies both run the balanced pair kernel
    # (int32 fixed-point sums, energies only in the second): both within the
    # force tolerance, repeat runs identical
    spec = maker()
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=False)
    pos, F = sys_.positions(), sys_.forces()
    ff.step(scalars=False)
    assert np.array_equal(sys_.forces(), F)
    ff.step(scalars=True)
    F_rot = sys_.forces()
    Fo, _, _, _ = O.forces(spec, pos)
    assert rms_rel(F, Fo) <= FORCE_RMS_TOL
    assert rms_rel(F, F_rot) <= 2e-6
    ff.close(), sys_.close()


def test_force_only_kernel_large_pair_forces(ctx):
    # pair force components above 0.06 hartree/bohr bypass the int32 shared
    # accumulators: an argon pair squeezed to 0.7 sigma
    spec = S.lj_argon()
    pos = spec.positions.copy()
    sigma = spec.meta["sigma"]
    d = pos[1] - pos[0]
    pos[1] = pos[0] + 0.7 * sigma * d / np.linalg.norm(d)
    spec.positions = pos
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=False)
    p, F = sys_.positions(), sys_.forces()
    Fo, _, _, _ = O.forces(spec, p)
    assert np.abs(Fo[0]).max() > 0.06
    assert rms_rel(F, Fo) <= FORCE_RMS_TOL
    assert np.abs(F[:2] - Fo[:2]).max() <= 1e-5 * np.abs(Fo[:2]).max()
    ff.close(), sys_.close()


@pytest.mark.parametrize("kernel", ["balanced", "exact"])
def test_small_cells_with_padding_slots(ctx, kernel):
    # 127 waters (381 atoms: the last tile and many list entries end in
    # padding slots) in cells so small that no tile fits a single periodic
    # copy, so every pair takes the minimum image; over a range of cell
    # sizes the padding slots' placeholder coordinates wrap to arbitrary
    # places under the minimum image and must still take part in no pair
    for density in (997.0, 985.0, 971.0, 958.0, 944.0, 930.0):
        spec = S.spc_water(127, density=density, r_cut_A=6.0, skin_A=1.0, seed=9)
        sys_ = hb.System.from_spec(ctx, spec)
        ff = hb.ForceField.from_spec(sys_, spec, exact_pairs=(kernel == "exact"))
        ff.step(scalars=False)
        pos, F = sys_.positions(), sys_.forces()
        ff.close(), sys_.close()
        assert np.isfinite(F).all()
        Fo, _, _, _ = O.forces(spec, pos)
        assert rms_rel(F, Fo) <= FORCE_RMS_TOL, (density, rms_rel(F, Fo))


@pytest.mark.parametrize("grid,order", [((64, 64, 60), 4), ((128, 128, 50), 8), ((48, 50, 45), 8)],
                         ids=["plane64-p4", "plane128-p8", "lines-p8"])
def test_triclinic_reciprocal_paths_match_oracle(ctx, grid, order):
    # a tilted cell through the whole-plane pass (64 x 64 and 128 x 128
    # (a, b) planes) and the line passes, with spline orders 4 and 8 (the
    # spread and gather with one thread per c offset): reciprocal energy
    # and total forces against the FP64 oracle
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=6)
    lx, ly, lz = spec.box[:3]
    spec.box = np.array([lx, ly, lz, 0.12 * lx, -0.08 * lx, 0.1 * ly])
    spec.grid = grid
    spec.order = order
    # a force-only step (no energy partials in the plane pass) and a step
    # with energies on the same positions
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=False)
    F0 = sys_.forces()
    ff.step(scalars=True)
    F, sc, pos = sys_.forces(), ff.scalars(), sys_.positions()
    ff.close(), sys_.close()
    assert rms_rel(F0, F) <= 2e-6
    Fo, _, _, _ = O.forces(spec, pos)
    assert rms_rel(F, Fo) <= FORCE_RMS_TOL, rms_rel(F, Fo)
    _, _, _, Tp = O.forces(spec, pos, poly_erfc=True)
    assert abs(sc["recip"] - Tp["recip"]) <= 1e-5 * abs(Tp["recip"])


def test_launch_shapes_keep_the_forces(ctx):
    """The autotuner's knobs change launch shapes, not results: any pair
    entry chunk or work quota gives byte-identical forces (integer sums); the line-pass
    transform and the per-atom gather agree with the defaults to f32
    rounding and with the FP64 oracle."""
    from heddle_b200 import _native as N

    spec = S.spc_water(8192, skin_A=2.0)
    assert spec.grid == (64, 64, 64)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=True)
    F0, e0 = sys_.forces(), ff.scalars()["potential"]
    for chunk in (1, 3, 16):
        ff.set_launch(pair_chunk=chunk)
        ff.step(scalars=True)
        assert np.array_equal(sys_.forces(), F0), chunk
    for quota in (1, 5, 0):
        ff.set_launch(pair_quota=quota)
        ff.step(scalars=True)
        assert np.array_equal(sys_.forces(), F0), quota
    Fo, _, _, _ = O.forces(spec, sys_.positions())
    for param in (N.HB_LAUNCH_FFT_PLANE, N.HB_LAUNCH_GATHER_FORM):
        N.check(ff.lib.hb_forcefield_set_launch(ff.h, param, 0))
        ff.step(scalars=True)
        F = sys_.forces()
        assert rms_rel(F, F0) < 2e-6
        assert rms_rel(F, Fo) <= FORCE_RMS_TOL
        assert abs(ff.scalars()["potential"] - e0) <= 1e-6 * abs(e0)
        N.check(ff.lib.hb_forcefield_set_launch(ff.h, param, 1))
    ff.close()
    sys_.close()
