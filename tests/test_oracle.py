"""The FP64 oracle pinned against the reference's known answers (CPU only).

The reference stores no golden numbers for this path; its tests check the
SPME pipeline against an explicit Ewald sum (tests/spme_pipeline.rs:101-190),
the spread against B-spline weights and charge conservation (:192-383), and
rely on Philox-4x32-10 (kernels/philox.cuh).  Those cases live in
tests/golden/reference_kat.json (regenerated by tests/golden/make_golden.py).
"""

import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from heddle_b200 import systems as S

GOLD = Path(__file__).resolve().parent / "golden"
KAT = json.loads((GOLD / "reference_kat.json").read_text())


class _Spec:
    def __init__(self, pos, q, L, alpha, grid, order):
        self.positions = np.asarray(pos, dtype=float)
        self.charges = np.asarray(q, dtype=float)
        self.types = np.zeros(len(q), dtype=np.int32)
        self.box = [L, L, L, 0.0, 0.0, 0.0]
        self.lj_sigma = None
        self.alpha = alpha
        self.r_cut_coul = 0.3 * L
        self.grid = tuple(grid)
        self.order = order
        self.excl_offsets = None


@pytest.mark.parametrize("case", KAT["spme_vs_ewald"], ids=lambda c: c["name"])
def test_spme_matches_explicit_ewald(case):
    # tests/spme_pipeline.rs:101-190 and :880-924 (orders 4-8), bound 5e-3
    L = case["box"]
    ref = case["ewald_energy_mmax8"]
    e_c = O.ewald_recip_energy(case["positions"], case["charges"], [L, L, L, 0, 0, 0], case["alpha"], 8)
    assert abs(e_c - ref) / abs(ref) < 1e-12
    for order in case["orders"]:
        sp = _Spec(case["positions"], case["charges"], L, case["alpha"], case["grid"], order)
        _, _, _, T = O.forces(sp)
        assert abs(T["recip"] - ref) / abs(ref) < case["rel_bound"], order


def test_spread_conserves_charge_and_single_particle_is_bspline():
    # tests/spme_pipeline.rs:192-232 and :320-383
    rng = np.random.default_rng(1)
    L = 1.0
    pos = rng.uniform(-0.5, 0.5, size=(5, 3))
    q = np.array([1.0, -0.5, 0.25, 0.75, -1.5])
    rho = O.spme_spread(pos, q, [L, L, L, 0, 0, 0], (12, 12, 12), 4)
    assert abs(rho.sum() - q.sum()) < 1e-12
    one = O.spme_spread(np.array([[0.013, -0.21, 0.37]]), np.array([1.0]), [L, L, L, 0, 0, 0], (16, 16, 16), 4)
    nz = one[one != 0]
    assert nz.size == 64
    u = (np.array([0.013, -0.21, 0.37]) + 0.5) * 16
    t = u - np.floor(u)
    w = [O.bspline_weights(4, x)[0] for x in t]
    expect = np.einsum("i,j,k->ijk", w[0], w[1], w[2])
    assert np.allclose(np.sort(nz), np.sort(expect.reshape(-1)), rtol=1e-13, atol=0)


@pytest.mark.parametrize("order", [4, 5, 6, 7, 8])
def test_bspline_partition_of_unity(order):
    for t in (0.0, 0.2, 0.5, 0.99):
        w, dw = O.bspline_weights(order, t)
        assert abs(w.sum() - 1.0) < 1e-14
        assert abs(dw.sum()) < 1e-13
        assert (w >= 0).all()


def test_b_factors_finite_and_even_orders_positive():
    # src/forces/spme.rs:1011-1033 (finite b-factors)
    for order in (4, 5, 6, 7, 8):
        for n in (16, 25, 64):
            b = O.b_factors(n, order)
            assert np.isfinite(b).all() and (b > 0).all()


@pytest.mark.parametrize("vec", KAT["philox4x32_10"], ids=["zeros", "ones", "pi"])
def test_philox_known_answers(vec):
    key = [int(x, 16) for x in vec["key"]]
    out = O.philox(key[0], key[1], [int(x, 16) for x in vec["ctr"]])
    assert [int(x, 16) for x in vec["out"]] == out.tolist()


def test_philox_gaussian_moments():
    g = np.array([O.philox_gaussian(7, s, p, a) for s in range(20) for p in range(50) for a in range(3)])
    assert abs(g.mean()) < 0.06 and abs(g.std() - 1.0) < 0.05


def test_water_forces_match_golden_and_finite_differences():
    gold = np.load(GOLD / "water_216.npz")
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3, velocity_seed=4)
    assert np.array_equal(spec.positions, gold["positions"])
    F, E, W, T = O.forces(spec)
    assert np.allclose(F, gold["forces"], rtol=0, atol=1e-12)
    assert np.allclose(E, gold["energies"], rtol=0, atol=1e-12)
    # force = -dE/dx (central differences) for a few coordinates
    rng = np.random.default_rng(0)
    for _ in range(3):
        i, d, h = int(rng.integers(spec.n)), int(rng.integers(3)), 1e-5
        p1, p2 = spec.positions.copy(), spec.positions.copy()
        p1[i, d] += h
        p2[i, d] -= h
        fd = -(O.forces(spec, p1)[1].sum() - O.forces(spec, p2)[1].sum()) / (2 * h)
        assert abs(fd - F[i, d]) < 1e-6 * max(1.0, abs(F[i, d])) + 1e-7


def test_neighbor_rule_matches_bruteforce():
    spec = S.spc_water(64, r_cut_A=5.0, skin_A=0.5)
    x = spec.positions.astype(np.float32)
    box = spec.box.astype(np.float32)
    rs = np.float32(spec.r_cut_coul + spec.r_skin)
    pairs = O.neighbor_pairs_f32(x, box, rs)
    # independent float32 evaluation of the same rule
    d = x[:, None, :] - x[None, :, :]
    L = box[0]
    s = (d / L).astype(np.float32)
    k = np.floor((s + np.float32(0.5)).astype(np.float32)).astype(np.float32)
    d = (d - (k * L).astype(np.float32)).astype(np.float32)
    r2 = ((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]).astype(np.float32) + d[..., 2] * d[..., 2]).astype(np.float32)
    i, j = np.nonzero(np.triu(r2 <= rs * rs, 1))
    assert np.array_equal(pairs, np.stack([i, j], axis=1).astype(np.uint32))


def test_settle_projection_restores_geometry():
    spec = S.spc_water(27, r_cut_A=3.0, skin_A=0.5)
    rng = np.random.default_rng(2)
    ref = spec.positions.copy()
    pos = ref + rng.normal(scale=0.02, size=ref.shape)
    vel = np.zeros_like(pos)
    p, v, vir, used = O.constrain_positions(spec, ref, pos, vel, spec.dt)
    assert used >= 0
    for m in range(27):
        o, h1, h2 = p[3 * m], p[3 * m + 1], p[3 * m + 2]
        assert abs(np.linalg.norm(o - h1) - spec.meta["r_oh"]) < 1e-10
        assert abs(np.linalg.norm(o - h2) - spec.meta["r_oh"]) < 1e-10
        assert abs(np.linalg.norm(h1 - h2) - spec.meta["d_hh"]) < 1e-10
    # the projection preserves each molecule's centre of mass
    m3 = spec.masses.reshape(-1, 3)
    c0 = (m3[..., None] * pos.reshape(-1, 3, 3)).sum(1) / m3.sum(1)[:, None]
    c1 = (m3[..., None] * p.reshape(-1, 3, 3)).sum(1) / m3.sum(1)[:, None]
    assert np.abs(c0 - c1).max() < 1e-12
    vv, _ = O.constrain_velocities(spec, p, rng.normal(size=pos.shape), spec.dt)
    for m in range(27):
        x = p[3 * m: 3 * m + 3]
        u = vv[3 * m: 3 * m + 3]
        for a, b in ((0, 1), (0, 2), (1, 2)):
            assert abs(np.dot(x[a] - x[b], u[a] - u[b])) < 1e-10


def test_mc_scale_com_keeps_molecules_rigid():
    # kernels/mc_barostat.cu:19-74: molecule centres scale about the origin;
    # a water split across the cell boundary stays rigid, and a molecule
    # inside the cell moves by exactly (s - 1) x its centre of mass
    L = 20.0
    box = np.array([L, L, L, 0.0, 0.0, 0.0])
    s = 1.01
    box1 = box * s
    inside = np.array([[1.0, 2.0, 3.0], [2.8, 2.0, 3.0], [0.5, 3.7, 3.0]])
    split = np.array([[9.9, 0.0, 0.0], [-9.6, 0.5, 0.0], [9.2, 1.6, 0.0]])  # H1 wrapped
    pos = np.vstack([inside, split])
    m = np.array([16.0, 1.0, 1.0, 16.0, 1.0, 1.0])
    off = np.array([0, 3, 6])
    atoms = np.arange(6)
    img = np.zeros((6, 3), dtype=np.int32)
    p1, i1 = O.mc_scale_com(off, atoms, m, box, box1, s, pos, img)
    com_in = (m[:3, None] * inside).sum(0) / m[:3].sum()
    assert np.allclose(p1[:3], inside + (s - 1) * com_in, atol=1e-12)
    contig = split.copy()
    contig[1, 0] += L
    com_sp = (m[3:, None] * contig).sum(0) / m[3:].sum()
    # rigid: the contiguous image rebuilt in the new cell is the old one
    # translated, and its centre of mass scaled by s
    d = p1[3:] - p1[3]
    d -= box1[:3] * np.round(d / box1[:3])
    new_contig = p1[3] + d
    assert np.allclose(new_contig - new_contig[0], contig - contig[0], atol=1e-12)
    assert np.allclose((m[3:, None] * new_contig).sum(0) / m[3:].sum(), s * com_sp, atol=1e-12)
    # image counts keep each atom's integer offset from its molecule's
    # contiguous image: x + img L' = contiguous + (img0 + K) L', K = -1 for
    # the wrapped H
    unwrapped = p1[3:] + i1[3:] * box1[:3]
    K = np.array([[0, 0, 0], [-1, 0, 0], [0, 0, 0]])
    assert np.allclose(unwrapped, new_contig + K * box1[:3], atol=1e-12)
    # every stored atom is inside the new cell
    assert np.all(np.abs(p1) <= 0.5 * box1[:3] + 1e-12)


def test_bonded_terms_are_energy_gradients():
    # bonds, angles and dihedrals of the solvated chain, each term alone:
    # F = -dE/dx by central differences (src/forces/*: analytic derivatives)
    import dataclasses

    spec = S.peptide_in_water()
    b = spec.meta["bonded"]
    p0 = spec.positions.copy()
    p0[:166] += np.random.default_rng(3).normal(scale=0.05, size=(166, 3))  # off the minimum
    for key in ("harmonic_bond", "harmonic_angle", "periodic_dihedral"):
        sp = dataclasses.replace(spec, lj_sigma=None, alpha=None, excl_offsets=None,
                                 meta={"bonded": {key: b[key]}})
        F, _, _, T = O.forces(sp, p0)
        assert T["bonded"] > 0.0
        h = 1e-5
        for a in (0, 3, 40, 100, 165):
            for d in range(3):
                pp = p0.copy()
                pp[a, d] += h
                pm = p0.copy()
                pm[a, d] -= h
                fd = -(O.forces(sp, pp)[3]["bonded"] - O.forces(sp, pm)[3]["bonded"]) / (2 * h)
                assert abs(F[a, d] - fd) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (key, a, d)


def test_topology_exclusion_rules():
    # src/forces/topology.rs:1185-1275 on a 6-atom chain 0-1-2-3-4-5 with a
    # constraint group {4, 5}, an explicit (0, 2) entry and two dihedrals
    # sharing the 1-4 pair (0, 3)
    from heddle_b200.topology import effective_exclusions, exclusion_csr

    bonds = [(0, 1), (1, 2), (2, 3), (3, 4)]
    angles = [(0, 1, 2), (1, 2, 3), (2, 3, 4)]
    dihedrals = [(0, 1, 2, 3), (1, 2, 3, 4), (0, 1, 2, 3)]
    scales = [(0.5, 0.8), (0.4, 0.7), (0.1, 0.1)]
    eff = effective_exclusions(6, bonds, angles, dihedrals, scales, constraint_groups=[(4, 5)],
                               explicit=[(2, 0, 0.9, 0.9)])
    assert eff[(0, 2)] == (0.9, 0.9)          # explicit wins over the angle rule
    assert eff[(0, 1)] == (0.0, 0.0) and eff[(1, 3)] == (0.0, 0.0)
    assert eff[(4, 5)] == (0.0, 0.0)          # constraint group pair
    assert eff[(0, 3)] == (0.5, 0.8)          # first dihedral in sorted order wins
    assert eff[(1, 4)] == (0.4, 0.7)
    assert (0, 4) not in eff and (2, 5) not in eff
    off, part, slj, sc = exclusion_csr(6, eff)
    assert off[-1] == 2 * len(eff)
    row0 = part[off[0]:off[1]].tolist()
    assert row0 == [1, 2, 3]


def test_mlp_oracle_gradients_match_finite_differences():
    # the CPU statement of the warm-start network: without the bf16 operand
    # rounding its gradient is the exact derivative of the loss
    from oracle import mlp as M

    rng = np.random.default_rng(7)
    p = rng.normal(scale=0.3, size=M.NPARAM)
    x = rng.normal(size=(40, M.NF))
    t = rng.normal(size=40)
    g, loss = M.gradients(p, x, t, use_bf16=False)
    h = 1e-6
    for q in list(range(0, M.NPARAM, 97)) + [M.NPARAM - 1]:
        pp = p.copy()
        pp[q] += h
        pm = p.copy()
        pm[q] -= h
        fd = (M.gradients(pp, x, t, use_bf16=False)[1] - M.gradients(pm, x, t, use_bf16=False)[1]) / (2 * h)
        assert abs(g[q] - fd) <= 1e-6 * max(1.0, abs(fd)), q
    # bf16 rounding is round-to-nearest-even on the top 16 bits
    assert M.bf16(1.0 + 2.0 ** -8) == 1.0 and M.bf16(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6


def test_coupling_philox_matches_the_pinned_c_oracle():
    from oracle import coupling as OC
    rng = np.random.default_rng(5)
    for _ in range(20):
        seed = int(rng.integers(0, 2 ** 63))
        ctr = rng.integers(0, 2 ** 32, size=4, dtype=np.uint64)
        o = OC.philox(seed, *ctr)
        ref = O.philox(seed & 0xFFFFFFFF, seed >> 32, ctr.astype(np.uint32))
        assert [int(x) for x in o] == [int(x) for x in ref]
        draw = int(rng.integers(0, 2 ** 40))
        i = int(rng.integers(0, 2 ** 32))
        assert OC.normal(seed, draw, i, 2) == pytest.approx(O.philox_gaussian(seed, draw, i, 2),
                                                            rel=1e-15, abs=1e-15)


def test_csvr_chain_samples_the_canonical_kinetic_energy():
    """Iterating the CSVR map leaves K Gamma(g/2, kT)-distributed: mean
    g kT / 2 and variance g (kT)^2 / 2 (Bussi et al. 2007)."""
    from oracle import coupling as OC
    g, kt = 12, 1.0
    k, ks = 0.1, []
    for draw in range(6000):
        k = OC.csvr(k, g, kt, 1.0, 5.0, 3, draw)["k_new"]
        ks.append(k)
    ks = np.array(ks[500:])
    assert ks.mean() == pytest.approx(0.5 * g * kt, rel=0.06)
    assert ks.var() == pytest.approx(0.5 * g * kt * kt, rel=0.25)
    # no coupling (tau -> infinity): factor 1
    assert OC.csvr(3.0, g, kt, 1.0, 1e30, 3, 0)["factor"] == pytest.approx(1.0, abs=1e-12)


def test_berendsen_andersen_and_pressure_coupling_limits():
    from oracle import coupling as OC
    f, inj = OC.berendsen_thermostat(2.0, 4, 1.0, 0.1, 1.0)  # K_target = 2: no change
    assert f == 1.0 and inj == 0.0
    f, inj = OC.berendsen_thermostat(4.0, 4, 1.0, 0.1, 1.0)
    assert f * f == pytest.approx(1.0 + 0.1 * (0.5 - 1.0)) and inj == pytest.approx(4.0 * (f * f - 1.0))
    rng = np.random.default_rng(2)
    v = rng.normal(size=(2000, 3))
    inv_m = np.full(2000, 0.5)
    same, hit = OC.andersen(v, inv_m, 2.0, 0.0, 7, 3)
    assert not hit.any() and np.array_equal(same, v)
    new, hit = OC.andersen(v, inv_m, 2.0, 1.0, 7, 3)
    assert hit.all() and new.std() == pytest.approx(1.0, rel=0.05)  # sqrt(kT / m)
    part, hit = OC.andersen(v, inv_m, 2.0, 0.25, 7, 3)
    assert 0.2 < hit.mean() < 0.3 and np.array_equal(part[~hit], v[~hit])
    box = np.array([30.0, 30.0, 30.0, 0.0, 0.0, 0.0])
    # P = P0 without noise: mu = 1
    k, w = 10.0, 50.0
    p = (2 * k + w) / (3 * 27000.0)
    b = OC.pressure_coupling("berendsen", k, w, box, p, 1.0, 1.0, 10.0, 2.0, 0, 0)
    assert b["mu"] == pytest.approx(1.0, abs=1e-15)
    # higher pressure than the target expands the box
    assert OC.pressure_coupling("berendsen", k, w, box, 0.5 * p, 1.0, 1.0, 10.0, 2.0, 0, 0)["mu"] > 1.0
    # the width guard keeps mu = 1 below 2 r_search
    g = OC.pressure_coupling("berendsen", k, w, box, 100.0, 1.0, 1.0, 10.0, 2.0, 0, 0, r_search=14.99)
    assert g["mu"] == 1.0


def test_reference_pair_source_regenerates():
    """The composed LJ + erfc pair kernel of the reference is rebuilt from
    its own templates (oracle/ref_build.py) with the four entry points the
    reference's launcher binds (src/forces/jit_composed.rs:84-87)."""
    from oracle import ref_build

    if not (ref_build.DEFAULT_REF / "src/forces/jit_composed.rs").exists():
        pytest.skip("reference tree absent")
    src = ref_build.compose_pair_source(ref_build.DEFAULT_REF, True, 17.0, 17.0)
    for entry in ("heddle_jit_composed_pair_force_f(", "heddle_jit_composed_pair_force_fev(",
                  "heddle_jit_composed_pair_force_single_f(", "heddle_jit_composed_pair_force_single_fev("):
        assert src.count(entry) == 1
    assert "struct LjPairFunctor" in src and "struct SpmeRealPairFunctor" in src
    assert "/*HEDDLE_JIT_" not in src
    # the same inputs give the same text
    assert src == ref_build.compose_pair_source(ref_build.DEFAULT_REF, True, 17.0, 17.0)


def _refcuda_case(name):
    if name == "refcuda_water512":
        spec = S.spc_water(512, r_cut_A=7.0, skin_A=1.0, seed=3)
    else:
        spec = S.spc_water(1000, r_cut_A=7.0, skin_A=1.0, seed=5)
        L = spec.box[0]
        spec.box = np.array([L, L, L, 0.10 * L, -0.06 * L, 0.08 * L])
    return spec


@pytest.mark.parametrize("name", ["refcuda_water512", "refcuda_water1000_tilted"])
def test_oracle_matches_reference_cuda_outputs(name):
    """The FP64 oracle against outputs of the reference itself: HeddleMD's
    own kernels (neighbour list, composed LJ + erfc pair kernel, SPME with
    cuFFT) run on a B200 by tests/golden/make_refcuda_golden.py.  Forces
    agree within the 1e-5 RMS contract (per class too), the potential
    energy to f32 resolution, and the reference's neighbour list, cut at
    r_search, is the oracle's f32 rule pair for pair."""
    import hashlib

    g = np.load(GOLD / f"{name}.npz")
    spec = _refcuda_case(name)
    assert np.allclose(spec.box, g["box"])
    pos = g["positions"].astype(np.float64)
    Fo, _, _, T = O.forces(spec, pos)
    Fo_real, _, _, _ = O.forces(spec, pos, recip=False)
    F = g["forces"].astype(np.float64)
    norm = np.sqrt((Fo ** 2).sum())
    assert np.sqrt(((F - Fo) ** 2).sum()) / norm <= 1e-5
    assert np.sqrt(((g["forces_pair"] - Fo_real) ** 2).sum()) / norm <= 1e-5
    assert np.sqrt(((g["forces_recip"] - (Fo - Fo_real)) ** 2).sum()) / norm <= 1e-5
    pe = T["lj"] + T["coulomb_real"] + T["recip"] - T["self"]
    assert abs(g["energy"].astype(np.float64).sum() - pe) <= 1e-6 * abs(pe)
    pairs = O.neighbor_pairs_f32(g["positions"], spec.box.astype(np.float32), g["r_search"])
    assert len(pairs) == int(g["n_pairs"])
    digest = hashlib.sha256(np.ascontiguousarray(pairs, dtype=np.uint32).tobytes()).hexdigest()
    assert digest == str(g["pairs_sha256"])
