"""Seeded synthetic systems of the benchmark configurations (no public data
set exists for this path; these generated inputs are the workloads).

All quantities are returned in Hartree atomic units.

  lj_argon       -- LJ argon, 10,000 atoms on the first sites of a 22^3
                    simple-cubic grid with +-0.05 a jitter, box 7.84e-9 m
                    (the 1374 kg/m^3 density the configuration names),
                    r_switch = r_cut, Maxwell-Boltzmann velocities at 94.4 K;
  spc_water      -- rigid SPC water on a cubic lattice (first N sites,
                    lexicographic) with seeded uniform random orientations at
                    997 kg/m^3; LJ on O-O, erfc real space with
                    beta = erfcinv(tol) / r_cut, SPME order 4 with ~1 A grid,
                    SETTLE groups and intramolecular exclusions.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import units as U
from .velocities import generate_velocities


@dataclass
class SystemSpec:
    name: str
    positions: np.ndarray
    velocities: np.ndarray
    masses: np.ndarray
    charges: np.ndarray
    types: np.ndarray
    box: np.ndarray
    # force field
    n_types: int = 1
    lj_sigma: np.ndarray | None = None
    lj_epsilon: np.ndarray | None = None
    lj_cutoff: np.ndarray | None = None
    lj_switch: np.ndarray | None = None
    alpha: float | None = None
    r_cut_coul: float | None = None
    grid: tuple | None = None
    order: int = 4
    excl_offsets: np.ndarray | None = None
    excl_partners: np.ndarray | None = None
    excl_lj: np.ndarray | None = None
    excl_coul: np.ndarray | None = None
    r_skin: float = 0.0
    # constraints
    group_offsets: np.ndarray | None = None
    group_atoms: np.ndarray | None = None
    group_kind: np.ndarray | None = None
    settle_ra: np.ndarray | None = None
    settle_rb: np.ndarray | None = None
    settle_rc: np.ndarray | None = None
    con_offsets: np.ndarray | None = None
    con_i: np.ndarray | None = None
    con_j: np.ndarray | None = None
    con_dist: np.ndarray | None = None
    # molecules (CSR over atom ids; the barostat scales their centres)
    mol_offsets: np.ndarray | None = None
    mol_atoms: np.ndarray | None = None
    # dynamics
    dt: float = 0.0
    temperature: float = 0.0
    friction: float = 0.0
    dt_fs: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])

    @property
    def n_constraints(self) -> int:
        if self.group_kind is None:
            return 0
        n = 0
        for g, k in enumerate(self.group_kind):
            if k == 0:
                n += 3
            else:
                n += int(self.con_offsets[g + 1] - self.con_offsets[g])
        return n


def fft_friendly(n: int) -> int:
    """Smallest m >= n whose only prime factors are 2, 3 and 5."""
    m = max(int(n), 1)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def lj_argon(seed: int = 2024, n_atoms: int = 10_000, n_side: int = 22,
             box_m: float = 7.84e-9, temperature_k: float = 94.4,
             velocity_seed: int = 7, skin_frac: float = 0.3) -> SystemSpec:
    L = U.length_au(box_m)
    a = L / n_side
    rng = np.random.default_rng(seed)
    idx = np.arange(n_atoms)
    ijk = np.stack([idx // (n_side * n_side), (idx // n_side) % n_side, idx % n_side], axis=1)
    pos = (ijk + 0.5) * a - 0.5 * L + rng.uniform(-0.05 * a, 0.05 * a, size=(n_atoms, 3))
    mass = np.full(n_atoms, U.mass_au_kg(6.6335e-26))
    sigma = U.length_au(3.405e-10)
    eps = U.energy_au_j(1.654e-21)
    rc = 2.5 * sigma
    kt = U.temperature_au_k(temperature_k)
    vel = generate_velocities(mass, kt, velocity_seed, 0)
    return SystemSpec(
        name="lj-argon-10000", positions=pos, velocities=vel, masses=mass,
        charges=np.zeros(n_atoms), types=np.zeros(n_atoms, dtype=np.uint32),
        box=np.array([L, L, L, 0.0, 0.0, 0.0]), n_types=1,
        lj_sigma=np.array([[sigma]]), lj_epsilon=np.array([[eps]]),
        lj_cutoff=np.array([[rc]]), lj_switch=np.array([[rc]]),
        r_skin=skin_frac * rc, dt=U.time_au_fs(5.0), dt_fs=5.0, temperature=kt,
        meta={"sigma": sigma, "epsilon": eps, "r_cut": rc})


def ionic_lattice(n_side: int = 32, spacing_A: float = 3.3, charge: float = 0.5,
                  sigma_A: float = 3.0, eps_kj_mol: float = 0.5, mass_amu: float = 22.99,
                  r_cut_A: float = 9.0, skin_A: float = 1.0, temperature_k: float = 300.0,
                  seed: int = 3, velocity_seed: int = 13) -> SystemSpec:
    """Rock-salt ordered +q/-q Lennard-Jones ions (one type, no constraints)
    in a cubic box, with SPME at ~1 A grid spacing: an unconstrained system
    that exercises the whole force path (pair kernel + reciprocal space)
    under the plain and lossless velocity-Verlet integrators."""
    n = n_side ** 3
    a = U.angstrom_au(spacing_A)
    L = n_side * a
    rng = np.random.default_rng(seed)
    idx = np.arange(n)
    ijk = np.stack([idx // (n_side * n_side), (idx // n_side) % n_side, idx % n_side], axis=1)
    pos = (ijk + 0.5) * a - 0.5 * L + rng.uniform(-0.02 * a, 0.02 * a, size=(n, 3))
    charges = np.where(ijk.sum(1) % 2 == 0, charge, -charge).astype(np.float64)
    mass = np.full(n, U.mass_au_amu(mass_amu))
    from scipy.special import erfcinv

    rc = U.angstrom_au(r_cut_A)
    alpha = float(erfcinv(1e-5)) / rc
    kt = U.temperature_au_k(temperature_k)
    grid_n = fft_friendly(int(math.ceil(L / U.angstrom_au(1.0) - 1e-9)))
    return SystemSpec(
        name=f"ionic-lattice-{n}", positions=pos, velocities=generate_velocities(mass, kt, velocity_seed, 0),
        masses=mass, charges=charges, types=np.zeros(n, dtype=np.uint32),
        box=np.array([L, L, L, 0.0, 0.0, 0.0]), n_types=1,
        lj_sigma=np.array([[U.angstrom_au(sigma_A)]]),
        lj_epsilon=np.array([[U.energy_au_kj_per_mol(eps_kj_mol)]]),
        lj_cutoff=np.array([[rc]]), lj_switch=np.array([[rc]]),
        alpha=alpha, r_cut_coul=rc, grid=(grid_n, grid_n, grid_n), order=4,
        r_skin=U.angstrom_au(skin_A), dt=U.time_au_fs(2.0), dt_fs=2.0, temperature=kt,
        meta={"spacing_A": spacing_A})


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform rotations from uniform unit quaternions (Shoemake 1992)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q0 = np.sqrt(1 - u1) * np.sin(2 * np.pi * u2)
    q1 = np.sqrt(1 - u1) * np.cos(2 * np.pi * u2)
    q2 = np.sqrt(u1) * np.sin(2 * np.pi * u3)
    q3 = np.sqrt(u1) * np.cos(2 * np.pi * u3)
    w, x, y, z = q3, q0, q1, q2
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


SPC = {
    "q_o": -0.82, "q_h": 0.41, "r_oh_A": 1.0, "hoh_deg": 109.47,
    "sigma_A": 3.166, "eps_kj_mol": 0.650, "m_o_amu": 15.9994, "m_h_amu": 1.008,
}


def settle_geometry(r_oh: float, hoh_deg: float, m_o: float, m_h: float):
    """(ra, rb, rc) of the canonical water triangle in its centre-of-mass
    frame: O at distance ra from the COM along the bisector, the H-H
    midpoint at rb on the other side, hydrogens at +-rc across
    (src/integrator/settle.rs:83-130)."""
    half = math.radians(hoh_deg) / 2.0
    h = r_oh * math.cos(half)
    rc = r_oh * math.sin(half)
    ra = 2.0 * m_h * h / (m_o + 2.0 * m_h)
    return ra, h - ra, rc


def spc_water(n_mol: int, seed: int = 11, density: float = 997.0, r_cut_A: float = 9.0,
              ewald_tol: float = 1.0e-5, grid_spacing_A: float = 1.0, order: int = 4,
              temperature_k: float = 300.0, switch_frac: float = 0.9,
              skin_A: float | None = None, velocity_seed: int = 5,
              dt_fs: float = 2.0, friction_per_ps: float = 1.0) -> SystemSpec:
    from scipy.special import erfcinv

    m_o = U.mass_au_amu(SPC["m_o_amu"])
    m_h = U.mass_au_amu(SPC["m_h_amu"])
    m_mol_kg = (SPC["m_o_amu"] + 2 * SPC["m_h_amu"]) * U.AMU_KG
    L_m = (n_mol * m_mol_kg / density) ** (1.0 / 3.0)
    L = U.length_au(L_m)
    n_side = int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    while n_side ** 3 < n_mol:
        n_side += 1
    a = L / n_side
    idx = np.arange(n_mol)
    ijk = np.stack([idx // (n_side * n_side), (idx // n_side) % n_side, idx % n_side], axis=1)
    o_pos = (ijk + 0.5) * a - 0.5 * L
    r_oh = U.angstrom_au(SPC["r_oh_A"])
    half = math.radians(SPC["hoh_deg"]) / 2.0
    body = np.array([[0.0, 0.0, 0.0],
                     [r_oh * math.sin(half), r_oh * math.cos(half), 0.0],
                     [-r_oh * math.sin(half), r_oh * math.cos(half), 0.0]])
    rng = np.random.default_rng(seed)
    R = _random_rotations(rng, n_mol)
    atoms = o_pos[:, None, :] + np.einsum("mij,aj->mai", R, body)
    pos = atoms.reshape(-1, 3)
    n = 3 * n_mol
    masses = np.tile([m_o, m_h, m_h], n_mol)
    charges = np.tile([SPC["q_o"], SPC["q_h"], SPC["q_h"]], n_mol)
    types = np.tile(np.array([0, 1, 1], dtype=np.uint32), n_mol)
    rc = U.angstrom_au(r_cut_A)
    alpha = float(erfcinv(ewald_tol)) / rc
    sigma = U.angstrom_au(SPC["sigma_A"])
    eps = U.energy_au_kj_per_mol(SPC["eps_kj_mol"])
    lj_sigma = np.array([[sigma, 1.0], [1.0, 1.0]])
    lj_eps = np.array([[eps, 0.0], [0.0, 0.0]])
    lj_cut = np.full((2, 2), rc)
    lj_sw = np.full((2, 2), switch_frac * rc)
    grid_n = fft_friendly(int(math.ceil(L / U.angstrom_au(grid_spacing_A) - 1e-9)))
    # exclusions: the three intramolecular pairs of every water, scale 0
    base = 3 * np.arange(n_mol)
    partners = np.stack([base + 1, base + 2, base, base + 2, base, base + 1], axis=1).reshape(-1)
    excl_off = (2 * np.arange(n + 1)).astype(np.uint32)
    ra, rb, rcs = settle_geometry(r_oh, SPC["hoh_deg"], m_o, m_h)
    kt = U.temperature_au_k(temperature_k)
    vel = generate_velocities(masses, kt, velocity_seed, 3 * n_mol)
    skin = (0.3 * rc) if skin_A is None else U.angstrom_au(skin_A)
    return SystemSpec(
        name=f"spc-water-{n_mol}", positions=pos, velocities=vel, masses=masses,
        charges=charges, types=types, box=np.array([L, L, L, 0.0, 0.0, 0.0]), n_types=2,
        lj_sigma=lj_sigma, lj_epsilon=lj_eps, lj_cutoff=lj_cut, lj_switch=lj_sw,
        alpha=alpha, r_cut_coul=rc, grid=(grid_n, grid_n, grid_n), order=order,
        excl_offsets=excl_off, excl_partners=partners.astype(np.uint32),
        excl_lj=np.zeros(2 * n), excl_coul=np.zeros(2 * n), r_skin=skin,
        group_offsets=(3 * np.arange(n_mol + 1)).astype(np.uint32),
        group_atoms=np.arange(n, dtype=np.uint32),
        group_kind=np.zeros(n_mol, dtype=np.uint32),
        settle_ra=np.full(n_mol, ra), settle_rb=np.full(n_mol, rb),
        settle_rc=np.full(n_mol, rcs),
        mol_offsets=(3 * np.arange(n_mol + 1)).astype(np.uint32),
        mol_atoms=np.arange(n, dtype=np.uint32),
        dt=U.time_au_fs(dt_fs), dt_fs=dt_fs, temperature=kt,
        friction=friction_per_ps / (1.0e-12 / U.AUT_S),
        meta={"L_A": L_m / U.ANGSTROM_M, "r_oh": r_oh, "hoh_deg": SPC["hoh_deg"],
              "d_hh": 2 * rcs})


def water_shake_groups(spec: SystemSpec) -> SystemSpec:
    """The same water as SHAKE groups (O-H1, O-H2, H1-H2 distance
    constraints) instead of SETTLE."""
    n_mol = spec.n // 3
    r_oh = spec.meta["r_oh"]
    d_hh = spec.meta["d_hh"]
    spec.group_kind = np.ones(n_mol, dtype=np.uint32)
    spec.con_offsets = (3 * np.arange(n_mol + 1)).astype(np.uint32)
    spec.con_i = np.tile(np.array([0, 0, 1], dtype=np.uint32), n_mol)
    spec.con_j = np.tile(np.array([1, 2, 2], dtype=np.uint32), n_mol)
    spec.con_dist = np.tile(np.array([r_oh, r_oh, d_hh]), n_mol)
    return spec


def replica_batch(seed: int = 2025, n_boxes: int = 64, lo: int = 256, hi: int = 8192,
                  r_cut_A: float = 9.0, skin_A: float = 1.2) -> list:
    """The uneven replica batch: n_boxes SPC water boxes with N_mol drawn
    log-uniform in [lo, hi] from `seed`, each built like the 8,192-molecule
    NVT box (300 K, own seeds), grid ~1 A rounded to a 5-smooth size.  The
    skin is capped per box so that 2 (r_cut + skin) fits the box width."""
    rng = np.random.default_rng(seed)
    n_mol = np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_boxes)).astype(int)
    specs = []
    for k, nm in enumerate(n_mol):
        probe = spc_water(int(nm), seed=1000 + k, velocity_seed=2000 + k, r_cut_A=r_cut_A,
                          skin_A=skin_A)
        width_A = probe.box[0] * U.BOHR_M / U.ANGSTROM_M
        cap = 0.5 * width_A * (1.0 - 2e-4) - r_cut_A - 0.01
        if cap < skin_A:
            probe.r_skin = U.angstrom_au(max(cap, 0.2))
        specs.append(probe)
    return specs


# ---------------------------------------------------------------------------
# solvated bonded chain (the learned-SHAKE configuration)
# ---------------------------------------------------------------------------
CHAIN = {
    "r_cc_A": 1.53, "r_ch_A": 1.09, "theta_deg": 109.5,
    "k_bond_kcal": 620.0,     # U = k/2 (r - r0)^2, kcal/mol/A^2
    "k_angle_kcal": 100.0,    # U = k/2 (theta - theta0)^2, kcal/mol/rad^2
    "k_dih_kcal": 0.15, "dih_n": 3, "dih_phi0_deg": 0.0,
    "lj14": 0.5, "coul14": 1.0 / 1.2,
    "m_c_amu": 12.011, "m_h_amu": 1.008,
    "sigma_c_A": 3.4, "eps_c_kj": 0.36, "sigma_h_A": 2.5, "eps_h_kj": 0.10,
}


def _grow_chain(rng, n_heavy: int, r_cc: float, theta: float, radius: float) -> np.ndarray:
    """Heavy-atom backbone: fixed bond length and angle, dihedrals drawn from
    the staggered set, kept within a sphere and 2.8 A from earlier atoms."""
    pts = [np.zeros(3), np.array([r_cc, 0.0, 0.0])]
    a = np.array([r_cc * (1 + math.cos(math.pi - theta)), r_cc * math.sin(math.pi - theta), 0.0])
    pts.append(a)
    min_d = U.angstrom_au(2.8)
    while len(pts) < n_heavy:
        for _attempt in range(200):
            phi = rng.choice([math.pi, math.pi / 3, -math.pi / 3], p=[0.5, 0.25, 0.25])
            phi += rng.normal(scale=0.2)
            p1, p2, p3 = pts[-3], pts[-2], pts[-1]
            b = p3 - p2
            b /= np.linalg.norm(b)
            nrm = np.cross(p2 - p1, b)
            nrm /= np.linalg.norm(nrm)
            m = np.cross(nrm, b)
            d2 = np.array([-r_cc * math.cos(theta), r_cc * math.sin(theta) * math.cos(phi),
                           r_cc * math.sin(theta) * math.sin(phi)])
            new = p3 + d2[0] * b + d2[1] * m + d2[2] * nrm
            if np.linalg.norm(new) > radius:
                continue
            if len(pts) > 3 and np.min(np.linalg.norm(np.array(pts[:-2]) - new, axis=1)) < min_d:
                continue
            pts.append(new)
            break
        else:
            raise RuntimeError("chain growth failed; change the seed")
    x = np.array(pts)
    return x - x.mean(axis=0)


def peptide_in_water(seed: int = 5, n_water: int = 1900, n_heavy: int = 56, box_A: float = 38.6,
                     r_cut_A: float = 9.0, skin_A: float = 1.2, temperature_k: float = 300.0,
                     dt_fs: float = 2.0, shake_rel_tol: float = 1e-8,
                     velocity_seed: int = 9) -> SystemSpec:
    """A 166-atom bonded chain (56 carbons: CH3 ends, 50 CH2 and 4 CH in the
    middle) with harmonic C-C bonds, harmonic angles, threefold dihedrals,
    charges uniform in [-0.5, 0.5] e shifted to a zero sum, every C-H bond a
    SHAKE constraint (one group per carbon), in n_water SPC waters (SETTLE)
    in a cubic box; SPME ~1 A grid, 1-2 / 1-3 exclusions and scaled 1-4
    pairs by the reference's topology rules."""
    from scipy.special import erfcinv

    from .topology import effective_exclusions, exclusion_csr

    rng = np.random.default_rng(seed)
    C = CHAIN
    L = U.angstrom_au(box_A)
    r_cc, r_ch = U.angstrom_au(C["r_cc_A"]), U.angstrom_au(C["r_ch_A"])
    theta = math.radians(C["theta_deg"])
    heavy = _grow_chain(rng, n_heavy, r_cc, theta, radius=0.3 * L)
    # hydrogens per carbon: 3 at the ends, 1 on four evenly spaced middle
    # carbons, 2 elsewhere -> 56 + 110 = 166 atoms
    n_h = [2] * n_heavy
    n_h[0] = n_h[-1] = 3
    for k in np.linspace(8, n_heavy - 9, 4).astype(int):
        n_h[k] = 1
    pos, mass, typ, heavy_idx, groups = [], [], [], [], []
    m_c, m_h = U.mass_au_amu(C["m_c_amu"]), U.mass_au_amu(C["m_h_amu"])
    h_ang = math.radians(70.5)
    for k in range(n_heavy):
        c = heavy[k]
        ci = len(pos)
        heavy_idx.append(ci)
        pos.append(c)
        mass.append(m_c)
        typ.append(2)
        nb = [heavy[q] for q in (k - 1, k + 1) if 0 <= q < n_heavy]
        dirs = [(v - c) / np.linalg.norm(v - c) for v in nb]
        hs = []
        if len(dirs) == 1:
            ax = -dirs[0]
            e1 = np.cross(ax, [0.3, 0.5, 0.8])
            e1 /= np.linalg.norm(e1)
            e2 = np.cross(ax, e1)
            for p in range(n_h[k]):
                phi = 2 * math.pi * p / 3
                hs.append(math.cos(h_ang) * ax + math.sin(h_ang) * (math.cos(phi) * e1 + math.sin(phi) * e2))
        else:
            bis = -(dirs[0] + dirs[1])
            bis /= np.linalg.norm(bis)
            perp = np.cross(dirs[0], dirs[1])
            perp /= np.linalg.norm(perp)
            half = math.radians(54.75)
            if n_h[k] == 1:
                hs.append(bis)
            else:
                hs.append(math.cos(half) * bis + math.sin(half) * perp)
                hs.append(math.cos(half) * bis - math.sin(half) * perp)
        g = [ci]
        for h in hs:
            g.append(len(pos))
            pos.append(c + r_ch * h)
            mass.append(m_h)
            typ.append(3)
        groups.append(g)
    n_pep = len(pos)
    pos = np.array(pos)
    # charges: uniform [-0.5, 0.5], shifted to sum 0
    q = rng.uniform(-0.5, 0.5, size=n_pep)
    q -= q.mean()
    # bonded terms
    adj = {i: [] for i in range(n_pep)}
    bonds_cc = [(heavy_idx[k], heavy_idx[k + 1]) for k in range(n_heavy - 1)]
    bonds_ch = [(g[0], h) for g in groups for h in g[1:]]
    for i, j in bonds_cc + bonds_ch:
        adj[i].append(j)
        adj[j].append(i)
    angles = []
    for j in range(n_pep):
        nb = sorted(adj[j])
        for x in range(len(nb)):
            for y in range(x + 1, len(nb)):
                angles.append((nb[x], j, nb[y]))
    dihedrals = []
    for j, k in bonds_cc:
        for i in sorted(adj[j]):
            if i == k:
                continue
            for l in sorted(adj[k]):
                if l == j:
                    continue
                dihedrals.append((i, j, k, l) if i < l else (l, k, j, i))
    # waters on a lattice, avoiding the chain
    m_o, m_hw = U.mass_au_amu(SPC["m_o_amu"]), U.mass_au_amu(SPC["m_h_amu"])
    n_side = int(math.ceil((n_water * 1.15) ** (1.0 / 3.0)))
    a = L / n_side
    sites = np.array([((i + 0.5) * a - 0.5 * L, (j + 0.5) * a - 0.5 * L, (k + 0.5) * a - 0.5 * L)
                      for i in range(n_side) for j in range(n_side) for k in range(n_side)])
    dmin = np.min(np.linalg.norm(sites[:, None, :] - pos[None, :, :], axis=2), axis=1)
    free = sites[dmin > U.angstrom_au(2.6)]
    if len(free) < n_water:
        raise RuntimeError("not enough free lattice sites for the waters")
    free = free[rng.permutation(len(free))[:n_water]]
    r_oh = U.angstrom_au(SPC["r_oh_A"])
    half = math.radians(SPC["hoh_deg"]) / 2.0
    body = np.array([[0.0, 0.0, 0.0], [r_oh * math.sin(half), r_oh * math.cos(half), 0.0],
                     [-r_oh * math.sin(half), r_oh * math.cos(half), 0.0]])
    R = _random_rotations(rng, n_water)
    wpos = (free[:, None, :] + np.einsum("mij,aj->mai", R, body)).reshape(-1, 3)
    all_pos = np.vstack([pos, wpos])
    n = len(all_pos)
    masses = np.concatenate([mass, np.tile([m_o, m_hw, m_hw], n_water)])
    charges = np.concatenate([q, np.tile([SPC["q_o"], SPC["q_h"], SPC["q_h"]], n_water)])
    types = np.concatenate([typ, np.tile([0, 1, 1], n_water)]).astype(np.uint32)
    # LJ tables, Lorentz-Berthelot over (water O, water H, C, H)
    sig = np.array([SPC["sigma_A"], 1.0, C["sigma_c_A"], C["sigma_h_A"]])
    eps = np.array([SPC["eps_kj_mol"], 0.0, C["eps_c_kj"], C["eps_h_kj"]])
    S_ = U.angstrom_au(0.5 * (sig[:, None] + sig[None, :]))
    E_ = U.energy_au_kj_per_mol(np.sqrt(eps[:, None] * eps[None, :]))
    rc = U.angstrom_au(r_cut_A)
    # exclusions: chain topology rules + the water triangles
    w_groups = [[n_pep + 3 * m, n_pep + 3 * m + 1, n_pep + 3 * m + 2] for m in range(n_water)]
    scales = [(C["lj14"], C["coul14"])] * len(dihedrals)
    eff = effective_exclusions(n, bonds=bonds_cc + bonds_ch, angles=angles, dihedrals=dihedrals,
                               dihedral_scales=scales, constraint_groups=groups + w_groups)
    off, part, slj, sc = exclusion_csr(n, eff)
    kcal = U.energy_au_kj_per_mol(4.184)
    bond_k = C["k_bond_kcal"] * kcal / U.angstrom_au(1.0) ** 2
    bonded = {
        "harmonic_bond": _bonded_params("bond", np.array(bonds_cc), np.full(len(bonds_cc), bond_k),
                                        np.full(len(bonds_cc), r_cc)),
        "harmonic_angle": _bonded_params("angle", np.array(angles),
                                         np.full(len(angles), C["k_angle_kcal"] * kcal),
                                         np.full(len(angles), theta)),
        "periodic_dihedral": _bonded_params("dihedral", np.array(dihedrals),
                                            np.full(len(dihedrals), C["k_dih_kcal"] * kcal),
                                            np.full(len(dihedrals), math.radians(C["dih_phi0_deg"])),
                                            np.full(len(dihedrals), C["dih_n"], dtype=np.uint32)),
    }
    # constraints: SETTLE waters, SHAKE groups for the C-H bonds
    ra, rb, rcs = settle_geometry(r_oh, SPC["hoh_deg"], m_o, m_hw)
    g_off, g_atoms, g_kind = [0], [], []
    c_off, c_i, c_j, c_d = [0], [], [], []
    for g in groups:
        g_atoms += g
        g_off.append(len(g_atoms))
        g_kind.append(1)
        for h in range(1, len(g)):
            c_i.append(0)
            c_j.append(h)
            c_d.append(r_ch)
        c_off.append(len(c_i))
    for wg in w_groups:
        g_atoms += wg
        g_off.append(len(g_atoms))
        g_kind.append(0)
        c_off.append(len(c_i))
    n_g = len(g_kind)
    kt = U.temperature_au_k(temperature_k)
    vel = generate_velocities(masses, kt, velocity_seed, len(c_i) + 3 * n_water)
    alpha = float(erfcinv(1e-5)) / rc
    grid_n = fft_friendly(int(math.ceil(L / U.angstrom_au(1.0) - 1e-9)))
    spec = SystemSpec(
        name=f"peptide-{n_pep}-water-{n_water}", positions=all_pos, velocities=vel,
        masses=masses, charges=charges, types=types, box=np.array([L, L, L, 0.0, 0.0, 0.0]),
        n_types=4, lj_sigma=S_, lj_epsilon=E_, lj_cutoff=np.full((4, 4), rc),
        lj_switch=np.full((4, 4), 0.9 * rc), alpha=alpha, r_cut_coul=rc,
        grid=(grid_n, grid_n, grid_n), order=4, excl_offsets=off, excl_partners=part,
        excl_lj=slj, excl_coul=sc, r_skin=U.angstrom_au(skin_A),
        group_offsets=np.array(g_off, dtype=np.uint32), group_atoms=np.array(g_atoms, dtype=np.uint32),
        group_kind=np.array(g_kind, dtype=np.uint32),
        settle_ra=np.full(n_g, ra), settle_rb=np.full(n_g, rb), settle_rc=np.full(n_g, rcs),
        con_offsets=np.array(c_off, dtype=np.uint32), con_i=np.array(c_i, dtype=np.uint32),
        con_j=np.array(c_j, dtype=np.uint32), con_dist=np.array(c_d),
        mol_offsets=None, mol_atoms=None,
        dt=U.time_au_fs(dt_fs), dt_fs=dt_fs, temperature=kt,
        friction=1.0 / (1.0e-12 / U.AUT_S),
        meta={"bonded": bonded, "n_peptide": n_pep, "shake_rel_tol": shake_rel_tol,
              "r_oh": r_oh, "d_hh": 2 * rcs, "r_ch": r_ch})
    return spec


def _bonded_params(kind, atoms, k, x0, mult=None):
    from .api import HarmonicAngleParams, HarmonicBondParams, PeriodicDihedralParams

    if kind == "bond":
        return HarmonicBondParams(atoms.astype(np.uint32), k, x0)
    if kind == "angle":
        return HarmonicAngleParams(atoms.astype(np.uint32), k, x0)
    return PeriodicDihedralParams(atoms.astype(np.uint32), k, x0, mult)
