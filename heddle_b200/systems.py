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
