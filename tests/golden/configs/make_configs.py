"""Generate the small schema-1 configuration fixtures of tests/test_io.py and
tests/test_gpu_run.py (SI units, extended XYZ, topology files):

  argon.in.toml / argon.in.xyz   256 LJ argon atoms, velocity Verlet NVE
  water.in.toml / water.in.xyz / water.in.topology
                                 216 SPC waters (SETTLE), SPME, Langevin,
                                 Monte-Carlo barostat
  argon_min.in.toml             the argon atoms (argon.in.xyz): a
                                 steepest-descent [[minimization]] phase, then
                                 a short velocity-Verlet [[phase]]
  water_cr.in.toml              the same waters (water.in.xyz / .topology),
                                 velocity Verlet + SETTLE with a CSVR
                                 thermostat and c-rescale pressure coupling
  chain.in.toml / chain.in.xyz / chain.in.topology
                                 a 14-atom bonded chain (harmonic bonds and
                                 angles, periodic dihedrals, SHAKE X-H
                                 groups) in SPC waters (216 minus the overlapping)

Run from this directory: python make_configs.py
"""

import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[2]))

from heddle_b200 import systems as S  # noqa: E402
from heddle_b200 import units as U  # noqa: E402
from heddle_b200.io import fmt_e  # noqa: E402


def write_xyz(path, species, pos_m, box_m):
    L = box_m
    with open(path, "w") as f:
        f.write(f"{len(species)}\n")
        f.write(f'Lattice="{fmt_e(L)} 0 0 0 {fmt_e(L)} 0 0 0 {fmt_e(L)}" '
                "Properties=species:S:1:pos:R:3\n")
        for s, p in zip(species, pos_m):
            f.write(f"{s} {fmt_e(p[0])} {fmt_e(p[1])} {fmt_e(p[2])}\n")


def argon():
    n_side, a = 7, 3.6e-10
    L = n_side * a
    rng = np.random.default_rng(1)
    idx = np.arange(256)
    ijk = np.stack([idx // 49, (idx // 7) % 7, idx % 7], axis=1)
    pos = (ijk + 0.5) * a - 0.5 * L + rng.uniform(-0.05 * a, 0.05 * a, size=(256, 3))
    write_xyz(HERE / "argon.in.xyz", ["Ar"] * 256, pos, L)
    (HERE / "argon.in.toml").write_text('''schema_version = 1
init = "argon.in.xyz"

[simulation]
seed = 1
temperature = 94.4

[[phase]]
name = "run"
n_steps = 100
dt = 5.0e-15

[phase.integrator]
kind = "velocity-verlet"
lossless = false

[phase.output]
trajectory_every = 20
include_velocities = true
log_every = 10

[[particle_types]]
name = "Ar"
mass = 6.6335e-26

[[pair_interactions]]
between = ["Ar", "Ar"]
potential = "lennard-jones"
sigma = 3.405e-10
epsilon = 1.654e-21
cutoff = 8.5125e-10
r_switch = 8.5125e-10

[neighbor_list]
mode = "cell-list"
r_skin = 1.0e-10
''')


WATER_TYPES = '''[[particle_types]]
name = "O"
mass = 2.6566e-26
charge = -1.3137845e-19

[[particle_types]]
name = "H"
mass = 1.6737e-27
charge = 6.5689224e-20

[[pair_interactions]]
between = ["O", "O"]
potential = "lennard-jones"
sigma = 3.166e-10
epsilon = 1.07935e-21
cutoff = 7.0e-10
r_switch = 6.3e-10

[[constraint_types]]
name = "SPC"
kind = "settle"
d_OH = 1.0e-10
d_HH = 1.633e-10

[spme]
alpha = 4.4620e9
r_cut_real = 7.0e-10
grid = [20, 20, 20]
spline_order = 4

[neighbor_list]
mode = "cell-list"
r_skin = 1.0e-10
'''


def water():
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3)
    pos = spec.positions * U.BOHR_M
    L = spec.box[0] * U.BOHR_M
    write_xyz(HERE / "water.in.xyz", ["O", "H", "H"] * 216, pos, L)
    with open(HERE / "water.in.topology", "w") as f:
        f.write("# 216 SPC waters, O at 3m\n[constraints]\n")
        for m in range(216):
            f.write(f"{3 * m} {3 * m + 1} {3 * m + 2} SPC\n")
    (HERE / "water.in.toml").write_text('''schema_version = 1
init = "water.in.xyz"
topology = "water.in.topology"

[simulation]
seed = 2
temperature = 300.0

[[phase]]
name = "npt"
n_steps = 60
dt = 2.0e-15

[phase.integrator]
kind = "langevin-baoab"
friction = 1.0e13
temperature = 300.0
seed = 5

[phase.barostat]
kind = "monte-carlo"
pressure = 1.0e5
temperature = 300.0
frequency = 10
seed = 7

[phase.output]
trajectory_every = 30
include_images = true
log_every = 10

''' + WATER_TYPES)


def argon_min():
    (HERE / "argon_min.in.toml").write_text('''schema_version = 1
init = "argon.in.xyz"

[simulation]
seed = 1
temperature = 94.4

[[minimization]]
name = "relax"

[minimization.algorithm]
kind = "steepest-descent"
force_tolerance = 1.0e-13
energy_tolerance = 1.0e-7
max_iterations = 2000

[minimization.output]
minlog_every = 5
trajectory_every = 10

[[phase]]
name = "run"
n_steps = 20
dt = 5.0e-15

[phase.integrator]
kind = "velocity-verlet"

[phase.output]
trajectory_every = 10
log_every = 10

[[particle_types]]
name = "Ar"
mass = 6.6335e-26

[[pair_interactions]]
between = ["Ar", "Ar"]
potential = "lennard-jones"
sigma = 3.405e-10
epsilon = 1.654e-21
cutoff = 8.5125e-10
r_switch = 7.5e-10

[neighbor_list]
mode = "cell-list"
r_skin = 1.0e-10
''')


def water_cr():
    (HERE / "water_cr.in.toml").write_text('''schema_version = 1
init = "water.in.xyz"
topology = "water.in.topology"

[simulation]
seed = 2
temperature = 300.0

[[phase]]
name = "npt"
n_steps = 60
dt = 2.0e-15

[phase.integrator]
kind = "velocity-verlet"
lossless = false

[phase.thermostat]
kind = "csvr"
temperature = 300.0
tau = 1.0e-13
seed = 11

[phase.barostat]
kind = "c-rescale"
pressure = 1.0e5
temperature = 300.0
tau = 1.0e-12
compressibility = 4.5e-10
seed = 13

[phase.output]
trajectory_every = 30
include_images = true
log_every = 10

''' + WATER_TYPES)


def chain():
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=4)
    Lw = spec.box[0]
    # a 4-carbon chain CH3-CH2-CH2-CH3 placed in a cavity at the origin
    r_cc, r_ch = 1.53e-10, 1.09e-10
    th = math.radians(111.0)
    c = [np.array([0.0, 0.0, 0.0]), np.array([r_cc, 0.0, 0.0])]
    c.append(c[1] + r_cc * np.array([-math.cos(th), math.sin(th), 0.0]))
    c.append(c[2] + r_cc * np.array([1.0, 0.0, 0.0]))
    c = [x - np.mean(c, axis=0) for x in c]
    atoms, species, groups = [], [], []
    for k, x in enumerate(c):
        ci = len(atoms)
        atoms.append(x)
        species.append("C")
        nh = 3 if k in (0, 3) else 2
        g = [ci]
        for h in range(nh):
            ang = 2 * math.pi * h / nh
            d = np.array([0.3 * (1 if k < 2 else -1), math.cos(ang), math.sin(ang)])
            d /= np.linalg.norm(d)
            g.append(len(atoms))
            atoms.append(x + r_ch * d)
            species.append("HC")
        groups.append(g)
    pep = np.array(atoms)
    wpos = spec.positions.reshape(-1, 3, 3) * U.BOHR_M
    keep = [m for m in range(216) if np.min(np.linalg.norm(wpos[m][0] - pep, axis=1)) > 2.8e-10]
    w = wpos[keep].reshape(-1, 3)
    pos = np.vstack([pep, w])
    species += ["O", "H", "H"] * len(keep)
    write_xyz(HERE / "chain.in.xyz", species, pos, Lw * U.BOHR_M)
    n_pep = len(pep)
    with open(HERE / "chain.in.topology", "w") as f:
        f.write("[bonds]\n")
        for k in range(3):
            f.write(f"{groups[k][0]} {groups[k + 1][0]} CC\n")
        f.write("[angles]\n")
        for k in range(1, 3):
            f.write(f"{groups[k - 1][0]} {groups[k][0]} {groups[k + 1][0]} CCC\n")
            for h in groups[k][1:]:
                f.write(f"{h} {groups[k][0]} {groups[k + 1][0]} HCC\n")
        f.write("[dihedrals]\n")
        f.write(f"{groups[0][0]} {groups[1][0]} {groups[2][0]} {groups[3][0]} X\n")
        f.write("[constraints]\n")
        for g in groups:
            f.write(" ".join(str(a) for a in g) + (" CH3\n" if len(g) == 4 else " CH2\n"))
        for m in range(len(keep)):
            o = n_pep + 3 * m
            f.write(f"{o} {o + 1} {o + 2} SPC\n")
        f.write("[charges]\n")
        for a in range(n_pep):
            q = -0.18 if species[a] == "C" else 0.06
            if a in (groups[1][0], groups[2][0]):
                q = -0.12
            f.write(f"{a} {fmt_e(q * 1.602176634e-19)}\n")
    (HERE / "chain.in.toml").write_text('''schema_version = 1
init = "chain.in.xyz"
topology = "chain.in.topology"

[simulation]
seed = 3
temperature = 300.0

[[phase]]
name = "run"
n_steps = 40
dt = 1.0e-15

[phase.integrator]
kind = "langevin-baoab"
friction = 5.0e13
temperature = 300.0
seed = 9

[phase.output]
trajectory_every = 20
log_every = 10

[[particle_types]]
name = "C"
mass = 1.9945e-26

[[particle_types]]
name = "HC"
mass = 1.6737e-27

[[pair_interactions]]
between = ["C", "C"]
potential = "lennard-jones"
sigma = 3.4e-10
epsilon = 5.98e-22
cutoff = 7.0e-10
r_switch = 6.3e-10

[[pair_interactions]]
between = ["C", "O"]
potential = "lennard-jones"
sigma = 3.28e-10
epsilon = 8.0e-22
cutoff = 7.0e-10
r_switch = 6.3e-10

[[bond_types]]
name = "CC"
potential = "harmonic"
k = 4.3e2
r0 = 1.53e-10

[[angle_types]]
name = "CCC"
potential = "harmonic"
k_theta = 7.0e-19
theta_0 = 1.937

[[angle_types]]
name = "HCC"
potential = "harmonic"
k_theta = 5.5e-19
theta_0 = 1.911

[[dihedral_types]]
name = "X"
potential = "periodic"
k_phi = 1.0e-21
n = 3
phi_0 = 0.0
scale_lj_14 = 0.5
scale_coul_14 = 0.8333333333

[[constraint_types]]
name = "CH3"
kind = "shake"
atoms = 4
constraints = [{ i = 0, j = 1, d = 1.09e-10 }, { i = 0, j = 2, d = 1.09e-10 }, { i = 0, j = 3, d = 1.09e-10 }]

[[constraint_types]]
name = "CH2"
kind = "shake"
atoms = 3
constraints = [{ i = 0, j = 1, d = 1.09e-10 }, { i = 0, j = 2, d = 1.09e-10 }]

''' + WATER_TYPES.replace('''[[constraint_types]]
name = "SPC"''', '''[[constraint_types]]
name = "SPC"''').replace('''[[pair_interactions]]
between = ["O", "O"]''', '''[[pair_interactions]]
between = ["O", "O"]'''))


if __name__ == "__main__":
    argon()
    argon_min()
    water()
    water_cr()
    chain()
