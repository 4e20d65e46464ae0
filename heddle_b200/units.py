"""SI <-> Hartree atomic unit conversion (CODATA 2018 values, the table of
src/units/atomic_constants.rs:11-35).  The force path works in atomic units;
conversion happens only at the configuration / file boundary."""

BOHR_M = 5.29177210903e-11          # m per bohr
ME_KG = 9.1093837015e-31            # kg per electron mass
E_C = 1.602176634e-19               # C per elementary charge
HARTREE_J = 4.359744722207101e-18   # J per hartree
AUT_S = 2.4188843265857195e-17      # s per atomic time unit
FORCE_N = 8.238723498254079e-08     # N per hartree/bohr
PRESSURE_PA = 29421015696522.1      # Pa per hartree/bohr^3
HARTREE_K = 315775.0248040668       # K per hartree (E_h / k_B)
VELOCITY_MS = 2187691.2636411153    # m/s per bohr/aut

AMU_KG = 1.66053906660e-27
AVOGADRO = 6.02214076e23
ANGSTROM_M = 1.0e-10
FS_S = 1.0e-15


def length_au(m: float) -> float:
    return m / BOHR_M


def angstrom_au(a: float) -> float:
    return a * ANGSTROM_M / BOHR_M


def mass_au_kg(kg: float) -> float:
    return kg / ME_KG


def mass_au_amu(amu: float) -> float:
    return amu * AMU_KG / ME_KG


def energy_au_j(j: float) -> float:
    return j / HARTREE_J


def energy_au_kj_per_mol(kj: float) -> float:
    return kj * 1.0e3 / AVOGADRO / HARTREE_J


def time_au_fs(fs: float) -> float:
    return fs * FS_S / AUT_S


def temperature_au_k(k: float) -> float:
    return k / HARTREE_K


def pressure_au_bar(bar: float) -> float:
    return bar * 1.0e5 / PRESSURE_PA


def ns_per_day(dt_fs: float, steps_per_s: float) -> float:
    """ns/day = dt[fs] * steps/s * 86400 s/day * 1e-6 ns/fs."""
    return dt_fs * steps_per_s * 0.0864
