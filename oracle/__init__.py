"""FP64 CPU oracle of HeddleMD's force-and-constraint path.

TEST INFRASTRUCTURE ONLY: the checker used by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference arm.  The product (heddle_b200) never
imports it.  The C restatement lives in oracle/heddle_oracle.c; this module
builds it on demand (oracle/Makefile) and wraps it with ctypes.
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

PD = C.POINTER(C.c_double)
PF = C.POINTER(C.c_float)
PI = C.POINTER(C.c_int32)
PU = C.POINTER(C.c_uint32)


class OrBox(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("lx", "ly", "lz", "xy", "xz", "yz")]


class OrFF(C.Structure):
    _fields_ = [
        ("lj_on", C.c_int), ("n_types", C.c_int),
        ("lj_sigma", PD), ("lj_epsilon", PD), ("lj_cutoff", PD), ("lj_switch", PD),
        ("coul_on", C.c_int), ("alpha", C.c_double), ("r_cut_coul", C.c_double),
        ("coul_poly_erfc", C.c_int),
        ("recip_on", C.c_int), ("grid", C.c_int * 3), ("order", C.c_int),
        ("excl_off", PI), ("excl_partner", PI), ("excl_lj_scale", PD), ("excl_coul_scale", PD),
        ("n_bonds", C.c_int32), ("bond_atoms", PI), ("bond_k", PD), ("bond_r0", PD),
        ("n_angles", C.c_int32), ("angle_atoms", PI), ("angle_k", PD), ("angle_theta0", PD),
        ("n_dihedrals", C.c_int32), ("dihedral_atoms", PI), ("dihedral_k", PD),
        ("dihedral_phi0", PD), ("dihedral_n", PI),
    ]


TERMS = ["lj", "coulomb_real", "recip", "self", "virial_pair", "virial_recip", "near_cut", "bonded"]

_lib = None


def build() -> Path:
    src = [HERE / "heddle_oracle.c", HERE / "heddle_oracle.h"]
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        L.or_neighbor_pairs_f32.restype = C.c_int64
        L.or_neighbor_pairs_f32.argtypes = [C.c_int32, PF, PF, C.c_float, PU, C.c_int64]
        L.or_pair_r2_f32.restype = None
        L.or_pair_r2_f32.argtypes = [C.c_int64, PU, PF, PF, PF]
        L.or_forces.restype = C.c_int
        L.or_forces.argtypes = [C.c_int32, PD, PD, PI, C.POINTER(OrBox), C.POINTER(OrFF), PD, PD, PD, PD, C.c_int]
        L.or_ewald_recip_energy.restype = C.c_double
        L.or_ewald_recip_energy.argtypes = [C.c_int32, PD, PD, C.POINTER(OrBox), C.c_double, C.c_int]
        L.or_bspline_weights.argtypes = [C.c_int, C.c_double, PD, PD]
        L.or_b_factors.argtypes = [C.c_int, C.c_int, PD]
        L.or_spme_spread.argtypes = [C.c_int32, PD, PD, C.POINTER(OrBox), C.c_int * 3, C.c_int, PD]
        L.or_constrain_positions.restype = C.c_int
        L.or_constrain_positions.argtypes = [C.c_int32, PI, PI, PI, PI, PI, PD, PD, C.POINTER(OrBox),
                                             PD, PD, PD, C.c_double, PD, C.c_double, C.c_int]
        L.or_constrain_velocities.restype = C.c_int
        L.or_constrain_velocities.argtypes = [C.c_int32, PI, PI, PI, PI, PI, PD, C.POINTER(OrBox),
                                              PD, PD, C.c_double, PD]
        L.or_philox4x32_10.argtypes = [C.c_uint32, C.c_uint32, PU, PU]
        L.or_philox_gaussian.restype = C.c_double
        L.or_philox_gaussian.argtypes = [C.c_uint32] * 6
        L.or_mc_scale_com.argtypes = [C.c_int32, PI, PI, PD, C.POINTER(OrBox), C.POINTER(OrBox), C.c_double,
                                      PD, PI]
        L.or_md_run.restype = C.c_int
        L.or_md_run.argtypes = [C.c_int32, PD, PD, PD, PD, PI, C.POINTER(OrBox), C.POINTER(OrFF),
                                C.c_int32, PI, PI, PI, PI, PI, PD, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_uint64, C.c_uint64, C.c_int, PD, C.c_int]
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(PD)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(PI)


def box_of(box) -> OrBox:
    return OrBox(*[float(x) for x in box])


class FF:
    """Force-field parameters for the oracle, built from a SystemSpec-like
    object (heddle_b200.systems.SystemSpec attributes)."""

    def __init__(self, spec, poly_erfc: bool = False, recip: bool = True):
        self.keep = []
        f = OrFF()
        if spec.lj_sigma is not None:
            f.lj_on = 1
            f.n_types = int(np.asarray(spec.lj_sigma).shape[0])
            for name, arr in (("lj_sigma", spec.lj_sigma), ("lj_epsilon", spec.lj_epsilon),
                              ("lj_cutoff", spec.lj_cutoff), ("lj_switch", spec.lj_switch)):
                a, p = _d(np.asarray(arr).reshape(-1))
                self.keep.append(a)
                setattr(f, name, p)
        if spec.alpha is not None:
            f.coul_on = 1
            f.alpha = float(spec.alpha)
            f.r_cut_coul = float(spec.r_cut_coul)
            f.coul_poly_erfc = 1 if poly_erfc else 0
            if recip and spec.grid is not None:
                f.recip_on = 1
                for k in range(3):
                    f.grid[k] = int(spec.grid[k])
                f.order = int(spec.order)
        if spec.excl_offsets is not None:
            for name, arr, conv in (("excl_off", spec.excl_offsets, _i),
                                    ("excl_partner", spec.excl_partners, _i),
                                    ("excl_lj_scale", spec.excl_lj, _d),
                                    ("excl_coul_scale", spec.excl_coul, _d)):
                a, p = conv(arr)
                self.keep.append(a)
                setattr(f, name, p)
        bonded = (getattr(spec, "meta", None) or {}).get("bonded") or {}
        for key, count, fields in (
                ("harmonic_bond", "n_bonds", (("bond_atoms", "atoms", _i), ("bond_k", "k", _d),
                                              ("bond_r0", "r0", _d))),
                ("harmonic_angle", "n_angles", (("angle_atoms", "atoms", _i), ("angle_k", "k", _d),
                                                ("angle_theta0", "theta0", _d))),
                ("periodic_dihedral", "n_dihedrals", (("dihedral_atoms", "atoms", _i),
                                                      ("dihedral_k", "k", _d),
                                                      ("dihedral_phi0", "phi0", _d),
                                                      ("dihedral_n", "n", _i)))):
            p = bonded.get(key)
            if p is None or len(p.k) == 0:
                continue
            setattr(f, count, len(p.k))
            for cname, attr, conv in fields:
                a, ptr = conv(np.asarray(getattr(p, attr)).reshape(-1))
                self.keep.append(a)
                setattr(f, cname, ptr)
        self.c = f


def forces(spec, positions=None, poly_erfc: bool = False, recip: bool = True, n_threads: int = 0):
    """F (n,3), E (n,), W (n,), terms dict at the given (default: spec) positions."""
    L = lib()
    pos = spec.positions if positions is None else positions
    n = int(np.asarray(pos).shape[0])
    p, pp = _d(np.asarray(pos).reshape(-1))
    q, qp = _d(spec.charges)
    t, tp = _i(spec.types)
    ff = FF(spec, poly_erfc, recip)
    F = np.zeros(3 * n)
    E = np.zeros(n)
    W = np.zeros(n)
    T = np.zeros(8)
    b = box_of(spec.box)
    rc = L.or_forces(n, pp, qp, tp, C.byref(b), C.byref(ff.c), F.ctypes.data_as(PD),
                     E.ctypes.data_as(PD), W.ctypes.data_as(PD), T.ctypes.data_as(PD), n_threads)
    if rc != 0:
        raise ValueError(f"or_forces failed with {rc}")
    return F.reshape(-1, 3), E, W, dict(zip(TERMS, T.tolist()))


def neighbor_pairs_f32(pos_f32: np.ndarray, box, r_search: float) -> np.ndarray:
    L = lib()
    x = np.ascontiguousarray(pos_f32, dtype=np.float32).reshape(-1)
    b = np.asarray(box, dtype=np.float32)
    n = x.shape[0] // 3
    cnt = L.or_neighbor_pairs_f32(n, x.ctypes.data_as(PF), b.ctypes.data_as(PF),
                                  C.c_float(np.float32(r_search)), None, 0)
    out = np.zeros(2 * max(cnt, 1), dtype=np.uint32)
    L.or_neighbor_pairs_f32(n, x.ctypes.data_as(PF), b.ctypes.data_as(PF),
                            C.c_float(np.float32(r_search)), out.ctypes.data_as(PU), cnt)
    return out[: 2 * cnt].reshape(-1, 2)


def pair_r2_f32(pos_f32: np.ndarray, box, pairs: np.ndarray) -> np.ndarray:
    """f32 squared minimum-image distances of the given (i, j) pairs by the
    neighbour rule of or_neighbor_pairs_f32 (kernels/pbc.cuh:18-43)."""
    x = np.ascontiguousarray(pos_f32, dtype=np.float32).reshape(-1)
    b = np.asarray(box, dtype=np.float32)
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
    out = np.zeros(p.size // 2, dtype=np.float32)
    lib().or_pair_r2_f32(p.size // 2, p.ctypes.data_as(PU), x.ctypes.data_as(PF),
                         b.ctypes.data_as(PF), out.ctypes.data_as(PF))
    return out


def ewald_recip_energy(pos, q, box, alpha: float, m_max: int = 8) -> float:
    p, pp = _d(np.asarray(pos).reshape(-1))
    qq, qp = _d(q)
    b = box_of(box)
    return lib().or_ewald_recip_energy(len(qq), pp, qp, C.byref(b), float(alpha), int(m_max))


def bspline_weights(order: int, t: float):
    w = np.zeros(order)
    dw = np.zeros(order)
    lib().or_bspline_weights(order, float(t), w.ctypes.data_as(PD), dw.ctypes.data_as(PD))
    return w, dw


def b_factors(n: int, order: int) -> np.ndarray:
    out = np.zeros(n)
    lib().or_b_factors(n, order, out.ctypes.data_as(PD))
    return out


def spme_spread(pos, q, box, grid, order: int) -> np.ndarray:
    p, pp = _d(np.asarray(pos).reshape(-1))
    qq, qp = _d(q)
    b = box_of(box)
    g = (C.c_int * 3)(*[int(x) for x in grid])
    rho = np.zeros(int(np.prod(grid)))
    lib().or_spme_spread(len(qq), pp, qp, C.byref(b), g, int(order), rho.ctypes.data_as(PD))
    return rho.reshape(tuple(int(x) for x in grid))


def _groups(spec):
    """CSR constraint groups (SETTLE groups expanded to their 3 distance
    constraints) in the oracle's int32 layout."""
    go = np.asarray(spec.group_offsets, dtype=np.int64)
    ng = len(go) - 1
    con_off = [0]
    ci, cj, cd = [], [], []
    for g in range(ng):
        if int(spec.group_kind[g]) == 0:
            ra, rb, rc = spec.settle_ra[g], spec.settle_rb[g], spec.settle_rc[g]
            d_oh2 = rc * rc + (ra + rb) ** 2
            d_hh2 = (2 * rc) ** 2
            ci += [0, 0, 1]
            cj += [1, 2, 2]
            cd += [d_oh2, d_oh2, d_hh2]
        else:
            c0, c1 = int(spec.con_offsets[g]), int(spec.con_offsets[g + 1])
            ci += [int(x) for x in spec.con_i[c0:c1]]
            cj += [int(x) for x in spec.con_j[c0:c1]]
            cd += [float(x) ** 2 for x in spec.con_dist[c0:c1]]
        con_off.append(len(ci))
    return (ng, np.asarray(go, dtype=np.int32), np.asarray(spec.group_atoms, dtype=np.int32),
            np.asarray(con_off, dtype=np.int32), np.asarray(ci, dtype=np.int32),
            np.asarray(cj, dtype=np.int32), np.asarray(cd, dtype=np.float64))


def constrain_positions(spec, ref_pos, pos, vel, dt: float, tol: float = 1e-13, max_iter: int = 10000):
    ng, go, ga, co, ci, cj, cd = _groups(spec)
    m, mp = _d(spec.masses)
    r, rp = _d(np.asarray(ref_pos).reshape(-1))
    p = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(-1)).copy()
    v = np.ascontiguousarray(np.asarray(vel, dtype=np.float64).reshape(-1)).copy()
    vir = np.zeros(len(ga))
    b = box_of(spec.box)
    used = lib().or_constrain_positions(
        ng, go.ctypes.data_as(PI), ga.ctypes.data_as(PI), co.ctypes.data_as(PI),
        ci.ctypes.data_as(PI), cj.ctypes.data_as(PI), cd.ctypes.data_as(PD), mp, C.byref(b),
        rp, p.ctypes.data_as(PD), v.ctypes.data_as(PD), float(dt), vir.ctypes.data_as(PD),
        float(tol), int(max_iter))
    return p.reshape(-1, 3), v.reshape(-1, 3), vir, used


def constrain_velocities(spec, pos, vel, dt: float):
    ng, go, ga, co, ci, cj, cd = _groups(spec)
    m, mp = _d(spec.masses)
    p, pp = _d(np.asarray(pos).reshape(-1))
    v = np.ascontiguousarray(np.asarray(vel, dtype=np.float64).reshape(-1)).copy()
    vir = np.zeros(len(ga))
    b = box_of(spec.box)
    lib().or_constrain_velocities(
        ng, go.ctypes.data_as(PI), ga.ctypes.data_as(PI), co.ctypes.data_as(PI),
        ci.ctypes.data_as(PI), cj.ctypes.data_as(PI), mp, C.byref(b), pp,
        v.ctypes.data_as(PD), float(dt), vir.ctypes.data_as(PD))
    return v.reshape(-1, 3), vir


def philox(key_lo: int, key_hi: int, ctr) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().or_philox4x32_10(key_lo, key_hi, c.ctypes.data_as(PU), o.ctypes.data_as(PU))
    return o


def philox_gaussian(seed: int, step: int, particle: int, axis: int) -> float:
    return lib().or_philox_gaussian(seed & 0xFFFFFFFF, seed >> 32, step & 0xFFFFFFFF, step >> 32,
                                    particle, axis)


def mc_scale_com(mol_offsets, mol_atoms, masses, box_old, box_new, scale: float, positions, images):
    """Monte-Carlo barostat centre-of-mass scaling (kernels/mc_barostat.cu:19-74,
    molecule translated as its contiguous image); returns (positions, images)."""
    off, po = _i(mol_offsets)
    at, pa = _i(mol_atoms)
    m, pm = _d(masses)
    pos, pp = _d(np.array(positions, dtype=np.float64).reshape(-1))
    img, pi = _i(np.array(images, dtype=np.int32).reshape(-1))
    b0 = box_of(box_old)
    b1 = box_of(box_new)
    lib().or_mc_scale_com(len(off) - 1, po, pa, pm, C.byref(b0), C.byref(b1), float(scale), pp, pi)
    return pos.reshape(-1, 3), img.reshape(-1, 3)


def md_run(spec, n_steps: int, integrator: str = "vv", positions=None, velocities=None,
           seed: int = 1, step0: int = 0, n_threads: int = 0, recip: bool = True):
    """Advance a copy of the state n_steps with the CPU driver; returns
    (positions, velocities, forces)."""
    n = spec.n
    pos = np.ascontiguousarray(np.asarray(spec.positions if positions is None else positions,
                                          dtype=np.float64).reshape(-1)).copy()
    vel = np.ascontiguousarray(np.asarray(spec.velocities if velocities is None else velocities,
                                          dtype=np.float64).reshape(-1)).copy()
    m, mp = _d(spec.masses)
    q, qp = _d(spec.charges)
    t, tp = _i(spec.types)
    ff = FF(spec, recip=recip)
    b = box_of(spec.box)
    F = np.zeros(3 * n)
    if spec.group_offsets is not None:
        ng, go, ga, co, ci, cj, cd = _groups(spec)
    else:
        ng = 0
        go = ga = co = ci = cj = np.zeros(1, dtype=np.int32)
        cd = np.zeros(1)
    rc = lib().or_md_run(
        n, pos.ctypes.data_as(PD), vel.ctypes.data_as(PD), mp, qp, tp, C.byref(b), C.byref(ff.c),
        ng, go.ctypes.data_as(PI), ga.ctypes.data_as(PI), co.ctypes.data_as(PI),
        ci.ctypes.data_as(PI), cj.ctypes.data_as(PI), cd.ctypes.data_as(PD),
        0 if integrator == "vv" else 1, float(spec.dt), float(spec.friction),
        float(spec.temperature), int(seed), int(step0), int(n_steps), F.ctypes.data_as(PD),
        int(n_threads))
    if rc != 0:
        raise ValueError(f"or_md_run failed with {rc}")
    return pos.reshape(-1, 3), vel.reshape(-1, 3), F.reshape(-1, 3)
