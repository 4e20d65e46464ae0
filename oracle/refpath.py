"""ctypes binding of the reference's own CUDA force path (test infrastructure).

oracle/ref_build.py compiles the reference's kernels into oracle/_ref/ and
oracle/ref_harness.cpp replays the reference's launch sequence on them; this
module feeds it a SystemSpec.  Tests use it to pin the product (and the
FP64 oracle) against the reference's own device arithmetic, and the bench
times it beside the product.  It needs a GPU and the built oracle/_ref/.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

REF = Path(__file__).resolve().parent / "_ref"
LIB = REF / "libhdref.so"

PF = C.POINTER(C.c_float)
PU = C.POINTER(C.c_uint32)
PD = C.POINTER(C.c_double)
PU64 = C.POINTER(C.c_uint64)

_lib = None

STAGES = ["eval", "clear", "tile_order", "pair", "single_pair", "finalize", "influence", "spread",
          "fft_forward", "apply_influence", "fft_inverse", "gather", "combine", "rebuild"]


def available() -> bool:
    return LIB.exists() and (REF / "neighbor.cubin").exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref is not built (python -m oracle.ref_build)")
        L = C.CDLL(str(LIB))
        L.hdref_last_error.restype = C.c_char_p
        L.hdref_init.argtypes = [C.c_char_p]
        L.hdref_ff_create.argtypes = [C.c_uint32, PF, PU, C.c_uint32, PF, PF, PF, PF, PU, PU, PF, PF,
                                      C.c_float, C.c_float, C.c_float, PU, C.c_uint32, PF, C.c_char_p,
                                      C.POINTER(C.c_void_p)]
        L.hdref_ff_set_positions.argtypes = [C.c_void_p, PF]
        L.hdref_ff_rebuild.argtypes = [C.c_void_p]
        L.hdref_ff_forces.argtypes = [C.c_void_p, C.c_int]
        L.hdref_ff_get.argtypes = [C.c_void_p, C.c_int, PF, PF, PF]
        L.hdref_ff_stats.argtypes = [C.c_void_p, PU64]
        L.hdref_ff_pairs.argtypes = [C.c_void_p, C.c_double, PU, C.c_uint64, PU64]
        L.hdref_ff_time.argtypes = [C.c_void_p, C.c_int, C.c_int, PD]
        L.hdref_ff_destroy.argtypes = [C.c_void_p]
        L.hdref_settle.argtypes = [C.c_uint32, PF, PF, PF, PF, PF, PF, PF, PF, PF, C.c_float, PF, PF]
        _check(L, L.hdref_init(str(REF).encode()))
        _lib = L
    return _lib


def _check(L, rc: int) -> None:
    if rc != 0:
        raise RuntimeError("reference path: " + L.hdref_last_error().decode())


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(PF)


def _u(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(PU)


def pair_module(spec) -> str:
    """Name of the composed pair module for this force field (built by
    oracle/ref_build.py for the water workloads)."""
    from oracle.ref_build import pair_variant_name

    live = spec.lj_epsilon != 0
    lj_c = float(np.max(spec.lj_cutoff[live]))
    sw = bool(np.any(spec.lj_switch[live] < spec.lj_cutoff[live]))
    name = pair_variant_name(sw, lj_c, spec.r_cut_coul)
    if not (REF / f"{name}.cubin").exists():
        raise RuntimeError(f"no composed pair module {name} in oracle/_ref")
    return name


class RefForceField:
    """The reference's force path (packed neighbour list, composed LJ +
    SPME-real pair kernel, SPME reciprocal with cuFFT) over one system."""

    def __init__(self, spec, positions=None, box=None, r_search=None):
        L = lib()
        self.L = L
        self.n = spec.n
        pos = spec.positions if positions is None else positions
        self.box = np.asarray(spec.box if box is None else box, dtype=np.float64)
        posq = np.zeros((spec.n, 4), dtype=np.float32)
        posq[:, :3] = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
        posq[:, 3] = spec.charges
        self._keep = []

        def f(a):
            a, p = _f(a)
            self._keep.append(a)
            return p

        def u(a):
            a, p = _u(a)
            self._keep.append(a)
            return p

        nt = spec.n_types
        rs = np.float32(r_search if r_search is not None else spec.r_cut_coul + spec.r_skin)
        self.r_search = float(rs)
        grid = np.asarray(spec.grid, dtype=np.uint32)
        h = C.c_void_p()
        _check(L, L.hdref_ff_create(
            spec.n, f(posq), u(spec.types), nt, f(spec.lj_sigma.reshape(-1)), f(spec.lj_epsilon.reshape(-1)),
            f(spec.lj_cutoff.reshape(-1)), f(spec.lj_switch.reshape(-1)), u(spec.excl_offsets),
            u(spec.excl_partners), f(spec.excl_lj), f(spec.excl_coul), C.c_float(spec.alpha),
            C.c_float(spec.r_cut_coul), C.c_float(rs), u(grid), spec.order, f(self.box),
            pair_module(spec).encode(), C.byref(h)))
        self.h = h
        self._posq = posq

    def set_positions(self, positions) -> None:
        self._posq[:, :3] = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        a, p = _f(self._posq)
        _check(self.L, self.L.hdref_ff_set_positions(self.h, p))

    def rebuild(self) -> None:
        _check(self.L, self.L.hdref_ff_rebuild(self.h))

    def evaluate(self, energies: bool = True) -> None:
        _check(self.L, self.L.hdref_ff_forces(self.h, 1 if energies else 0))

    def result(self, which: str = "total"):
        """(forces (n, 3), per-atom energy, per-atom virial) of the last
        evaluation; which = total, pair (the fast class) or recip (slow)."""
        k = {"total": 0, "pair": 1, "recip": 2}[which]
        F = np.zeros(3 * self.n, dtype=np.float32)
        E = np.zeros(self.n, dtype=np.float32)
        W = np.zeros(self.n, dtype=np.float32)
        _check(self.L, self.L.hdref_ff_get(self.h, k, F.ctypes.data_as(PF), E.ctypes.data_as(PF),
                                           W.ctypes.data_as(PF)))
        return F.reshape(-1, 3).astype(np.float64), E.astype(np.float64), W.astype(np.float64)

    def stats(self) -> dict:
        o = np.zeros(6, dtype=np.uint64)
        _check(self.L, self.L.hdref_ff_stats(self.h, o.ctypes.data_as(PU64)))
        return dict(zip(["entries", "single_pairs", "entry_capacity", "single_capacity", "blocks", "cells"],
                        (int(x) for x in o)))

    def pairs(self, r_keep: float) -> np.ndarray:
        """Deduplicated canonical pairs (i < j) of the reference's list whose
        f64 minimum-image distance is at most r_keep."""
        cnt = C.c_uint64()
        _check(self.L, self.L.hdref_ff_pairs(self.h, float(r_keep), None, 0, C.byref(cnt)))
        out = np.zeros(2 * max(cnt.value, 1), dtype=np.uint32)
        _check(self.L, self.L.hdref_ff_pairs(self.h, float(r_keep), out.ctypes.data_as(PU), cnt.value,
                                             C.byref(cnt)))
        return out[: 2 * cnt.value].reshape(-1, 2)

    def time(self, reps: int = 20, energies: bool = False) -> dict:
        """Mean device ms of one evaluation and of each stage, and of one
        neighbour rebuild."""
        ms = np.zeros(14, dtype=np.float64)
        _check(self.L, self.L.hdref_ff_time(self.h, int(reps), 1 if energies else 0, ms.ctypes.data_as(PD)))
        return dict(zip(STAGES, ms.tolist()))

    def close(self) -> None:
        if self.h:
            self.L.hdref_ff_destroy(self.h)
            self.h = None


def settle(spec, pos0, pos1, vel, dt: float, box=None):
    """The reference's SETTLE position step: snapshot pos0, constrain pos1
    (velocities corrected by the displacement / dt).  Waters only (atoms
    3g, 3g+1, 3g+2).  Returns (positions, velocities, constraint virial)."""
    L = lib()
    ng = spec.n // 3
    m = np.asarray(spec.masses).reshape(-1, 3)
    b = np.asarray(spec.box if box is None else box, dtype=np.float64)
    p0 = np.zeros((spec.n, 4), np.float32)
    p1 = np.zeros((spec.n, 4), np.float32)
    p0[:, :3] = np.asarray(pos0).reshape(-1, 3)
    p1[:, :3] = np.asarray(pos1).reshape(-1, 3)
    p0[:, 3] = p1[:, 3] = spec.charges
    v = np.ascontiguousarray(np.asarray(vel, dtype=np.float32).reshape(-1))
    out = np.zeros_like(p1)
    vir = np.zeros(spec.n, np.float32)
    keep = [_f(a) for a in (p0, p1, spec.settle_ra, spec.settle_rb, spec.settle_rc, m[:, 0], m[:, 1], b)]
    _check(L, L.hdref_settle(ng, keep[0][1], keep[1][1], v.ctypes.data_as(PF), keep[2][1], keep[3][1],
                             keep[4][1], keep[5][1], keep[6][1], keep[7][1], C.c_float(dt),
                             out.ctypes.data_as(PF), vir.ctypes.data_as(PF)))
    return out[:, :3].astype(np.float64), v.reshape(-1, 3).astype(np.float64), vir.astype(np.float64)
