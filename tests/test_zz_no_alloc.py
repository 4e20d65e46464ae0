"""The allocation-free SPME entry point (hb_spme_recip_noalloc).

Some callers cannot let this library call cudaMalloc: a process whose
device memory belongs to another allocator (a framework's caching pool, a
fixed-budget serving process) must not have memory taken behind its back,
and cudaMalloc / cudaFree would stall its device.  Those callers pass their
own input and output buffers, and the library's scratch is a fixed
file-scope device array.  Here torch plays that caller: it owns the
buffers.

Each case calls the entry point twice in a row and checks both results
against the force field's own reciprocal part (the existing entry point,
within the force tolerance of the other tests) and against the FP64
oracle's reciprocal forces and energy.  The cases cover spline orders 4, 6
and 8, a tilted cell and grids that are not powers of two.  The file is
named to run last, and works both alone and after the other tests.
"""

import ctypes as C

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import _native as N
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5


def make_case(name):
    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3)
    if name == "ortho-p4":
        pass
    elif name == "tilted-p8-20x24x18":
        lx, ly, lz = spec.box[:3]
        spec.box = np.array([lx, ly, lz, 0.12 * lx, -0.08 * lx, 0.1 * ly])
        spec.grid = (20, 24, 18)
        spec.order = 8
    elif name == "ortho-p6-32^3":
        spec.grid = (32, 32, 32)
        spec.order = 6
    return spec


@pytest.mark.parametrize("name", ["ortho-p4", "tilted-p8-20x24x18", "ortho-p6-32^3"])
def test_noalloc_recip_matches_force_field_and_oracle_twice(ctx, name):
    import torch

    spec = make_case(name)
    assert int(np.prod(spec.grid)) <= 32768 and max(spec.grid) <= 64
    sys_ = hb.System.from_spec(ctx, spec)
    full = hb.ForceField.from_spec(sys_, spec)
    full.step(scalars=True)
    f_full = sys_.forces()
    e_recip = full.scalars()["recip"]
    full.close()
    real = hb.ForceField.from_spec(sys_, spec, reciprocal=False)
    real.step(scalars=False)
    f_recip_ref = f_full - sys_.forces()
    real.close()
    pos = sys_.positions()
    sys_.close()
    # the FP64 oracle's reciprocal part at the same (f32-rounded) positions
    Fo_all, _, _, To = O.forces(spec, pos)
    Fo_real, _, _, _ = O.forces(spec, pos, recip=False)
    f_recip_oracle = Fo_all - Fo_real
    norm_total = np.sqrt((Fo_all ** 2).sum())

    posq = torch.tensor(np.concatenate([pos, spec.charges[:, None]], axis=1), dtype=torch.float32,
                        device="cuda:0").contiguous()
    lib = N.load()
    box = np.ascontiguousarray(spec.box, dtype=np.float64)
    grid = np.ascontiguousarray(spec.grid, dtype=np.uint32)
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for _ in range(2):
        out = torch.full((spec.n, 4), float("nan"), dtype=torch.float32, device="cuda:0")
        energy = C.c_double(0.0)
        N.check(lib.hb_spme_recip_noalloc(C.c_void_p(posq.data_ptr()), spec.n, N.dptr(box),
                                          N.u32ptr(grid), spec.order, float(spec.alpha),
                                          C.c_void_p(out.data_ptr()), C.byref(energy),
                                          C.c_void_p(stream)))
        torch.cuda.synchronize()
        o = out.cpu().numpy().astype(np.float64)
        results.append((o, energy.value))
    for o, e in results:
        assert np.isfinite(o).all()
        f = o[:, :3]
        # against the existing entry point (same kernels, same tolerance as
        # the force tests)
        rms = np.sqrt(((f - f_recip_ref) ** 2).sum() / (f_recip_ref ** 2).sum())
        assert rms <= FORCE_RMS_TOL, rms
        assert abs(e - e_recip) <= 1e-9 * abs(e_recip)
        # against the FP64 oracle: the reciprocal part's error measured
        # against the total force (the force contract), and on its own
        assert np.sqrt(((f - f_recip_oracle) ** 2).sum()) / norm_total <= FORCE_RMS_TOL
        assert np.sqrt(((f - f_recip_oracle) ** 2).sum() / (f_recip_oracle ** 2).sum()) <= 1e-4
        assert abs(e - To["recip"]) <= 1e-5 * abs(To["recip"])
    # the scratch keeps the last call's contents; every call clears what
    # must start at zero, so both calls agree exactly
    assert np.array_equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]


def test_noalloc_rejects_grids_beyond_its_limit():
    lib = N.load()
    box = np.array([30.0, 30.0, 30.0, 0.0, 0.0, 0.0])
    grid = np.array([64, 64, 64], dtype=np.uint32)
    rc = lib.hb_spme_recip_noalloc(None, 0, N.dptr(box), N.u32ptr(grid), 4, 0.3, None, None, None)
    assert rc == 5  # HB_ERR_INVALID_GRID
    assert b"32768" in lib.hb_last_error()
    grid = np.array([80, 16, 16], dtype=np.uint32)
    rc = lib.hb_spme_recip_noalloc(None, 0, N.dptr(box), N.u32ptr(grid), 4, 0.3, None, None, None)
    assert rc == 5
    assert b"64 points per axis" in lib.hb_last_error()
