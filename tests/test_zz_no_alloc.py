"""The allocation-free SPME entry point (hb_spme_recip_noalloc) against the
force field's own reciprocal part.

Callers that cannot allocate device memory -- code running during CUDA
graph capture, or a process whose device memory is owned by another
allocator -- pass their own input and output buffers; the library's scratch
is a fixed file-scope device array.  Here torch plays that caller: it owns
the buffers.  The file is named to run last, and works both alone and after
the other tests.
"""

import ctypes as C

import numpy as np
import pytest

import heddle_b200 as hb
from heddle_b200 import _native as N
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def test_noalloc_recip_matches_force_field_twice(ctx):
    import torch

    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3)
    assert int(np.prod(spec.grid)) <= 32768
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
        f = o[:, :3]
        rms = np.sqrt(((f - f_recip_ref) ** 2).sum() / (f_recip_ref ** 2).sum())
        assert rms <= 1e-5, rms
        assert abs(e - e_recip) <= 1e-9 * abs(e_recip)
        assert np.isfinite(o).all()
    # the scratch keeps the last call's contents; the second call clears
    # what must start at zero, so both calls agree exactly
    assert np.array_equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]


def test_noalloc_rejects_grids_beyond_its_limit():
    lib = N.load()
    box = np.array([30.0, 30.0, 30.0, 0.0, 0.0, 0.0])
    grid = np.array([64, 64, 64], dtype=np.uint32)
    rc = lib.hb_spme_recip_noalloc(None, 0, N.dptr(box), N.u32ptr(grid), 4, 0.3, None, None, None)
    assert rc == 5  # HB_ERR_INVALID_GRID
    assert b"32768" in lib.hb_last_error()
