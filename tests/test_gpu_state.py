"""GPU checks of the state exchange (C ABI hb_system_set_state /
hb_system_get_state): positions shifted by whole lattice vectors of a
triclinic cell come back wrapped to the same place with the image counts
moved by the shift; velocities alone leave positions and images untouched; a
non-finite position is rejected and changes nothing; page-locked output
arrays are filled in place."""

import numpy as np
import pytest

import heddle_b200 as hb

pytestmark = pytest.mark.gpu

BOX = np.array([30.0, 27.0, 25.0, 4.0, -3.0, 2.5])  # lx, ly, lz, xy, xz, yz (bohr)


def lattice(box):
    lx, ly, lz, xy, xz, yz = box
    return np.array([[lx, 0.0, 0.0], [xy, ly, 0.0], [xz, yz, lz]])


def make(ctx, n=500, seed=1):
    rng = np.random.default_rng(seed)
    frac = rng.uniform(-0.5, 0.5, size=(n, 3))
    pos = frac @ lattice(BOX)
    return hb.System(ctx, pos, np.full(n, 1000.0), rng.uniform(-0.5, 0.5, n),
                     np.zeros(n, dtype=np.uint32), BOX, velocities=rng.normal(size=(n, 3)) * 1e-4)


def test_lattice_shifts_wrap_back_with_image_counts(ctx):
    sys_ = make(ctx)
    p0, v0, i0, _ = sys_.state()
    rng = np.random.default_rng(7)
    k = rng.integers(-3, 4, size=p0.shape)
    shifted = p0 + k @ lattice(BOX)
    for rep in range(2):  # twice: the staging buffers are reused
        sys_.set_state(shifted, None)
        p1, v1, i1, _ = sys_.state()
        assert np.abs(p1 - p0).max() < 1e-5
        assert np.array_equal(i1, i0 + (rep + 1) * k)  # counts carry on
        assert np.array_equal(v1, v0)
        # positions already in the cell: nothing moves, the counts stay
        sys_.set_state(p1, None)
        p2, _, i2, _ = sys_.state()
        assert np.array_equal(p2, p1) and np.array_equal(i2, i1)
    sys_.close()


def test_velocities_alone_and_rejected_positions(ctx):
    sys_ = make(ctx, seed=2)
    p0, v0, i0, f0 = sys_.state()
    v_new = np.random.default_rng(3).normal(size=v0.shape) * 1e-3
    sys_.set_state(None, v_new)
    p1, v1, i1, _ = sys_.state()
    assert np.array_equal(p1, p0) and np.array_equal(i1, i0)
    assert np.array_equal(v1, v_new.astype(np.float32).astype(np.float64))
    bad = p0.copy()
    bad[123, 1] = np.nan
    with pytest.raises(hb.HeddleError, match="non-finite position for atom 123"):
        sys_.set_state(bad, np.zeros_like(v0))
    p2, v2, i2, _ = sys_.state()
    assert np.array_equal(p2, p0) and np.array_equal(v2, v1) and np.array_equal(i2, i0)
    sys_.close()


def test_state_into_page_locked_arrays(ctx):
    import torch

    sys_ = make(ctx, seed=4)
    ref = sys_.state()
    host = tuple(torch.empty((sys_.n, 3), dtype=dt, pin_memory=True).numpy()
                 for dt in (torch.float64, torch.float64, torch.int32, torch.float64))
    out = sys_.state(out=host)
    for a, b, h in zip(out, ref, host):
        assert np.array_equal(a, b)
        assert np.shares_memory(a, h)
    with pytest.raises(ValueError):
        sys_.state(out=(host[0], host[1], host[0], host[3]))  # wrong dtype for the images
    sys_.close()


def test_single_precision_exchange(ctx):
    """hb_system_set_state_f32 / hb_system_get_state_f32: the same state as
    the FP64 exchange (the device holds f32), a round trip changes nothing,
    and a non-finite position is rejected with nothing changed."""
    sys_ = make(ctx, seed=6)
    p64, v64, i64, f64 = sys_.state()
    out = tuple(np.zeros((sys_.n, 3), dtype=dt) for dt in (np.float32, np.float32, np.int32, np.float32))
    sys_.state_f32(out)
    assert np.array_equal(out[0].astype(np.float64), p64)
    assert np.array_equal(out[1].astype(np.float64), v64)
    assert np.array_equal(out[2], i64)
    assert np.array_equal(out[3].astype(np.float64), f64)
    sys_.set_state_f32(out[0], out[1])
    p1, v1, i1, _ = sys_.state()
    assert np.array_equal(p1, p64) and np.array_equal(v1, v64) and np.array_equal(i1, i64)
    bad = out[0].copy()
    bad[7, 2] = np.inf
    with pytest.raises(hb.HeddleError, match="non-finite position for atom 7"):
        sys_.set_state_f32(bad, np.zeros_like(out[1]))
    p2, v2, i2, _ = sys_.state()
    assert np.array_equal(p2, p64) and np.array_equal(v2, v64) and np.array_equal(i2, i64)
    with pytest.raises(ValueError):
        sys_.set_state_f32(p64, None)  # float64 arrays belong to set_state
    sys_.close()
