"""Packed neighbour-list capacity behaviour on the GPU, after the reference's
tests/packed_neighbour_capacity.rs:165-230: high water grows the slabs
geometrically and reports a reallocation, the grown list is the same list,
and an overflow halts the force field with HB_ERR_NL_OVERFLOW.

The slab size is set from the host (HB_LAUNCH_NL_SLAB), which rebuilds the
list at once into slabs of that size; the fill pass never writes past a slab
(it raises the overflow bit instead), so no case here writes out of bounds.
"""

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def rms_rel(F, R):
    return float(np.sqrt(((F - R) ** 2).sum() / (R ** 2).sum()))


@pytest.fixture(scope="module")
def water():
    return S.spc_water(512, skin_A=2.0)


def oracle_pairs(spec, sys_):
    pos = sys_.positions().astype(np.float32)
    return O.neighbor_pairs_f32(pos, spec.box.astype(np.float32),
                                np.float32(spec.r_cut_coul + spec.r_skin))


def test_high_water_grows_slab_and_keeps_the_list(ctx, water):
    spec = water
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    cap0 = ff.capacity()
    mx = cap0["max_tile_entries"]
    assert cap0["slab"] >= mx and cap0["status"] & 10 == 0
    ref_pairs = oracle_pairs(spec, sys_)
    rebuilds0 = ff.stats()["rebuilds"]
    # slabs 1.2 x the fullest tile: the rebuild fits but is above 3/4 full,
    # so the library grows them (1.5 x the fullest tile + 4) and rebuilds
    tight = (6 * mx + 4) // 5
    assert 4 * mx > 3 * tight and mx <= tight
    ff.set_launch(nl_slab=tight)
    cap1 = ff.capacity()
    assert cap1["reallocations"] == cap0["reallocations"] + 2  # the tight slab, then the growth
    assert cap1["slab"] == mx + mx // 2 + 4
    assert cap1["status"] & 10 == 0
    assert ff.stats()["rebuilds"] > rebuilds0
    pairs, dups = ff.neighbor_pairs()
    assert dups == 0 and np.array_equal(pairs, ref_pairs)
    ff.step(scalars=False)
    Fo, _, _, _ = O.forces(spec, sys_.positions())
    assert rms_rel(sys_.forces(), Fo) <= 1e-5
    ff.close(), sys_.close()


def test_slab_with_headroom_reports_no_growth(ctx, water):
    spec = water
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    mx = ff.capacity()["max_tile_entries"]
    roomy = 2 * mx + 8
    ff.set_launch(nl_slab=roomy)
    cap = ff.capacity()
    assert cap["slab"] == roomy and cap["status"] & 10 == 0
    r0 = cap["reallocations"]
    ff.pre_step(force=True)
    assert ff.capacity()["reallocations"] == r0  # a rebuild that fits reuses the slabs
    ff.close(), sys_.close()


def test_overflow_halts_with_nl_overflow_until_a_larger_slab(ctx, water):
    spec = water
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    mx = ff.capacity()["max_tile_entries"]
    with pytest.raises(hb.HeddleError) as e:
        ff.set_launch(nl_slab=max(2, mx // 2))
    assert e.value.name == "HB_ERR_NL_OVERFLOW"
    assert ff.capacity()["status"] & 8
    # the overflow bit is sticky: every later call halts the same way
    with pytest.raises(hb.HeddleError) as e:
        ff.step(scalars=False)
    assert e.value.name == "HB_ERR_NL_OVERFLOW"
    # recovery (beyond the reference, which stops the run): a larger slab
    ff.set_launch(nl_slab=mx + mx // 2 + 4)
    assert ff.capacity()["status"] & 10 == 0
    ff.step(scalars=False)
    Fo, _, _, _ = O.forces(spec, sys_.positions())
    assert rms_rel(sys_.forces(), Fo) <= 1e-5
    pairs, dups = ff.neighbor_pairs()
    assert dups == 0 and np.array_equal(pairs, oracle_pairs(spec, sys_))
    ff.close(), sys_.close()


def test_tile_build_bounded_wait_times_out_and_the_next_rebuild_works(ctx, water):
    """The tile build stages candidate tiles with bulk copies completing on
    mbarriers; every wait is bounded.  With the test knob no copy is issued,
    so the first wait runs out: the kernel flags it, drains its copies and
    returns, the call reports HB_ERR_DEVICE_TIMEOUT, and once the knob is
    cleared the next rebuild gives the exact list and forces again (no GPU
    fault is involved)."""
    from heddle_b200 import _native as N

    spec = water
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=False)
    F0 = sys_.forces()
    N.check(ff.lib.hb_forcefield_set_launch(ff.h, N.HB_LAUNCH_NL_WAIT_TEST, 256))
    with pytest.raises(hb.HeddleError) as e:
        ff.pre_step(force=True)
    assert e.value.name == "HB_ERR_DEVICE_TIMEOUT"
    N.check(ff.lib.hb_forcefield_set_launch(ff.h, N.HB_LAUNCH_NL_WAIT_TEST, 0))
    ff.pre_step(force=True)
    pairs, dups = ff.neighbor_pairs()
    assert dups == 0
    assert np.array_equal(pairs, oracle_pairs(spec, sys_))
    ff.step(scalars=False)
    assert np.array_equal(sys_.forces(), F0)
    ff.close()
    sys_.close()
