"""GPU parity of the bonded terms (harmonic bonds, angles, periodic
dihedrals) and the scaled 1-4 exclusions on the solvated chain, against the
FP64 oracle."""

import dataclasses

import numpy as np
import pytest

import heddle_b200 as hb
import oracle as O
from heddle_b200 import systems as S

pytestmark = pytest.mark.gpu


def rms_rel(F, R):
    return float(np.sqrt(((F - R) ** 2).sum() / (R ** 2).sum()))


@pytest.mark.parametrize("only_bonded", [True, False], ids=["bonded", "full"])
def test_chain_forces_match_oracle(ctx, only_bonded):
    spec = S.peptide_in_water()
    rng = np.random.default_rng(4)
    spec.positions = spec.positions.copy()
    spec.positions[:166] += rng.normal(scale=0.05, size=(166, 3))  # off the ideal geometry
    if only_bonded:
        spec = dataclasses.replace(spec, lj_sigma=None, alpha=None, excl_offsets=None)
    sys_ = hb.System.from_spec(ctx, spec)
    ff = hb.ForceField.from_spec(sys_, spec)
    ff.step(scalars=True)
    pos, F, sc = sys_.positions(), sys_.forces(), ff.scalars()
    Fo, _, _, To = O.forces(spec, pos)
    if only_bonded:
        assert rms_rel(F[:166], Fo[:166]) < 1e-5
        assert np.abs(F[166:]).max() == 0.0
    else:
        assert rms_rel(F, Fo) < 1e-5
    assert abs(sc["bonded"] - To["bonded"]) <= 1e-5 * abs(To["bonded"])
    # repeat: byte-identical
    ff.step(scalars=True)
    assert np.array_equal(sys_.forces(), F)
    ff.close(), sys_.close()
