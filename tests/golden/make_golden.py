"""Regenerate the golden fixtures under tests/golden/.

  reference_kat.json -- the known-answer cases the reference's own tests use
      for this path, restated as data: the two- and four-charge SPME vs
      explicit-Ewald fixtures of tests/spme_pipeline.rs:101-190 (1 nm box,
      alpha 4e9 1/m, grid 16^3, orders 4-8, bound 5e-3) with their Ewald
      energies from an independent numpy evaluation below; and the published
      Philox-4x32-10 known-answer vectors (Salmon et al., Random123
      kat_vectors) for the RNG of kernels/philox.cuh.
  water_216.npz -- a 216-molecule SPC water configuration (r_cut 7 A,
      skin 1 A, grid 20^3) with its FP64 oracle forces, per-atom energies and
      energy terms, frozen so later oracle changes are caught.

Run from the repository root:  python tests/golden/make_golden.py
"""

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def ewald_numpy(pos, q, L, alpha, m_max=8):
    m = np.arange(-m_max, m_max + 1)
    ma, mb, mc = np.meshgrid(m, m, m, indexing="ij")
    mask = ~((ma == 0) & (mb == 0) & (mc == 0))
    k = 2 * np.pi * np.stack([ma[mask], mb[mask], mc[mask]], axis=1) / L
    k2 = (k * k).sum(axis=1)
    phase = k @ np.asarray(pos).T
    s = (np.asarray(q)[None, :] * np.exp(-1j * phase)).sum(axis=1)
    return float((4 * np.pi / k2 * np.exp(-k2 / (4 * alpha * alpha)) * np.abs(s) ** 2).sum() / (2 * L ** 3))


def main():
    cases = [
        {"name": "two_charge_pair", "positions": [[0.2e-9, 0.0, 0.0], [-0.2e-9, 0.0, 0.0]],
         "charges": [1.0, -1.0]},
        {"name": "four_charges", "positions": [[0.1e-9, 0.0, 0.0], [-0.1e-9, 0.2e-9, 0.0],
                                               [0.0, -0.2e-9, 0.15e-9], [-0.15e-9, 0.1e-9, -0.1e-9]],
         "charges": [1.0, -1.0, 2.0, -2.0]},
    ]
    for c in cases:
        c["box"] = 1.0e-9
        c["alpha"] = 4.0e9
        c["grid"] = [16, 16, 16]
        c["orders"] = [4, 5, 6, 7, 8]
        c["rel_bound"] = 5.0e-3
        c["ewald_energy_mmax8"] = ewald_numpy(c["positions"], c["charges"], 1.0e-9, 4.0e9)
    kat = {
        "spme_vs_ewald": cases,
        "philox4x32_10": [
            {"ctr": ["00000000"] * 4, "key": ["00000000"] * 2,
             "out": ["6627e8d5", "e169c58d", "bc57ac4c", "9b00dbd8"]},
            {"ctr": ["ffffffff"] * 4, "key": ["ffffffff"] * 2,
             "out": ["408f276d", "41c83b0e", "a20bc7c6", "6d5451fd"]},
            {"ctr": ["243f6a88", "85a308d3", "13198a2e", "03707344"], "key": ["a4093822", "299f31d0"],
             "out": ["d16cfe09", "94fdcceb", "5001e420", "24126ea1"]},
        ],
    }
    (HERE / "reference_kat.json").write_text(json.dumps(kat, indent=1) + "\n")

    import oracle as O
    from heddle_b200 import systems as S

    spec = S.spc_water(216, r_cut_A=7.0, skin_A=1.0, seed=3, velocity_seed=4)
    F, E, W, T = O.forces(spec)
    np.savez_compressed(
        HERE / "water_216.npz", positions=spec.positions, charges=spec.charges,
        box=spec.box, grid=np.array(spec.grid), alpha=spec.alpha, r_cut=spec.r_cut_coul,
        forces=F, energies=E, virials=W,
        terms=np.array([T[k] for k in ("lj", "coulomb_real", "recip", "self", "virial_pair", "virial_recip")]))
    print("wrote", HERE / "reference_kat.json", HERE / "water_216.npz")


if __name__ == "__main__":
    main()
