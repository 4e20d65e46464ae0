"""Golden vectors from the reference's own CUDA path (needs a GPU and oracle/_ref).

Runs HeddleMD's kernels (built by oracle/ref_build.py, replayed by
oracle/ref_harness.cpp) on seeded SPC water boxes and stores the inputs and
the reference's outputs, so that CPU tests can check the FP64 oracle
against the reference itself without a GPU:

  python tests/golden/make_refcuda_golden.py [OUT_DIR]

writes (by default into tests/golden/) OUT_DIR/refcuda_water512.npz (orthorhombic, r_c 7 A) and
OUT_DIR/refcuda_water1000_tilted.npz (triclinic, r_c 7 A): f32 positions and
box, reference total / pair / reciprocal forces, per-atom energies and
virials, and the reference's canonical pair list cut at r_search (stored as
its length and the SHA-256 of the sorted (i, j) uint32 array).
"""

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from heddle_b200 import systems as S  # noqa: E402
from oracle import refpath as R  # noqa: E402


def tilted(spec):
    L = spec.box[0]
    spec.box = np.array([L, L, L, 0.10 * L, -0.06 * L, 0.08 * L])
    return spec


CASES = {
    "refcuda_water512": lambda: S.spc_water(512, r_cut_A=7.0, skin_A=1.0, seed=3),
    "refcuda_water1000_tilted": lambda: tilted(S.spc_water(1000, r_cut_A=7.0, skin_A=1.0, seed=5)),
}


def wrap(pos, box):
    """Positions wrapped into the primary cell, rounded to f32."""
    lx, ly, lz, xy, xz, yz = box
    p = np.array(pos, dtype=np.float64)
    sc = np.floor(p[:, 2] / lz)
    p -= np.outer(sc, [xz, yz, lz])
    sb = np.floor(p[:, 1] / ly)
    p -= np.outer(sb, [xy, ly, 0.0])
    sa = np.floor(p[:, 0] / lx)
    p[:, 0] -= sa * lx
    return p.astype(np.float32)


def main(out_dir: str) -> None:
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    for name, make in CASES.items():
        spec = make()
        pos = wrap(spec.positions, spec.box).astype(np.float64)
        ref = R.RefForceField(spec, positions=pos)
        ref.rebuild()
        ref.evaluate(energies=True)
        F, E, W = ref.result("total")
        Fp, _, _ = ref.result("pair")
        Fr, _, _ = ref.result("recip")
        rs = ref.r_search
        cand = ref.pairs(rs * (1 + 1e-4) + 1e-6)
        st = ref.stats()
        ref.close()
        r2 = O.pair_r2_f32(pos.astype(np.float32), spec.box.astype(np.float32), cand)
        pairs = np.ascontiguousarray(cand[r2 <= np.float32(rs) * np.float32(rs)], dtype=np.uint32)
        np.savez_compressed(out / f"{name}.npz", positions=pos.astype(np.float32),
                            box=spec.box, forces=F.astype(np.float32), forces_pair=Fp.astype(np.float32),
                            forces_recip=Fr.astype(np.float32), energy=E.astype(np.float32),
                            virial=W.astype(np.float32), n_pairs=np.int64(len(pairs)),
                            pairs_sha256=np.array(hashlib.sha256(pairs.tobytes()).hexdigest()),
                            r_search=np.float32(rs),
                            entries=st["entries"], single_pairs=st["single_pairs"])
        print(name, spec.n, "atoms,", len(pairs), "pairs,", st)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent))
