"""Build recipe for the reference's own CUDA force path (test infrastructure).

HeddleMD's host is Rust and cannot be built here, but its device code can:

* the static kernels `kernels/{neighbor,spme_recip,settle,forces}.cu` compile
  from their own sources (the reference's build.rs runs `nvcc --ptx
  -std=c++17` on each, `build.rs:95-110`); here each becomes an sm_100a cubin;
* the order-specialised SPME spread / gather is `#define PME_ORDER p` in
  front of `kernels/precision.cuh`, `kernels/pbc.cuh` and
  `kernels/spme_spread_gather.cuh` (`src/forces/spme.rs:166-172`), compiled
  with `--use_fast_math` as the reference's NVRTC call does
  (`src/forces/jit_composed.rs:34-60`);
* the composed LJ + erfc pair kernel is assembled from the reference's own
  string templates -- the `PREAMBLE`, `OUTER_LOOP_TEMPLATE` and
  `SINGLE_PAIR_LOOP_TEMPLATE` constants (`src/forces/jit_composed.rs:1350-1921`),
  the Lennard-Jones functor (`src/forces/lj.rs:225-310`) and the SPME
  real-space functor (`src/forces/spme.rs:708-765`) -- read from the
  reference tree at build time, in the canonical slot order LJ, SPME-real,
  with the composite struct, the per-pair sum and the four entry points
  laid out as `compose_source` / `emit_entry_point` describe
  (`src/forces/jit_composed.rs:1076-1343`).

Everything is written to `oracle/_ref/` (git-ignored; it travels with the
built library).  `oracle/ref_harness.cpp` (own code) loads the cubins and
replays the reference's launch sequence; `oracle/refpath.py` binds it.
Nothing here is part of the product: only tests and the bench's
reference-CUDA timing use it.

  python -m oracle.ref_build [--reference /root/reference]
"""

from __future__ import annotations

import argparse
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_REF = Path("/root/reference")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
STATIC_KERNELS = ["neighbor", "spme_recip", "settle", "forces"]
SPME_ORDERS = [4, 5, 6, 7, 8]


def _nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _raw_string_after(text: str, anchor: str, nth: int = 0) -> str:
    """The body of the nth Rust raw string literal r#"..."# that follows
    `anchor` in `text`."""
    pos = text.index(anchor)
    for _ in range(nth + 1):
        start = text.index('r#"', pos) + 3
        end = text.index('"#', start)
        pos = end + 2
    return text[start:end]


def _const_raw(text: str, name: str) -> str:
    return _raw_string_after(text, f"const {name}: &str = ")


def _unformat(s: str, **subs: str) -> str:
    """Expand a Rust format! template: named {fields}, then {{ / }} escapes."""
    for k, v in subs.items():
        s = s.replace("{" + k + "}", "\x00" + k + "\x00")
    s = s.replace("{{", "{").replace("}}", "}")
    for k, v in subs.items():
        s = s.replace("\x00" + k + "\x00", v)
    return s


# Kernel argument schemas of the two pair fragments, as declared by
# lj_arg_schema (src/forces/lj.rs:135-150) and spme_real_arg_schema
# (src/forces/spme.rs:691-704): (kernel parameter, C type, functor field).
LJ_ARGS = [("lj_n_types", "unsigned int ", "n_types"),
           ("lj_type_sigma", "const Real *", "type_sigma"),
           ("lj_type_epsilon", "const Real *", "type_epsilon"),
           ("lj_type_cutoff", "const Real *", "type_cutoff"),
           ("lj_type_switch", "const Real *", "type_switch"),
           ("lj_excl_offsets", "const unsigned int *", "excl_offsets"),
           ("lj_excl_partners", "const unsigned int *", "excl_partners"),
           ("lj_excl_scales", "const Real *", "excl_scales")]
SPME_ARGS = [("spme_real_k_coulomb", "Real ", "k_coulomb"),
             ("spme_real_alpha", "Real ", "alpha"),
             ("spme_real_r_cut", "Real ", "r_cut_real"),
             ("spme_real_excl_offsets", "const unsigned int *", "excl_offsets"),
             ("spme_real_excl_partners", "const unsigned int *", "excl_partners"),
             ("spme_real_excl_scales", "const Real *", "excl_scales")]


def compose_pair_source(ref: Path, lj_switch: bool, lj_cutoff: float, coul_cutoff: float) -> str:
    """The composed pair-force translation unit for the fragment set
    (lennard_jones, spme_real), both with uniform cut-offs."""
    import numpy as np

    jc = (ref / "src/forces/jit_composed.rs").read_text()
    lj = (ref / "src/forces/lj.rs").read_text()
    sp = (ref / "src/forces/spme.rs").read_text()
    preamble = _const_raw(jc, "PREAMBLE")
    outer = _const_raw(jc, "OUTER_LOOP_TEMPLATE")
    single = _const_raw(jc, "SINGLE_PAIR_LOOP_TEMPLATE")
    body = _raw_string_after(lj, "let evaluate_body = if switch_degenerate {", 1 if lj_switch else 0)
    lj_functor = _unformat(_raw_string_after(lj, "let functor_source = format!("), eval_body=body)
    sp_functor = _raw_string_after(sp, "pub fn spme_real_pair_force_fragment(")
    # the cut-offs are f32 values printed as f64 (jit_composed.rs:1088-1098)
    lj_c = float(np.float32(lj_cutoff))
    co_c = float(np.float32(coul_cutoff))
    max_c = max(lj_c, co_c)
    frags = [("functor_lennard_jones", "LjPairFunctor", lj_functor, LJ_ARGS, lj_c),
             ("functor_spme_real", "SpmeRealPairFunctor", sp_functor, SPME_ARGS, co_c)]
    out = [preamble,
           "\n#define HEDDLE_JIT_MAX_CUTOFF R(%.17e)\n\n" % max_c,
           "\n#define HEDDLE_JIT_MAX_CUTOFF_SQUARED R(%.17e)\n\n" % (max_c * max_c)]
    for field, _, src, _, _ in frags:
        out.append(f"// fragment: {field}\n{src}\n")
    out.append("\nstruct HeddleJitComposedPairFunc {\n")
    out += [f"    {struct} {field};\n" for field, struct, _, _, _ in frags]
    out.append("};\n")
    # per-pair sum over the fragments in canonical order, each scaled by its
    # own exclusion factor; a fragment whose uniform cut-off is below the
    # outer maximum gets a constant guard
    out.append("\ntemplate <bool WriteEv>\n__device__ static inline void heddle_jit_eval_pair_sum(\n"
               "    const HeddleJitComposedPairFunc &composite,\n"
               "    Real r2, Real inv_r, Real r, Real qi, Real qj, unsigned int i_type, "
               "unsigned int j_type, unsigned int i, unsigned int j,\n"
               "    Real &factor, Real &energy, Real &virial)\n{\n"
               "    factor = R(0.0); energy = R(0.0); virial = R(0.0);\n")
    for field, _, _, _, cut in frags:
        term = (f"Real s_factor, s_energy, s_virial;\n"
                f"        composite.{field}.evaluate(r2, inv_r, r, qi, qj, i_type, j_type, i, j, "
                f"s_factor, s_energy, s_virial);\n"
                f"        Real ex_scale = composite.{field}.exclusion_scale(i, j);\n"
                f"        factor += s_factor * ex_scale;\n"
                f"        if (WriteEv) {{ energy += s_energy * ex_scale; virial += s_virial * ex_scale; }}")
        if cut == max_c:
            out.append(f"    {{\n        {term}\n    }}\n")
        else:
            out.append(f"    {{\n        if (r2 <= R({cut * cut:.17e})) {{\n        {term}\n        }}\n    }}\n")
    out.append("}\n")
    out.append(outer)
    out.append(single)

    def entry(name: str, ev: bool, single_pair: bool) -> str:
        s = []
        if single_pair:
            s.append(f'\nextern "C" __global__ void {name}(\n')
            common = ["const Real4 *posq", "const unsigned int *type_indices",
                      "const unsigned int *single_pair_atoms",
                      "const unsigned int *interaction_count_ptr", "const Real *lattice"]
        else:
            # 256 threads, at least 4 resident blocks (jit_composed.rs:88-102)
            s.append(f'\nextern "C" __global__ void __launch_bounds__(256, 4) {name}(\n')
            common = ["const Real4 *posq", "const unsigned int *type_indices",
                      "const Real4 *tile_sorted_posq", "const Real *block_centre",
                      "const Real *block_bbox", "const unsigned int *sorted_particle_ids",
                      "const unsigned int *iblock_offset",
                      "const unsigned int *sorted_interacting_atoms", "unsigned int n_iblocks",
                      "const Real *lattice"]
        common += [f"unsigned long long *fast_{k}_fp" for k in
                   ("force_x", "force_y", "force_z", "energy", "virial")]
        s += [f"    {c},\n" for c in common]
        for field, _, _, args, _ in frags:
            s += [f"    {ty}{nm},\n" for nm, ty, _ in args]
        s.append("    unsigned int n)\n{\n    HeddleJitComposedPairFunc composite;\n")
        for field, _, _, args, _ in frags:
            s += [f"    composite.{field}.{fld} = {nm};\n" for nm, _, fld in args]
        flag = "true" if ev else "false"
        if single_pair:
            s.append(f"    heddle_jit_single_pair_loop<{flag}>(\n"
                     "        composite, single_pair_atoms, interaction_count_ptr, posq, type_indices, lattice,\n"
                     "        fast_force_x_fp, fast_force_y_fp, fast_force_z_fp, fast_energy_fp, "
                     "fast_virial_fp, n);\n}\n")
        else:
            s.append(f"    heddle_jit_outer_loop<{flag}>(\n"
                     "        composite, iblock_offset, n_iblocks, posq, type_indices, tile_sorted_posq,\n"
                     "        block_centre, block_bbox, sorted_particle_ids, sorted_interacting_atoms, lattice,\n"
                     "        fast_force_x_fp, fast_force_y_fp, fast_force_z_fp, fast_energy_fp, "
                     "fast_virial_fp, n);\n}\n")
        return "".join(s)

    out.append(entry("heddle_jit_composed_pair_force_f", False, False))
    out.append(entry("heddle_jit_composed_pair_force_fev", True, False))
    out.append(entry("heddle_jit_composed_pair_force_single_f", False, True))
    out.append(entry("heddle_jit_composed_pair_force_single_fev", True, True))
    src = "".join(out)
    # LJ consumes the per-atom type index, so the loop templates' type-load
    # markers become loads (jit_composed.rs:1217-1241)
    src = (src.replace("/*HEDDLE_JIT_ITYPE_LOAD*/", "i_type = i_valid ? type_indices[i_atom_id] : 0u;")
              .replace("/*HEDDLE_JIT_JTYPE_LOAD*/", "j_type = j_valid ? type_indices[j_atom_id] : 0u;")
              .replace("/*HEDDLE_JIT_JTYPE_SHUFFLE*/", "j_type = __shfl_sync(0xFFFFFFFFu, j_type, src_lane);")
              .replace("/*HEDDLE_JIT_TYPE_LOAD_PERPAIR*/",
                       "i_type = type_indices[atom_i]; j_type = type_indices[atom_j];"))
    return src


def pair_variant_name(lj_switch: bool, lj_cutoff: float, coul_cutoff: float) -> str:
    import numpy as np

    a = np.float32(lj_cutoff).view(np.uint32)
    b = np.float32(coul_cutoff).view(np.uint32)
    return f"pair_sw{int(lj_switch)}_{int(a):08x}_{int(b):08x}"


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build_pair_variant(ref: Path, lj_switch: bool, lj_cutoff: float, coul_cutoff: float) -> Path:
    OUT.mkdir(exist_ok=True)
    name = pair_variant_name(lj_switch, lj_cutoff, coul_cutoff)
    cubin = OUT / f"{name}.cubin"
    if cubin.exists():
        return cubin
    src = OUT / f"{name}.cu"
    src.write_text(compose_pair_source(ref, lj_switch, lj_cutoff, coul_cutoff))
    _run([_nvcc(), "-cubin", *ARCH, "-std=c++17", "--use_fast_math", "-o", str(cubin), str(src)])
    return cubin


def pair_variants() -> list[tuple[bool, float, float]]:
    """(LJ switch, LJ cut-off, Coulomb cut-off) of the workloads the tests and
    the bench compare: SPC water at r_c = 7 and 9 A with the LJ switch at
    0.9 r_c (bohr)."""
    sys.path.insert(0, str(HERE.parent))
    from heddle_b200 import units as U

    return [(True, U.angstrom_au(r), U.angstrom_au(r)) for r in (7.0, 9.0)]


def build(ref: Path = DEFAULT_REF, verbose: bool = False) -> bool:
    """Compile everything into oracle/_ref; False when the reference tree is absent."""
    if not (ref / "kernels" / "neighbor.cu").exists():
        return False
    OUT.mkdir(exist_ok=True)
    kdir = ref / "kernels"
    nvcc = _nvcc()
    for k in STATIC_KERNELS:
        cubin = OUT / f"{k}.cubin"
        if not cubin.exists():
            if verbose:
                print("nvcc", k)
            _run([nvcc, "-cubin", *ARCH, "-std=c++17", "-I", str(kdir), "-o", str(cubin),
                  str(kdir / f"{k}.cu")])
    for p in SPME_ORDERS:
        cubin = OUT / f"spme_sg_p{p}.cubin"
        if not cubin.exists():
            if verbose:
                print("nvcc spread/gather p", p)
            _run([nvcc, "-cubin", *ARCH, "-std=c++17", "--use_fast_math", f"-DPME_ORDER={p}",
                  "-I", str(kdir), "-include", str(kdir / "precision.cuh"), "-include",
                  str(kdir / "pbc.cuh"), "-x", "cu", "-o", str(cubin),
                  str(kdir / "spme_spread_gather.cuh")])
    for sw, a, b in pair_variants():
        build_pair_variant(ref, sw, a, b)
    lib = OUT / "libhdref.so"
    src = HERE / "ref_harness.cpp"
    if not lib.exists() or src.stat().st_mtime > lib.stat().st_mtime:
        cuda = Path(nvcc).resolve().parent.parent
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(cuda / "include"),
              "-o", str(lib), str(src), "-L", str(cuda / "lib64"), "-L", str(cuda / "lib64/stubs"),
              "-lcudart", "-lcuda", "-lcufft", f"-Wl,-rpath,{cuda / 'lib64'}"])
    return True


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(DEFAULT_REF))
    a = ap.parse_args()
    ok = build(Path(a.reference), verbose=True)
    print("built" if ok else "reference tree not found; nothing built")
    return 0


if __name__ == "__main__":
    sys.exit(main())
