"""Host-side checks that need no GPU: the C-ABI library loads and exports
every entry point the public header declares, the ctypes layouts match the
header, velocity generation, synthetic systems, and the error path of a
GPU-less context."""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from heddle_b200 import _native as N
from heddle_b200 import systems as S
from heddle_b200 import units as U
from heddle_b200.velocities import ChaCha8, chacha_blocks, generate_velocities

from conftest import gpu_available

ROOT = Path(__file__).resolve().parents[1]
HEADER = (ROOT / "include" / "heddle_b200.h").read_text()


def declared_symbols():
    return sorted(set(re.findall(r"\b(hb_[a-z_0-9]+)\s*\(", HEADER)))


def test_library_exports_every_declared_symbol():
    lib = N.load()
    syms = declared_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(N.SIGNATURES), set(syms) ^ set(N.SIGNATURES)
    assert lib.hb_version().startswith(b"heddle_b200")


def test_struct_layouts_match_header_field_order():
    for struct, cname in ((N.SystemDesc, "hb_system_desc"), (N.ForceFieldDesc, "hb_forcefield_desc"),
                          (N.ConstraintsDesc, "hb_constraints_desc"), (N.IntegratorDesc, "hb_integrator_desc"),
                          (N.BarostatDesc, "hb_barostat_desc"), (N.ThermostatDesc, "hb_thermostat_desc"),
                          (N.PcoupleDesc, "hb_pcouple_desc"), (N.MinimizerDesc, "hb_minimizer_desc"),
                          (N.MinReport, "hb_min_report")):
        body = re.search(r"typedef struct \{([^}]*)\}\s*" + cname + ";", HEADER).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            for part in decl.split(","):
                m = re.search(r"\*?\s*([a-z_0-9]+)\s*(\[\d+\])?\s*$", part.strip())
                names.append(m.group(1))
        assert names == [f[0] for f in struct._fields_], cname


@pytest.mark.skipif(gpu_available(), reason="checks the GPU-less error path")
def test_context_without_gpu_fails_loudly():
    import heddle_b200 as hb

    with pytest.raises(hb.HeddleError) as e:
        hb.Context(0)
    assert e.value.name == "HB_ERR_CUDA"


def test_chacha_block_function_rfc7539_vector():
    # RFC 7539 section 2.3.2: the 20-round block function on the IETF layout
    key = np.frombuffer(bytes(range(32)), dtype="<u4").astype(np.uint32)
    words = chacha_blocks(key, 1, 1, rounds=20, stream=(0x4A000000 << 32) | 0x09000000)
    # counter word 13 carries the first nonce word in the IETF layout
    blk = chacha_blocks_ietf(key, 1, [0x09000000, 0x4A000000, 0x00000000])
    expect = [0xE4E7F110, 0x15593BD1, 0x1FDD0F50, 0xC47120A3, 0xC7F4D1C7, 0x0368C033, 0x9AAA2204,
              0x4E6CD4C3, 0x466482D2, 0x09AA9F07, 0x05D7C214, 0xA2028BD9, 0xD19C12B5, 0xB94E16DE,
              0xE883D0CB, 0x4E3C50A2]
    assert blk.tolist() == expect
    assert words.shape == (1, 16)


def chacha_blocks_ietf(key, counter, nonce):
    # same quarter-round core as heddle_b200.velocities with the IETF state
    # layout (32-bit counter, 96-bit nonce) used by the RFC test vector
    st = np.zeros(16, dtype=np.uint32)
    st[:4] = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574]
    st[4:12] = key
    st[12] = counter
    st[13:16] = nonce
    x = st.copy()

    def rotl(v, n):
        return np.uint32(((int(v) << n) | (int(v) >> (32 - n))) & 0xFFFFFFFF)

    def qr(a, b, c, d):
        x[a] = np.uint32((int(x[a]) + int(x[b])) & 0xFFFFFFFF); x[d] = rotl(x[d] ^ x[a], 16)
        x[c] = np.uint32((int(x[c]) + int(x[d])) & 0xFFFFFFFF); x[b] = rotl(x[b] ^ x[c], 12)
        x[a] = np.uint32((int(x[a]) + int(x[b])) & 0xFFFFFFFF); x[d] = rotl(x[d] ^ x[a], 8)
        x[c] = np.uint32((int(x[c]) + int(x[d])) & 0xFFFFFFFF); x[b] = rotl(x[b] ^ x[c], 7)

    for _ in range(10):
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
    return ((x.astype(np.uint64) + st.astype(np.uint64)) & 0xFFFFFFFF).astype(np.uint32)


def test_chacha_core_matches_ietf_reference_layout_when_nonce_is_zero():
    key = np.arange(8, dtype=np.uint32) * 0x01020304
    a = chacha_blocks(key, 5, 1, rounds=20)[0]
    b = chacha_blocks_ietf(key, 5, [0, 0, 0])
    assert a.tolist() == b.tolist()


def test_velocities_deterministic_exact_temperature_zero_momentum():
    m = np.tile([29000.0, 1837.0, 1837.0], 300)
    kt = U.temperature_au_k(300.0)
    v1 = generate_velocities(m, kt, 42, 3 * 300)
    v2 = generate_velocities(m, kt, 42, 3 * 300)
    v3 = generate_velocities(m, kt, 43, 3 * 300)
    assert np.array_equal(v1, v2) and not np.array_equal(v1, v3)
    ke = 0.5 * (m[:, None] * v1 ** 2).sum()
    ndof = 3 * len(m) - 3 * 300 - 3
    assert abs(ke / (0.5 * ndof * kt) - 1.0) < 1e-6
    p = (m[:, None] * v1).sum(0)
    assert np.abs(p).max() < 1e-6 * np.sqrt(m.sum() * kt)
    r = ChaCha8(1).next_f64(100000)
    assert 0.0 <= r.min() and r.max() < 1.0 and abs(r.mean() - 0.5) < 0.01


def test_synthetic_systems_match_their_definitions():
    w = S.spc_water(8192)
    assert w.n == 24576
    L_nm = w.box[0] * U.BOHR_M * 1e9
    assert abs(L_nm - 6.2641) < 2e-4
    assert w.grid == (64, 64, 64)
    rho = 8192 * (15.9994 + 2 * 1.008) * U.AMU_KG / (w.box[0] * U.BOHR_M) ** 3
    assert abs(rho - 997.0) < 1e-6
    beta_nm = w.alpha / (U.BOHR_M * 1e9)
    assert abs(beta_nm - 3.4705) < 1e-3
    big = S.spc_water(65536, r_cut_A=9.0)
    assert big.grid == (128, 128, 128) and abs(big.box[0] * U.BOHR_M * 1e9 - 12.528) < 1e-3
    ar = S.lj_argon()
    assert ar.n == 10000 and abs(ar.box[0] * U.BOHR_M - 7.84e-9) < 1e-20
    assert np.abs(ar.positions).max() <= 0.5 * ar.box[0]
    # SETTLE geometry reproduces the O-H and H-H distances
    ra, rb, rc = w.settle_ra[0], w.settle_rb[0], w.settle_rc[0]
    assert abs(np.sqrt(rc * rc + (ra + rb) ** 2) - w.meta["r_oh"]) < 1e-12


def test_fft_friendly_sizes():
    assert S.fft_friendly(63) == 64 and S.fft_friendly(126) == 128 and S.fft_friendly(25) == 25


def test_package_exports_every_name_the_tests_use():
    import re
    from pathlib import Path

    import heddle_b200 as hb

    root = Path(__file__).resolve().parent.parent
    names = set()
    for f in list((root / "tests").glob("*.py")) + [root / "bench.py", root / "__graft_entry__.py"]:
        names |= set(re.findall(r"\bhb\.([A-Za-z_]+)", f.read_text()))
    assert sorted(n for n in names if not hasattr(hb, n)) == []
