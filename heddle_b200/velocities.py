"""Maxwell-Boltzmann initial velocities, the procedure of the reference's
generate_velocities (src/runner.rs:3194-3283): ChaCha8 stream seeded from a
u64, Box-Muller per (atom, axis), centre-of-mass drift removed, one global
rescale to the exact equipartition kinetic energy with
N_dof = 3N - n_constraints - 3.

The random stream restates the published algorithms the reference pulls from
its Rust dependencies (rand_chacha 0.3.1 / rand_core 0.6.4 / rand 0.8.6):
  * seed_from_u64 fills the 32-byte key with PCG32 outputs
    (multiplier 6364136223846793005, increment 11634580027462260723,
    XSH-RR output), state advanced before each output;
  * ChaCha with 8 rounds, 64-bit block counter in words 12-13 and a zero
    64-bit stream id in words 14-15, blocks consumed in counter order;
  * next_u64 = word[k] | word[k+1] << 32;
  * a uniform f64 in [0, 1) is (u64 >> 11) * 2^-53.
No test vector of the reference pins this stream (its tests check only
determinism in the seed), so parity of the exact velocities is unpinned; the
statistical properties and exact-temperature rescale are tested.
"""

from __future__ import annotations

import numpy as np

_MASK32 = 0xFFFFFFFF


def _pcg32_seed_words(state: int) -> np.ndarray:
    mul, inc = 6364136223846793005, 11634580027462260723
    words = []
    for _ in range(8):
        state = (state * mul + inc) & 0xFFFFFFFFFFFFFFFF
        xorshifted = (((state >> 18) ^ state) >> 27) & _MASK32
        rot = state >> 59
        x = ((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & _MASK32
        words.append(x)
    return np.array(words, dtype=np.uint32)


def _rotl(x: np.ndarray, n: int) -> np.ndarray:
    return (x << np.uint32(n)) | (x >> np.uint32(32 - n))


def chacha_blocks(key: np.ndarray, first_block: int, n_blocks: int, rounds: int = 8,
                  stream: int = 0) -> np.ndarray:
    """ChaCha block function for blocks first_block .. first_block+n_blocks-1;
    returns uint32 words shaped (n_blocks, 16)."""
    ctr = np.arange(first_block, first_block + n_blocks, dtype=np.uint64)
    st = np.zeros((16, n_blocks), dtype=np.uint32)
    st[0], st[1], st[2], st[3] = 0x61707865, 0x3320646E, 0x79622D32, 0x6B206574
    for k in range(8):
        st[4 + k] = key[k]
    st[12] = (ctr & np.uint64(_MASK32)).astype(np.uint32)
    st[13] = (ctr >> np.uint64(32)).astype(np.uint32)
    st[14] = stream & _MASK32
    st[15] = (stream >> 32) & _MASK32
    x = st.copy()

    def qr(a, b, c, d):
        x[a] += x[b]; x[d] ^= x[a]; x[d] = _rotl(x[d], 16)
        x[c] += x[d]; x[b] ^= x[c]; x[b] = _rotl(x[b], 12)
        x[a] += x[b]; x[d] ^= x[a]; x[d] = _rotl(x[d], 8)
        x[c] += x[d]; x[b] ^= x[c]; x[b] = _rotl(x[b], 7)

    with np.errstate(over="ignore"):
        for _ in range(rounds // 2):
            qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
            qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
        x += st
    return x.T.copy()


class ChaCha8:
    """Sequential u64 / f64 stream of ChaCha8 seeded like seed_from_u64."""

    def __init__(self, seed: int):
        self.key = _pcg32_seed_words(seed & 0xFFFFFFFFFFFFFFFF)
        self.block = 0

    def next_u64(self, count: int) -> np.ndarray:
        n_blocks = (2 * count + 15) // 16
        words = chacha_blocks(self.key, self.block, n_blocks).reshape(-1)
        self.block += n_blocks
        words = words[: 2 * count].astype(np.uint64)
        return words[0::2] | (words[1::2] << np.uint64(32))

    def next_f64(self, count: int) -> np.ndarray:
        return (self.next_u64(count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def generate_velocities(masses: np.ndarray, temperature: float, seed: int,
                        n_constraints: int = 0) -> np.ndarray:
    """Velocities (n, 3) in atomic units; temperature is k_B T in hartree."""
    m = np.asarray(masses, dtype=np.float64)
    n = m.shape[0]
    v = np.zeros((n, 3), dtype=np.float32)
    if temperature == 0.0 or n == 0:
        return v.astype(np.float64)
    rng = ChaCha8(seed)
    # draws are consumed atom by atom, axis by axis, two per sample
    u = rng.next_f64(6 * n).reshape(n, 3, 2)
    u1 = 1.0 - u[:, :, 0]
    u2 = u[:, :, 1]
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    sigma = np.sqrt(temperature / m)
    v = (z * sigma[:, None]).astype(np.float32)
    total = m.sum()
    if total > 0.0:
        for ax in range(3):
            vcom = float(np.sum(m * v[:, ax].astype(np.float64))) / total
            v[:, ax] = (v[:, ax].astype(np.float64) - vcom).astype(np.float32)
    ndof = 3 * n - n_constraints - 3
    if ndof <= 0:
        return np.zeros((n, 3))
    ke = 0.5 * float(np.sum(m[:, None] * v.astype(np.float64) ** 2))
    if ke > 0.0:
        scale = np.sqrt(0.5 * ndof * temperature / ke)
        v = (v.astype(np.float64) * scale).astype(np.float32)
    return v.astype(np.float64)
