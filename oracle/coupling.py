"""CPU restatement of the thermostats and per-step pressure couplings (test
infrastructure only: the checker of heddle_b200's hb_couple.cu kernels).

Follows the reference's device formulas in FP64:
  * Philox-4x32-10 (Salmon et al., SC11) as kernels/philox.cuh:21-55,
    vectorised over the third counter word;
  * normals by the Box-Muller cosine branch on u = (x + 1/2) 2^-32
    (philox_gaussian_f64, kernels/philox.cuh:135-155);
  * CSVR: csvr_sample_and_factor (kernels/nose_hoover.cu:145-255), the sum of
    squares over counters (draw, 0, i, 0), i = 1 .. g-1, r at i = 0;
  * Berendsen: berendsen_compute_factor (kernels/nose_hoover.cu:390-415);
  * Andersen: andersen_resample (kernels/andersen.cu), Bernoulli on counter
    (draw, 0, id, 3), velocities on (draw, 0, id, 0..2);
  * c-rescale / Berendsen barostat: c_rescale_compute_mu /
    berendsen_compute_mu (kernels/barostat.cu:140-255), with the box-width
    guard of the engine (a step that would take the narrowest perpendicular
    width below 2 r_search keeps mu = 1).
"""

from __future__ import annotations

import math

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox(seed: int, c0, c1, c2, c3):
    """Philox-4x32-10 of key (seed lo, seed hi) on counters (c0, c1, c2, c3)
    (numpy arrays broadcast together); returns the four output words."""
    k0 = np.uint64(seed & MASK)
    k1 = np.uint64((seed >> 32) & MASK)
    c = [np.asarray(x, dtype=np.uint64) & np.uint64(MASK) for x in np.broadcast_arrays(c0, c1, c2, c3)]
    for _ in range(10):
        p0 = c[0] * np.uint64(M0)
        p2 = c[2] * np.uint64(M1)
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(MASK)
        hi2, lo2 = p2 >> np.uint64(32), p2 & np.uint64(MASK)
        c = [hi2 ^ c[1] ^ k0, lo2, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(W0)) & np.uint64(MASK)
        k1 = (k1 + np.uint64(W1)) & np.uint64(MASK)
    return c


def uniform(x) -> np.ndarray:
    return (np.asarray(x, dtype=np.float64) + 0.5) * (1.0 / 4294967296.0)


def normal(seed: int, draw: int, idx, axis: int = 0) -> np.ndarray:
    """Standard normals for counters (draw lo, draw hi, idx, axis)."""
    o = philox(seed, draw & MASK, draw >> 32, np.asarray(idx, dtype=np.uint64), axis)
    u1, u2 = uniform(o[0]), uniform(o[1])
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)


def csvr(k: float, g: int, kt: float, dt: float, tau: float, seed: int, draw: int) -> dict:
    """CSVR chain for kinetic energy k with g degrees of freedom."""
    c = math.exp(-dt / tau)
    xi = normal(seed, draw, np.arange(1, max(g, 1), dtype=np.uint64))
    s = float(np.sum(xi * xi))
    r = float(normal(seed, draw, 0))
    kt_half = 0.5 * kt
    cross = 2.0 * r * math.sqrt(c * (1.0 - c) * k * kt_half) if k > 0.0 else 0.0
    kn = c * k + kt_half * (1.0 - c) * (s + r * r) + cross
    if not math.isfinite(kn) or kn <= 0.0:
        kn = k
    f = math.sqrt(kn / k) if (k > 0.0 and kn != k) else 1.0
    return {"factor": f, "k_new": kn, "s": s, "r": r}


def berendsen_thermostat(k: float, g: int, kt: float, dt: float, tau: float):
    """(factor, injected energy) of one Berendsen thermostat step."""
    if not k > 0.0:
        return 1.0, 0.0
    lam2 = 1.0 + dt / tau * (0.5 * g * kt / k - 1.0)
    lam2 = max(lam2, 0.0)
    return math.sqrt(lam2), k * (lam2 - 1.0)


def andersen(vel, inv_mass, kt: float, p_coll: float, seed: int, draw: int):
    """(new velocities, resampled mask) of one Andersen collision step;
    p_coll is compared in the single precision the kernel receives."""
    vel = np.array(vel, dtype=np.float64).reshape(-1, 3)
    n = len(vel)
    ids = np.arange(n, dtype=np.uint64)
    u = uniform(philox(seed, draw & MASK, draw >> 32, ids, 3)[0])
    hit = (u < float(np.float32(p_coll))) & (np.asarray(inv_mass) > 0)
    sig = np.sqrt(kt * np.asarray(inv_mass, dtype=np.float64))
    out = vel.copy()
    for a in range(3):
        out[hit, a] = sig[hit] * normal(seed, draw, ids[hit], a)
    return out, hit


def perp_widths(box) -> np.ndarray:
    lx, ly, lz, xy, xz, yz = (float(x) for x in box)
    a = np.array([lx, 0.0, 0.0])
    b = np.array([xy, ly, 0.0])
    c = np.array([xz, yz, lz])
    v = lx * ly * lz
    return np.array([v / np.linalg.norm(np.cross(b, c)), v / np.linalg.norm(np.cross(c, a)),
                     v / np.linalg.norm(np.cross(a, b))])


def pressure_coupling(kind: str, k: float, w: float, box, p0: float, kt: float, dt: float,
                      tau: float, kappa: float, seed: int, draw: int, r_search: float = 0.0) -> dict:
    """One c-rescale ("c_rescale") or Berendsen step: pressure, mu and the
    new box from the kinetic energy k and the total virial w."""
    box = np.asarray(box, dtype=np.float64)
    v = box[0] * box[1] * box[2]
    p = (2.0 * k + w) / (3.0 * v)
    r = float(normal(seed, draw, 0)) if kind == "c_rescale" else 0.0
    mu3 = 1.0 - kappa * (dt / tau) * (p0 - p)
    if kind == "c_rescale":
        mu3 += math.sqrt(2.0 * kappa * kt * dt / (tau * v)) * r
    mu3 = max(mu3, 1.0e-18)
    mu = mu3 ** (1.0 / 3.0)
    if r_search > 0.0 and mu * perp_widths(box).min() < 2.0 * r_search:
        mu, mu3 = 1.0, 1.0
    return {"pressure": p, "mu": mu, "r": r, "volume": v * mu3, "box": box * mu,
            "injection": p0 * (v * mu3 - v)}
