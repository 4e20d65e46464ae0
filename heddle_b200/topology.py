"""Topology bookkeeping on the host: effective exclusion lists.

Restates the reference's rules (src/forces/topology.rs:1185-1275) for the
exclusion CSR the force field takes:
  1. explicit entries are kept as given;
  2. every bond (i, j) without an entry adds (i, j) with scales 0;
  3. every angle's 1-3 pair (i, k) without an entry adds scales 0;
  4. every constraint group adds each distinct intra-group pair not yet
     covered, scales 0;
  5. dihedrals, walked in canonical sorted order, add their (i, l) 1-4 pair
     with the dihedral type's LJ / Coulomb 1-4 scales when no entry covers
     it yet (first wins).
Pairs are canonical (min, max).  The result is returned as a symmetric CSR
(offsets [n+1], partners, LJ scales, Coulomb scales), the layout of
hb_forcefield_desc.
"""

from __future__ import annotations

import numpy as np


def _canon(i: int, j: int) -> tuple:
    return (i, j) if i < j else (j, i)


def effective_exclusions(n_atoms: int, bonds=(), angles=(), dihedrals=(), dihedral_scales=(),
                         constraint_groups=(), explicit=()) -> dict:
    """Map (i, j) -> (scale_lj, scale_coul) under the five rules.

    bonds: iterable of (i, j); angles: (i, j, k) with the vertex j;
    dihedrals: (i, j, k, l) with dihedral_scales[q] = (lj14, coul14);
    constraint_groups: iterables of atom ids; explicit: (i, j, s_lj, s_c)."""
    eff: dict = {}
    for i, j, slj, sc in explicit:
        eff[_canon(int(i), int(j))] = (float(slj), float(sc))
    for i, j in bonds:
        eff.setdefault(_canon(int(i), int(j)), (0.0, 0.0))
    for a in angles:
        eff.setdefault(_canon(int(a[0]), int(a[2])), (0.0, 0.0))
    for g in constraint_groups:
        g = [int(x) for x in g]
        for x in range(len(g)):
            for y in range(x + 1, len(g)):
                eff.setdefault(_canon(g[x], g[y]), (0.0, 0.0))
    order = sorted(range(len(dihedrals)), key=lambda q: tuple(int(v) for v in dihedrals[q]))
    for q in order:
        d = dihedrals[q]
        key = _canon(int(d[0]), int(d[3]))
        if key not in eff:
            slj, sc = dihedral_scales[q]
            eff[key] = (float(slj), float(sc))
    return eff


def exclusion_csr(n_atoms: int, eff: dict):
    """Symmetric CSR of an exclusion map: (offsets, partners, s_lj, s_coul)."""
    rows: list = [[] for _ in range(n_atoms)]
    for (i, j), (slj, sc) in sorted(eff.items()):
        rows[i].append((j, slj, sc))
        rows[j].append((i, slj, sc))
    off = np.zeros(n_atoms + 1, dtype=np.uint32)
    for a in range(n_atoms):
        rows[a].sort()
        off[a + 1] = off[a] + len(rows[a])
    part = np.array([p for r in rows for p, _, _ in r], dtype=np.uint32)
    slj = np.array([s for r in rows for _, s, _ in r], dtype=np.float64)
    sc = np.array([s for r in rows for _, _, s in r], dtype=np.float64)
    return off, part, slj, sc
