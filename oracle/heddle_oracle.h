/*
 * heddle_oracle.h -- FP64 CPU restatement of HeddleMD's per-timestep
 * force-and-constraint path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the
 * smoke() entry and bench.py's CPU-baseline / reference arm may load it.
 * The product (heddle_b200) never links, imports or calls it.
 *
 * Units: Hartree atomic units (a0, Eh, m_e, e; k_Coulomb = 1, k_B = 1),
 * as the reference uses internally (src/gpu/kernels.rs:176,
 * src/units/atomic_constants.rs:11-35).
 *
 * Box: lower-triangular lattice (lx, ly, lz, xy, xz, yz), as
 * src/pbc.rs:11-60.
 */
#ifndef HEDDLE_ORACLE_H
#define HEDDLE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double lx, ly, lz, xy, xz, yz;
} or_box;

typedef struct {
  /* Lennard-Jones slot (src/forces/lj.rs:237-283); per type-pair tables
   * of size n_types * n_types, row-major [ti * n_types + tj]. */
  int lj_on;
  int n_types;
  const double *lj_sigma;
  const double *lj_epsilon;
  const double *lj_cutoff;
  const double *lj_switch;
  /* erfc-screened real-space Coulomb (src/forces/spme.rs:730-759). */
  int coul_on;
  double alpha;
  double r_cut_coul;
  /* 0: exact erfc (FP64).  1: Abramowitz-Stegun 7.1.26 polynomial, the
   * form the reference's f32 build evaluates (src/forces/spme.rs:742-751). */
  int coul_poly_erfc;
  /* SPME reciprocal (src/forces/spme.rs:228-503). */
  int recip_on;
  int grid[3];
  int order;
  /* exclusions: CSR over atoms, partners + separate LJ / Coulomb scales
   * (src/forces/topology.rs:312-440). NULL excl_off = no exclusions. */
  const int32_t *excl_off;
  const int32_t *excl_partner;
  const double *excl_lj_scale;
  const double *excl_coul_scale;
  /* bonded terms, one row per term: harmonic bonds
   * (src/forces/harmonic_bond.rs:283-307), harmonic angles with the vertex
   * in the middle (src/forces/angle.rs:260-313), periodic dihedrals
   * (src/forces/dihedral.rs:383-467). */
  int32_t n_bonds;
  const int32_t *bond_atoms;
  const double *bond_k, *bond_r0;
  int32_t n_angles;
  const int32_t *angle_atoms;
  const double *angle_k, *angle_theta0;
  int32_t n_dihedrals;
  const int32_t *dihedral_atoms;
  const double *dihedral_k, *dihedral_phi0;
  const int32_t *dihedral_n;
} or_ff;

/* terms[] layout written by or_forces */
enum {
  OR_E_LJ = 0,
  OR_E_COUL_REAL = 1,
  OR_E_RECIP = 2,      /* 0.5 * sum_k G |rho_hat|^2 */
  OR_E_SELF = 3,       /* sum_i alpha/sqrt(pi) q_i^2 */
  OR_W_PAIR = 4,       /* sum over pairs factor * r^2 */
  OR_W_RECIP = 5,      /* 0.5 * sum_k vf |rho_hat|^2 */
  OR_N_PAIRS_NEAR_CUT = 6, /* pairs within 1e-6 relative of a cutoff */
  OR_E_BONDED = 7,     /* bonds + angles + dihedrals (their virial is in OR_W_PAIR) */
  OR_N_TERMS = 8
};

/* ---- periodic boundary helpers (kernels/pbc.cuh:18-93) ---- */
void or_min_image(const or_box *b, double *dx, double *dy, double *dz);
void or_wrap_with_image(const or_box *b, double *x, double *y, double *z,
                        int *ka, int *kb, int *kc);

/* ---- neighbour set under the stated f32 rule ----
 * All unordered pairs (i < j) whose single-precision minimum-image r^2,
 * evaluated operation by operation with IEEE round-to-nearest and no
 * fused multiply-add, satisfies r^2 <= r_search^2 (the membership test of
 * kernels/neighbor.cu:509-529).  xyz holds float positions [3n].
 * Writes min(count, cap) pairs as (i, j) into out_pairs[2*cap], sorted
 * lexicographically; returns the total count. */
void or_pair_r2_f32(int64_t n_pairs, const uint32_t *pairs, const float *xyz,
                    const float *box6, float *out_r2);
int64_t or_neighbor_pairs_f32(int32_t n, const float *xyz, const float *box6,
                              float r_search, uint32_t *out_pairs, int64_t cap);

/* ---- forces ----
 * pos[3n], q[n], type[n] -> F[3n], E[n] (per-atom energy shares),
 * W[n] (per-atom virial shares), terms[OR_N_TERMS].
 * Per-atom conventions follow the reference: pair energy and virial split
 * 1/2 to each atom (jit_composed.rs:1755-1769); reciprocal energy share
 * 1/2 q phi - u_self (spme_spread_gather.cuh:328-333); reciprocal virial
 * share W_recip / N uniform.  Excluded pairs keep their reciprocal-space
 * interaction (no excluded-pair correction), as the reference does.
 * Returns 0 on success, negative on invalid input. */
int or_forces(int32_t n, const double *pos, const double *q,
              const int32_t *type, const or_box *box, const or_ff *ff,
              double *F, double *E, double *W, double *terms, int n_threads);

/* Explicit Ewald reciprocal energy truncated to |m_d| <= m_max, for an
 * orthorhombic box (the independent check of tests/spme_pipeline.rs:46-83). */
double or_ewald_recip_energy(int32_t n, const double *pos, const double *q,
                             const or_box *box, double alpha, int m_max);

/* SPME pieces exposed for unit checks. */
void or_bspline_weights(int order, double t, double *w, double *dw);
void or_b_factors(int n, int order, double *out);
/* real grid rho[n_a*n_b*n_c] of the charge spread (row-major, c fastest) */
void or_spme_spread(int32_t n, const double *pos, const double *q,
                    const or_box *box, const int grid[3], int order,
                    double *rho);

/* ---- SETTLE / SHAKE / RATTLE (kernels/settle.cu, kernels/shake.cu) ----
 * Groups: CSR group_off[n_groups+1] into group_atoms[]; constraints per
 * group: CSR con_off[n_groups+1] into con_i/con_j (local indices) and
 * con_d2 (target squared distances).
 * or_constrain_positions: converged Gauss-Seidel SHAKE with constraint
 * gradients taken at the pre-drift snapshot ref_pos[3n]; updates pos[3n]
 * in place, adds (dx / dt) to vel[3n], writes the position-level constraint
 * virial per atom slot into vir_slot (may be NULL).
 * Returns max sweeps used (or -1 if tol not reached within max_iter). */
int or_constrain_positions(int32_t n_groups, const int32_t *group_off,
                           const int32_t *group_atoms, const int32_t *con_off,
                           const int32_t *con_i, const int32_t *con_j,
                           const double *con_d2, const double *mass,
                           const or_box *box, const double *ref_pos,
                           double *pos, double *vel, double dt,
                           double *vir_slot, double tol, int max_iter);
/* RATTLE velocity projection by a direct dense solve of the constraint
 * velocity equations of each group (exact to round-off); adds the
 * velocity-level constraint virial into vir_slot (may be NULL, dt > 0). */
int or_constrain_velocities(int32_t n_groups, const int32_t *group_off,
                            const int32_t *group_atoms, const int32_t *con_off,
                            const int32_t *con_i, const int32_t *con_j,
                            const double *mass, const or_box *box,
                            const double *pos, double *vel, double dt,
                            double *vir_slot);

/* ---- Philox-4x32-10 and the Box-Muller Gaussian (kernels/philox.cuh) ---- */
void or_philox4x32_10(uint32_t key_lo, uint32_t key_hi, const uint32_t ctr[4],
                      uint32_t out[4]);
double or_philox_gaussian(uint32_t seed_lo, uint32_t seed_hi, uint32_t step_lo,
                          uint32_t step_hi, uint32_t particle, uint32_t axis);

/* ---- Monte-Carlo barostat centre-of-mass scaling
 * (kernels/mc_barostat.cu:19-74, src/integrator/mc_barostat.rs:300-318) ----
 * Each molecule (CSR off/atoms) is rebuilt as its contiguous image about its
 * first atom (minimum-image displacements in box_old, the cell the positions
 * live in), its mass-weighted centre c is computed, every atom is translated
 * by (scale - 1) c and wrapped into box_new; img[3n] keeps each atom's
 * integer offset from its molecule's contiguous image.  (The reference translates the stored, per-atom wrapped
 * positions instead, which agrees for molecules that do not straddle the
 * cell boundary.) */
void or_mc_scale_com(int32_t n_mol, const int32_t *off, const int32_t *atoms,
                     const double *mass, const or_box *box_old, const or_box *box_new,
                     double scale, double *pos, int32_t *img);

/* ---- CPU MD driver used as the timed CPU baseline ----
 * One velocity-Verlet or Langevin-middle step per iteration with SETTLE/SHAKE
 * groups, forces from or_forces.  integrator: 0 = velocity Verlet,
 * 1 = Langevin (BAOAB, middle scheme).  State arrays are updated in place. */
int or_md_run(int32_t n, double *pos, double *vel, const double *mass,
              const double *q, const int32_t *type, const or_box *box,
              const or_ff *ff, int32_t n_groups, const int32_t *group_off,
              const int32_t *group_atoms, const int32_t *con_off,
              const int32_t *con_i, const int32_t *con_j, const double *con_d2,
              int integrator, double dt, double friction, double kt,
              uint64_t seed, uint64_t step0, int n_steps, double *F,
              int n_threads);

#ifdef __cplusplus
}
#endif
#endif
