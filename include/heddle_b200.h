/*
 * heddle_b200.h -- C ABI of the B200-native HeddleMD force-and-constraint
 * path.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (HB_OK or an HB_ERR_* code) and leaves a thread-local message readable
 * through hb_last_error().  Units are Hartree atomic units (bohr, hartree,
 * electron mass, elementary charge, atomic time; k_Coulomb = k_B = 1), the
 * reference's internal units (src/units/atomic_constants.rs:11-35).
 * The box is the lower-triangular lattice (lx, ly, lz, xy, xz, yz) of
 * src/pbc.rs:11-60.
 *
 * Threading: a context and everything created from it is single-threaded
 * and runs on the context's stream(s), as the reference runs on one default
 * stream (src/runner.rs:2441-2447).
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the HeddleMD project root).
 */
#ifndef HEDDLE_B200_H
#define HEDDLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (errors of rqm/error-handling.md:13-115) ---- */
enum {
  HB_OK = 0,
  HB_ERR_INVALID_ARGUMENT = 1,   /* malformed descriptor / null pointer */
  HB_ERR_CUDA = 2,               /* CUDA runtime failure (GpuError) */
  HB_ERR_NL_OVERFLOW = 3,        /* NeighborListError::PackedNeighborOverflow */
  HB_ERR_BOX_TOO_SMALL = 4,      /* NeighborListError::BoxTooSmallForCells */
  HB_ERR_INVALID_GRID = 5,       /* SpmeError::InvalidGrid */
  HB_ERR_CONSTRAINT_SHAPE = 6,   /* ConstraintError (group too large, bad kind) */
  HB_ERR_DEVICE_TIMEOUT = 7,     /* a bounded device-side wait gave up */
  HB_ERR_UNSUPPORTED = 8,        /* combination the reference rejects
                                    (e.g. all-pairs + SPME, src/io/config.rs:85-88) */
  HB_ERR_NOT_FINITE = 9          /* non-finite position / box value */
};

/* aggregate level of ForceField::step (src/forces/mod.rs:662-717) */
enum { HB_FORCES_ONLY = 0, HB_FORCES_AND_SCALARS = 1 };

/* integrator kinds (registry names of src/integrator/mod.rs:627-677) */
enum {
  HB_INTEGRATOR_VV = 0,          /* "velocity-verlet" */
  HB_INTEGRATOR_VV_LOSSLESS = 1, /* velocity Verlet, lossless (f32 + f64) mode */
  HB_INTEGRATOR_LANGEVIN = 2     /* "langevin-baoab" (middle scheme) */
};

/* launch-shape parameters of hb_forcefield_set_launch (autotuned) */
enum {
  HB_LAUNCH_PAIR_BLOCKS_PER_SM = 0, /* resident blocks of the persistent pair kernel
                                       per SM (1..8, default 8); fewer leave room
                                       for the concurrent reciprocal-space chain */
  HB_LAUNCH_NL_SLAB = 1,            /* packed entries per i-tile slab (>= 2): the
                                       list is rebuilt at once into slabs of this
                                       size; more than 3/4 full grows them again
                                       (the reference's high-water growth,
                                       src/forces/neighbor_list.rs:400-446), an
                                       overflow returns HB_ERR_NL_OVERFLOW and
                                       halts the force field until a larger slab
                                       is set */
  HB_LAUNCH_PAIR_CHUNK = 2,         /* packed entries per work item of the
                                       persistent pair kernel (1..64, default 4):
                                       shorter items balance better, longer ones
                                       reload the i-tile less often */
  HB_LAUNCH_FFT_PLANE = 3,          /* 1 (default where supported: 64 x 64 and
                                       128 x 128 (a, b) planes): whole-plane FFT
                                       pass; 0: line passes */
  HB_LAUNCH_GATHER_FORM = 4,        /* spline orders 4 and 8: 1 (default) one
                                       thread per (atom, c offset); 0 one thread
                                       per atom */
  HB_LAUNCH_PAIR_QUOTA = 5,         /* work items per pair-kernel warp (0..4096):
                                       0 (default) persistent blocks; q > 0
                                       blocks that retire after q items each, so
                                       the concurrent reciprocal-space kernels
                                       are scheduled between them */
  HB_LAUNCH_NL_WAIT_TEST = 6        /* failure-path test of the tile build's
                                       bounded waits: v > 0 issues no bulk
                                       copies and gives up after v polls (the
                                       next rebuild returns HB_ERR_DEVICE_TIMEOUT);
                                       0 restores normal operation */
};

/* pair accumulation modes (hb_forcefield_desc.pair_mode) */
enum { HB_PAIRS_FAST = 0, HB_PAIRS_EXACT = 1 };

/* constraint kinds (src/integrator/constraint.rs:205-212) */
enum { HB_CONSTRAINT_SETTLE = 0, HB_CONSTRAINT_SHAKE = 1 };

typedef struct hb_context hb_context;
typedef struct hb_system hb_system;
typedef struct hb_forcefield hb_forcefield;
typedef struct hb_constraints hb_constraints;
typedef struct hb_integrator hb_integrator;
typedef struct hb_barostat hb_barostat;
typedef struct hb_thermostat hb_thermostat;
typedef struct hb_pcouple hb_pcouple;
typedef struct hb_minimizer hb_minimizer;
typedef struct hb_batch hb_batch;
typedef struct hb_shake_mlp hb_shake_mlp;

/* Message of the last failing call on this thread ("" when none). */
const char *hb_last_error(void);

/* Library version string. */
const char *hb_version(void);

/* ---- context: replaces init_device (src/gpu/device.rs:67-74) ---- */
int hb_context_create(int device_ordinal, hb_context **out);
int hb_context_destroy(hb_context *ctx);
int hb_context_synchronize(hb_context *ctx);

/* ---- system state: replaces ParticleBuffers::new (src/gpu/buffers.rs:11-38)
 * and SimulationBox::new (src/pbc.rs:142-170).  The library copies the host
 * arrays into device structure-of-arrays and owns them. */
typedef struct {
  uint32_t n_atoms;
  const double *positions;   /* [3n] */
  const double *velocities;  /* [3n] or NULL (zero) */
  const double *masses;      /* [n] */
  const double *charges;     /* [n] */
  const uint32_t *types;     /* [n] particle-type indices */
  const int32_t *images;     /* [3n] or NULL (zero) */
  double box[6];             /* lx, ly, lz, xy, xz, yz */
} hb_system_desc;

int hb_system_create(hb_context *ctx, const hb_system_desc *desc,
                     hb_system **out);
int hb_system_destroy(hb_system *sys);
/* Overwrite positions / velocities from host ([3n] each, NULL = keep).
 * Positions are wrapped into the cell on the device (FP64, image counts
 * carried on); a non-finite position is rejected before anything changes.
 * The arrays are copied as they are (page-locked host memory copies
 * fastest) and may be reused when the call returns. */
int hb_system_set_state(hb_system *sys, const double *positions,
                        const double *velocities);
/* Download positions, velocities, images, forces (any may be NULL); the
 * conversion to FP64 runs on the device. */
int hb_system_get_state(hb_system *sys, double *positions, double *velocities,
                        int32_t *images, double *forces);
/* The same exchange with single-precision host arrays -- the precision of
 * the reference's own particle buffers (ParticleBuffers, Real = f32,
 * src/gpu/buffers.rs) -- at half the PCIe bytes; the wrap into the cell
 * still runs in FP64 on the device. */
int hb_system_set_state_f32(hb_system *sys, const float *positions,
                            const float *velocities);
int hb_system_get_state_f32(hb_system *sys, float *positions, float *velocities,
                            int32_t *images, float *forces);
int hb_system_set_box(hb_system *sys, const double box[6]);
/* Velocity flip v <- -v of both halves of the lossless (f32 + f64) state:
 * step 3 of the reversal protocol (rqm/pipeline-reversibility.md,
 * tests/integration_lossless.rs:302-395). */
int hb_system_flip_velocities(hb_system *sys);
int hb_system_get_box(hb_system *sys, double box[6]);

/* ---- force field: replaces ForceField::new (src/forces/mod.rs:355-621)
 * with the LJ slot (src/forces/lj.rs), SPME real (src/forces/spme.rs:620-781)
 * and SPME reciprocal (src/forces/spme.rs:228-503, :862-917). */
typedef struct {
  /* Lennard-Jones: tables [n_types * n_types], row-major (ti * n + tj). */
  int lj_enabled;
  uint32_t n_types;
  const double *lj_sigma;
  const double *lj_epsilon;
  const double *lj_cutoff;
  const double *lj_switch;
  /* erfc-screened real-space Coulomb */
  int coulomb_enabled;
  double alpha;
  double r_cut_coulomb;
  /* SPME reciprocal */
  int recip_enabled;
  uint32_t grid[3];
  uint32_t spline_order;     /* 4..8 */
  /* exclusions: CSR over atoms (offsets [n+1]), partner ids, scales */
  const uint32_t *excl_offsets;  /* NULL = none */
  const uint32_t *excl_partners;
  const double *excl_lj_scale;
  const double *excl_coulomb_scale;
  /* neighbour list */
  double r_skin;
  /* pair accumulation: HB_PAIRS_FAST sums each neighbour entry's 32 pair
   * forces in f32 before the fixed-point add (the reference's scheme,
   * src/forces/jit_composed.rs:1696-1786); HB_PAIRS_EXACT converts every
   * pair force to fixed point and takes the minimum image per pair, so the
   * forces are a function of the positions alone, independent of when the
   * neighbour list was rebuilt and of how it packed the pairs -- what
   * bit-exact time reversal of the lossless integrator needs. */
  int pair_mode;
  /* bonded terms, one row per term (the reference's HarmonicBond,
   * HarmonicAngle and PeriodicDihedral slots, src/forces/harmonic_bond.rs,
   * src/forces/angle.rs, src/forces/dihedral.rs, expanded from their type
   * tables): U = k/2 (r - r0)^2; U = k/2 (theta - theta0)^2 with the angle
   * at the middle atom; U = k (1 + cos(n phi - phi0)).  Their exclusions
   * (1-2, 1-3, scaled 1-4, src/forces/topology.rs:1185-1275) are the
   * caller's, in the exclusion CSR above. */
  uint32_t n_bonds;
  const uint32_t *bond_atoms;        /* [2 n_bonds] */
  const double *bond_k;
  const double *bond_r0;
  uint32_t n_angles;
  const uint32_t *angle_atoms;       /* [3 n_angles]: i, j (vertex), k */
  const double *angle_k;
  const double *angle_theta0;
  uint32_t n_dihedrals;
  const uint32_t *dihedral_atoms;    /* [4 n_dihedrals]: i, j, k, l */
  const double *dihedral_k;
  const double *dihedral_phi0;
  const uint32_t *dihedral_n;        /* multiplicity */
} hb_forcefield_desc;

int hb_forcefield_create(hb_system *sys, const hb_forcefield_desc *desc,
                         hb_forcefield **out);
int hb_forcefield_destroy(hb_forcefield *ff);
/* ForceField::step (src/forces/mod.rs:662-670): neighbour pre-step (rebuild
 * when any atom moved more than r_skin / 2), pair forces, SPME, combine.
 * Forces land in the system's force buffer; level HB_FORCES_AND_SCALARS
 * also produces per-atom energies / virials and the FP64 scalars. */
int hb_forcefield_step(hb_forcefield *ff, int level);
/* NeighborListState::pre_step (src/forces/neighbor_list.rs:1265-1354):
 * rebuild if needed (force != 0 forces a rebuild); *rebuilt = 1 if so. */
int hb_forcefield_pre_step(hb_forcefield *ff, int force, int *rebuilt);
/* FP64 scalars of the last HB_FORCES_AND_SCALARS step:
 * out[0] LJ energy, [1] real-space Coulomb, [2] reciprocal (k-space sum),
 * [3] self energy (subtracted), [4] total potential, [5] pair + bonded
 * virial, [6] reciprocal virial, [7] total virial, [8] bonded energy,
 * [9] reserved (0). */
int hb_forcefield_scalars(hb_forcefield *ff, double out[10]);
/* Set a launch-shape parameter (HB_LAUNCH_*); captured graphs of the force
 * field's integrators are re-captured on their next call. */
int hb_forcefield_set_launch(hb_forcefield *ff, int param, int value);
/* per-atom energy and virial shares of the last scalar step ([n] each). */
int hb_forcefield_get_per_atom(hb_forcefield *ff, double *energy,
                               double *virial);
/* Canonical neighbour pairs (i < j) held by the packed list whose f32
 * minimum-image distance is within r_cut + r_skin: the analogue of
 * NeighborListState::pair_snapshot (src/forces/neighbor_list.rs:1366-1560).
 * Writes min(count, cap) pairs (i, j) sorted; *count = total;
 * *duplicates = pairs represented more than once (must be 0). */
int hb_neighbor_pairs(hb_forcefield *ff, uint32_t *pairs, uint64_t cap,
                      uint64_t *count, uint64_t *duplicates);
/* Neighbour-list statistics: out[0] tiles, [1] entries, [2] entry capacity,
 * [3] rebuild count, [4] status word, [5] pair slots per step. */
int hb_neighbor_stats(hb_forcefield *ff, uint64_t out[6]);
/* Packed-list capacity (the reference's capacity status,
 * src/forces/neighbor_list.rs:1080-1262 and kernels/neighbor.cu:643-669):
 * out[0] entries per i-tile slab, [1] most entries of one i-tile in the last
 * build, [2] slab reallocations so far (high-water growth included), [3]
 * status word (HB_ST bits: 1 displaced, 2 high water, 8 overflow). */
int hb_neighbor_capacity(hb_forcefield *ff, uint64_t out[4]);

/* ---- constraints: replaces the Constraint hooks
 * (src/integrator/constraint.rs:43-122) of SETTLE (src/integrator/settle.rs)
 * and SHAKE/RATTLE (src/integrator/shake.rs).  Groups are CSR lists of atom
 * ids; SETTLE groups are (O, H1, H2) with geometry (ra, rb, rc); SHAKE groups
 * carry local constraint pairs with target distances. */
typedef struct {
  uint32_t n_groups;
  const uint32_t *group_offsets;   /* [n_groups + 1] into group_atoms */
  const uint32_t *group_atoms;
  const uint32_t *group_kind;      /* HB_CONSTRAINT_* per group */
  /* SETTLE geometry per group (ignored for SHAKE groups) */
  const double *settle_ra;
  const double *settle_rb;
  const double *settle_rc;
  /* SHAKE constraints: CSR per group into (local i, local j, distance) */
  const uint32_t *con_offsets;     /* [n_groups + 1] */
  const uint32_t *con_i;
  const uint32_t *con_j;
  const double *con_dist;
  double shake_tol;                /* tolerance on |r|^2 - d^2 (bohr^2) */
  uint32_t shake_max_iter;
  int shake_tol_relative;          /* != 0: tolerance relative to d^2 */
} hb_constraints_desc;

int hb_constraints_create(hb_system *sys, const hb_constraints_desc *desc,
                          hb_constraints **out);
int hb_constraints_destroy(hb_constraints *c);
/* Constraint::apply_before_drift: snapshot pre-drift positions. */
int hb_constraints_before_drift(hb_constraints *c);
/* Constraint::apply_after_drift: position reset + velocity correction. */
int hb_constraints_after_drift(hb_constraints *c, double dt);
/* Constraint::apply_after_kick: velocity projection (+ virial when dt > 0). */
int hb_constraints_after_kick(hb_constraints *c, double dt);
/* per-atom constraint virial of the last step ([n]) */
int hb_constraints_get_virial(hb_constraints *c, double *virial);
/* SHAKE sweep statistics since creation or the last reset: out[0]
 * group-sweeps (sweeps that still moved something, summed over groups and
 * calls), out[1] group solves, out[2] mean sweeps per solve. */
int hb_constraints_shake_stats(hb_constraints *c, double out[3], int reset);
/* Training data of the learned warm start: while recording, every SHAKE
 * position call stores per SHAKE constraint (in group order) 8 geometry
 * features, the first Gauss-Seidel multiplier lam1, the multiplier-to-sigma
 * scale ls and the converged multiplier lam; get_record copies those of the
 * last call (features [8 m], the others [m], m = SHAKE constraints). */
int hb_constraints_record(hb_constraints *c, int enable);
int hb_constraints_get_record(hb_constraints *c, float *features, double *lam1, double *lscale,
                              double *lam, uint32_t *m);
/* With a Langevin integrator and every atom in a SETTLE water (no SHAKE
 * group), a step's kick, velocity projection, drift / O / drift and
 * position reset run as one kernel, one thread per water, with the same
 * per-atom arithmetic as the four separate kernels (enable = 1, the
 * default); enable = 0 launches the four.  No reference counterpart: the
 * reference launches them in turn (kernels/langevin.cu:13-80,
 * kernels/settle.cu:145-492). */
int hb_constraints_fuse_head(hb_constraints *c, int enable);
/* Warm-start SHAKE from the network (NULL switches it off): features ->
 * network -> lam0 = lam1 + prediction / ls, then the usual sweeps to the
 * same tolerance. */
int hb_constraints_set_warm_start(hb_constraints *c, hb_shake_mlp *m);

/* ---- learned SHAKE warm start (no reference counterpart: the reference's
 * SHAKE starts from zero multipliers, kernels/shake.cu:108-348).  A
 * 8 -> 64 -> 64 -> 1 tanh network; its hidden layers run as BF16 tcgen05
 * tensor-core GEMMs with FP32 accumulation, forward and backward, trained by
 * Adam in one deterministic CTA.  Parameters (FP32, packed): W1 [64][8], b1
 * [64], W2 [64][64], b2 [64], w3 [64], b3.  Inputs are standardised by
 * (x - mean) * inv_std and targets divided by target_scale inside. */
int hb_shake_mlp_create(hb_context *ctx, uint64_t seed, hb_shake_mlp **out);
int hb_shake_mlp_destroy(hb_shake_mlp *m);
uint32_t hb_shake_mlp_param_count(void);
int hb_shake_mlp_get_params(hb_shake_mlp *m, float *out, uint32_t n);
int hb_shake_mlp_set_params(hb_shake_mlp *m, const float *in, uint32_t n);
int hb_shake_mlp_set_normalization(hb_shake_mlp *m, const float *mean, const float *inv_std,
                                   float target_scale);
/* host rows in, host predictions out (target units) */
int hb_shake_mlp_predict(hb_shake_mlp *m, const float *features, uint64_t n, float *out);
/* gradients of the mean squared error (normalised units) over n <= 4096
 * rows, no update; *loss = that error */
int hb_shake_mlp_gradients(hb_shake_mlp *m, const float *features, const float *targets,
                           uint32_t n, float *grads, double *loss);
/* Bounded waits: every mbarrier wait of the network's kernels gives up after
 * `polls` polls (default 2^22), the kernel frees its tensor memory and the
 * call (or the integrator step that ran the inference) returns
 * HB_ERR_DEVICE_TIMEOUT; the rows of a timed-out inference get no
 * correction.  issue = 0 makes inference issue no tensor-core work, so its
 * first wait runs out with nothing in flight: the failure-path test, with
 * no GPU fault.  No reference counterpart. */
int hb_shake_mlp_set_wait_limit(hb_shake_mlp *m, uint32_t polls, int issue);
/* epochs of minibatch Adam (seeded shuffles); loss_per_epoch [epochs] */
int hb_shake_mlp_train(hb_shake_mlp *m, const float *features, const float *targets,
                       uint64_t n, uint32_t epochs, uint32_t batch, double lr, uint64_t seed,
                       double *loss_per_epoch);

/* ---- integrator: replaces integrator::run_step (src/integrator/mod.rs:344)
 * for velocity Verlet (src/integrator/velocity_verlet.rs) and Langevin
 * (src/integrator/langevin_baoab.rs). */
typedef struct {
  int kind;                 /* HB_INTEGRATOR_* */
  double dt;
  double friction;          /* Langevin gamma (1 / time) */
  double temperature;       /* k_B T in hartree */
  uint64_t seed;
  uint64_t step0;           /* first Philox draw counter */
} hb_integrator_desc;

int hb_integrator_create(hb_system *sys, const hb_integrator_desc *desc,
                         hb_integrator **out);
int hb_integrator_destroy(hb_integrator *it);
/* Advance n_steps steps.  cons may be NULL.  scalar_every > 0 evaluates
 * forces with scalars on every scalar_every-th step (0 = never). */
int hb_integrator_step(hb_integrator *it, hb_forcefield *ff,
                       hb_constraints *cons, uint32_t n_steps,
                       uint32_t scalar_every);
/* Same as hb_integrator_step, launched as CUDA graphs of one step each
 * (captured on first use; the neighbour rebuild is a device-side IF node
 * taken when an atom moved more than r_skin / 2; the Langevin draw counter
 * lives on the device, so replays draw fresh noise). */
int hb_integrator_step_graph(hb_integrator *it, hb_forcefield *ff,
                             hb_constraints *cons, uint32_t n_steps);
/* Upload, steps and read-out in one call: replaces the runner's steps
 * followed by ParticleState::download_from (src/runner.rs:2709-2716,
 * src/state.rs:140-216).  positions_in / velocities_in (f32 [3n], either may
 * be NULL) are uploaded as by hb_system_set_state_f32 (the forces of the
 * last evaluation are kept); n_steps >= 1 steps run as by
 * hb_integrator_step_graph; then the state after the last step is written
 * to positions / velocities / forces (f32 [3n]) and images (i32 [3n]), any
 * of which may be NULL.  With page-locked host arrays the last step is one
 * CUDA graph whose positions and image counts (and the Langevin velocities)
 * are copied out while its force evaluation runs; a step that ends with a
 * barostat move or scales positions in its tail copies them at its end.
 * The graph is captured again when a host pointer changes.  Pageable host
 * arrays are filled after the steps instead.  The input arrays may be the
 * output arrays (the upload completes before the steps).  Returns when the
 * host arrays are filled. */
int hb_integrator_step_exchange_f32(hb_integrator *it, hb_forcefield *ff,
                                    hb_constraints *cons, uint32_t n_steps,
                                    const float *positions_in,
                                    const float *velocities_in, float *positions,
                                    float *velocities, int32_t *images,
                                    float *forces);

/* Kernel launches of one step: the step is captured into a throwaway CUDA
 * graph (nothing runs) and its kernel nodes are counted: kernels[0] = the
 * kernels every step launches, kernels[1] = the kernels of a neighbour
 * rebuild (a conditional node taken only on rebuild steps), kernels[2] =
 * the kernels of one barostat volume move (0 without a barostat). */
int hb_integrator_count_launches(hb_integrator *it, hb_forcefield *ff,
                                 hb_constraints *cons, uint64_t *kernels);

/* ---- Monte-Carlo barostat: replaces McBarostat
 * (src/integrator/mc_barostat.rs:218-360, "monte-carlo" in the barostat
 * registry) and mc_barostat_scale_molecule_com (kernels/mc_barostat.cu:19-74).
 * A move: draw (Philox-4x32-10, key = seed, counter = move number),
 * dV = max_dV (2 u1 - 1), isotropic lattice scale (V'/V)^(1/3) in FP64,
 * molecule centres of mass scaled about the origin with every molecule kept
 * rigid, a forces + scalars evaluation, Metropolis test on
 * w = dU + P dV - n_mol kT ln(V'/V), and on rejection the box, positions,
 * images, forces and scalars of the pre-move state restored.  A contraction
 * that would take the narrowest perpendicular width below 2 (r_cut + r_skin)
 * is rejected before any work.  Every 10 attempts max_dV is divided by 1.1
 * (acceptance < 25 %) or multiplied by 1.1 up to 0.3 V (> 75 %).  The whole
 * move runs on the device (no host read), so it also runs inside a graph. */
typedef struct {
  double pressure;           /* hartree / bohr^3 */
  double temperature;        /* k_B T in hartree */
  uint32_t frequency;        /* a move after every frequency-th step (>= 1) */
  double volume_step;        /* initial max |dV| in bohr^3; <= 0: 1 % of V */
  uint64_t seed;
  uint32_t n_molecules;      /* 0: every atom is its own molecule */
  const uint32_t *mol_offsets;   /* [n_molecules + 1] */
  const uint32_t *mol_atoms;     /* [n_atoms]: each atom exactly once */
} hb_barostat_desc;

int hb_barostat_create(hb_system *sys, const hb_barostat_desc *desc, hb_barostat **out);
int hb_barostat_destroy(hb_barostat *b);
/* Barostat::apply_move.  The force field's last evaluation must have been
 * HB_FORCES_AND_SCALARS at the current configuration (its potential energy
 * is U_old), as the reference's runner arranges on the step before a move. */
int hb_barostat_mc_move(hb_barostat *b, hb_forcefield *ff);
/* out[0] volume, [1] acceptance ratio, [2] max_dV, [3] P V - cumulative
 * P dV (the barostat's term of the conserved quantity), [4] attempted,
 * [5] accepted, [6] last dV, [7] last w, [8] last U_old, [9] last U_new,
 * [10] last scale, [11] last move accepted (0/1), [12] last trial applied
 * (0/1), [13] last u2, [14] move counter. */
int hb_barostat_stats(hb_barostat *b, double out[15]);
/* Attach (or detach with NULL) a barostat to an integrator: the step whose
 * number is a multiple of the barostat's frequency evaluates scalars and is
 * followed by a move (src/runner.rs:2693-2708). */
int hb_integrator_set_barostat(hb_integrator *it, hb_barostat *b);

/* ---- velocity thermostats for velocity Verlet: replace CsvrThermostat
 * (src/integrator/csvr.rs:45-260, csvr_sample_and_factor /
 * csvr_sample_partials / csvr_finish_from_partials in
 * kernels/nose_hoover.cu:145-385), AndersenThermostat
 * (src/integrator/andersen.rs:110-260, kernels/andersen.cu) and the
 * Berendsen thermostat (src/integrator/berendsen.rs,
 * berendsen_compute_factor in kernels/nose_hoover.cu:390-415).
 * Each step, after the force evaluation and the constraint velocity
 * projection and before the final half kick (the reference's composed
 * post-force order, src/runner.rs:2661-2686):
 *   CSVR:      K = sum m v^2 / 2 of the current velocities (FP64), then
 *              K' = c K + (kT/2)(1 - c)(s + r^2) + 2 r sqrt(c (1 - c) K kT / 2)
 *              with c = exp(-dt / tau), r and the g - 1 terms of s = sum xi^2
 *              the Box-Muller normals of Philox (key seed, counter
 *              (draw, 0, i, 0)), g = 3N - n_constraints - 3; factor
 *              sqrt(K'/K) (1 when K' is not finite and positive or K = 0);
 *   Berendsen: factor sqrt(max(0, 1 + dt/tau (g kT / 2K - 1)));
 *   Andersen:  after the kick, every atom whose uniform (counter (draw, 0,
 *              id, 3)) is below p = clamp(rate dt, 0, 1) gets the velocity
 *              sqrt(kT / m) (xi_0, xi_1, xi_2) (counters (draw, 0, id, 0..2)).
 * The draw counter lives on the device and advances once per step, so a
 * captured step draws fresh numbers on every replay. */
#define HB_THERMOSTAT_CSVR 0
#define HB_THERMOSTAT_ANDERSEN 1
#define HB_THERMOSTAT_BERENDSEN 2
typedef struct {
  int kind;                  /* HB_THERMOSTAT_* */
  double temperature;        /* k_B T in hartree */
  double tau;                /* coupling time (a.u.), CSVR and Berendsen */
  double collision_rate;     /* collisions per a.u. time, Andersen */
  uint64_t seed;
  uint32_t n_constraints;    /* removed from the degrees of freedom */
} hb_thermostat_desc;

int hb_thermostat_create(hb_system *sys, const hb_thermostat_desc *desc, hb_thermostat **out);
int hb_thermostat_destroy(hb_thermostat *t);
/* out[0] cumulative injected energy sum (K' - K) (CSVR, Berendsen), [1] last
 * K, [2] last factor, [3] last sum of squares s, [4] last r, [5] draws,
 * [6] degrees of freedom g. */
int hb_thermostat_stats(hb_thermostat *t, double out[7]);
/* Attach (or detach with NULL) a thermostat; velocity Verlet only. */
int hb_integrator_set_thermostat(hb_integrator *it, hb_thermostat *t);

/* ---- per-step pressure coupling for velocity Verlet: replaces
 * CRescaleBarostat (src/integrator/c_rescale_barostat.rs:60-300,
 * c_rescale_compute_mu in kernels/barostat.cu:140-214) and the Berendsen
 * barostat (src/integrator/berendsen_barostat.rs, berendsen_compute_mu in
 * kernels/barostat.cu:216-255).  Every step evaluates energies and virial;
 * after the constraint velocity projection, P = (2K + W) / 3V with W the
 * force-field virial plus the constraint virial of the step, then
 *   mu^3 = 1 - kappa dt/tau (P0 - P) [+ sqrt(2 kappa kT dt / (tau V)) r]
 * (the noise term for c-rescale, r from Philox counter (draw, 0, 0, 0)),
 * clamped below at 1e-18, the lattice scaled by mu (FP64) and, after the
 * final half kick, every position scaled by mu about the origin.  A step
 * that would take the narrowest perpendicular width below
 * 2 (r_cut + r_skin) keeps mu = 1 and counts a guard. */
#define HB_PCOUPLE_C_RESCALE 0
#define HB_PCOUPLE_BERENDSEN 1
typedef struct {
  int kind;                  /* HB_PCOUPLE_* */
  double pressure;           /* hartree / bohr^3 */
  double temperature;        /* k_B T in hartree (c-rescale noise) */
  double tau;                /* coupling time, a.u. */
  double compressibility;    /* bohr^3 / hartree */
  uint64_t seed;
} hb_pcouple_desc;

int hb_pcouple_create(hb_system *sys, const hb_pcouple_desc *desc, hb_pcouple **out);
int hb_pcouple_destroy(hb_pcouple *p);
/* out[0] last pressure, [1] volume after the last step, [2] cumulative
 * P0 dV, [3] last mu, [4] draws, [5] last K, [6] last W, [7] guarded
 * steps. */
int hb_pcouple_stats(hb_pcouple *p, double out[8]);
/* Attach (or detach with NULL); velocity Verlet only, and not together
 * with a Monte-Carlo barostat. */
int hb_integrator_set_pcouple(hb_integrator *it, hb_pcouple *p);

/* ---- steepest-descent minimisation: replaces SteepestDescentMinimizer
 * (src/minimizer/steepest_descent.rs:123-300, kernels/minimize.cu) and the
 * runner's minimisation loop (src/runner.rs:1804-2140).  An iteration:
 * F_max = max |F_i| (single precision), x += s F / F_max, the constraint
 * groups projected back onto their manifold (position-only Gauss-Seidel with
 * gradients at the current positions; settle_positions_no_velocity /
 * shake_positions_no_velocity), forces + energy; accepted when the energy
 * drops (s = min(s * step_increase, max_step)), else the previous state is
 * restored (s = s * step_decrease).  Convergence: F_max = 0, F_max <=
 * force_tolerance (when > 0), or on an accepted iteration |E - E_prev| <=
 * energy_tolerance max(|E|, |E_prev|, 1e-30) (when > 0).  Every decision is
 * made on the device; a call runs up to n iterations with one host read. */
#define HB_MIN_FORCE_TOLERANCE 1
#define HB_MIN_ENERGY_TOLERANCE 2
#define HB_MIN_FORCE_ZERO 3
typedef struct {
  double initial_step;       /* bohr (> 0) */
  double max_step;           /* bohr (>= initial_step) */
  double step_increase;      /* >= 1 */
  double step_decrease;      /* in (0, 1) */
  double force_tolerance;    /* hartree / bohr; 0 disables */
  double energy_tolerance;   /* relative; 0 disables */
  uint64_t max_iterations;   /* > 0 */
} hb_minimizer_desc;

typedef struct {
  uint64_t iteration;        /* 0: the state before the first iteration */
  double energy;             /* hartree: accepted energy after the iteration */
  double max_force;          /* hartree / bohr at the accepted configuration */
  double step;               /* bohr: the step the iteration tried (0 for 0) */
  int accepted;
  int converged;             /* HB_MIN_* once converged, else 0 */
} hb_min_report;

/* cons may be NULL.  The minimiser evaluates ff (with energies) itself. */
int hb_minimizer_create(hb_forcefield *ff, hb_constraints *cons, const hb_minimizer_desc *desc,
                        hb_minimizer **out);
int hb_minimizer_destroy(hb_minimizer *m);
/* Forces and energy at the current positions; the iteration-0 report. */
int hb_minimizer_begin(hb_minimizer *m, hb_min_report *out);
/* Up to n iterations (stopping at convergence or max_iterations); their
 * reports in out[0 .. *n_done). */
int hb_minimizer_iterate(hb_minimizer *m, uint32_t n, hb_min_report *out, uint32_t *n_done);

/* ---- batched replicas: the runner's captured-graph replay
 * (src/runner.rs:2803-3000, src/gpu/graph.rs:222-242) extended to many
 * independent systems of uneven sizes.  Every member's whole step is
 * captured into ONE CUDA graph, each member on its own parallel branch
 * (the streams of the member's context), so one graph launch advances every
 * system by one step; each member keeps its device-side rebuild decision.
 * Members keep their own force fields, constraints and integrators
 * (velocity Verlet or Langevin; no barostat); members that share a context
 * share its streams and run one after another inside the graph.  cons may
 * be NULL or hold NULL entries.  Members must outlive the batch; a member's
 * list growth (or any capacity change) makes the next call recapture. */
int hb_batch_create(hb_context *ctx, uint32_t n_members, hb_integrator *const *its,
                    hb_forcefield *const *ffs, hb_constraints *const *cons, hb_batch **out);
int hb_batch_destroy(hb_batch *b);
/* n_steps graph launches; the device time is reported by hb_timing_get on
 * the batch's context (out[0]) when timing is enabled there. */
int hb_batch_step(hb_batch *b, uint32_t n_steps);
/* kernels[0] = kernels of one batch step (all members), kernels[1] = sum
 * over members of the kernels of one neighbour rebuild. */
int hb_batch_count_launches(hb_batch *b, uint64_t kernels[2]);
/* Pair-kernel form of a batch step (no reference counterpart; the
 * reference replays one graph per system, src/runner.rs:2803-3000).
 * one_launch != 0: when the members share the pair physics (types, tables,
 * cut-offs, alpha), take force-only steps and each have a context of their
 * own, every member runs its step up to the pair kernel, one persistent
 * pair kernel then covers the work items of all members (each item finds
 * its member in a table), and each member finishes its step after it.
 * one_launch = 0 (the default; about 5 % faster on 64 uneven water boxes,
 * since members that skip a rebuild start their pair kernels without
 * waiting for the others) and members that do not qualify: each member
 * launches its own pair kernel in its graph branch.  Both forms give the
 * same forces bit for bit (integer accumulation).  The next hb_batch_step
 * recaptures. */
int hb_batch_set_pair_form(hb_batch *b, int one_launch);
/* *one_launch = 1 when the next step uses the one-launch form. */
int hb_batch_pair_form(hb_batch *b, int *one_launch);

/* ---- FP64 deterministic scalar reductions (kernels/nose_hoover.cu:22-103,
 * kernels/barostat.cu:11-78): kinetic energy and the mass-weighted
 * velocity sum. out[0] = KE, out[1..3] = total momentum. */
int hb_reduce_kinetic(hb_system *sys, double out[4]);

/* ---- allocation-free SPME reciprocal evaluation.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory --
 * a process whose device memory belongs to another allocator (a framework's
 * caching pool, a fixed-budget serving process), where a cudaMalloc would
 * take memory that allocator counts on, and cudaMalloc / cudaFree would
 * stall the device.
 *
 * posq: device [4n] floats (x, y, z, q) in any atom order; out: device
 * [4n] floats receiving (fx, fy, fz, per-atom energy share 1/2 q phi -
 * alpha/sqrt(pi) q^2) of the reciprocal part; energy: host pointer for the
 * FP64 reciprocal energy, or NULL (non-NULL synchronises the stream);
 * stream: a cudaStream_t, or NULL for the legacy default stream.
 *
 * Limits: at most 64 grid points per axis and 32768 in total (e.g. 32^3);
 * larger grids are rejected with HB_ERR_INVALID_GRID.  All scratch lives in
 * one file-scope device array (about 0.7 MB) that every GPU loading the
 * library holds until the process exits; the call allocates nothing.  The
 * first call on a device looks up that array's address (cudaGetSymbolAddress)
 * and caches it for the device's primary context: make that first call
 * before any stream capture, and make no call after cudaDeviceReset (the
 * cached address would be stale).  Every call shares the one array, which
 * keeps the last call's contents (each call clears what must start at
 * zero), so calls whose GPU work overlaps (different streams or threads)
 * race; serialise them. */
int hb_spme_recip_noalloc(const float *posq, uint32_t n, const double box[6],
                          const uint32_t grid[3], uint32_t order, double alpha,
                          float *out, double *energy, void *stream);

/* ---- device timing of the last hb_integrator_step call, in ms:
 * out[0] total, out[1] pair kernel (sum), out[2] SPME (sum), out[3]
 * neighbour rebuilds (sum), out[4] integrator + constraints (sum);
 * instrumentation is on when enable != 0. */
int hb_timing_enable(hb_context *ctx, int enable);
int hb_timing_get(hb_context *ctx, double out[8]);

#ifdef __cplusplus
}
#endif
#endif /* HEDDLE_B200_H */
