// hb_internal.cuh -- shared types and device helpers of the B200-native
// HeddleMD force-and-constraint path.  Everything here is internal to
// libheddle_b200.so; the public surface is include/heddle_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/heddle_b200.h"

// ---------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------
void hb_set_error(const std::string &msg);
int hb_fail(int code, const std::string &msg);

#define HB_CUDA(call)                                                       \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      return hb_fail(HB_ERR_CUDA, std::string(#call) + ": " +               \
                                      cudaGetErrorString(e_));              \
    }                                                                       \
  } while (0)

#define HB_REQUIRE(cond, code, msg)               \
  do {                                            \
    if (!(cond)) return hb_fail((code), (msg));   \
  } while (0)

#define HB_TRY(call)                                                        \
  do {                                                                      \
    int r_ = (call);                                                        \
    if (r_ != HB_OK) return r_;                                             \
  } while (0)

// fixed-point scales: pair/recip force, energy and virial accumulate as
// two's-complement int64 with 2^40 fractional bits (resolution 9.1e-13,
// range +-8.4e6 in atomic units); the SPME charge grid uses 2^32 as the
// reference's spread does (kernels/spme_spread_gather.cuh:31).
#define HB_FP_SCALE 1099511627776.0f        /* 2^40 */
#define HB_FP_INV_SCALE (1.0 / 1099511627776.0)
#define HB_RHO_SCALE 4294967296.0f          /* 2^32 */
#define HB_N_SCALARS 10                     /* doubles of hb_forcefield_scalars */
/* largest isotropic lattice scaling |mu - 1| since the last neighbour
 * rebuild under which the list is kept (the tile boxes carry this margin) */
#define HB_BOX_SLACK 0.01f
#define HB_XFIX_SCALE 1099511627776.0       /* 2^40 per bohr */
#define HB_VFIX_SCALE 72057594037927936.0   /* 2^56 per bohr / aut */

#define HB_TILE 32
#define HB_SENTINEL 0xFFFFFFFFu

// status word bits (kernels/neighbor.cu:634-669 layout, plus build bits)
#define HB_ST_DISPLACED 1u        /* an atom moved more than r_skin / 2 */
#define HB_ST_ENTRY_OVERFLOW 8u   /* entry capacity exceeded on a rebuild */
#define HB_ST_ENTRY_HIGHWATER 2u  /* entry count above 3/4 of capacity */
#define HB_ST_DEVICE_TIMEOUT 16u  /* a bounded wait of the tile build ran out */

// ---------------------------------------------------------------------
// device box: lattice plus reciprocal helpers, kept in device memory so a
// barostat can change it inside a captured graph
// ---------------------------------------------------------------------
struct DBox {
  float lx, ly, lz, xy, xz, yz;
  float ilx, ily, ilz;   // 1 / lx etc.
  int ortho;             // xy == xz == yz == 0
};

// Operation-by-operation single-precision minimum image, no contraction:
// the membership rule of the neighbour set (same operation order as the
// reference's kernels/pbc.cuh:18-43).  Used only where exactness matters.
__device__ __forceinline__ float hb_exact_r2(float dx, float dy, float dz,
                                             const DBox &b) {
  float sc = __fdiv_rn(dz, b.lz);
  float sb = __fdiv_rn(__fsub_rn(dy, __fmul_rn(sc, b.yz)), b.ly);
  float sa = __fdiv_rn(
      __fsub_rn(__fsub_rn(dx, __fmul_rn(sb, b.xy)), __fmul_rn(sc, b.xz)), b.lx);
  float ka = floorf(__fadd_rn(sa, 0.5f));
  float kb = floorf(__fadd_rn(sb, 0.5f));
  float kc = floorf(__fadd_rn(sc, 0.5f));
  dx = __fsub_rn(dx, __fadd_rn(__fadd_rn(__fmul_rn(ka, b.lx), __fmul_rn(kb, b.xy)),
                               __fmul_rn(kc, b.xz)));
  dy = __fsub_rn(dy, __fadd_rn(__fmul_rn(kb, b.ly), __fmul_rn(kc, b.yz)));
  dz = __fsub_rn(dz, __fmul_rn(kc, b.lz));
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)),
                   __fmul_rn(dz, dz));
}

// fast minimum image (contraction allowed) for force arithmetic
__device__ __forceinline__ void hb_min_image(float &dx, float &dy, float &dz,
                                             const DBox &b) {
  float sc = dz * b.ilz;
  float sb = (dy - sc * b.yz) * b.ily;
  float sa = (dx - sb * b.xy - sc * b.xz) * b.ilx;
  float ka = rintf(sa), kb = rintf(sb), kc = rintf(sc);
  dx -= ka * b.lx + kb * b.xy + kc * b.xz;
  dy -= kb * b.ly + kc * b.yz;
  dz -= kc * b.lz;
}

// wrap into the primary cell [-1/2, 1/2)^3 (fractional) and return the
// image triple (kernels/pbc.cuh:73-91 semantics)
__device__ __forceinline__ void hb_wrap(float &x, float &y, float &z, int &ka,
                                        int &kb, int &kc, const DBox &b) {
  float sc = z / b.lz;
  float sb = (y - sc * b.yz) / b.ly;
  float sa = (x - sb * b.xy - sc * b.xz) / b.lx;
  float fa = floorf(sa + 0.5f), fb = floorf(sb + 0.5f), fc = floorf(sc + 0.5f);
  x -= fa * b.lx + fb * b.xy + fc * b.xz;
  y -= fb * b.ly + fc * b.yz;
  z -= fc * b.lz;
  ka = (int)fa;
  kb = (int)fb;
  kc = (int)fc;
}

// Philox-4x32-10 (Salmon et al. 2011) as kernels/philox.cuh and
// src/integrator/philox.rs:21-50 use it: key (k0, k1), counter (c0..c3);
// returns the first two output words.
__host__ __device__ inline void hb_philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                                          uint32_t c2, uint32_t c3, uint32_t &o0,
                                          uint32_t &o1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)c0 * 0xD2511F53u, p2 = (uint64_t)c2 * 0xCD9E8D57u;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi2 = (uint32_t)(p2 >> 32), lo2 = (uint32_t)p2;
    const uint32_t n0 = hi2 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo2;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  o0 = c0;
  o1 = c1;
}

#ifdef __CUDACC__
// Box-Muller cosine branch on the first two words, u = (x + 1/2) 2^-32
// (kernels/philox.cuh:135-150), evaluated in single precision.
__device__ __forceinline__ float hb_gaussian(uint32_t s_lo, uint32_t s_hi, uint64_t step,
                                             uint32_t atom, uint32_t axis) {
  uint32_t o0, o1;
  hb_philox(s_lo, s_hi, (uint32_t)step, (uint32_t)(step >> 32), atom, axis, o0, o1);
  const float u1 = ((float)(o0 >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float u2 = ((float)(o1 >> 8) + 0.5f) * (1.0f / 16777216.0f);
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Langevin middle scheme, per atom (kernels/langevin.cu:13-80): the full
// kick v += F dt / m ...
__device__ __forceinline__ void hb_lang_kick(float4 &v, const float4 &f, float dt) {
  const float h = dt * v.w;
  v.x += f.x * h;
  v.y += f.y * h;
  v.z += f.z * h;
}

// ... and half drift, O step (friction factor a, k_B T, the atom's Philox
// stream at the step's draw counter), half drift and the wrap into the
// cell with the image counts carried
__device__ __forceinline__ void hb_lang_drift_ou(float4 &p, float4 &v, int4 &im, float dt,
                                                 float a, float kt, uint32_t s_lo, uint32_t s_hi,
                                                 uint64_t step, uint32_t i, const DBox &b) {
  const float hdt = 0.5f * dt;
  p.x += v.x * hdt;
  p.y += v.y * hdt;
  p.z += v.z * hdt;
  const float sig = sqrtf((1.0f - a * a) * kt * v.w);
  v.x = a * v.x + sig * hb_gaussian(s_lo, s_hi, step, i, 0u);
  v.y = a * v.y + sig * hb_gaussian(s_lo, s_hi, step, i, 1u);
  v.z = a * v.z + sig * hb_gaussian(s_lo, s_hi, step, i, 2u);
  p.x += v.x * hdt;
  p.y += v.y * hdt;
  p.z += v.z * hdt;
  int ka, kb, kc;
  hb_wrap(p.x, p.y, p.z, ka, kb, kc, b);
  im.x += ka;
  im.y += kb;
  im.z += kc;
}
#endif

// lower-triangular lattice (lx, ly, lz, xy, xz, yz) -> the single-precision
// box the kernels read
__host__ __device__ inline DBox hb_make_dbox(const double b[6]) {
  DBox d;
  d.lx = (float)b[0];
  d.ly = (float)b[1];
  d.lz = (float)b[2];
  d.xy = (float)b[3];
  d.xz = (float)b[4];
  d.yz = (float)b[5];
  d.ilx = (float)(1.0 / b[0]);
  d.ily = (float)(1.0 / b[1]);
  d.ilz = (float)(1.0 / b[2]);
  d.ortho = (b[3] == 0.0 && b[4] == 0.0 && b[5] == 0.0) ? 1 : 0;
  return d;
}

// perpendicular widths of the cell spanned by a = (lx,0,0), b = (xy,ly,0),
// c = (xz,yz,lz): volume / |b x c|, volume / |c x a|, volume / |a x b|
__host__ __device__ inline void hb_perp_widths(const double b[6], double w[3]) {
  const double ax = b[0], bx = b[3], by = b[1], cx = b[4], cy = b[5], cz = b[2];
  const double vol = ax * by * cz;
  // b x c, c x a, a x b with a = (ax,0,0), b = (bx,by,0), c = (cx,cy,cz)
  const double bc0 = by * cz, bc1 = -bx * cz, bc2 = bx * cy - by * cx;
  const double ca1 = cz * ax, ca2 = -cy * ax;
  const double ab2 = ax * by;
  w[0] = vol / sqrt(bc0 * bc0 + bc1 * bc1 + bc2 * bc2);
  w[1] = vol / sqrt(ca1 * ca1 + ca2 * ca2);
  w[2] = vol / sqrt(ab2 * ab2);
}

__device__ __forceinline__ void hb_frac(float x, float y, float z,
                                        const DBox &b, float &sa, float &sb,
                                        float &sc) {
  sc = z / b.lz;
  sb = (y - sc * b.yz) / b.ly;
  sa = (x - sb * b.xy - sc * b.xz) / b.lx;
}

// ---------------------------------------------------------------------
// host-side objects
// ---------------------------------------------------------------------
struct hb_context {
  int device = 0;
  int n_sm = 148;
  cudaStream_t stream = nullptr;    // main stream
  cudaStream_t stream2 = nullptr;   // SPME runs here, overlapping the pair kernel
  cudaStream_t stream3 = nullptr;   // captures the bodies of conditional graph nodes
  cudaStream_t stream4 = nullptr;   // host read-out overlapping a step's force evaluation
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_xfork = nullptr, ev_xjoin = nullptr;
  bool timing = false;
  // stage timers (accumulated over the last hb_integrator_step call)
  std::vector<cudaEvent_t> tev;
  double t_ms[8] = {0};
};

struct hb_system {
  hb_context *ctx = nullptr;
  uint32_t n = 0;
  double box[6] = {0};            // host mirror of d_box64 (refresh before use)
  double *d_box64 = nullptr;       // [6] FP64 lattice, the authoritative box
  DBox *d_box = nullptr;           // single-precision view of d_box64
  float4 *d_posq = nullptr;      // x, y, z, q (wrapped into the primary cell)
  float4 *d_vel = nullptr;       // vx, vy, vz, 1/m
  int4 *d_image = nullptr;       // image counts a, b, c, type
  float4 *d_force = nullptr;     // fx, fy, fz, 0 (total force, atom order)
  float4 *d_pos_prev = nullptr;  // pre-drift positions (constraint snapshot)
  // lossless mode: the state as 64-bit fixed point ([3n] each), positions
  // in 2^-40 bohr, velocities in 2^-56 bohr/aut; the f32 posq / vel are
  // derived from it.  fix_valid: the fixed state mirrors posq / vel (any
  // other writer of positions or velocities clears it).
  long long *d_xfix = nullptr;
  long long *d_vfix = nullptr;
  bool fix_valid = false;
  std::vector<double> h_mass;
  std::vector<double> h_charge;
  std::vector<uint32_t> h_type;
  // FP64 reduction scratch
  double *d_red = nullptr;       // partials
  double *h_red = nullptr;       // pinned
  // state transfer staging (allocated at the first set_state / get_state):
  // [3n] positions, [3n] velocities, [3n] forces as FP64, [3n] images, and
  // the first non-finite atom index of an upload
  double *d_stage = nullptr;
  int32_t *d_stage_img = nullptr;
  uint32_t *d_bad = nullptr;
};

// SPME reciprocal state
struct SpmeState {
  int on = 0;
  int na = 0, nb = 0, nc = 0, nch = 0, order = 4;
  float alpha = 0.f;
  unsigned long long *d_rho_fixed = nullptr;  // [na*nb*nc] int64 grid
  float2 *d_grid = nullptr;                   // [na*nb*nch] complex
  float *d_v = nullptr;                       // [na*nb*nc] real potential
  float *d_bfac = nullptr;                    // b-factors a | b | c
  float2 *d_tw = nullptr;                     // twiddles a | b | c
  double *d_part = nullptr;                   // energy / virial partials
  int n_part = 0;
  int use_plane = 0;                          // kc-major planes + whole-plane pass
  int gather_c = 1;                           // orders 4, 8: thread per (atom, c offset)
  double *d_sums = nullptr;                   // [2] E_recip, W_recip
  float4 *d_recip = nullptr;                  // per sorted atom fx, fy, fz, e
  float self_pref = 0.f;                      // alpha / sqrt(pi)
};

struct hb_shake_mlp;

// process-wide creation counter: objects that captured graphs refer to are
// compared by this id, never by address (a freed object's address can be
// reused by a new one)
uint64_t hb_next_uid();

struct hb_forcefield {
  hb_system *sys = nullptr;
  uint64_t uid = hb_next_uid();
  // ---- parameters
  int lj_on = 0, coul_on = 0;
  uint32_t n_types = 0;
  std::vector<float4> h_lj;        // per type pair: sigma^2, 24 eps, cut^2, r_switch^2
  float4 *d_lj = nullptr;
  float *d_lj_invd = nullptr;      // per type pair: 1 / (cut^2 - r_switch^2) (0: no switch)
  float alpha = 0.f, coul_rc2 = 0.f;
  bool exact_pairs = false;        // per-pair fixed point and minimum image (lossless mode)
  float rc_max = 0.f, r_skin = 0.f, r_search = 0.f;
  int any_switch = 0;
  int excl_scaled = 0;             // some exclusion has a non-zero scale
  uint32_t *d_excl_off = nullptr;  // CSR over original ids
  uint32_t *d_excl_partner = nullptr;
  float2 *d_excl_scale = nullptr;  // (lj, coulomb)
  uint32_t n_excl = 0;
  // ---- neighbour list (sorted-index space)
  uint32_t n_tiles = 0, n_pad = 0;
  int nv_log2 = 5;                 // voxel grid 2^nv_log2 per axis
  uint32_t *d_vox_key = nullptr;   // per atom
  uint32_t *d_vox_count = nullptr; // per voxel (+1)
  uint32_t *d_vox_off = nullptr;
  uint32_t *d_scan_tmp = nullptr;
  uint32_t *d_sorted_ids = nullptr;  // sorted slot -> atom id (pad = sentinel)
  uint32_t *d_inv_perm = nullptr;    // atom id -> sorted slot
  float4 *d_tile_posq = nullptr;     // positions in sorted order
  int *d_tile_type = nullptr;
  float4 *d_tile_center = nullptr;   // per tile: centre xyz, spc flag in w
  float4 *d_tile_half = nullptr;     // per tile: half extents
  uint32_t *d_tile_nent = nullptr;   // entries held by each tile
  uint32_t slab = 0;                 // entry capacity per tile
  uint32_t maxc = 1024;              // candidate j-tiles per i-tile (shared memory)
  uint32_t *d_entry_j = nullptr;     // [n_tiles * slab * 32] sorted j slots
  uint32_t *d_entry_excl = nullptr;  // [n_tiles * slab * 32] exclusion masks
  uint64_t entry_cap = 0;            // n_tiles * slab
  uint32_t reallocations = 0;        // slab (re)allocations after the first
  uint64_t layout_gen = 0;           // bumped when list buffers or sizes change:
                                     // captured graphs older than it are stale
  float4 *d_ref_pos = nullptr;       // positions at the last rebuild
  DBox *d_ref_box = nullptr;         // box at the last rebuild
  uint32_t *d_status = nullptr;      // status word
  uint32_t *d_counters = nullptr;    // [0] rebuilds, [1] entries of the last
                                     // build, [2] running count of a build,
                                     // [3] largest candidate count seen
  uint32_t *h_status = nullptr;      // pinned mirror
  int pair_blocks_per_sm = 8;        // persistent pair kernel residency (tunable)
  int pair_chunk = 4;                // packed entries per pair work item (tunable)
  int pair_quota = 0;                // work items per pair warp (0: persistent; tunable)
  uint32_t nl_polls = 1u << 20;      // poll limit of the tile build's bounded waits
  uint32_t nl_issue = 1;             // 0 (test only): issue no bulk copies, so the waits run out
  uint32_t *d_work = nullptr;        // work counter of the balanced pair kernel
                                     // (zeroed by the combine kernel)
  uint64_t rebuilds_host = 0;
  bool built = false;
  // ---- accumulators (sorted-slot space)
  unsigned long long *d_fp = nullptr;  // [5][n_pad]: fx fy fz e w
  // ---- SPME
  SpmeState spme;
  // ---- scalars
  double *d_scalars = nullptr;       // [HB_N_SCALARS]
  unsigned long long *d_acc = nullptr;  // int64 totals: [0] LJ energy, [1] pair +
                                        // bonded energy, [2] pair + bonded virial,
                                        // [3] bonded energy
  // ---- bonded terms (per term: atoms and parameters)
  uint32_t n_bonds = 0, n_angles = 0, n_dihedrals = 0;
  uint2 *d_bond_atoms = nullptr;
  float2 *d_bond_par = nullptr;      // k, r0
  uint4 *d_angle_atoms = nullptr;    // i, j (vertex), k
  float2 *d_angle_par = nullptr;     // k, theta0
  uint4 *d_dih_atoms = nullptr;      // i, j, k, l
  float4 *d_dih_par = nullptr;       // k, phi0, n
  double h_scalars[HB_N_SCALARS] = {0};
  float *d_energy = nullptr;         // per atom (atom order)
  float *d_virial = nullptr;
};

struct hb_constraints {
  hb_system *sys = nullptr;
  uint64_t uid = hb_next_uid();
  uint32_t n_settle = 0, n_shake = 0;
  // SETTLE: per group (O, H1, H2) atom ids and geometry
  uint4 *d_settle_atoms = nullptr;   // o, h1, h2, 0
  float4 *d_settle_geom = nullptr;   // ra, rb, rc, 0
  float2 *d_settle_mass = nullptr;   // m_o, m_h
  // SHAKE: per group CSR
  uint32_t *d_shake_aoff = nullptr, *d_shake_atoms = nullptr;
  uint32_t *d_shake_coff = nullptr;
  uint2 *d_shake_pairs = nullptr;    // local i, j
  double *d_shake_d2 = nullptr;
  double shake_tol = 3.57e-6;
  int shake_rel = 0;                 // tolerance relative to d^2
  uint32_t shake_max_iter = 32;
  uint32_t n_shake_cons = 0;         // constraints of the SHAKE groups
  // learned warm start and its training data (per SHAKE constraint)
  hb_shake_mlp *mlp = nullptr;       // warm start when set
  bool record = false;               // write features and converged multipliers
  bool fuse_head = true;             // Langevin head in one kernel where it applies
  float *d_feat = nullptr;           // [n_shake_cons * 8]
  double *d_lam1 = nullptr;          // first Gauss-Seidel multiplier
  double *d_lsc = nullptr;           // multiplier -> sigma-unit scale
  double *d_lam = nullptr;           // converged total multiplier
  float *d_pred = nullptr;           // network output
  unsigned long long *d_stats = nullptr;  // [0] group-sweeps, [1] group solves
  uint32_t n_slots = 0;
  float *d_virial = nullptr;         // per atom
  uint32_t *d_iters = nullptr;       // max sweeps of the last SHAKE call
};

struct hb_integrator {
  hb_system *sys = nullptr;
  int kind = HB_INTEGRATOR_VV;
  double dt = 0.0, friction = 0.0, temperature = 0.0;
  uint64_t seed = 0, step = 0;
  uint64_t *d_step = nullptr;   // Philox draw counter read by the O step
  uint32_t *d_done = nullptr;   // completion counter of the fused Langevin + SETTLE head
  bool forces_valid = false;
  // graph mode
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t g_ev0 = nullptr, g_ev1 = nullptr;
  uint64_t graph_ff = 0;        // uids of the objects the graphs were captured with
  uint64_t graph_cons = 0;
  uint64_t graph_gen = 0;       // the force field's layout_gen at capture
  // Monte-Carlo barostat attached to the step loop (may be null) and the
  // graph of a step that ends with a volume move
  hb_barostat *baro = nullptr;
  cudaGraphExec_t graph_exec_move = nullptr;
  uint64_t graph_baro = 0;
  // velocity thermostat and per-step pressure coupling (velocity Verlet)
  hb_thermostat *thermo = nullptr;
  hb_pcouple *pc = nullptr;
  uint64_t graph_thermo = 0, graph_pc = 0;
  // exchange steps (hb_integrator_step_exchange_f32): the last step of a
  // call as a graph that also copies the state into page-locked host arrays
  // (with and without a volume move), captured for one set of host pointers
  cudaGraphExec_t graph_exec_x = nullptr, graph_exec_x_move = nullptr;
  const void *graph_x_key[4] = {nullptr, nullptr, nullptr, nullptr};
};

// Device-resident state of the Monte-Carlo barostat (FP64).  The whole move
// -- draw, proposal, trial force evaluation, Metropolis test, revert and
// step-size adaptation -- runs on the device with no host read.
struct BaroState {
  double lattice_pre[6];   // lattice before the trial
  double scalars_pre[HB_N_SCALARS];  // force-field scalars before the trial
  double max_dv;           // current maximum volume displacement
  double u_old, u_new, dv, v_old, v_new, scale, u1, u2, w;
  double injection;        // sum of P dV over accepted moves
  double volume;           // volume after the last move
  unsigned long long draw, attempted, accepted;
  unsigned int win_attempted, win_accepted;
  int trial, last_accepted;
};

struct hb_barostat {
  hb_system *sys = nullptr;
  uint64_t uid = hb_next_uid();
  double pressure = 0.0, kt = 0.0;
  uint32_t frequency = 25;
  uint64_t seed = 0;
  uint32_t n_mol = 0;
  uint32_t *d_mol_off = nullptr;     // [n_mol + 1]
  uint32_t *d_mol_atoms = nullptr;   // [n]
  double *d_mass = nullptr;          // [n] FP64 masses
  BaroState *d_state = nullptr;
  float4 *d_snap_pos = nullptr;      // pre-move positions, images, forces
  int4 *d_snap_img = nullptr;
  float4 *d_snap_force = nullptr;
};

// Device-resident state of a thermostat or a pressure coupling (FP64), so
// a captured step reads and advances it with no host work.
struct CoupleState {
  double injection;        // thermostat: sum (K' - K); pressure: sum P0 dV
  double k, factor, s, r;  // last kinetic energy, rescale factor, sum xi^2, r
  double pressure, volume, w, mu;
  unsigned long long draws, guarded;
};

struct hb_thermostat {
  hb_system *sys = nullptr;
  uint64_t uid = hb_next_uid();
  int kind = 0;
  double kt = 0.0, tau = 0.0, rate = 0.0;
  uint64_t seed = 0;
  uint32_t g_dof = 1;
  CoupleState *d_st = nullptr;
  double *d_part = nullptr;   // per-block partial sums of the CSVR draw
};

struct hb_pcouple {
  hb_system *sys = nullptr;
  uint64_t uid = hb_next_uid();
  int kind = 0;
  double pressure = 0.0, kt = 0.0, tau = 0.0, kappa = 0.0;
  uint64_t seed = 0;
  CoupleState *d_st = nullptr;
  double *d_part = nullptr;   // partial sums of the constraint virial
};

// Device state of the steepest-descent minimiser (hb_min.cu)
struct MinState {
  double last_energy;      // energy of the accepted configuration
  double prev_energy;      // accepted energy before the current iteration
  double e_trial;
  float step, step_used, fmax, scale;
  int skip, reject, converged, pad;
  unsigned long long iteration;
};

struct hb_minimizer {
  hb_forcefield *ff = nullptr;
  hb_constraints *cons = nullptr;
  float initial_step = 0.f, max_step = 0.f, inc = 1.f, dec = 0.5f;
  double ftol = 0.0, etol = 0.0;
  uint64_t max_iter = 0, done = 0;
  bool begun = false;
  int converged = 0;
  MinState *d_st = nullptr;
  hb_min_report *d_rep = nullptr;   // [rep_cap] reports of the current call
  uint32_t rep_cap = 256;
  float *d_part = nullptr;          // per-block |F|^2 maxima
  float4 *d_snap_pos = nullptr, *d_snap_force = nullptr;
  int4 *d_snap_img = nullptr;
  double *d_snap_scal = nullptr;
};

// ---------------------------------------------------------------------
// internal entry points implemented across the translation units
// ---------------------------------------------------------------------
// neighbour list (hb_nlist.cu)
int nl_setup(hb_forcefield *ff);
int nl_free(hb_forcefield *ff);
// Rebuild the list.  gated: kernels run only when the status word has the
// displacement bit set (a device-side decision, no host read).
int nl_rebuild(hb_forcefield *ff, bool gated, cudaStream_t s);
int nl_kernel_count();
// During stream capture: the rebuild as a device-side conditional graph node.
int nl_rebuild_conditional(hb_forcefield *ff, cudaStream_t s);
int nl_displacement_check(hb_forcefield *ff, cudaStream_t s);
int nl_gather_positions(hb_forcefield *ff, cudaStream_t s);
int nl_first_build(hb_forcefield *ff);
int nl_set_slab(hb_forcefield *ff, uint32_t slab);
int nl_pairs(hb_forcefield *ff, std::vector<uint32_t> &pairs, uint64_t &dups);
// bonded terms (hb_bonded.cu): fixed-point adds into fp (sorted slots)
int bonded_setup(hb_forcefield *ff, const hb_forcefield_desc *d);
int bonded_free(hb_forcefield *ff);
int bonded_launch(hb_forcefield *ff, bool ev, cudaStream_t s);
// pair kernel (hb_pair.cu)
int pair_launch(hb_forcefield *ff, bool ev, cudaStream_t s);
// SPME (hb_spme.cu)
int spme_setup(hb_forcefield *ff, const hb_forcefield_desc *d);
int spme_free(hb_forcefield *ff);
int spme_launch(hb_forcefield *ff, bool ev, cudaStream_t s);
// multi-system pair launch of replica batches (hb_pair.cu)
size_t pair_member_bytes();
bool pair_batchable(hb_forcefield *const *ffs, uint32_t n);
int pair_batch_table(hb_forcefield *const *ffs, uint32_t n, void *d_table, uint32_t *items_total);
int pair_launch_batch(hb_forcefield *const *ffs, uint32_t n, const void *d_table,
                      uint32_t items_total, uint32_t *d_work, cudaStream_t s);
// HB_LAUNCH_FFT_PLANE / HB_LAUNCH_GATHER_FORM (hb_forcefield_set_launch)
int spme_set_form(hb_forcefield *ff, int param, int value);
// combine (hb_integ.cu): fixed-point + reciprocal -> force (atom order)
int forces_finalize(hb_forcefield *ff, bool ev, cudaStream_t s);
int scalars_reduce(hb_forcefield *ff, cudaStream_t s);
// integrators (hb_integ.cu)
int integ_vv_kick_drift(hb_integrator *it, cudaStream_t s);
int integ_vv_kick(hb_integrator *it, cudaStream_t s);
int integ_lang_kick(hb_integrator *it, cudaStream_t s);
int integ_lang_drift_ou(hb_integrator *it, cudaStream_t s);
int reduce_kinetic(hb_system *sys, double out[4]);
// the same reduction left on the device: [0] kinetic energy, [1..3] momentum
int reduce_kinetic_device(hb_system *sys, cudaStream_t s, const double **d_out);
// thermostat / pressure coupling of a velocity-Verlet step (hb_couple.cu):
// the factors after the velocity projection, then the final half kick with
// the rescale, Andersen collisions and position scaling fused in
int couple_prepare(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, cudaStream_t s);
int couple_final_kick(hb_integrator *it, cudaStream_t s);
int integ_flip_velocities(hb_system *sys, cudaStream_t s);
// lossless mode: fixed-point state from posq / vel (and posq / vel snapped to it)
int integ_fix_derive(hb_system *sys, cudaStream_t s);
// system (hb_api.cu): copy the device FP64 lattice into the host mirror
int sys_refresh_box(hb_system *sys);
// Monte-Carlo barostat (hb_baro.cu): propose + scale, then (after a force
// evaluation with scalars) decide + revert
int baro_propose(hb_barostat *b, hb_forcefield *ff, cudaStream_t s);
int baro_decide(hb_barostat *b, hb_forcefield *ff, cudaStream_t s);
// learned SHAKE warm start (hb_mlp.cu): network on device features
int mlp_infer(hb_shake_mlp *m, const float *d_feat, uint32_t n, float *d_out, cudaStream_t s);
int mlp_status(hb_shake_mlp *m);
// constraints (hb_cons.cu)
int cons_positions(hb_constraints *c, double dt, cudaStream_t s);
int cons_velocities(hb_constraints *c, double dt, bool virial, cudaStream_t s);
// Langevin head (kick, velocity projection, drift / O / drift, position
// reset) in one kernel when every atom is in a SETTLE water and there is no
// SHAKE group
bool cons_lang_head_fusable(const hb_constraints *c);
int cons_lang_settle_head(hb_constraints *c, float dt, float a, float kt, uint32_t s_lo,
                          uint32_t s_hi, uint64_t *d_step, uint32_t *d_done, cudaStream_t s);
// position-only projection (minimiser); skip: optional device no-op flag
int cons_project(hb_constraints *c, const int *skip, cudaStream_t s);
// steepest descent (hb_min.cu): warm-up report, trial step, decision + report
int min_alloc(hb_minimizer *m);
void min_free(hb_minimizer *m);
int min_init(hb_minimizer *m, cudaStream_t s);
int min_trial(hb_minimizer *m, cudaStream_t s);
int min_finish(hb_minimizer *m, uint32_t slot, cudaStream_t s);

static inline unsigned int hb_div_up(uint64_t a, uint64_t b) {
  return (unsigned int)((a + b - 1) / b);
}
