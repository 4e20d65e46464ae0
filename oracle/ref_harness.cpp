// Launcher for the reference's own CUDA force path (test infrastructure).
//
// Loads the cubins that oracle/ref_build.py compiles from the reference's
// kernels/*.cu and its regenerated composed pair kernel, and replays the
// reference's per-step launch sequence on given inputs:
//
//   neighbour rebuild  NeighborListState::rebuild_impl + rebuild_packed_neighbour
//                      (src/forces/neighbor_list.rs:945-1262), launch shapes of
//                      src/gpu/kernels.rs:1741-2260 (256-thread blocks; 4 warps
//                      per block for find_blocks_with_interactions, 8 for the
//                      block boxes and the entry scatter)
//   pair forces        ForceField::run (src/forces/mod.rs:757-1020): tile-order
//                      position scatter + padding, the composed _f/_fev kernel
//                      (one 256-thread block per i-block), the single-pair kernel
//                      over the single-pair capacity, finalize_packed_forces
//   SPME reciprocal    SpmeReciprocalGrid::compute (src/forces/spme.rs:391-480)
//                      and SpmeReciprocalState::compute (:858-900): influence
//                      function every step, atom bin sort after a rebuild,
//                      fixed-point spread, cuFFT R2C / C2R (src/gpu/cufft.rs:
//                      110-135), apply_influence, reduce_partials (scale 0.5/N),
//                      order-specialised gather
//   combine            combine_class_totals (kernels/forces.cu)
//   SETTLE             settle_snapshot + settle_positions (kernels/settle.cu,
//                      hooks src/integrator/settle.rs:313-370)
//
// Buffers hold the reference's layouts (SoA Real arrays, i64 fixed point);
// Real is float (the reference's default build).  Only tests and the
// bench's reference-CUDA timing use this library.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;
std::string g_dir;
std::map<std::string, CUmodule> g_mods;

int fail(const std::string &m) {
  g_err = m;
  return 1;
}

#define CU(x)                                                                   \
  do {                                                                          \
    CUresult r_ = (x);                                                          \
    if (r_ != CUDA_SUCCESS) {                                                   \
      const char *s_ = nullptr;                                                 \
      cuGetErrorString(r_, &s_);                                                \
      return fail(std::string(#x) + ": " + (s_ ? s_ : "?"));                    \
    }                                                                           \
  } while (0)
#define RT(x)                                                                   \
  do {                                                                          \
    cudaError_t r_ = (x);                                                       \
    if (r_ != cudaSuccess) return fail(std::string(#x) + ": " + cudaGetErrorString(r_)); \
  } while (0)
#define FFT(x)                                                                  \
  do {                                                                          \
    cufftResult r_ = (x);                                                       \
    if (r_ != CUFFT_SUCCESS) return fail(std::string(#x) + ": cufft " + std::to_string((int)r_)); \
  } while (0)
#define TRY(x)                                                                  \
  do {                                                                          \
    if ((x) != 0) return 1;                                                     \
  } while (0)

int module(const std::string &name, CUmodule *out) {
  auto it = g_mods.find(name);
  if (it != g_mods.end()) {
    *out = it->second;
    return 0;
  }
  CUmodule m;
  std::string path = g_dir + "/" + name + ".cubin";
  CU(cuModuleLoad(&m, path.c_str()));
  g_mods[name] = m;
  *out = m;
  return 0;
}

int func(const std::string &mod, const char *name, CUfunction *f) {
  CUmodule m;
  TRY(module(mod, &m));
  CU(cuModuleGetFunction(f, m, name));
  return 0;
}

// Launch with by-value arguments; the addresses of the parameters stay
// valid for the duration of cuLaunchKernel, which copies them.
template <class... A>
int launch(CUfunction f, unsigned grid, unsigned block, cudaStream_t s, A... a) {
  if (grid == 0) return 0;
  void *params[] = {(void *)&a...};
  CU(cuLaunchKernel(f, grid, 1, 1, block, 1, 1, 0, (CUstream)s, params, nullptr));
  return 0;
}

unsigned cdiv(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

template <class T>
int dalloc(T **p, size_t count) {
  RT(cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1)));
  RT(cudaMemset(*p, 0, sizeof(T) * std::max<size_t>(count, 1)));
  return 0;
}

// lengths of the block-total levels of the recursive scan
// (src/forces/neighbor_list.rs:1611-1624)
std::vector<uint32_t> scan_levels(uint32_t len) {
  std::vector<uint32_t> out;
  for (;;) {
    uint32_t blocks = (len + 255u) / 256u;
    out.push_back(blocks);
    if (blocks <= 1u) break;
    len = blocks;
  }
  return out;
}

// cardinal B-spline M_p(x) by the Cox-de Boor recursion and the squared
// structure-factor moduli of Essmann et al. (1995), eq. 4.4, with near-zero
// moduli (odd orders) replaced by the mean of their periodic neighbours, as
// compute_b_factors does (src/forces/spme.rs:524-585)
double bspline(int p, double x) {
  std::vector<double> v(p);
  for (int i = 0; i < p; ++i) v[i] = (x - i >= 0.0 && x - i < 1.0) ? 1.0 : 0.0;
  for (int k = 2; k <= p; ++k) {
    double inv = 1.0 / (k - 1.0);
    for (int i = 0; i + k <= p; ++i) {
      double xi = x - i;
      v[i] = xi * inv * v[i] + (k - xi) * inv * v[i + 1];
    }
  }
  return v[0];
}

std::vector<float> b_factors(int n, int p) {
  std::vector<double> mod(n);
  for (int k = 0; k < n; ++k) {
    double th = 2.0 * M_PI * k / n, re = 0.0, im = 0.0;
    for (int j = 1; j < p; ++j) {
      double m = bspline(p, (double)j), a = th * (j - 1);
      re += m * std::cos(a);
      im += m * std::sin(a);
    }
    mod[k] = re * re + im * im;
  }
  for (int k = 0; k < n; ++k)
    if (mod[k] < 1.0e-7) mod[k] = 0.5 * (mod[(k + n - 1) % n] + mod[(k + 1) % n]);
  std::vector<float> out(n);
  for (int k = 0; k < n; ++k) out[k] = mod[k] > 0.0 ? (float)(1.0 / mod[k]) : 0.0f;
  return out;
}

}  // namespace

struct hdref_ff {
  uint32_t n = 0, n_types = 0, order = 4, grid[3] = {0, 0, 0};
  float alpha = 0, r_cut = 0, r_search = 0, lat[6] = {0, 0, 0, 0, 0, 0};
  cudaStream_t s = nullptr;
  // kernels
  CUfunction k_cells, k_scan_local, k_scan_apply, k_scan_fin, k_scan_fin_dev, k_scatter, k_sort_cells,
      k_tile_pos, k_tile_pad, k_bbox, k_find, k_status, k_hist, k_scat_entries, k_finalize;
  CUfunction k_pair_f, k_pair_fev, k_single_f, k_single_fev;
  CUfunction k_influence, k_binkey, k_finish, k_apply, k_reduce, k_spread, k_gather, k_combine;
  // system
  float *lattice = nullptr;
  float4 *posq = nullptr;
  uint32_t *types = nullptr;
  float *lj_sigma = nullptr, *lj_eps = nullptr, *lj_cut = nullptr, *lj_sw = nullptr;
  uint32_t *ex_off = nullptr, *ex_part = nullptr;
  float *ex_lj = nullptr, *ex_coul = nullptr;
  // cell list
  uint32_t nc[3] = {0, 0, 0}, nct = 0;
  uint32_t *cell_idx = nullptr, *cell_counts = nullptr, *cell_offsets = nullptr, *cursors = nullptr,
           *sorted_ids = nullptr;
  std::vector<uint32_t *> cscan;
  std::vector<uint32_t> cscan_len;
  // packed entries
  uint32_t n_blocks = 0, cap_tiles = 0, cap_sp = 0;
  uint32_t *tile_count = nullptr;
  float4 *tile_posq = nullptr;
  float *centre = nullptr, *bbox = nullptr;
  uint32_t *itiles = nullptr, *iatoms = nullptr, *sorted_iatoms = nullptr, *sp_atoms = nullptr,
           *icount = nullptr, *status = nullptr, *ib_count = nullptr, *ib_offset = nullptr,
           *ib_cursor = nullptr;
  std::vector<uint32_t *> iscan;
  std::vector<uint32_t> iscan_len;
  // force classes
  unsigned long long *fp[5] = {};
  float *fast[5] = {}, *slow[5] = {}, *out[5] = {};
  // SPME
  uint32_t M = 0, Mc = 0, n_vpart = 0;
  float *bfac[3] = {}, *G = nullptr, *vfac = nullptr, *rho = nullptr, *rho_hat = nullptr, *V = nullptr,
        *vpart = nullptr, *w_pp = nullptr, *u_self = nullptr;
  long long *rho_fixed = nullptr;
  uint32_t *bin_key = nullptr, *bin_counts = nullptr, *bin_offsets = nullptr, *bin_cursor = nullptr,
           *spme_sorted = nullptr;
  std::vector<uint32_t *> bscan;
  std::vector<uint32_t> bscan_len;
  cufftHandle fwd = 0, inv = 0;
  bool have_fft = false;
};

namespace {

int scan(hdref_ff *f, const uint32_t *in, uint32_t *out, std::vector<uint32_t *> &lv,
         std::vector<uint32_t> &lens, uint32_t len, const uint32_t *dev_total, uint32_t host_total) {
  // prefix_scan_cell_counts (src/gpu/kernels.rs:1814-1920)
  TRY(launch(f->k_scan_local, cdiv(len, 256), 256, f->s, in, out, lv[0], len));
  size_t descent = lv.size() - 1;
  for (size_t l = 0; l < descent; ++l) {
    uint32_t n = lens[l];
    TRY(launch(f->k_scan_local, cdiv(n, 256), 256, f->s, (const uint32_t *)lv[l], lv[l], lv[l + 1], n));
  }
  for (size_t l = descent; l-- > 0;) {
    if (l == 0) {
      TRY(launch(f->k_scan_apply, cdiv(len, 256), 256, f->s, (const uint32_t *)lv[0], out, len));
    } else {
      uint32_t n = lens[l - 1];
      TRY(launch(f->k_scan_apply, cdiv(n, 256), 256, f->s, (const uint32_t *)lv[l], lv[l - 1], n));
    }
  }
  if (dev_total)
    TRY(launch(f->k_scan_fin_dev, 1, 256, f->s, out, len, dev_total));
  else
    TRY(launch(f->k_scan_fin, 1, 256, f->s, out, len, host_total));
  return 0;
}

int alloc_levels(std::vector<uint32_t *> &lv, std::vector<uint32_t> &lens, uint32_t len) {
  lens = scan_levels(len);
  lv.assign(lens.size(), nullptr);
  for (size_t i = 0; i < lens.size(); ++i) TRY(dalloc(&lv[i], lens[i]));
  return 0;
}

int alloc_entries(hdref_ff *f) {
  cudaFree(f->itiles);
  cudaFree(f->iatoms);
  cudaFree(f->sorted_iatoms);
  cudaFree(f->sp_atoms);
  TRY(dalloc(&f->itiles, f->cap_tiles));
  TRY(dalloc(&f->iatoms, (size_t)f->cap_tiles * 32));
  TRY(dalloc(&f->sorted_iatoms, (size_t)f->cap_tiles * 32));
  TRY(dalloc(&f->sp_atoms, (size_t)f->cap_sp * 2));
  return 0;
}

int rebuild(hdref_ff *f) {
  uint32_t n = f->n;
  cudaStream_t s = f->s;
  RT(cudaMemsetAsync(f->status, 0, 4, s));
  // cell list (neighbor_list.rs:1003-1040)
  RT(cudaMemsetAsync(f->cell_counts, 0, 4ull * f->nct, s));
  TRY(launch(f->k_cells, cdiv(n, 256), 256, s, (const float4 *)f->posq, (const float *)f->lattice, f->nc[0],
             f->nc[1], f->nc[2], f->cell_idx, f->cell_counts, n));
  TRY(scan(f, f->cell_counts, f->cell_offsets, f->cscan, f->cscan_len, f->nct, nullptr, n));
  RT(cudaMemsetAsync(f->cursors, 0, 4ull * f->nct, s));
  TRY(launch(f->k_scatter, cdiv(n, 256), 256, s, (const uint32_t *)f->cell_idx,
             (const uint32_t *)f->cell_offsets, f->cursors, f->sorted_ids, n));
  TRY(launch(f->k_sort_cells, cdiv(f->nct, 256), 256, s, (const uint32_t *)f->cell_offsets, f->sorted_ids,
             f->nct));
  // packed construction (neighbor_list.rs:1080-1262)
  uint32_t padded = f->n_blocks * 32;
  TRY(launch(f->k_tile_pos, cdiv(n, 256), 256, s, (const float4 *)f->posq, (const uint32_t *)f->sorted_ids,
             f->tile_posq, n));
  TRY(launch(f->k_tile_pad, cdiv(padded - n, 256), 256, s, f->tile_posq, n, padded));
  TRY(launch(f->k_bbox, cdiv(f->n_blocks, 8), 256, s, (const float4 *)f->tile_posq,
             (const uint32_t *)f->tile_count, f->centre, f->bbox, f->n_blocks));
  float rs2 = f->r_search * f->r_search;
  for (int attempt = 0;; ++attempt) {
    RT(cudaMemsetAsync(f->icount, 0, 8, s));
    RT(cudaMemsetAsync(f->status, 0, 4, s));
    TRY(launch(f->k_find, cdiv(f->n_blocks, 4), 128, s, (const float4 *)f->tile_posq,
               (const uint32_t *)f->sorted_ids, (const float *)f->centre, (const float *)f->bbox,
               (const float *)f->lattice, rs2, f->n_blocks, n, f->cap_tiles, f->cap_sp, f->itiles,
               f->iatoms, f->sp_atoms, f->icount));
    uint32_t hw_t = (uint32_t)std::floor(f->cap_tiles * 0.8), hw_s = (uint32_t)std::floor(f->cap_sp * 0.8);
    TRY(launch(f->k_status, 1, 1, s, (const uint32_t *)f->icount, f->cap_tiles, f->cap_sp, hw_t, hw_s,
               f->status));
    uint32_t st = 0;
    RT(cudaMemcpyAsync(&st, f->status, 4, cudaMemcpyDeviceToHost, s));
    RT(cudaStreamSynchronize(s));
    // the probe rebuild's geometric growth (factor 1.5) until neither a
    // high-water nor an overflow bit is set
    bool gt = (st & (2u | 8u)) != 0, gs = (st & (4u | 16u)) != 0;
    if (!gt && !gs) break;
    if (attempt > 64) return fail("neighbour capacity did not converge");
    if (gt) f->cap_tiles = std::max<uint32_t>((uint32_t)std::ceil(f->cap_tiles * 1.5), f->cap_tiles + 1);
    if (gs) f->cap_sp = std::max<uint32_t>((uint32_t)std::ceil(f->cap_sp * 1.5), f->cap_sp + 1);
    TRY(alloc_entries(f));
  }
  RT(cudaMemsetAsync(f->ib_count, 0, 4ull * f->n_blocks, s));
  TRY(launch(f->k_hist, cdiv(f->cap_tiles, 256), 256, s, (const uint32_t *)f->itiles,
             (const uint32_t *)f->icount, f->ib_count, f->n_blocks));
  TRY(scan(f, f->ib_count, f->ib_offset, f->iscan, f->iscan_len, f->n_blocks, f->icount, 0));
  RT(cudaMemsetAsync(f->ib_cursor, 0, 4ull * f->n_blocks, s));
  TRY(launch(f->k_scat_entries, cdiv(f->cap_tiles, 8), 256, s, (const uint32_t *)f->itiles,
             (const uint32_t *)f->iatoms, (const uint32_t *)f->icount, (const uint32_t *)f->ib_offset,
             f->ib_cursor, f->sorted_iatoms, f->n_blocks));
  // SPME atom bin sort after every rebuild (spme.rs:413-428,
  // src/gpu/kernels.rs:518-598)
  if (f->have_fft) {
    RT(cudaMemsetAsync(f->bin_counts, 0, 4ull * f->M, s));
    RT(cudaMemsetAsync(f->bin_cursor, 0, 4ull * f->M, s));
    TRY(launch(f->k_binkey, cdiv(n, 256), 256, s, (const float4 *)f->posq, (const float *)f->lattice,
               f->grid[0], f->grid[1], f->grid[2], f->bin_key, f->bin_counts, n));
    TRY(scan(f, f->bin_counts, f->bin_offsets, f->bscan, f->bscan_len, f->M, nullptr, n));
    TRY(launch(f->k_scatter, cdiv(n, 256), 256, s, (const uint32_t *)f->bin_key,
               (const uint32_t *)f->bin_offsets, f->bin_cursor, f->spme_sorted, n));
    TRY(launch(f->k_sort_cells, cdiv(f->M, 256), 256, s, (const uint32_t *)f->bin_offsets, f->spme_sorted,
               f->M));
  }
  return 0;
}

// the stages of one force evaluation, each recordable with an event
enum Stage { ST_MEMSET, ST_TILEPOS, ST_PAIR, ST_SINGLE, ST_FINALIZE, ST_INFLUENCE, ST_SPREAD, ST_FFT_FWD,
             ST_APPLY, ST_FFT_INV, ST_GATHER, ST_COMBINE, ST_COUNT };

int evaluate(hdref_ff *f, int ev, cudaEvent_t *marks) {
  uint32_t n = f->n;
  cudaStream_t s = f->s;
  auto mark = [&](int i) -> int {
    if (marks) RT(cudaEventRecord(marks[i], s));
    return 0;
  };
  TRY(mark(0));
  // class accumulators (mod.rs:777-833) and fixed-point buffers (:838-854)
  for (int k = 0; k < 5; ++k) {
    if (k < 3 || ev) {
      RT(cudaMemsetAsync(f->fast[k], 0, 4ull * n, s));
      if (f->have_fft) RT(cudaMemsetAsync(f->slow[k], 0, 4ull * n, s));
    }
    RT(cudaMemsetAsync(f->fp[k], 0, 8ull * n, s));
  }
  TRY(mark(1));
  uint32_t padded = f->n_blocks * 32;
  TRY(launch(f->k_tile_pos, cdiv(n, 256), 256, s, (const float4 *)f->posq, (const uint32_t *)f->sorted_ids,
             f->tile_posq, n));
  TRY(launch(f->k_tile_pad, cdiv(padded - n, 256), 256, s, f->tile_posq, n, padded));
  TRY(mark(2));
  float kc = 1.0f;  // K_COULOMB_F32 in atomic units (src/gpu/kernels.rs:176)
  const float *lat = f->lattice;
  TRY(launch(ev ? f->k_pair_fev : f->k_pair_f, f->n_blocks, 256, s, (const float4 *)f->posq,
             (const uint32_t *)f->types, (const float4 *)f->tile_posq, (const float *)f->centre,
             (const float *)f->bbox, (const uint32_t *)f->sorted_ids, (const uint32_t *)f->ib_offset,
             (const uint32_t *)f->sorted_iatoms, f->n_blocks, lat, f->fp[0], f->fp[1], f->fp[2], f->fp[3],
             f->fp[4], f->n_types, (const float *)f->lj_sigma, (const float *)f->lj_eps,
             (const float *)f->lj_cut, (const float *)f->lj_sw, (const uint32_t *)f->ex_off,
             (const uint32_t *)f->ex_part, (const float *)f->ex_lj, kc, f->alpha, f->r_cut,
             (const uint32_t *)f->ex_off, (const uint32_t *)f->ex_part, (const float *)f->ex_coul, n));
  TRY(mark(3));
  TRY(launch(ev ? f->k_single_fev : f->k_single_f, cdiv(f->cap_sp, 256), 256, s, (const float4 *)f->posq,
             (const uint32_t *)f->types, (const uint32_t *)f->sp_atoms, (const uint32_t *)f->icount, lat,
             f->fp[0], f->fp[1], f->fp[2], f->fp[3], f->fp[4], f->n_types, (const float *)f->lj_sigma,
             (const float *)f->lj_eps, (const float *)f->lj_cut, (const float *)f->lj_sw,
             (const uint32_t *)f->ex_off, (const uint32_t *)f->ex_part, (const float *)f->ex_lj, kc, f->alpha,
             f->r_cut, (const uint32_t *)f->ex_off, (const uint32_t *)f->ex_part, (const float *)f->ex_coul, n));
  TRY(mark(4));
  TRY(launch(f->k_finalize, cdiv(n, 256), 256, s, (const unsigned long long *)f->fp[0],
             (const unsigned long long *)f->fp[1], (const unsigned long long *)f->fp[2],
             (const unsigned long long *)f->fp[3], (const unsigned long long *)f->fp[4], f->fast[0], f->fast[1],
             f->fast[2], f->fast[3], f->fast[4], n, (uint32_t)(ev ? 1u : 0u)));
  TRY(mark(5));
  if (f->have_fft) {
    TRY(launch(f->k_influence, cdiv(f->Mc, 256), 256, s, (const float *)f->bfac[0], (const float *)f->bfac[1],
               (const float *)f->bfac[2], f->G, f->vfac, lat, f->grid[0], f->grid[1], f->grid[2], kc, f->alpha,
               f->Mc));
    TRY(mark(6));
    RT(cudaMemsetAsync(f->rho_fixed, 0, 8ull * f->M, s));
    TRY(launch(f->k_spread, cdiv((uint64_t)n * f->order, 256), 256, s, (const float4 *)f->posq,
               (const uint32_t *)f->spme_sorted, lat, f->grid[0], f->grid[1], f->grid[2], f->order, f->rho_fixed,
               n));
    TRY(launch(f->k_finish, cdiv(f->M, 256), 256, s, (const long long *)f->rho_fixed, f->rho, f->M));
    TRY(mark(7));
    FFT(cufftExecR2C(f->fwd, f->rho, (cufftComplex *)f->rho_hat));
    TRY(mark(8));
    uint32_t ncc = f->grid[2] / 2 + 1;
    TRY(launch(f->k_apply, cdiv(f->Mc, 256), 256, s, (const float *)f->G, (const float *)f->vfac, f->rho_hat,
               f->vpart, f->grid[2], ncc, f->Mc));
    TRY(mark(9));
    FFT(cufftExecC2R(f->inv, (cufftComplex *)f->rho_hat, f->V));
    TRY(mark(10));
    float scale = 0.5f / (float)n;
    TRY(launch(f->k_reduce, 1, 256, s, (const float *)f->vpart, f->w_pp, f->n_vpart, scale));
    TRY(launch(f->k_gather, cdiv(n, 256), 256, s, (const float4 *)f->posq, (const float *)f->V,
               (const float *)f->u_self, (const float *)f->w_pp, (const uint32_t *)f->spme_sorted, lat,
               f->grid[0], f->grid[1], f->grid[2], f->order, f->slow[0], f->slow[1], f->slow[2], f->slow[3],
               f->slow[4], n));
    TRY(mark(11));
  } else {
    for (int i = 6; i <= 11; ++i) TRY(mark(i));
  }
  TRY(launch(f->k_combine, cdiv(n, 256), 256, s, (const float *)f->fast[0], (const float *)f->fast[1],
             (const float *)f->fast[2], (const float *)f->fast[3], (const float *)f->fast[4],
             (const float *)f->slow[0], (const float *)f->slow[1], (const float *)f->slow[2],
             (const float *)f->slow[3], (const float *)f->slow[4], f->out[0], f->out[1], f->out[2], f->out[3],
             f->out[4], n));
  TRY(mark(12));
  return 0;
}

}  // namespace

extern "C" {

const char *hdref_last_error(void) { return g_err.c_str(); }

// dir: the folder holding the cubins written by oracle/ref_build.py
int hdref_init(const char *dir) {
  g_dir = dir;
  RT(cudaSetDevice(0));
  RT(cudaFree(nullptr));  // the primary context is current from here on
  CUmodule m;
  TRY(module("neighbor", &m));
  return 0;
}

// One reference force field over n atoms.  posq: host [4n] floats; types
// [n]; LJ tables [n_types^2] (sigma, epsilon, cut-off, switch radius);
// exclusions: CSR over atoms with separate LJ / Coulomb scales; lattice
// (lx, ly, lz, xy, xz, yz); r_search = r_cut + r_skin (f32); grid[3] = 0
// disables SPME; pair_cubin names the composed pair module.
int hdref_ff_create(uint32_t n, const float *posq, const uint32_t *types, uint32_t n_types,
                    const float *lj_sigma, const float *lj_eps, const float *lj_cut, const float *lj_sw,
                    const uint32_t *excl_off, const uint32_t *excl_partners, const float *excl_lj,
                    const float *excl_coul, float alpha, float r_cut, float r_search, const uint32_t grid[3],
                    uint32_t order, const float lattice[6], const char *pair_cubin, hdref_ff **out) {
  *out = nullptr;
  if (n == 0) return fail("empty system");
  hdref_ff *f = new hdref_ff();
  f->n = n;
  f->n_types = n_types;
  f->order = order;
  f->alpha = alpha;
  f->r_cut = r_cut;
  f->r_search = r_search;
  std::memcpy(f->lat, lattice, sizeof(f->lat));
  RT(cudaStreamCreateWithFlags(&f->s, cudaStreamNonBlocking));
  const std::string nb = "neighbor", pr = pair_cubin;
  TRY(func(nb, "compute_cell_indices_and_histogram", &f->k_cells));
  TRY(func(nb, "prefix_scan_local_blocks", &f->k_scan_local));
  TRY(func(nb, "prefix_scan_apply_block_totals", &f->k_scan_apply));
  TRY(func(nb, "prefix_scan_finalize_offsets", &f->k_scan_fin));
  TRY(func(nb, "prefix_scan_finalize_offsets_dev", &f->k_scan_fin_dev));
  TRY(func(nb, "scatter_atoms_into_cells", &f->k_scatter));
  TRY(func(nb, "sort_cells_by_particle_id", &f->k_sort_cells));
  TRY(func(nb, "scatter_positions_to_tile_order", &f->k_tile_pos));
  TRY(func(nb, "fill_tile_position_padding", &f->k_tile_pad));
  TRY(func(nb, "compute_block_bbox", &f->k_bbox));
  TRY(func(nb, "find_blocks_with_interactions", &f->k_find));
  TRY(func(nb, "set_neighbor_status_bits", &f->k_status));
  TRY(func(nb, "histogram_entries_by_iblock", &f->k_hist));
  TRY(func(nb, "scatter_entries_by_iblock", &f->k_scat_entries));
  TRY(func(nb, "finalize_packed_forces", &f->k_finalize));
  TRY(func(pr, "heddle_jit_composed_pair_force_f", &f->k_pair_f));
  TRY(func(pr, "heddle_jit_composed_pair_force_fev", &f->k_pair_fev));
  TRY(func(pr, "heddle_jit_composed_pair_force_single_f", &f->k_single_f));
  TRY(func(pr, "heddle_jit_composed_pair_force_single_fev", &f->k_single_fev));
  TRY(func("forces", "combine_class_totals", &f->k_combine));
  // device copies of the inputs
  TRY(dalloc(&f->lattice, 6));
  RT(cudaMemcpy(f->lattice, lattice, 24, cudaMemcpyHostToDevice));
  TRY(dalloc(&f->posq, n));
  RT(cudaMemcpy(f->posq, posq, 16ull * n, cudaMemcpyHostToDevice));
  TRY(dalloc(&f->types, n));
  RT(cudaMemcpy(f->types, types, 4ull * n, cudaMemcpyHostToDevice));
  uint32_t nt2 = n_types * n_types;
  float **tabs[4] = {&f->lj_sigma, &f->lj_eps, &f->lj_cut, &f->lj_sw};
  const float *src[4] = {lj_sigma, lj_eps, lj_cut, lj_sw};
  for (int k = 0; k < 4; ++k) {
    TRY(dalloc(tabs[k], nt2));
    RT(cudaMemcpy(*tabs[k], src[k], 4ull * nt2, cudaMemcpyHostToDevice));
  }
  uint32_t ne = excl_off[n];
  TRY(dalloc(&f->ex_off, n + 1));
  RT(cudaMemcpy(f->ex_off, excl_off, 4ull * (n + 1), cudaMemcpyHostToDevice));
  TRY(dalloc(&f->ex_part, ne));
  TRY(dalloc(&f->ex_lj, ne));
  TRY(dalloc(&f->ex_coul, ne));
  if (ne) {
    RT(cudaMemcpy(f->ex_part, excl_partners, 4ull * ne, cudaMemcpyHostToDevice));
    RT(cudaMemcpy(f->ex_lj, excl_lj, 4ull * ne, cudaMemcpyHostToDevice));
    RT(cudaMemcpy(f->ex_coul, excl_coul, 4ull * ne, cudaMemcpyHostToDevice));
  }
  // cell layout: floor(perpendicular width / r_search) >= 3 per direction
  // (neighbor_list.rs:1563-1584; widths src/pbc.rs:308-325), in f32
  float lx = lattice[0], ly = lattice[1], lz = lattice[2], xy = lattice[3], xz = lattice[4], yz = lattice[5];
  float vol = lx * ly * lz, lylz = ly * lz, xylz = xy * lz, c3 = xy * yz - ly * xz;
  float w[3] = {vol / std::sqrt(lylz * lylz + xylz * xylz + c3 * c3), lylz / std::sqrt(lz * lz + yz * yz), lz};
  for (int d = 0; d < 3; ++d) {
    int64_t c = (int64_t)std::floor(w[d] / r_search);
    if (c < 3) return fail("BoxTooSmallForCells: a box width holds fewer than 3 cells of r_search");
    f->nc[d] = (uint32_t)c;
  }
  f->nct = f->nc[0] * f->nc[1] * f->nc[2];
  TRY(dalloc(&f->cell_idx, n));
  TRY(dalloc(&f->cell_counts, f->nct));
  TRY(dalloc(&f->cursors, f->nct));
  TRY(dalloc(&f->cell_offsets, f->nct + 1));
  TRY(dalloc(&f->sorted_ids, n));
  TRY(alloc_levels(f->cscan, f->cscan_len, f->nct));
  // packed data (neighbor_list.rs:286-390): 32-atom blocks, seed capacity
  // 128 entries per block capped at n_blocks^2 for both lists
  f->n_blocks = (n + 31) / 32;
  std::vector<uint32_t> cnt(f->n_blocks, 32u);
  if (n % 32) cnt.back() = n % 32;
  TRY(dalloc(&f->tile_count, f->n_blocks));
  RT(cudaMemcpy(f->tile_count, cnt.data(), 4ull * f->n_blocks, cudaMemcpyHostToDevice));
  TRY(dalloc(&f->tile_posq, (size_t)f->n_blocks * 32));
  TRY(dalloc(&f->centre, (size_t)f->n_blocks * 4));
  TRY(dalloc(&f->bbox, (size_t)f->n_blocks * 3));
  uint64_t seed = std::min<uint64_t>((uint64_t)f->n_blocks * 128, (uint64_t)f->n_blocks * f->n_blocks);
  f->cap_tiles = f->cap_sp = (uint32_t)std::max<uint64_t>(seed, 1);
  TRY(alloc_entries(f));
  TRY(dalloc(&f->icount, 2));
  TRY(dalloc(&f->status, 1));
  TRY(dalloc(&f->ib_count, f->n_blocks));
  TRY(dalloc(&f->ib_offset, f->n_blocks + 1));
  TRY(dalloc(&f->ib_cursor, f->n_blocks));
  TRY(alloc_levels(f->iscan, f->iscan_len, f->n_blocks));
  for (int k = 0; k < 5; ++k) {
    TRY(dalloc(&f->fp[k], n));
    TRY(dalloc(&f->fast[k], n));
    TRY(dalloc(&f->slow[k], n));
    TRY(dalloc(&f->out[k], n));
  }
  // SPME reciprocal grid (spme.rs:228-389)
  if (grid && grid[0] && grid[1] && grid[2]) {
    f->have_fft = true;
    for (int d = 0; d < 3; ++d) f->grid[d] = grid[d];
    f->M = grid[0] * grid[1] * grid[2];
    f->Mc = grid[0] * grid[1] * (grid[2] / 2 + 1);
    std::string sg = "spme_sg_p" + std::to_string(order);
    TRY(func(sg, "spme_spread_fixed_point", &f->k_spread));
    TRY(func(sg, "spme_force_gather", &f->k_gather));
    const std::string sr = "spme_recip";
    TRY(func(sr, "spme_recip_compute_influence", &f->k_influence));
    TRY(func(sr, "spme_compute_bin_key", &f->k_binkey));
    TRY(func(sr, "spme_spread_finish", &f->k_finish));
    TRY(func(sr, "spme_recip_apply_influence", &f->k_apply));
    TRY(func(sr, "spme_recip_reduce_partials", &f->k_reduce));
    for (int d = 0; d < 3; ++d) {
      std::vector<float> b = b_factors((int)grid[d], (int)order);
      TRY(dalloc(&f->bfac[d], grid[d]));
      RT(cudaMemcpy(f->bfac[d], b.data(), 4ull * grid[d], cudaMemcpyHostToDevice));
    }
    TRY(dalloc(&f->G, f->Mc));
    TRY(dalloc(&f->vfac, f->Mc));
    TRY(dalloc(&f->rho_fixed, f->M));
    TRY(dalloc(&f->rho, f->M));
    TRY(dalloc(&f->rho_hat, 2ull * f->Mc));
    TRY(dalloc(&f->V, f->M));
    f->n_vpart = cdiv(f->Mc, 256);
    TRY(dalloc(&f->vpart, f->n_vpart));
    TRY(dalloc(&f->w_pp, 1));
    // u_self = k_C alpha / sqrt(pi) q^2 in f64, stored as f32 (spme.rs:786-800)
    std::vector<float> us(n);
    double pre = 1.0 * (double)alpha / std::sqrt(M_PI);
    for (uint32_t i = 0; i < n; ++i) us[i] = (float)(pre * (double)posq[4 * i + 3] * (double)posq[4 * i + 3]);
    TRY(dalloc(&f->u_self, n));
    RT(cudaMemcpy(f->u_self, us.data(), 4ull * n, cudaMemcpyHostToDevice));
    TRY(dalloc(&f->bin_key, n));
    TRY(dalloc(&f->bin_counts, f->M));
    TRY(dalloc(&f->bin_offsets, f->M + 1));
    TRY(dalloc(&f->bin_cursor, f->M));
    TRY(dalloc(&f->spme_sorted, n));
    TRY(alloc_levels(f->bscan, f->bscan_len, f->M));
    FFT(cufftPlan3d(&f->fwd, (int)grid[0], (int)grid[1], (int)grid[2], CUFFT_R2C));
    FFT(cufftPlan3d(&f->inv, (int)grid[0], (int)grid[1], (int)grid[2], CUFFT_C2R));
    FFT(cufftSetStream(f->fwd, f->s));
    FFT(cufftSetStream(f->inv, f->s));
  }
  *out = f;
  return 0;
}

// Replace the positions (host [4n] floats, same atom order).
int hdref_ff_set_positions(hdref_ff *f, const float *posq) {
  RT(cudaMemcpyAsync(f->posq, posq, 16ull * f->n, cudaMemcpyHostToDevice, f->s));
  RT(cudaStreamSynchronize(f->s));
  return 0;
}

// Neighbour rebuild (and the SPME atom sort that follows a rebuild).
int hdref_ff_rebuild(hdref_ff *f) {
  TRY(rebuild(f));
  RT(cudaStreamSynchronize(f->s));
  return 0;
}

// One force evaluation (ev != 0: energies and virials too).
int hdref_ff_forces(hdref_ff *f, int ev) {
  TRY(evaluate(f, ev, nullptr));
  RT(cudaStreamSynchronize(f->s));
  return 0;
}

// Results of the last evaluation, atom order: which = 0 total, 1 fast class
// (pair kernels), 2 slow class (SPME reciprocal).  fxyz: [3n] interleaved;
// energy, virial: [n] (either may be NULL).
int hdref_ff_get(hdref_ff *f, int which, float *fxyz, float *energy, float *virial) {
  float **b = which == 0 ? f->out : which == 1 ? f->fast : f->slow;
  uint32_t n = f->n;
  std::vector<float> t(n);
  for (int k = 0; k < 3; ++k) {
    RT(cudaMemcpy(t.data(), b[k], 4ull * n, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) fxyz[3 * i + k] = t[i];
  }
  if (energy) RT(cudaMemcpy(energy, b[3], 4ull * n, cudaMemcpyDeviceToHost));
  if (virial) RT(cudaMemcpy(virial, b[4], 4ull * n, cudaMemcpyDeviceToHost));
  return 0;
}

// out[0] packed entries, [1] single pairs, [2] entry capacity, [3]
// single-pair capacity, [4] 32-atom blocks, [5] cells
int hdref_ff_stats(hdref_ff *f, uint64_t out[6]) {
  uint32_t c[2];
  RT(cudaMemcpy(c, f->icount, 8, cudaMemcpyDeviceToHost));
  out[0] = c[0];
  out[1] = c[1];
  out[2] = f->cap_tiles;
  out[3] = f->cap_sp;
  out[4] = f->n_blocks;
  out[5] = f->nct;
  return 0;
}

// The canonical deduplicated pair list of pair_snapshot /
// decode_canonical_pairs (neighbor_list.rs:1366-1500): every (i-block atom,
// entry j-atom) pair of the packed entries plus the single pairs, as
// (min, max).  Only pairs whose f64 minimum-image distance is at most
// r_keep are returned (a prefilter for the caller's exact test); writes up
// to cap pairs, *count = number kept.
int hdref_ff_pairs(hdref_ff *f, double r_keep, uint32_t *pairs, uint64_t cap, uint64_t *count) {
  uint32_t c[2];
  RT(cudaMemcpy(c, f->icount, 8, cudaMemcpyDeviceToHost));
  uint32_t n = f->n;
  std::vector<uint32_t> tiles(c[0]), atoms((size_t)c[0] * 32), single((size_t)c[1] * 2), ids(n);
  std::vector<float> pq(4ull * n);
  if (c[0]) {
    RT(cudaMemcpy(tiles.data(), f->itiles, 4ull * c[0], cudaMemcpyDeviceToHost));
    RT(cudaMemcpy(atoms.data(), f->sorted_iatoms, 128ull * c[0], cudaMemcpyDeviceToHost));
  }
  if (c[1]) RT(cudaMemcpy(single.data(), f->sp_atoms, 8ull * c[1], cudaMemcpyDeviceToHost));
  RT(cudaMemcpy(ids.data(), f->sorted_ids, 4ull * n, cudaMemcpyDeviceToHost));
  RT(cudaMemcpy(pq.data(), f->posq, 16ull * n, cudaMemcpyDeviceToHost));
  // The i-block of sorted entry e is not stored with the sorted copy; the
  // i-block offsets give it (entries are grouped by i-block).
  std::vector<uint32_t> off(f->n_blocks + 1);
  RT(cudaMemcpy(off.data(), f->ib_offset, 4ull * (f->n_blocks + 1), cudaMemcpyDeviceToHost));
  const double L[6] = {f->lat[0], f->lat[1], f->lat[2], f->lat[3], f->lat[4], f->lat[5]};
  auto near = [&](uint32_t a, uint32_t b) {
    double dx = (double)pq[4 * a] - pq[4 * b], dy = (double)pq[4 * a + 1] - pq[4 * b + 1],
           dz = (double)pq[4 * a + 2] - pq[4 * b + 2];
    double sc = dz / L[2], sb = (dy - sc * L[5]) / L[1], sa = (dx - sb * L[3] - sc * L[4]) / L[0];
    double ka = std::floor(sa + 0.5), kb = std::floor(sb + 0.5), kc = std::floor(sc + 0.5);
    dx -= ka * L[0] + kb * L[3] + kc * L[4];
    dy -= kb * L[1] + kc * L[5];
    dz -= kc * L[2];
    return dx * dx + dy * dy + dz * dz <= r_keep * r_keep;
  };
  std::vector<uint64_t> keys;
  for (uint32_t b = 0; b < f->n_blocks; ++b) {
    for (uint32_t e = off[b]; e < off[b + 1] && e < c[0]; ++e) {
      for (uint32_t l = 0; l < 32; ++l) {
        uint32_t sid = b * 32 + l;
        uint32_t ia = sid < n ? ids[sid] : n;
        if (ia >= n) continue;
        for (uint32_t r = 0; r < 32; ++r) {
          uint32_t ja = atoms[(size_t)e * 32 + ((l + r) & 31)];
          if (ja >= n || ja == ia) continue;
          uint32_t lo = std::min(ia, ja), hi = std::max(ia, ja);
          if (near(lo, hi)) keys.push_back(((uint64_t)lo << 32) | hi);
        }
      }
    }
  }
  for (uint32_t k = 0; k < c[1]; ++k) {
    uint32_t a = single[2 * k], b = single[2 * k + 1];
    if (a >= n || b >= n || a == b) continue;
    uint32_t lo = std::min(a, b), hi = std::max(a, b);
    if (near(lo, hi)) keys.push_back(((uint64_t)lo << 32) | hi);
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  *count = keys.size();
  for (uint64_t k = 0; k < keys.size() && k < cap; ++k) {
    pairs[2 * k] = (uint32_t)(keys[k] >> 32);
    pairs[2 * k + 1] = (uint32_t)keys[k];
  }
  return 0;
}

// Device time of the path: reps evaluations after one warm-up, events on
// the harness stream.  ms[0] whole evaluation (no events inside, mean),
// ms[1..12] per stage (means): accumulator clears, tile-order scatter,
// packed pair kernel, single-pair kernel, finalize, influence function,
// spread (+ clear + finish), forward FFT, apply influence, inverse FFT,
// reduce + gather, class combine; ms[13] one neighbour rebuild (probe-free,
// mean of `reps` rebuilds, SPME sort included).
int hdref_ff_time(hdref_ff *f, int reps, int ev, double ms[14]) {
  if (reps < 1) reps = 1;
  cudaEvent_t e[ST_COUNT + 1];
  for (auto &x : e) RT(cudaEventCreate(&x));
  TRY(evaluate(f, ev, nullptr));
  RT(cudaStreamSynchronize(f->s));
  RT(cudaEventRecord(e[0], f->s));
  for (int r = 0; r < reps; ++r) TRY(evaluate(f, ev, nullptr));
  RT(cudaEventRecord(e[1], f->s));
  RT(cudaEventSynchronize(e[1]));
  float t = 0;
  RT(cudaEventElapsedTime(&t, e[0], e[1]));
  for (int i = 0; i < 14; ++i) ms[i] = 0.0;
  ms[0] = t / reps;
  for (int r = 0; r < reps; ++r) {
    TRY(evaluate(f, ev, e));
    RT(cudaEventSynchronize(e[ST_COUNT]));
    for (int i = 0; i < ST_COUNT; ++i) {
      RT(cudaEventElapsedTime(&t, e[i], e[i + 1]));
      ms[1 + i] += t / reps;
    }
  }
  // steady-state rebuilds: capacities are already sized
  RT(cudaEventRecord(e[0], f->s));
  for (int r = 0; r < reps; ++r) TRY(rebuild(f));
  RT(cudaEventRecord(e[1], f->s));
  RT(cudaEventSynchronize(e[1]));
  RT(cudaEventElapsedTime(&t, e[0], e[1]));
  ms[13] = t / reps;
  for (auto &x : e) cudaEventDestroy(x);
  return 0;
}

int hdref_ff_destroy(hdref_ff *f) {
  if (!f) return 0;
  if (f->have_fft) {
    cufftDestroy(f->fwd);
    cufftDestroy(f->inv);
  }
  void *bufs[] = {f->lattice, f->posq, f->types, f->lj_sigma, f->lj_eps, f->lj_cut, f->lj_sw, f->ex_off,
                  f->ex_part, f->ex_lj, f->ex_coul, f->cell_idx, f->cell_counts, f->cell_offsets, f->cursors,
                  f->sorted_ids, f->tile_count, f->tile_posq, f->centre, f->bbox, f->itiles, f->iatoms,
                  f->sorted_iatoms, f->sp_atoms, f->icount, f->status, f->ib_count, f->ib_offset, f->ib_cursor,
                  f->G, f->vfac, f->rho, f->rho_hat, f->V, f->vpart, f->w_pp, f->u_self, f->rho_fixed,
                  f->bin_key, f->bin_counts, f->bin_offsets, f->bin_cursor, f->spme_sorted, f->bfac[0],
                  f->bfac[1], f->bfac[2]};
  for (void *p : bufs) cudaFree(p);
  for (int k = 0; k < 5; ++k) {
    cudaFree(f->fp[k]);
    cudaFree(f->fast[k]);
    cudaFree(f->slow[k]);
    cudaFree(f->out[k]);
  }
  for (auto *p : f->cscan) cudaFree(p);
  for (auto *p : f->iscan) cudaFree(p);
  for (auto *p : f->bscan) cudaFree(p);
  cudaStreamDestroy(f->s);
  delete f;
  return 0;
}

// SETTLE position step of the reference on n_groups waters (atoms
// 3g, 3g+1, 3g+2 = O, H, H): settle_snapshot of pos0, then settle_positions
// on pos1 with the velocities vel (host [3n], updated in place), dt, and
// per-group geometry.  pos0/pos1: host [4n] floats; pos_out: [4n];
// virial_out: [n] constraint virial per atom slot (may be NULL).
int hdref_settle(uint32_t n_groups, const float *pos0, const float *pos1, float *vel, const float *ra,
                 const float *rb, const float *rc, const float *m_o, const float *m_h, const float lattice[6],
                 float dt, float *pos_out, float *virial_out) {
  uint32_t n = 3 * n_groups;
  CUfunction k_snap, k_pos;
  TRY(func("settle", "settle_snapshot", &k_snap));
  TRY(func("settle", "settle_positions", &k_pos));
  std::vector<uint32_t> atoms(n), offs(n_groups), cnts(n_groups, 3u);
  for (uint32_t i = 0; i < n; ++i) atoms[i] = i;
  for (uint32_t g = 0; g < n_groups; ++g) offs[g] = 3 * g;
  float4 *posq;
  float *lat, *v[3], *snap[3], *geo[5], *vir;
  uint32_t *d_atoms, *d_offs, *d_cnts;
  TRY(dalloc(&posq, n));
  TRY(dalloc(&lat, 6));
  for (int k = 0; k < 3; ++k) {
    TRY(dalloc(&v[k], n));
    TRY(dalloc(&snap[k], n));
  }
  const float *gsrc[5] = {ra, rb, rc, m_o, m_h};
  for (int k = 0; k < 5; ++k) {
    TRY(dalloc(&geo[k], n_groups));
    RT(cudaMemcpy(geo[k], gsrc[k], 4ull * n_groups, cudaMemcpyHostToDevice));
  }
  TRY(dalloc(&vir, n));
  TRY(dalloc(&d_atoms, n));
  TRY(dalloc(&d_offs, n_groups));
  TRY(dalloc(&d_cnts, n_groups));
  RT(cudaMemcpy(d_atoms, atoms.data(), 4ull * n, cudaMemcpyHostToDevice));
  RT(cudaMemcpy(d_offs, offs.data(), 4ull * n_groups, cudaMemcpyHostToDevice));
  RT(cudaMemcpy(d_cnts, cnts.data(), 4ull * n_groups, cudaMemcpyHostToDevice));
  RT(cudaMemcpy(lat, lattice, 24, cudaMemcpyHostToDevice));
  std::vector<float> t(n);
  for (int k = 0; k < 3; ++k) {
    for (uint32_t i = 0; i < n; ++i) t[i] = vel[3 * i + k];
    RT(cudaMemcpy(v[k], t.data(), 4ull * n, cudaMemcpyHostToDevice));
  }
  RT(cudaMemcpy(posq, pos0, 16ull * n, cudaMemcpyHostToDevice));
  TRY(launch(k_snap, cdiv(n_groups, 256), 256, (cudaStream_t)0, (const float4 *)posq, (const uint32_t *)d_atoms,
             (const uint32_t *)d_offs, (const uint32_t *)d_cnts, snap[0], snap[1], snap[2], n_groups));
  RT(cudaMemcpy(posq, pos1, 16ull * n, cudaMemcpyHostToDevice));
  TRY(launch(k_pos, cdiv(n_groups, 256), 256, (cudaStream_t)0, posq, v[0], v[1], v[2], (const float *)snap[0],
             (const float *)snap[1], (const float *)snap[2], (const uint32_t *)d_atoms, (const uint32_t *)d_offs,
             (const uint32_t *)d_cnts, (const float *)geo[0], (const float *)geo[1], (const float *)geo[2],
             (const float *)geo[3], (const float *)geo[4], (const float *)lat, dt, vir, n_groups));
  RT(cudaDeviceSynchronize());
  RT(cudaMemcpy(pos_out, posq, 16ull * n, cudaMemcpyDeviceToHost));
  for (int k = 0; k < 3; ++k) {
    RT(cudaMemcpy(t.data(), v[k], 4ull * n, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) vel[3 * i + k] = t[i];
  }
  if (virial_out) RT(cudaMemcpy(virial_out, vir, 4ull * n, cudaMemcpyDeviceToHost));
  void *bufs[] = {posq, lat, v[0], v[1], v[2], snap[0], snap[1], snap[2], geo[0], geo[1], geo[2], geo[3], geo[4],
                  vir, d_atoms, d_offs, d_cnts};
  for (void *p : bufs) cudaFree(p);
  return 0;
}

}  // extern "C"
