// hb_baro.cu -- Monte-Carlo barostat for the B200 force path.
//
// Replaces McBarostat::apply_move (src/integrator/mc_barostat.rs:218-360)
// and mc_barostat_scale_molecule_com (kernels/mc_barostat.cu:19-74).  The
// reference orchestrates a move from the host (two device->host reads of
// the potential energy, a host Metropolis test, device-to-device restores).
// Here the move is four kernels around one force evaluation and never
// synchronises:
//   k_baro_propose   1 thread: U_old from the scalars, Philox draw, dV, the
//                    width guard, FP64 lattice scale;
//   k_baro_scale     1 thread per molecule: snapshot of the molecule's
//                    positions/images/forces, FP64 centre of mass, rigid
//                    translation by (s - 1) COM, wrap into the new cell;
//   (force evaluation with scalars; the neighbour list is kept when the
//    scaling is within its tolerance, else rebuilt against the new box)
//   k_baro_decide    1 thread: Metropolis test in FP64, box/scalars revert on
//                    rejection, step-size adaptation, diagnostics;
//   k_baro_restore   1 thread per atom: positions/images/forces revert.
// so a move also runs inside a captured CUDA graph.
//
// One deliberate difference from the reference kernel: it translates each
// stored (per-atom wrapped) position by the molecule's shift, which for a
// molecule split across the cell boundary leaves the atoms on the far side
// displaced by (s - 1) x lattice vector relative to their partners.  This
// kernel translates the molecule's contiguous image (atom = reference atom +
// minimum-image displacement) and wraps each atom back into the new cell,
// updating its image counts, so every molecule stays rigid.  For molecules
// that do not straddle the boundary the two agree.
#include <cmath>
#include <cstring>
#include <vector>

#include "hb_internal.cuh"

namespace {

__device__ __forceinline__ double baro_volume(const double *lat) {
  return lat[0] * lat[1] * lat[2];
}

__global__ void k_baro_propose(BaroState *__restrict__ st, double *__restrict__ lat,
                               DBox *__restrict__ dbox, const double *__restrict__ scalars,
                               double r_search, uint32_t seed_lo, uint32_t seed_hi) {
  st->u_old = scalars[4];
  for (int q = 0; q < HB_N_SCALARS; ++q) st->scalars_pre[q] = scalars[q];
  st->draw += 1ull;
  uint32_t o0, o1;
  hb_philox(seed_lo, seed_hi, (uint32_t)st->draw, (uint32_t)(st->draw >> 32), 0u, 0u, o0, o1);
  const double inv32 = 1.0 / 4294967296.0;
  const double u1 = ((double)o0 + 0.5) * inv32;
  const double u2 = ((double)o1 + 0.5) * inv32;
  const double v_old = baro_volume(lat);
  const double dv = st->max_dv * (2.0 * u1 - 1.0);
  const double v_new = v_old + dv;
  double w[3];
  hb_perp_widths(lat, w);
  const double min_w = fmin(w[0], fmin(w[1], w[2]));
  bool trial = v_new > 0.0;
  double scale = 1.0;
  if (trial) {
    scale = cbrt(v_new / v_old);
    if (r_search > 0.0 && scale * min_w < 2.0 * r_search) trial = false;
  }
  if (trial) {
    for (int d = 0; d < 6; ++d) {
      st->lattice_pre[d] = lat[d];
      lat[d] *= scale;
    }
    *dbox = hb_make_dbox(lat);
  }
  st->u1 = u1;
  st->u2 = u2;
  st->dv = dv;
  st->v_old = v_old;
  st->v_new = v_new;
  st->scale = trial ? scale : 1.0;
  st->trial = trial ? 1 : 0;
  st->last_accepted = 0;
}

// One thread per molecule.  Centre of mass of the contiguous image about
// the molecule's first atom (single-precision minimum image in the cell the
// positions live in, i.e. the pre-move box; FP64 mass-weighted sum in stored
// order, so the result is deterministic), then every atom is translated by
// (s - 1) COM and wrapped into the new cell.
__global__ void k_baro_scale(const BaroState *__restrict__ st,
                             const uint32_t *__restrict__ off, const uint32_t *__restrict__ atoms,
                             const double *__restrict__ mass, float4 *__restrict__ posq,
                             int4 *__restrict__ image, const float4 *__restrict__ force,
                             float4 *__restrict__ snap_pos, int4 *__restrict__ snap_img,
                             float4 *__restrict__ snap_force, const DBox *__restrict__ dbox,
                             uint32_t n_mol) {
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_mol) return;
  const uint32_t lo = off[m], hi = off[m + 1];
  for (uint32_t k = lo; k < hi; ++k) {
    const uint32_t a = atoms[k];
    snap_pos[a] = posq[a];
    snap_img[a] = image[a];
    snap_force[a] = force[a];
  }
  if (!st->trial || hi == lo) return;
  const DBox b = hb_make_dbox(st->lattice_pre);  // the positions' cell
  const DBox bn = *dbox;                         // the trial cell
  const float4 ref = posq[atoms[lo]];
  double mt = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
  for (uint32_t k = lo; k < hi; ++k) {
    const uint32_t a = atoms[k];
    const float4 p = posq[a];
    float dx = p.x - ref.x, dy = p.y - ref.y, dz = p.z - ref.z;
    hb_min_image(dx, dy, dz, b);
    const double ma = mass[a];
    cx += ma * (double)dx;
    cy += ma * (double)dy;
    cz += ma * (double)dz;
    mt += ma;
  }
  const double f = st->scale - 1.0;
  const double sx = f * ((double)ref.x + cx / mt);
  const double sy = f * ((double)ref.y + cy / mt);
  const double sz = f * ((double)ref.z + cz / mt);
  for (uint32_t k = lo; k < hi; ++k) {
    const uint32_t a = atoms[k];
    float4 p = posq[a];
    // contiguous image: p - K L with K the lattice shift the minimum image
    // applied to p - ref
    float dx = p.x - ref.x, dy = p.y - ref.y, dz = p.z - ref.z;
    const float ox = dx, oy = dy, oz = dz;
    hb_min_image(dx, dy, dz, b);
    float sa, sb, sc;  // K L = (p - ref) - d, recovered as lattice counts
    {
      const float rx = ox - dx, ry = oy - dy, rz = oz - dz;
      hb_frac(rx, ry, rz, b, sa, sb, sc);
    }
    const int ka = (int)rintf(sa), kb = (int)rintf(sb), kc = (int)rintf(sc);
    float x = (float)((double)ref.x + (double)dx + sx);
    float y = (float)((double)ref.y + (double)dy + sy);
    float z = (float)((double)ref.z + (double)dz + sz);
    int wa, wb, wc;
    hb_wrap(x, y, z, wa, wb, wc, bn);
    p.x = x;
    p.y = y;
    p.z = z;
    posq[a] = p;
    int4 im = image[a];
    im.x += ka + wa;
    im.y += kb + wb;
    im.z += kc + wc;
    image[a] = im;
  }
}

__global__ void k_baro_decide(BaroState *__restrict__ st, double *__restrict__ lat,
                              DBox *__restrict__ dbox, double *__restrict__ scalars,
                              double pressure, double kt, double n_mol) {
  bool accepted = false;
  double v_post = st->v_old;
  st->u_new = st->u_old;
  st->w = 0.0;
  if (st->trial) {
    const double u_new = scalars[4];
    const double w = (u_new - st->u_old) + pressure * st->dv -
                     n_mol * kt * log(st->v_new / st->v_old);
    accepted = w <= 0.0 || st->u2 < exp(-w / kt);
    st->u_new = u_new;
    st->w = w;
    if (accepted) {
      v_post = st->v_new;
    } else {
      for (int d = 0; d < 6; ++d) lat[d] = st->lattice_pre[d];
      *dbox = hb_make_dbox(lat);
      for (int q = 0; q < HB_N_SCALARS; ++q) scalars[q] = st->scalars_pre[q];
    }
  }
  // adaptive step (src/integrator/mc_barostat.rs:157-179)
  st->attempted += 1ull;
  st->win_attempted += 1u;
  if (accepted) {
    st->accepted += 1ull;
    st->win_accepted += 1u;
  }
  if (st->win_attempted >= 10u) {
    const double att = (double)st->win_attempted, acc = (double)st->win_accepted;
    if (acc < 0.25 * att) st->max_dv /= 1.1;
    else if (acc > 0.75 * att) st->max_dv = fmin(st->max_dv * 1.1, 0.3 * v_post);
    st->win_attempted = 0u;
    st->win_accepted = 0u;
  }
  if (accepted) st->injection += pressure * (v_post - st->v_old);
  st->volume = v_post;
  st->last_accepted = accepted ? 1 : 0;
}

__global__ void k_baro_restore(const BaroState *__restrict__ st, float4 *__restrict__ posq,
                               int4 *__restrict__ image, float4 *__restrict__ force,
                               const float4 *__restrict__ snap_pos,
                               const int4 *__restrict__ snap_img,
                               const float4 *__restrict__ snap_force, uint32_t n) {
  if (!st->trial || st->last_accepted) return;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  posq[i] = snap_pos[i];
  image[i] = snap_img[i];
  force[i] = snap_force[i];
}

}  // namespace

int baro_propose(hb_barostat *b, hb_forcefield *ff, cudaStream_t s) {
  hb_system *sys = b->sys;
  const double r_search = ff ? (double)ff->r_search : 0.0;
  k_baro_propose<<<1, 1, 0, s>>>(b->d_state, sys->d_box64, sys->d_box, ff->d_scalars, r_search,
                                 (uint32_t)b->seed, (uint32_t)(b->seed >> 32));
  if (b->n_mol)
    k_baro_scale<<<hb_div_up(b->n_mol, 128), 128, 0, s>>>(
        b->d_state, b->d_mol_off, b->d_mol_atoms, b->d_mass, sys->d_posq, sys->d_image,
        sys->d_force, b->d_snap_pos, b->d_snap_img, b->d_snap_force, sys->d_box, b->n_mol);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int baro_decide(hb_barostat *b, hb_forcefield *ff, cudaStream_t s) {
  hb_system *sys = b->sys;
  k_baro_decide<<<1, 1, 0, s>>>(b->d_state, sys->d_box64, sys->d_box, ff->d_scalars, b->pressure,
                                b->kt, (double)b->n_mol);
  if (sys->n)
    k_baro_restore<<<hb_div_up(sys->n, 256), 256, 0, s>>>(b->d_state, sys->d_posq, sys->d_image,
                                                          sys->d_force, b->d_snap_pos,
                                                          b->d_snap_img, b->d_snap_force, sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

extern "C" int hb_barostat_destroy(hb_barostat *b) {
  if (!b) return HB_OK;
  cudaSetDevice(b->sys->ctx->device);
  cudaStreamSynchronize(b->sys->ctx->stream);
  cudaFree(b->d_mol_off);
  cudaFree(b->d_mol_atoms);
  cudaFree(b->d_mass);
  cudaFree(b->d_state);
  cudaFree(b->d_snap_pos);
  cudaFree(b->d_snap_img);
  cudaFree(b->d_snap_force);
  delete b;
  return HB_OK;
}

extern "C" int hb_barostat_create(hb_system *sys, const hb_barostat_desc *d, hb_barostat **out) {
  HB_REQUIRE(sys && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  // validation of McBarostatBuilder::validate_params (mc_barostat.rs:388-405)
  HB_REQUIRE(std::isfinite(d->pressure), HB_ERR_INVALID_ARGUMENT,
             "barostat.pressure: value must be finite");
  HB_REQUIRE(std::isfinite(d->temperature) && d->temperature > 0.0, HB_ERR_INVALID_ARGUMENT,
             "barostat.temperature: value must be finite and strictly positive");
  HB_REQUIRE(d->frequency >= 1, HB_ERR_INVALID_ARGUMENT, "barostat.frequency: value must be >= 1, got 0");
  HB_REQUIRE(std::isfinite(d->volume_step), HB_ERR_INVALID_ARGUMENT,
             "barostat.volume_step: value must be finite");
  const uint32_t n = sys->n;
  std::vector<uint32_t> off, atoms;
  if (d->n_molecules == 0) {
    off.resize(n + 1);
    atoms.resize(n);
    for (uint32_t i = 0; i <= n; ++i) off[i] = i;
    for (uint32_t i = 0; i < n; ++i) atoms[i] = i;
  } else {
    HB_REQUIRE(d->mol_offsets && d->mol_atoms, HB_ERR_INVALID_ARGUMENT, "null molecule table");
    off.assign(d->mol_offsets, d->mol_offsets + d->n_molecules + 1);
    HB_REQUIRE(off[0] == 0 && off[d->n_molecules] == n, HB_ERR_INVALID_ARGUMENT,
               "molecule table must cover every atom exactly once");
    std::vector<uint8_t> seen(n, 0);
    for (uint32_t m = 0; m < d->n_molecules; ++m)
      HB_REQUIRE(off[m] <= off[m + 1], HB_ERR_INVALID_ARGUMENT, "molecule offsets must not decrease");
    atoms.assign(d->mol_atoms, d->mol_atoms + n);
    for (uint32_t a : atoms) {
      HB_REQUIRE(a < n && !seen[a], HB_ERR_INVALID_ARGUMENT,
                 "molecule table must cover every atom exactly once");
      seen[a] = 1;
    }
  }
  hb_barostat *b = new hb_barostat();
  b->sys = sys;
  b->pressure = d->pressure;
  b->kt = d->temperature;
  b->frequency = d->frequency;
  b->seed = d->seed;
  b->n_mol = d->n_molecules ? d->n_molecules : n;
  double lat[6];
  int rc = HB_OK;
  cudaSetDevice(sys->ctx->device);
  cudaStreamSynchronize(sys->ctx->stream);
  if (cudaMemcpy(lat, sys->d_box64, sizeof(lat), cudaMemcpyDeviceToHost) != cudaSuccess) rc = HB_ERR_CUDA;
  BaroState st;
  std::memset(&st, 0, sizeof(st));
  const double v0 = lat[0] * lat[1] * lat[2];
  st.max_dv = d->volume_step > 0.0 ? d->volume_step : 0.01 * v0;
  st.volume = v0;
  const size_t nn = std::max(n, 1u);
  auto ok = [](cudaError_t e) { return e == cudaSuccess; };
  if (rc == HB_OK &&
      !(ok(cudaMalloc(&b->d_mol_off, sizeof(uint32_t) * (b->n_mol + 1))) &&
        ok(cudaMalloc(&b->d_mol_atoms, sizeof(uint32_t) * nn)) &&
        ok(cudaMalloc(&b->d_mass, sizeof(double) * nn)) &&
        ok(cudaMalloc(&b->d_state, sizeof(BaroState))) &&
        ok(cudaMalloc(&b->d_snap_pos, sizeof(float4) * nn)) &&
        ok(cudaMalloc(&b->d_snap_img, sizeof(int4) * nn)) &&
        ok(cudaMalloc(&b->d_snap_force, sizeof(float4) * nn)) &&
        ok(cudaMemcpy(b->d_mol_off, off.data(), sizeof(uint32_t) * off.size(), cudaMemcpyHostToDevice)) &&
        (n == 0 || ok(cudaMemcpy(b->d_mol_atoms, atoms.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice))) &&
        (n == 0 || ok(cudaMemcpy(b->d_mass, sys->h_mass.data(), sizeof(double) * n, cudaMemcpyHostToDevice))) &&
        ok(cudaMemcpy(b->d_state, &st, sizeof(st), cudaMemcpyHostToDevice))))
    rc = HB_ERR_CUDA;
  if (rc != HB_OK) {
    hb_barostat_destroy(b);
    return hb_fail(rc, "barostat state allocation failed");
  }
  *out = b;
  return HB_OK;
}

extern "C" int hb_barostat_stats(hb_barostat *b, double out[15]) {
  HB_REQUIRE(b && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_CUDA(cudaStreamSynchronize(b->sys->ctx->stream));
  BaroState st;
  HB_CUDA(cudaMemcpy(&st, b->d_state, sizeof(st), cudaMemcpyDeviceToHost));
  out[0] = st.volume;
  out[1] = st.attempted ? (double)st.accepted / (double)st.attempted : 0.0;
  out[2] = st.max_dv;
  out[3] = b->pressure * st.volume - st.injection;
  out[4] = (double)st.attempted;
  out[5] = (double)st.accepted;
  out[6] = st.dv;
  out[7] = st.w;
  out[8] = st.u_old;
  out[9] = st.u_new;
  out[10] = st.scale;
  out[11] = st.last_accepted;
  out[12] = st.trial;
  out[13] = st.u2;
  out[14] = (double)st.draw;
  return HB_OK;
}
