// hb_couple.cu -- velocity thermostats (CSVR, Andersen, Berendsen) and
// per-step pressure coupling (c-rescale, Berendsen) for velocity Verlet.
//
// The reference runs these as host-orchestrated slots around its composed
// post-force kernel (src/runner.rs:2661-2686): thermostat.apply_post and
// barostat.apply compute device scalars from the velocities after the
// constraint projection, then one per-particle kernel applies the final
// half kick, the thermostat's rescale / resample and the barostat's
// position scaling.  Here the same order is kept with every scalar on the
// device:
//   * the kinetic energy is a fixed-grid FP64 reduction (deterministic);
//   * the CSVR sum of g - 1 squared normals is split over 148 blocks with a
//     fixed chunking and a fixed tree (csvr_sample_partials /
//     csvr_finish_from_partials, kernels/nose_hoover.cu:263-385);
//   * the draw counter advances in the finishing kernel (CSVR, c-rescale) or
//     in a one-thread kernel after the resample (Andersen), never inside a
//     kernel whose other threads read it;
//   * k_vv_final fuses the final kick with the rescale factor, the Andersen
//     collisions and the position scaling, so coupling costs one extra
//     elementwise pass at most.
#include <algorithm>
#include <cmath>

#include "hb_internal.cuh"

namespace {

#define CPL_BLOCKS 148
#define CPL_THREADS 256

// One standard normal from Philox-4x32-10 (key seed, counter (draw lo,
// draw hi, i, axis)) by the Box-Muller cosine branch on u = (x + 1/2) 2^-32,
// in double precision (philox_gaussian_f64, kernels/philox.cuh:135-155).
__device__ double gauss64(uint32_t s_lo, uint32_t s_hi, unsigned long long draw, uint32_t i,
                          uint32_t axis) {
  uint32_t o0, o1;
  hb_philox(s_lo, s_hi, (uint32_t)draw, (uint32_t)(draw >> 32), i, axis, o0, o1);
  const double u1 = ((double)o0 + 0.5) * (1.0 / 4294967296.0);
  const double u2 = ((double)o1 + 0.5) * (1.0 / 4294967296.0);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// fixed-shape block tree over CPL_THREADS values
__device__ double block_sum(double v, double *sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int st = CPL_THREADS / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// CSVR: block b sums xi_i^2 over its contiguous chunk of i in [1, g)
__global__ void __launch_bounds__(CPL_THREADS)
    k_csvr_part(const CoupleState *__restrict__ st, double *__restrict__ part, uint32_t s_lo,
                uint32_t s_hi, uint32_t g) {
  __shared__ double sh[CPL_THREADS];
  const unsigned long long draw = st->draws;
  const uint32_t m = g > 0u ? g - 1u : 0u;
  const uint32_t chunk = (m + gridDim.x - 1u) / gridDim.x;
  const uint32_t start = blockIdx.x * chunk;
  const uint32_t end = min(start + chunk, m);
  double s = 0.0;
  for (uint32_t j = start + threadIdx.x; j < end; j += CPL_THREADS) {
    const double xi = gauss64(s_lo, s_hi, draw, j + 1u, 0u);
    s += xi * xi;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// CSVR chain (Bussi, Donadio and Parrinello 2007) in FP64
__global__ void __launch_bounds__(CPL_THREADS)
    k_csvr_finish(CoupleState *__restrict__ st, const double *__restrict__ part, uint32_t nb,
                  const double *__restrict__ ke, uint32_t s_lo, uint32_t s_hi, double c,
                  double one_minus_c, double kt_half) {
  __shared__ double sh[CPL_THREADS];
  double a = 0.0;
  for (uint32_t b = threadIdx.x; b < nb; b += CPL_THREADS) a += part[b];
  const double s = block_sum(a, sh);
  if (threadIdx.x == 0) {
    const unsigned long long draw = st->draws;
    const double r = gauss64(s_lo, s_hi, draw, 0u, 0u);
    const double k = ke[0];
    const double cross = k > 0.0 ? 2.0 * r * sqrt(c * one_minus_c * k * kt_half) : 0.0;
    double kn = c * k + kt_half * one_minus_c * (s + r * r) + cross;
    if (!isfinite(kn) || kn <= 0.0) kn = k;
    const double f = (k > 0.0 && kn != k) ? sqrt(kn / k) : 1.0;
    st->k = k;
    st->s = s;
    st->r = r;
    st->factor = f;
    st->injection += kn - k;
    st->draws = draw + 1ull;
  }
}

// Berendsen weak coupling: lambda^2 = 1 + dt/tau (K_target / K - 1)
__global__ void k_berendsen_factor(CoupleState *__restrict__ st, const double *__restrict__ ke,
                                   double k_target, double dt_over_tau) {
  const double k = ke[0];
  st->k = k;
  if (!(k > 0.0)) {
    st->factor = 1.0;
    return;
  }
  double lam2 = 1.0 + dt_over_tau * (k_target / k - 1.0);
  if (!(lam2 > 0.0)) lam2 = 0.0;
  st->factor = sqrt(lam2);
  st->injection += k * (lam2 - 1.0);
}

__global__ void k_draw_inc(CoupleState *st) { st->draws += 1ull; }

// per-block FP64 partial sums of a float array (the constraint virial)
__global__ void __launch_bounds__(CPL_THREADS)
    k_sum_part(const float *__restrict__ x, uint32_t n, double *__restrict__ part) {
  __shared__ double sh[CPL_THREADS];
  double a = 0.0;
  for (uint32_t i = blockIdx.x * CPL_THREADS + threadIdx.x; i < n; i += gridDim.x * CPL_THREADS)
    a += (double)x[i];
  a = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// Pressure coupling: P from the kinetic energy and the total virial, then
// mu^3 = 1 - kappa dt/tau (P0 - P) [+ noise], the FP64 lattice scaled by mu
// (c_rescale_compute_mu / berendsen_compute_mu, kernels/barostat.cu:140-255)
__global__ void __launch_bounds__(CPL_THREADS)
    k_pc_mu(CoupleState *__restrict__ st, const double *__restrict__ part, uint32_t nb,
            const double *__restrict__ ke, const double *__restrict__ scalars,
            double *__restrict__ lat, DBox *__restrict__ dbox, int noise, uint32_t s_lo,
            uint32_t s_hi, double p0, double dt_over_tau, double kappa, double noise_num,
            double r_search) {
  __shared__ double sh[CPL_THREADS];
  double a = 0.0;
  if (part)
    for (uint32_t b = threadIdx.x; b < nb; b += CPL_THREADS) a += part[b];
  const double w_cons = block_sum(a, sh);
  if (threadIdx.x != 0) return;
  const double v = lat[0] * lat[1] * lat[2];
  const double k = ke[0];
  const double w = scalars[7] + w_cons;
  const double p = (2.0 * k + w) / (3.0 * v);
  double r = 0.0;
  if (noise) {
    const unsigned long long draw = st->draws;
    r = gauss64(s_lo, s_hi, draw, 0u, 0u);
    st->draws = draw + 1ull;
  }
  double mu3 = 1.0 - kappa * dt_over_tau * (p0 - p);
  if (noise) mu3 += sqrt(noise_num / v) * r;
  const double mu3_min = 1.0e-18;  // (1e-6)^3
  if (!(mu3 > mu3_min)) mu3 = mu3_min;
  double mu = cbrt(mu3);
  double wd[3];
  hb_perp_widths(lat, wd);
  const double min_w = fmin(wd[0], fmin(wd[1], wd[2]));
  if (r_search > 0.0 && mu * min_w < 2.0 * r_search) {
    mu = 1.0;
    mu3 = 1.0;
    st->guarded += 1ull;
  }
  if (mu != 1.0) {
    for (int d = 0; d < 6; ++d) lat[d] *= mu;
    *dbox = hb_make_dbox(lat);
  }
  st->k = k;
  st->w = w;
  st->pressure = p;
  st->mu = mu;
  st->r = r;
  st->volume = v * mu3;
  st->injection += p0 * (v * mu3 - v);
}

// Final half kick with the coupling fused in.  TK: 0 none, 1 rescale by the
// thermostat factor, 2 Andersen collisions.  PC: scale positions by mu.
template <int TK, bool PC>
__global__ void k_vv_final(float4 *__restrict__ vel, float4 *__restrict__ posq,
                           const float4 *__restrict__ force, float dt,
                           const CoupleState *__restrict__ th, const CoupleState *__restrict__ pc,
                           uint32_t s_lo, uint32_t s_hi, float p_coll, double kt, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = vel[i];
  const float4 f = force[i];
  const float h = 0.5f * dt * v.w;
  v.x += f.x * h;
  v.y += f.y * h;
  v.z += f.z * h;
  if (TK == 1) {
    const float fac = (float)th->factor;
    v.x *= fac;
    v.y *= fac;
    v.z *= fac;
  } else if (TK == 2) {
    // andersen_resample (kernels/andersen.cu): Bernoulli on counter
    // (draw, id, 3), Maxwell-Boltzmann velocity on counters (draw, id, 0..2)
    const unsigned long long draw = th->draws;
    uint32_t o0, o1;
    hb_philox(s_lo, s_hi, (uint32_t)draw, (uint32_t)(draw >> 32), i, 3u, o0, o1);
    const double u = ((double)o0 + 0.5) * (1.0 / 4294967296.0);
    if (u < (double)p_coll && v.w > 0.0f) {
      const double sig = sqrt(kt * (double)v.w);
      v.x = (float)(sig * gauss64(s_lo, s_hi, draw, i, 0u));
      v.y = (float)(sig * gauss64(s_lo, s_hi, draw, i, 1u));
      v.z = (float)(sig * gauss64(s_lo, s_hi, draw, i, 2u));
    }
  }
  vel[i] = v;
  if (PC) {
    const float mu = (float)pc->mu;
    float4 p = posq[i];
    p.x *= mu;
    p.y *= mu;
    p.z *= mu;
    posq[i] = p;
  }
}

template <int TK, bool PC>
void launch_final(hb_integrator *it, cudaStream_t s, float p_coll) {
  hb_system *sys = it->sys;
  const hb_thermostat *t = it->thermo;
  k_vv_final<TK, PC><<<hb_div_up(sys->n, 256), 256, 0, s>>>(
      sys->d_vel, sys->d_posq, sys->d_force, (float)it->dt, t ? t->d_st : nullptr,
      it->pc ? it->pc->d_st : nullptr, t ? (uint32_t)t->seed : 0u,
      t ? (uint32_t)(t->seed >> 32) : 0u, p_coll, t ? t->kt : 0.0, sys->n);
}

}  // namespace

int couple_prepare(hb_integrator *it, hb_forcefield *ff, hb_constraints *cons, cudaStream_t s) {
  hb_system *sys = it->sys;
  hb_thermostat *t = it->thermo;
  hb_pcouple *pc = it->pc;
  const bool need_ke = pc || (t && t->kind != HB_THERMOSTAT_ANDERSEN);
  const double *ke = nullptr;
  if (need_ke) HB_TRY(reduce_kinetic_device(sys, s, &ke));
  if (t && t->kind == HB_THERMOSTAT_CSVR) {
    const double c = std::exp(-it->dt / t->tau);
    k_csvr_part<<<CPL_BLOCKS, CPL_THREADS, 0, s>>>(t->d_st, t->d_part, (uint32_t)t->seed,
                                                   (uint32_t)(t->seed >> 32), t->g_dof);
    k_csvr_finish<<<1, CPL_THREADS, 0, s>>>(t->d_st, t->d_part, CPL_BLOCKS, ke,
                                            (uint32_t)t->seed, (uint32_t)(t->seed >> 32), c,
                                            1.0 - c, 0.5 * t->kt);
  } else if (t && t->kind == HB_THERMOSTAT_BERENDSEN) {
    k_berendsen_factor<<<1, 1, 0, s>>>(t->d_st, ke, 0.5 * (double)t->g_dof * t->kt,
                                       it->dt / t->tau);
  }
  if (pc) {
    const bool with_cons = cons && sys->n > 0;
    if (with_cons)
      k_sum_part<<<CPL_BLOCKS, CPL_THREADS, 0, s>>>(cons->d_virial, sys->n, pc->d_part);
    const bool noise = pc->kind == HB_PCOUPLE_C_RESCALE;
    k_pc_mu<<<1, CPL_THREADS, 0, s>>>(
        pc->d_st, with_cons ? pc->d_part : nullptr, CPL_BLOCKS, ke, ff->d_scalars, sys->d_box64,
        sys->d_box, noise ? 1 : 0, (uint32_t)pc->seed, (uint32_t)(pc->seed >> 32), pc->pressure,
        it->dt / pc->tau, pc->kappa, 2.0 * pc->kappa * pc->kt * it->dt / pc->tau,
        (double)ff->r_search);
  }
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int couple_final_kick(hb_integrator *it, cudaStream_t s) {
  hb_system *sys = it->sys;
  if (sys->n == 0) return HB_OK;
  const hb_thermostat *t = it->thermo;
  const int tk = !t ? 0 : (t->kind == HB_THERMOSTAT_ANDERSEN ? 2 : 1);
  // p = clamp(rate dt, 0, 1), held in single precision like the reference's
  // Real argument (src/integrator/andersen.rs:154-162)
  const float p_coll = t ? (float)std::min(std::max(t->rate * it->dt, 0.0), 1.0) : 0.0f;
  const bool pc = it->pc != nullptr;
  if (tk == 0 && pc) launch_final<0, true>(it, s, p_coll);
  else if (tk == 1 && !pc) launch_final<1, false>(it, s, p_coll);
  else if (tk == 1 && pc) launch_final<1, true>(it, s, p_coll);
  else if (tk == 2 && !pc) launch_final<2, false>(it, s, p_coll);
  else if (tk == 2 && pc) launch_final<2, true>(it, s, p_coll);
  else launch_final<0, false>(it, s, p_coll);
  if (tk == 2) k_draw_inc<<<1, 1, 0, s>>>(t->d_st);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

// ---------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------
extern "C" int hb_thermostat_create(hb_system *sys, const hb_thermostat_desc *d,
                                    hb_thermostat **out) {
  HB_REQUIRE(sys && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(d->kind == HB_THERMOSTAT_CSVR || d->kind == HB_THERMOSTAT_ANDERSEN ||
                 d->kind == HB_THERMOSTAT_BERENDSEN,
             HB_ERR_INVALID_ARGUMENT, "unknown thermostat kind");
  HB_REQUIRE(std::isfinite(d->temperature) && d->temperature > 0.0, HB_ERR_INVALID_ARGUMENT,
             "thermostat.temperature must be finite and strictly positive");
  if (d->kind == HB_THERMOSTAT_ANDERSEN)
    HB_REQUIRE(std::isfinite(d->collision_rate) && d->collision_rate >= 0.0,
               HB_ERR_INVALID_ARGUMENT, "thermostat.collision_rate must be finite and >= 0");
  else
    HB_REQUIRE(std::isfinite(d->tau) && d->tau > 0.0, HB_ERR_INVALID_ARGUMENT,
               "thermostat.tau must be finite and strictly positive");
  hb_thermostat *t = new hb_thermostat();
  t->sys = sys;
  t->kind = d->kind;
  t->kt = d->temperature;
  t->tau = d->tau;
  t->rate = d->collision_rate;
  t->seed = d->seed;
  const long long g = 3ll * (long long)sys->n - (long long)d->n_constraints - 3ll;
  t->g_dof = (uint32_t)std::max(g, 1ll);
  CoupleState zero{};
  zero.factor = 1.0;
  zero.mu = 1.0;
  if (cudaMalloc(&t->d_st, sizeof(CoupleState)) != cudaSuccess ||
      cudaMemcpy(t->d_st, &zero, sizeof(CoupleState), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMalloc(&t->d_part, sizeof(double) * CPL_BLOCKS) != cudaSuccess) {
    hb_thermostat_destroy(t);
    return hb_fail(HB_ERR_CUDA, "thermostat state allocation failed");
  }
  *out = t;
  return HB_OK;
}

extern "C" int hb_thermostat_destroy(hb_thermostat *t) {
  if (!t) return HB_OK;
  cudaStreamSynchronize(t->sys->ctx->stream);
  cudaFree(t->d_st);
  cudaFree(t->d_part);
  delete t;
  return HB_OK;
}

extern "C" int hb_thermostat_stats(hb_thermostat *t, double out[7]) {
  HB_REQUIRE(t && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  CoupleState h;
  HB_CUDA(cudaStreamSynchronize(t->sys->ctx->stream));
  HB_CUDA(cudaMemcpy(&h, t->d_st, sizeof(CoupleState), cudaMemcpyDeviceToHost));
  out[0] = h.injection;
  out[1] = h.k;
  out[2] = h.factor;
  out[3] = h.s;
  out[4] = h.r;
  out[5] = (double)h.draws;
  out[6] = (double)t->g_dof;
  return HB_OK;
}

extern "C" int hb_integrator_set_thermostat(hb_integrator *it, hb_thermostat *t) {
  HB_REQUIRE(it, HB_ERR_INVALID_ARGUMENT, "null integrator");
  HB_REQUIRE(!t || t->sys == it->sys, HB_ERR_INVALID_ARGUMENT,
             "integrator and thermostat must share one system");
  HB_REQUIRE(!t || it->kind == HB_INTEGRATOR_VV, HB_ERR_UNSUPPORTED,
             "a thermostat needs the (non-lossless) velocity-Verlet integrator");
  it->thermo = t;
  return HB_OK;
}

extern "C" int hb_pcouple_create(hb_system *sys, const hb_pcouple_desc *d, hb_pcouple **out) {
  HB_REQUIRE(sys && d && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  HB_REQUIRE(d->kind == HB_PCOUPLE_C_RESCALE || d->kind == HB_PCOUPLE_BERENDSEN,
             HB_ERR_INVALID_ARGUMENT, "unknown pressure coupling kind");
  HB_REQUIRE(std::isfinite(d->pressure), HB_ERR_INVALID_ARGUMENT,
             "barostat.pressure must be finite");
  HB_REQUIRE(std::isfinite(d->tau) && d->tau > 0.0, HB_ERR_INVALID_ARGUMENT,
             "barostat.tau must be finite and strictly positive");
  HB_REQUIRE(std::isfinite(d->compressibility) && d->compressibility > 0.0,
             HB_ERR_INVALID_ARGUMENT, "barostat.compressibility must be finite and strictly positive");
  if (d->kind == HB_PCOUPLE_C_RESCALE)
    HB_REQUIRE(std::isfinite(d->temperature) && d->temperature > 0.0, HB_ERR_INVALID_ARGUMENT,
               "barostat.temperature must be finite and strictly positive");
  hb_pcouple *p = new hb_pcouple();
  p->sys = sys;
  p->kind = d->kind;
  p->pressure = d->pressure;
  p->kt = d->temperature;
  p->tau = d->tau;
  p->kappa = d->compressibility;
  p->seed = d->seed;
  CoupleState zero{};
  zero.factor = 1.0;
  zero.mu = 1.0;
  zero.volume = sys->box[0] * sys->box[1] * sys->box[2];
  if (cudaMalloc(&p->d_st, sizeof(CoupleState)) != cudaSuccess ||
      cudaMemcpy(p->d_st, &zero, sizeof(CoupleState), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMalloc(&p->d_part, sizeof(double) * CPL_BLOCKS) != cudaSuccess) {
    hb_pcouple_destroy(p);
    return hb_fail(HB_ERR_CUDA, "pressure coupling state allocation failed");
  }
  *out = p;
  return HB_OK;
}

extern "C" int hb_pcouple_destroy(hb_pcouple *p) {
  if (!p) return HB_OK;
  cudaStreamSynchronize(p->sys->ctx->stream);
  cudaFree(p->d_st);
  cudaFree(p->d_part);
  delete p;
  return HB_OK;
}

extern "C" int hb_pcouple_stats(hb_pcouple *p, double out[8]) {
  HB_REQUIRE(p && out, HB_ERR_INVALID_ARGUMENT, "null argument");
  CoupleState h;
  HB_CUDA(cudaStreamSynchronize(p->sys->ctx->stream));
  HB_CUDA(cudaMemcpy(&h, p->d_st, sizeof(CoupleState), cudaMemcpyDeviceToHost));
  out[0] = h.pressure;
  out[1] = h.volume;
  out[2] = h.injection;
  out[3] = h.mu;
  out[4] = (double)h.draws;
  out[5] = h.k;
  out[6] = h.w;
  out[7] = (double)h.guarded;
  return HB_OK;
}

extern "C" int hb_integrator_set_pcouple(hb_integrator *it, hb_pcouple *p) {
  HB_REQUIRE(it, HB_ERR_INVALID_ARGUMENT, "null integrator");
  HB_REQUIRE(!p || p->sys == it->sys, HB_ERR_INVALID_ARGUMENT,
             "integrator and pressure coupling must share one system");
  HB_REQUIRE(!p || it->kind == HB_INTEGRATOR_VV, HB_ERR_UNSUPPORTED,
             "pressure coupling needs the (non-lossless) velocity-Verlet integrator");
  HB_REQUIRE(!p || !it->baro, HB_ERR_UNSUPPORTED,
             "one barostat per integrator: detach the Monte-Carlo barostat first");
  it->pc = p;
  return HB_OK;
}
