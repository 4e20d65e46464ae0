// hb_min.cu -- steepest-descent energy minimisation on the device.
//
// Replaces SteepestDescentMinimizer (src/minimizer/steepest_descent.rs:123-300)
// and its kernels (kernels/minimize.cu): trial step x + s F / F_max, the
// constraint projection, a forces + energy evaluation, accept when the
// energy drops (s <- min(s * increase, max_step)), else restore
// (s <- s * decrease).  The reference decides each iteration on the host
// after two device-to-host reads; here every decision is a one-thread
// kernel on device state, so a call runs many iterations back to back with
// one read of their reports at the end:
//   * F_max is a max over |F|^2 in single precision (order-free, so the
//     multi-block reduction is exact), square-rooted once;
//   * a rejected trial restores positions, images, forces and scalars from
//     a snapshot instead of evaluating the forces again (the evaluation is
//     deterministic, so the restored state is the one it would recompute);
//   * once an iteration reports convergence, the following iterations of
//     the call are no-ops on the device (the skip flag gates the trial, the
//     projection, the decision and the report; the force evaluation of a
//     skipped iteration sees unchanged positions).
#include <algorithm>
#include <cmath>

#include "hb_internal.cuh"

namespace {

#define MIN_BLOCKS 148
#define MIN_THREADS 256

__device__ float block_max(float v, float *sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int st = MIN_THREADS / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + st]);
    __syncthreads();
  }
  const float r = sh[0];
  __syncthreads();
  return r;
}

// per-block maximum of |F_i|^2 (sd_f_max_reduction, kernels/minimize.cu:70-113)
__global__ void __launch_bounds__(MIN_THREADS)
    k_min_fmax_part(const float4 *__restrict__ force, uint32_t n, float *__restrict__ part) {
  __shared__ float sh[MIN_THREADS];
  float m = 0.0f;
  for (uint32_t i = blockIdx.x * MIN_THREADS + threadIdx.x; i < n; i += gridDim.x * MIN_THREADS) {
    const float4 f = force[i];
    const float m2 = f.x * f.x + f.y * f.y + f.z * f.z;
    if (m2 > m) m = m2;
  }
  m = block_max(m, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = m;
}

__device__ float fmax_of(const float *part, uint32_t nb, float *sh) {
  float m = 0.0f;
  for (uint32_t b = threadIdx.x; b < nb; b += MIN_THREADS) m = fmaxf(m, part[b]);
  return sqrtf(block_max(m, sh));
}

__device__ int force_criteria(float fmax, double ftol) {
  if (fmax == 0.0f) return HB_MIN_FORCE_ZERO;
  if (ftol > 0.0 && (double)fmax <= ftol) return HB_MIN_FORCE_TOLERANCE;
  return 0;
}

// initial_state + the runner's pre-loop check (src/runner.rs:1896-1965):
// iteration-0 report, only force criteria
__global__ void __launch_bounds__(MIN_THREADS)
    k_min_init(MinState *__restrict__ st, const float *__restrict__ part, uint32_t nb,
               const double *__restrict__ scal, float step0, double ftol,
               hb_min_report *__restrict__ rep) {
  __shared__ float sh[MIN_THREADS];
  const float fm = fmax_of(part, nb, sh);
  if (threadIdx.x != 0) return;
  st->last_energy = scal[4];
  st->prev_energy = scal[4];
  st->step = step0;
  st->step_used = 0.0f;
  st->fmax = fm;
  st->iteration = 0;
  st->skip = 0;
  st->reject = 0;
  st->converged = force_criteria(fm, ftol);
  rep->iteration = 0;
  rep->energy = scal[4];
  rep->max_force = fm;
  rep->step = 0.0;
  rep->accepted = 1;
  rep->converged = st->converged;
}

__global__ void k_min_begin(MinState *__restrict__ st, const double *__restrict__ scal,
                            double *__restrict__ snap) {
  const bool skip = st->converged != 0 || !(st->fmax > 0.0f);
  st->skip = skip ? 1 : 0;
  st->reject = 0;
  if (skip) return;
  st->prev_energy = st->last_energy;
  st->step_used = st->step;
  // x_trial = x + step F / F_max with 1 / F_max taken once
  // (steepest_descent.rs:193-197, sd_compute_step kernels/minimize.cu:8-27)
  st->scale = st->step * (1.0f / st->fmax);
  for (int q = 0; q < HB_N_SCALARS; ++q) snap[q] = scal[q];
}

__global__ void k_min_trial(float4 *__restrict__ posq, int4 *__restrict__ image,
                            const float4 *__restrict__ force, float4 *__restrict__ sp,
                            int4 *__restrict__ si, float4 *__restrict__ sf,
                            const DBox *__restrict__ box, const MinState *__restrict__ st,
                            uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || st->skip) return;
  const float scale = st->scale;
  float4 p = posq[i];
  int4 im = image[i];
  const float4 f = force[i];
  sp[i] = p;
  si[i] = im;
  sf[i] = f;
  p.x = p.x + f.x * scale;
  p.y = p.y + f.y * scale;
  p.z = p.z + f.z * scale;
  int ka, kb, kc;
  hb_wrap(p.x, p.y, p.z, ka, kb, kc, *box);
  im.x += ka;
  im.y += kb;
  im.z += kc;
  posq[i] = p;
  image[i] = im;
}

__global__ void k_min_decide(MinState *__restrict__ st, double *__restrict__ scal,
                             const double *__restrict__ snap, float inc, float dec,
                             float max_step) {
  if (st->skip) return;
  const double e = scal[4];
  st->e_trial = e;
  if (e < st->last_energy) {
    st->last_energy = e;
    st->step = fminf(st->step * inc, max_step);
    st->reject = 0;
  } else {
    for (int q = 0; q < HB_N_SCALARS; ++q) scal[q] = snap[q];
    st->step = st->step * dec;
    st->reject = 1;
  }
}

__global__ void k_min_restore(float4 *__restrict__ posq, int4 *__restrict__ image,
                              float4 *__restrict__ force, const float4 *__restrict__ sp,
                              const int4 *__restrict__ si, const float4 *__restrict__ sf,
                              const MinState *__restrict__ st, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || st->skip || !st->reject) return;
  posq[i] = sp[i];
  image[i] = si[i];
  force[i] = sf[i];
}

// MinimizerStepReport and check_convergence (steepest_descent.rs:210-283)
__global__ void __launch_bounds__(MIN_THREADS)
    k_min_report(MinState *__restrict__ st, const float *__restrict__ part, uint32_t nb,
                 double ftol, double etol, hb_min_report *__restrict__ rep, uint32_t slot) {
  __shared__ float sh[MIN_THREADS];
  const float fm = fmax_of(part, nb, sh);
  if (threadIdx.x != 0 || st->skip) return;
  const bool acc = !st->reject;
  st->iteration += 1ull;
  st->fmax = fm;
  const double e = acc ? st->e_trial : st->prev_energy;
  int reason = force_criteria(fm, ftol);
  if (!reason && acc && etol > 0.0 &&
      fabs(e - st->prev_energy) <= etol * fmax(fmax(fabs(e), fabs(st->prev_energy)), 1.0e-30))
    reason = HB_MIN_ENERGY_TOLERANCE;
  st->converged = reason;
  hb_min_report r;
  r.iteration = st->iteration;
  r.energy = e;
  r.max_force = fm;
  r.step = st->step_used;
  r.accepted = acc ? 1 : 0;
  r.converged = reason;
  rep[slot] = r;
}

}  // namespace

int min_fmax(hb_minimizer *m, cudaStream_t s) {
  hb_system *sys = m->ff->sys;
  k_min_fmax_part<<<MIN_BLOCKS, MIN_THREADS, 0, s>>>(sys->d_force, sys->n, m->d_part);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int min_init(hb_minimizer *m, cudaStream_t s) {
  HB_TRY(min_fmax(m, s));
  k_min_init<<<1, MIN_THREADS, 0, s>>>(m->d_st, m->d_part, MIN_BLOCKS, m->ff->d_scalars,
                                       m->initial_step, m->ftol, m->d_rep);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int min_trial(hb_minimizer *m, cudaStream_t s) {
  hb_system *sys = m->ff->sys;
  k_min_begin<<<1, 1, 0, s>>>(m->d_st, m->ff->d_scalars, m->d_snap_scal);
  if (sys->n)
    k_min_trial<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_posq, sys->d_image, sys->d_force,
                                                       m->d_snap_pos, m->d_snap_img,
                                                       m->d_snap_force, sys->d_box, m->d_st,
                                                       sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int min_finish(hb_minimizer *m, uint32_t slot, cudaStream_t s) {
  hb_system *sys = m->ff->sys;
  k_min_decide<<<1, 1, 0, s>>>(m->d_st, m->ff->d_scalars, m->d_snap_scal, m->inc, m->dec,
                               m->max_step);
  if (sys->n)
    k_min_restore<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_posq, sys->d_image,
                                                         sys->d_force, m->d_snap_pos,
                                                         m->d_snap_img, m->d_snap_force,
                                                         m->d_st, sys->n);
  HB_TRY(min_fmax(m, s));
  k_min_report<<<1, MIN_THREADS, 0, s>>>(m->d_st, m->d_part, MIN_BLOCKS, m->ftol, m->etol,
                                         m->d_rep, slot);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int min_alloc(hb_minimizer *m) {
  const uint32_t n = std::max(m->ff->sys->n, 1u);
  HB_CUDA(cudaMalloc(&m->d_st, sizeof(MinState)));
  HB_CUDA(cudaMemset(m->d_st, 0, sizeof(MinState)));
  HB_CUDA(cudaMalloc(&m->d_rep, sizeof(hb_min_report) * m->rep_cap));
  HB_CUDA(cudaMalloc(&m->d_part, sizeof(float) * MIN_BLOCKS));
  HB_CUDA(cudaMalloc(&m->d_snap_pos, sizeof(float4) * n));
  HB_CUDA(cudaMalloc(&m->d_snap_force, sizeof(float4) * n));
  HB_CUDA(cudaMalloc(&m->d_snap_img, sizeof(int4) * n));
  HB_CUDA(cudaMalloc(&m->d_snap_scal, sizeof(double) * HB_N_SCALARS));
  return HB_OK;
}

void min_free(hb_minimizer *m) {
  cudaFree(m->d_st);
  cudaFree(m->d_rep);
  cudaFree(m->d_part);
  cudaFree(m->d_snap_pos);
  cudaFree(m->d_snap_force);
  cudaFree(m->d_snap_img);
  cudaFree(m->d_snap_scal);
}
