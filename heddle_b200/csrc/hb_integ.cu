// hb_integ.cu -- force combine, FP64 scalar reductions and the integrator
// kernels of the B200 force-and-constraint path.
//
//   * k_finalize: int64 fixed-point pair sums + SPME reciprocal terms ->
//     f32 force per atom (atom order), clearing the accumulators for the
//     next step (replaces finalize_packed_forces + combine_class_totals,
//     kernels/neighbor.cu:728-760, kernels/forces.cu:13-41);
//   * energy / virial totals are exact int64 sums of the fixed-point
//     per-atom shares (order-independent), the reciprocal terms are FP64
//     fixed-shape trees -> byte-identical scalars run to run
//     (kernels/nose_hoover.cu:22-103, kernels/barostat.cu:11-78);
//   * velocity Verlet kick-drift / kick (kernels/integrate.cu:24-265) with
//     a lossless variant, and the Langevin
//     middle scheme whose O step draws Philox-4x32-10 Gaussians keyed by
//     (seed, step, atom, axis) (kernels/langevin.cu:13-80,
//     kernels/philox.cuh).
#include <cmath>

#include "hb_internal.cuh"

namespace {

__device__ __forceinline__ float from_fixed(unsigned long long v) {
  return (float)((double)(long long)v * HB_FP_INV_SCALE);
}

template <bool EV>
__global__ void k_finalize(unsigned long long *__restrict__ fp, const float4 *__restrict__ recip,
                           const uint32_t *__restrict__ sorted_ids, float4 *__restrict__ force,
                           float *__restrict__ energy, float *__restrict__ virial,
                           const double *__restrict__ spme_sums,
                           unsigned long long *__restrict__ acc, uint32_t *__restrict__ work,
                           uint32_t n, uint32_t np) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0) *work = 0u;  // the pair kernel's work counter, for the next evaluation
  long long e_fix = 0, w_fix = 0;
  if (k < n) {
    const uint32_t id = sorted_ids[k];
    float fx = from_fixed(fp[k]);
    float fy = from_fixed(fp[np + k]);
    float fz = from_fixed(fp[2 * np + k]);
    fp[k] = 0ull;
    fp[np + k] = 0ull;
    fp[2 * np + k] = 0ull;
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (recip) r = recip[k];
    force[id] = make_float4(fx + r.x, fy + r.y, fz + r.z, 0.0f);
    if (EV) {
      e_fix = (long long)fp[3 * np + k];
      w_fix = (long long)fp[4 * np + k];
      fp[3 * np + k] = 0ull;
      fp[4 * np + k] = 0ull;
      float wr = spme_sums ? (float)(spme_sums[1] / (double)n) : 0.0f;
      energy[id] = (float)((double)e_fix * HB_FP_INV_SCALE) + r.w;
      virial[id] = (float)((double)w_fix * HB_FP_INV_SCALE) + wr;
    }
  }
  if (EV) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e_fix += __shfl_xor_sync(0xFFFFFFFFu, e_fix, o);
      w_fix += __shfl_xor_sync(0xFFFFFFFFu, w_fix, o);
    }
    if ((threadIdx.x & 31u) == 0u) {
      if (e_fix) atomicAdd(&acc[1], (unsigned long long)e_fix);
      if (w_fix) atomicAdd(&acc[2], (unsigned long long)w_fix);
    }
  }
}

__global__ void k_scalars(unsigned long long *__restrict__ acc,
                          const double *__restrict__ spme_sums, double e_self,
                          const float4 *__restrict__ recip_unused, double *__restrict__ out) {
  const double lj = (double)(long long)acc[0] * HB_FP_INV_SCALE;
  const double pair = (double)(long long)acc[1] * HB_FP_INV_SCALE;
  const double wp = (double)(long long)acc[2] * HB_FP_INV_SCALE;
  const double eb = (double)(long long)acc[3] * HB_FP_INV_SCALE;
  const double er = spme_sums ? spme_sums[0] : 0.0;
  const double wr = spme_sums ? spme_sums[1] : 0.0;
  out[0] = lj;
  out[1] = pair - lj - eb;
  out[2] = er;
  out[3] = spme_sums ? e_self : 0.0;
  out[4] = pair + er - (spme_sums ? e_self : 0.0);
  out[5] = wp;
  out[6] = wr;
  out[7] = wp + wr;
  out[8] = eb;
  out[9] = 0.0;
  acc[0] = 0ull;
  acc[1] = 0ull;
  acc[2] = 0ull;
  acc[3] = 0ull;
}


__global__ void k_vv_kick_drift(float4 *__restrict__ posq, float4 *__restrict__ vel,
                                int4 *__restrict__ image, const float4 *__restrict__ force,
                                float4 *__restrict__ prev, const DBox *__restrict__ box, float dt,
                                uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DBox b = *box;
  float4 p = posq[i];
  float4 v = vel[i];
  const float4 f = force[i];
  prev[i] = p;
  const float h = 0.5f * dt * v.w;
  v.x += f.x * h;
  v.y += f.y * h;
  v.z += f.z * h;
  p.x += v.x * dt;
  p.y += v.y * dt;
  p.z += v.z * dt;
  int ka, kb, kc;
  hb_wrap(p.x, p.y, p.z, ka, kb, kc, b);
  int4 im = image[i];
  im.x += ka;
  im.y += kb;
  im.z += kc;
  image[i] = im;
  posq[i] = p;
  vel[i] = v;
}

__global__ void k_vv_kick(float4 *__restrict__ vel, const float4 *__restrict__ force, float dt,
                          uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = vel[i];
  const float4 f = force[i];
  const float h = 0.5f * dt * v.w;
  v.x += f.x * h;
  v.y += f.y * h;
  v.z += f.z * h;
  vel[i] = v;
}

// Lossless variant.  The reference carries (f32 value, f64 low part) pairs
// (kernels/integrate.cu:46-110); their round trip is exact only while no
// f64 rounding error crosses an f32 rounding boundary.  Here the state is
// 64-bit fixed point -- X in 2^-40 bohr, V in 2^-56 bohr/aut -- and one
// step is
//   V += K(X),  X += g(V),  wrap X by integer lattice vectors,  V += K(X)
// with K(X) = rint(F(X) dt / 2m * 2^56) and g(V) = rint(V dt 2^-16), g odd.
// Every update is an integer addition, so flipping V and stepping again
// retraces the trajectory exactly (bit-exact time reversal by
// construction, given forces that are a function of the positions alone).
// posq / vel are the f32 images of X / V.
__device__ __forceinline__ long long fix_kick(float f, double kc) {
  return llrint((double)f * kc);
}

__global__ void k_fix_derive(float4 *__restrict__ posq, float4 *__restrict__ vel,
                             long long *__restrict__ xfix, long long *__restrict__ vfix,
                             uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = posq[i], v = vel[i];
  const long long X[3] = {llrint((double)p.x * HB_XFIX_SCALE), llrint((double)p.y * HB_XFIX_SCALE),
                          llrint((double)p.z * HB_XFIX_SCALE)};
  const long long V[3] = {llrint((double)v.x * HB_VFIX_SCALE), llrint((double)v.y * HB_VFIX_SCALE),
                          llrint((double)v.z * HB_VFIX_SCALE)};
  for (int d = 0; d < 3; ++d) {
    xfix[3 * i + d] = X[d];
    vfix[3 * i + d] = V[d];
  }
  p.x = (float)((double)X[0] / HB_XFIX_SCALE);
  p.y = (float)((double)X[1] / HB_XFIX_SCALE);
  p.z = (float)((double)X[2] / HB_XFIX_SCALE);
  v.x = (float)((double)V[0] / HB_VFIX_SCALE);
  v.y = (float)((double)V[1] / HB_VFIX_SCALE);
  v.z = (float)((double)V[2] / HB_VFIX_SCALE);
  posq[i] = p;
  vel[i] = v;
}

__global__ void k_vvl_kick_drift(float4 *__restrict__ posq, float4 *__restrict__ vel,
                                 int4 *__restrict__ image, const float4 *__restrict__ force,
                                 float4 *__restrict__ prev, long long *__restrict__ xfix,
                                 long long *__restrict__ vfix, const double *__restrict__ lat,
                                 double dt, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = posq[i];
  float4 v = vel[i];
  const float4 f = force[i];
  prev[i] = p;
  const double kc = 0.5 * dt * (double)v.w * HB_VFIX_SCALE;
  const double gc = dt * (HB_XFIX_SCALE / HB_VFIX_SCALE);
  long long X[3], V[3];
  const float fa3[3] = {f.x, f.y, f.z};
  for (int d = 0; d < 3; ++d) {
    V[d] = vfix[3 * i + d] + fix_kick(fa3[d], kc);
    X[d] = xfix[3 * i + d] + llrint((double)V[d] * gc);
  }
  // wrap by integer lattice vectors of the FP64 lattice
  const double lx = lat[0], ly = lat[1], lz = lat[2], xy = lat[3], xz = lat[4], yz = lat[5];
  const double x = (double)X[0] / HB_XFIX_SCALE, y = (double)X[1] / HB_XFIX_SCALE,
               z = (double)X[2] / HB_XFIX_SCALE;
  const double sc = z / lz, sb = (y - sc * yz) / ly, sa = (x - sb * xy - sc * xz) / lx;
  const long long ka = (long long)floor(sa + 0.5), kb = (long long)floor(sb + 0.5),
                  kcc = (long long)floor(sc + 0.5);
  if (ka | kb | kcc) {
    const long long LX = llrint(lx * HB_XFIX_SCALE), LY = llrint(ly * HB_XFIX_SCALE),
                    LZ = llrint(lz * HB_XFIX_SCALE), XY = llrint(xy * HB_XFIX_SCALE),
                    XZ = llrint(xz * HB_XFIX_SCALE), YZ = llrint(yz * HB_XFIX_SCALE);
    X[0] -= ka * LX + kb * XY + kcc * XZ;
    X[1] -= kb * LY + kcc * YZ;
    X[2] -= kcc * LZ;
    int4 im = image[i];
    im.x += (int)ka;
    im.y += (int)kb;
    im.z += (int)kcc;
    image[i] = im;
  }
  for (int d = 0; d < 3; ++d) {
    xfix[3 * i + d] = X[d];
    vfix[3 * i + d] = V[d];
  }
  p.x = (float)((double)X[0] / HB_XFIX_SCALE);
  p.y = (float)((double)X[1] / HB_XFIX_SCALE);
  p.z = (float)((double)X[2] / HB_XFIX_SCALE);
  v.x = (float)((double)V[0] / HB_VFIX_SCALE);
  v.y = (float)((double)V[1] / HB_VFIX_SCALE);
  v.z = (float)((double)V[2] / HB_VFIX_SCALE);
  posq[i] = p;
  vel[i] = v;
}

__global__ void k_vvl_kick(float4 *__restrict__ vel, const float4 *__restrict__ force,
                           long long *__restrict__ vfix, double dt, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = vel[i];
  const float4 f = force[i];
  const double kc = 0.5 * dt * (double)v.w * HB_VFIX_SCALE;
  const long long V0 = vfix[3 * i] + fix_kick(f.x, kc);
  const long long V1 = vfix[3 * i + 1] + fix_kick(f.y, kc);
  const long long V2 = vfix[3 * i + 2] + fix_kick(f.z, kc);
  vfix[3 * i] = V0;
  vfix[3 * i + 1] = V1;
  vfix[3 * i + 2] = V2;
  v.x = (float)((double)V0 / HB_VFIX_SCALE);
  v.y = (float)((double)V1 / HB_VFIX_SCALE);
  v.z = (float)((double)V2 / HB_VFIX_SCALE);
  vel[i] = v;
}

// v <- -v on the f32 velocity and its fixed-point state
__global__ void k_flip_velocities(float4 *__restrict__ vel, long long *__restrict__ vfix,
                                  uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = vel[i];
  v.x = -v.x;
  v.y = -v.y;
  v.z = -v.z;
  vel[i] = v;
  vfix[3 * i] = -vfix[3 * i];
  vfix[3 * i + 1] = -vfix[3 * i + 1];
  vfix[3 * i + 2] = -vfix[3 * i + 2];
}

__global__ void k_lang_kick(float4 *__restrict__ vel, const float4 *__restrict__ force, float dt,
                            uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = vel[i];
  hb_lang_kick(v, force[i], dt);
  vel[i] = v;
}

__global__ void k_lang_drift_ou(float4 *__restrict__ posq, float4 *__restrict__ vel,
                                int4 *__restrict__ image, float4 *__restrict__ prev,
                                const DBox *__restrict__ box, float dt, float a, float kt,
                                uint32_t s_lo, uint32_t s_hi, const uint64_t *__restrict__ step_ptr,
                                uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t step = *step_ptr;
  const DBox b = *box;
  float4 p = posq[i];
  float4 v = vel[i];
  prev[i] = p;
  int4 im = image[i];
  hb_lang_drift_ou(p, v, im, dt, a, kt, s_lo, s_hi, step, i, b);
  image[i] = im;
  posq[i] = p;
  vel[i] = v;
}

// the Philox draw counter lives on the device so a captured step advances
// it on every replay
__global__ void k_step_inc(uint64_t *step) { *step += 1ull; }

#define RED_BLOCKS 296
// kinetic energy and momentum, FP64, fixed grid and fixed tree shape
__global__ void k_kinetic_part(const float4 *__restrict__ vel, double *__restrict__ part,
                               uint32_t n) {
  __shared__ double s[4][256];
  double ke = 0.0, px = 0.0, py = 0.0, pz = 0.0;
  for (uint32_t i = blockIdx.x * 256u + threadIdx.x; i < n; i += gridDim.x * 256u) {
    const float4 v = vel[i];
    if (v.w > 0.0f) {
      const double m = 1.0 / (double)v.w;
      ke += 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
      px += m * v.x;
      py += m * v.y;
      pz += m * v.z;
    }
  }
  s[0][threadIdx.x] = ke;
  s[1][threadIdx.x] = px;
  s[2][threadIdx.x] = py;
  s[3][threadIdx.x] = pz;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int q = 0; q < 4; ++q) s[q][threadIdx.x] += s[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[4 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_kinetic_final(const double *__restrict__ part, int nb, double *__restrict__ out) {
  __shared__ double s[4][256];
  double a[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += 256)
    for (int q = 0; q < 4; ++q) a[q] += part[4 * b + q];
  for (int q = 0; q < 4; ++q) s[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int q = 0; q < 4; ++q) s[q][threadIdx.x] += s[q][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = s[threadIdx.x][0];
}

}  // namespace

int forces_finalize(hb_forcefield *ff, bool ev, cudaStream_t s) {
  hb_system *sys = ff->sys;
  const uint32_t n = sys->n;
  const float4 *recip = ff->spme.on ? ff->spme.d_recip : nullptr;
  const double *sums = ff->spme.on ? ff->spme.d_sums : nullptr;
  if (n > 0) {
    if (ev)
      k_finalize<true><<<hb_div_up(n, 256), 256, 0, s>>>(ff->d_fp, recip, ff->d_sorted_ids,
                                                         sys->d_force, ff->d_energy, ff->d_virial,
                                                         sums, ff->d_acc, ff->d_work, n, ff->n_pad);
    else
      k_finalize<false><<<hb_div_up(n, 256), 256, 0, s>>>(ff->d_fp, recip, ff->d_sorted_ids,
                                                          sys->d_force, ff->d_energy,
                                                          ff->d_virial, sums, ff->d_acc,
                                                          ff->d_work, n, ff->n_pad);
  }
  if (ev) {
    double e_self = 0.0;
    if (ff->spme.on) {
      for (double q : sys->h_charge) e_self += q * q;
      e_self *= (double)ff->spme.alpha / std::sqrt(M_PI);
    }
    k_scalars<<<1, 1, 0, s>>>(ff->d_acc, sums, e_self, nullptr, ff->d_scalars);
  }
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int integ_vv_kick_drift(hb_integrator *it, cudaStream_t s) {
  hb_system *sys = it->sys;
  if (sys->n == 0) return HB_OK;
  if (it->kind == HB_INTEGRATOR_VV_LOSSLESS)
    k_vvl_kick_drift<<<hb_div_up(sys->n, 256), 256, 0, s>>>(
        sys->d_posq, sys->d_vel, sys->d_image, sys->d_force, sys->d_pos_prev, sys->d_xfix,
        sys->d_vfix, sys->d_box64, it->dt, sys->n);
  else
    k_vv_kick_drift<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_posq, sys->d_vel, sys->d_image,
                                                           sys->d_force, sys->d_pos_prev,
                                                           sys->d_box, (float)it->dt, sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int integ_flip_velocities(hb_system *sys, cudaStream_t s) {
  if (sys->n == 0) return HB_OK;
  k_flip_velocities<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_vel, sys->d_vfix, sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int integ_fix_derive(hb_system *sys, cudaStream_t s) {
  if (sys->n)
    k_fix_derive<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_posq, sys->d_vel, sys->d_xfix,
                                                        sys->d_vfix, sys->n);
  HB_CUDA(cudaGetLastError());
  sys->fix_valid = true;
  return HB_OK;
}

int integ_vv_kick(hb_integrator *it, cudaStream_t s) {
  hb_system *sys = it->sys;
  if (sys->n == 0) return HB_OK;
  if (it->kind == HB_INTEGRATOR_VV_LOSSLESS)
    k_vvl_kick<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_vel, sys->d_force, sys->d_vfix,
                                                      it->dt, sys->n);
  else
    k_vv_kick<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_vel, sys->d_force, (float)it->dt,
                                                     sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int integ_lang_kick(hb_integrator *it, cudaStream_t s) {
  hb_system *sys = it->sys;
  if (sys->n == 0) return HB_OK;
  k_lang_kick<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_vel, sys->d_force, (float)it->dt,
                                                     sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int integ_lang_drift_ou(hb_integrator *it, cudaStream_t s) {
  hb_system *sys = it->sys;
  if (sys->n == 0) return HB_OK;
  const float a = (float)std::exp(-it->friction * it->dt);
  k_lang_drift_ou<<<hb_div_up(sys->n, 256), 256, 0, s>>>(
      sys->d_posq, sys->d_vel, sys->d_image, sys->d_pos_prev, sys->d_box, (float)it->dt, a,
      (float)it->temperature, (uint32_t)it->seed, (uint32_t)(it->seed >> 32), it->d_step, sys->n);
  k_step_inc<<<1, 1, 0, s>>>(it->d_step);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int reduce_kinetic_device(hb_system *sys, cudaStream_t s, const double **d_out) {
  // with n = 0 the partial sums are zero and the result is zero
  k_kinetic_part<<<RED_BLOCKS, 256, 0, s>>>(sys->d_vel, sys->d_red, sys->n);
  k_kinetic_final<<<1, 256, 0, s>>>(sys->d_red, RED_BLOCKS, sys->d_red + 4 * RED_BLOCKS);
  HB_CUDA(cudaGetLastError());
  *d_out = sys->d_red + 4 * RED_BLOCKS;
  return HB_OK;
}

int reduce_kinetic(hb_system *sys, double out[4]) {
  cudaStream_t s = sys->ctx->stream;
  if (sys->n == 0) {
    for (int q = 0; q < 4; ++q) out[q] = 0.0;
    return HB_OK;
  }
  const double *d_ke = nullptr;
  HB_TRY(reduce_kinetic_device(sys, s, &d_ke));
  HB_CUDA(cudaMemcpyAsync(sys->h_red, sys->d_red + 4 * RED_BLOCKS, sizeof(double) * 4,
                          cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  for (int q = 0; q < 4; ++q) out[q] = sys->h_red[q];
  return HB_OK;
}
