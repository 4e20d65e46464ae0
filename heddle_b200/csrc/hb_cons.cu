// hb_cons.cu -- SETTLE and SHAKE/RATTLE constraint kernels.
//
// SETTLE (kernels/settle.cu:145-510, src/integrator/settle.rs:313-404):
// the analytical rigid-water reset of Miyamoto & Kollman (J. Comput. Chem.
// 13, 952-962, 1992) with the pre-drift snapshot as reference frame, the
// H-H width correction used by common SETTLE implementations, the velocity
// correction dx / dt and the position-level constraint virial; the velocity
// projection solves the 3x3 bond-impulse system exactly.  One thread per
// water, every working value in registers.
//
// SHAKE / RATTLE (kernels/shake.cu:108-556, src/integrator/shake.rs:397-495):
// Gauss-Seidel sweeps over the group's pair constraints with the
// constraint gradients frozen at the pre-drift snapshot, absolute tolerance
// on |r|^2 - d^2; the group is solved in FP64 (positions relative to the
// group's first atom), the multiplier solve the reference runs in f32.
// RATTLE iterates the velocity conditions (v_i - v_j) . r_ij = 0 in FP64.
#include <cmath>

#include "hb_internal.cuh"

namespace {

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float csqrt(float x) { return sqrtf(fmaxf(x, 0.0f)); }
__device__ __forceinline__ V3 mi(V3 d, const DBox &b) {
  hb_min_image(d.x, d.y, d.z, b);
  return d;
}
__device__ __forceinline__ V3 unit(V3 a) {
  float l = sqrtf(dot(a, a));
  return l > 0.0f ? (1.0f / l) * a : v3(0.f, 0.f, 0.f);
}

// SETTLE position reset of one water in registers: P = pre-drift snapshot,
// Q = drifted positions (reset in place), V = velocities (corrected by
// dx / dt in place), vir = the position-level virial of each atom
__device__ __forceinline__ void settle_pos_core(const float4 &P0, const float4 &P1,
                                                const float4 &P2, float4 (&Q)[3], float4 (&V)[3],
                                                const float4 &ge, float mo, float mh,
                                                const DBox &bx, float dt, float (&vir)[3]) {
  const float ra = ge.x, rb = ge.y, rc = ge.z;
  const float4 Q0 = Q[0], Q1 = Q[1], Q2 = Q[2];
  // reference frame: snapshot bond vectors relative to the snapshot oxygen
  const V3 b0 = mi(v3(P1.x - P0.x, P1.y - P0.y, P1.z - P0.z), bx);
  const V3 c0 = mi(v3(P2.x - P0.x, P2.y - P0.y, P2.z - P0.z), bx);
  // unconstrained positions relative to the snapshot oxygen
  const V3 ua = mi(v3(Q0.x - P0.x, Q0.y - P0.y, Q0.z - P0.z), bx);
  const V3 ub = b0 + mi(v3(Q1.x - P1.x, Q1.y - P1.y, Q1.z - P1.z), bx);
  const V3 uc = c0 + mi(v3(Q2.x - P2.x, Q2.y - P2.y, Q2.z - P2.z), bx);
  const float inv_m = 1.0f / (mo + 2.0f * mh);
  const V3 com = inv_m * (mo * ua + mh * ub + mh * uc);
  const V3 a1 = ua - com, b1 = ub - com, c1 = uc - com;
  // primed frame: Z' normal of the reference plane, X' from the moved oxygen
  const V3 ez = unit(cross(b0, c0));
  const V3 ex = unit(cross(a1, ez));
  const V3 ey = unit(cross(ez, ex));
  const float b0x = dot(b0, ex), b0y = dot(b0, ey);
  const float c0x = dot(c0, ex), c0y = dot(c0, ey);
  const float a1z = dot(a1, ez);
  const float b1x = dot(b1, ex), b1y = dot(b1, ey), b1z = dot(b1, ez);
  const float c1x = dot(c1, ex), c1y = dot(c1, ey), c1z = dot(c1, ez);
  // tilt of the canonical triangle
  const float sphi = a1z / ra;
  const float cphi = csqrt(1.0f - sphi * sphi);
  const float spsi = (b1z - c1z) / (2.0f * rc * cphi);
  const float cpsi = csqrt(1.0f - spsi * spsi);
  const float a2y = ra * cphi;
  float b2x = -rc * cpsi;
  const float t1 = -rb * cphi, t2 = rc * spsi * sphi;
  const float b2y = t1 - t2, c2y = t1 + t2;
  // width correction so |H1 - H2| equals 2 rc exactly
  const float hh2 = 4.0f * b2x * b2x + (b2y - c2y) * (b2y - c2y) + (b1z - c1z) * (b1z - c1z);
  b2x -= 0.5f * (2.0f * b2x + csqrt(4.0f * b2x * b2x - hh2 + 4.0f * rc * rc));
  // in-plane rotation
  const float al = b2x * (b0x - c0x) + b0y * b2y + c0y * c2y;
  const float be = b2x * (c0y - b0y) + b0x * b2y + c0x * c2y;
  const float ga = b0x * b1y - b1x * b0y + c0x * c1y - c1x * c0y;
  const float ab2 = al * al + be * be;
  const float sth = ab2 > 0.0f ? (al * ga - be * csqrt(ab2 - ga * ga)) / ab2 : 0.0f;
  const float cth = csqrt(1.0f - sth * sth);
  const V3 a3 = v3(-a2y * sth, a2y * cth, a1z);
  const V3 b3 = v3(b2x * cth - b2y * sth, b2x * sth + b2y * cth, b1z);
  const V3 c3 = v3(-b2x * cth - c2y * sth, -b2x * sth + c2y * cth, c1z);
  // back to the lab frame (relative to the centre of mass)
  const V3 ra3 = a3.x * ex + a3.y * ey + a3.z * ez;
  const V3 rb3 = b3.x * ex + b3.y * ey + b3.z * ez;
  const V3 rc3 = c3.x * ex + c3.y * ey + c3.z * ez;
  const V3 corr[3] = {(com + ra3) - ua, (com + rb3) - ub, (com + rc3) - uc};
  const V3 rel[3] = {ra3, rb3, rc3};
  const float ms[3] = {mo, mh, mh};
  const float inv_dt = dt != 0.0f ? 1.0f / dt : 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    Q[a].x += corr[a].x;
    Q[a].y += corr[a].y;
    Q[a].z += corr[a].z;
    V[a].x += corr[a].x * inv_dt;
    V[a].y += corr[a].y * inv_dt;
    V[a].z += corr[a].z * inv_dt;
    vir[a] = ms[a] * inv_dt * inv_dt * dot(corr[a], rel[a]);
  }
}

__global__ void k_settle_pos(const uint4 *__restrict__ atoms, const float4 *__restrict__ geom,
                             const float2 *__restrict__ mass, float4 *__restrict__ posq,
                             float4 *__restrict__ vel, const float4 *__restrict__ prev,
                             const DBox *__restrict__ box, float dt, float *__restrict__ virial,
                             uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const DBox bx = *box;
  const uint4 at = atoms[g];
  const uint32_t id[3] = {at.x, at.y, at.z};
  float4 Q[3] = {posq[at.x], posq[at.y], posq[at.z]};
  float4 V[3] = {vel[at.x], vel[at.y], vel[at.z]};
  float vir[3];
  settle_pos_core(prev[at.x], prev[at.y], prev[at.z], Q, V, geom[g], mass[g].x, mass[g].y, bx,
                  dt, vir);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    posq[id[a]] = Q[a];
    vel[id[a]] = V[a];
    if (virial) virial[id[a]] = vir[a];
  }
}

__device__ __forceinline__ bool solve3(const float m[3][3], const float r[3], float g[3]) {
  const float det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                    m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                    m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if (det == 0.0f) return false;
  const float id = 1.0f / det;
  g[0] = (r[0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
          m[0][1] * (r[1] * m[2][2] - m[1][2] * r[2]) +
          m[0][2] * (r[1] * m[2][1] - m[1][1] * r[2])) * id;
  g[1] = (m[0][0] * (r[1] * m[2][2] - m[1][2] * r[2]) -
          r[0] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
          m[0][2] * (m[1][0] * r[2] - r[1] * m[2][0])) * id;
  g[2] = (m[0][0] * (m[1][1] * r[2] - r[1] * m[2][1]) -
          m[0][1] * (m[1][0] * r[2] - r[1] * m[2][0]) +
          r[0] * (m[1][0] * m[2][1] - m[1][1] * m[2][0])) * id;
  return true;
}

// velocity projection: impulses g_k along r_k (O-H1, O-H2, H1-H2) that
// zero the relative velocity along every bond
// velocity projection of one water in registers (W in place); with dt > 0
// the impulses' virial of each atom goes to vir
__device__ __forceinline__ void settle_vel_core(const float4 &p0, const float4 &p1,
                                                const float4 &p2, float4 &w0, float4 &w1,
                                                float4 &w2, float mo, float mh, const DBox &bx,
                                                float dt, float (&vir)[3]) {
  const float io = 1.0f / mo, ih = 1.0f / mh;
  const V3 x0 = v3(p0.x, p0.y, p0.z);
  const V3 x1 = x0 + mi(v3(p1.x - p0.x, p1.y - p0.y, p1.z - p0.z), bx);
  const V3 x2 = x0 + mi(v3(p2.x - p0.x, p2.y - p0.y, p2.z - p0.z), bx);
  const V3 v0 = v3(w0.x, w0.y, w0.z), v1 = v3(w1.x, w1.y, w1.z), v2 = v3(w2.x, w2.y, w2.z);
  const V3 r1 = x0 - x1, r2 = x0 - x2, r3 = x1 - x2;
  const float d11 = dot(r1, r1), d22 = dot(r2, r2), d33 = dot(r3, r3);
  const float d12 = dot(r1, r2), d13 = dot(r1, r3), d23 = dot(r2, r3);
  const float m[3][3] = {{d11 * (io + ih), d12 * io, -d13 * ih},
                         {d12 * io, d22 * (io + ih), d23 * ih},
                         {-d13 * ih, d23 * ih, 2.0f * d33 * ih}};
  const float rhs[3] = {-dot(v0 - v1, r1), -dot(v0 - v2, r2), -dot(v1 - v2, r3)};
  float gg[3] = {0.f, 0.f, 0.f};
  solve3(m, rhs, gg);
  const V3 dv0 = io * (gg[0] * r1 + gg[1] * r2);
  const V3 dv1 = ih * ((-gg[0]) * r1 + gg[2] * r3);
  const V3 dv2 = ih * ((-gg[1]) * r2 - gg[2] * r3);
  w0.x += dv0.x; w0.y += dv0.y; w0.z += dv0.z;
  w1.x += dv1.x; w1.y += dv1.y; w1.z += dv1.z;
  w2.x += dv2.x; w2.y += dv2.y; w2.z += dv2.z;
  if (dt > 0.0f) {
    const float inv_dt = 1.0f / dt;
    const V3 com = (1.0f / (mo + 2.0f * mh)) * (mo * x0 + mh * x1 + mh * x2);
    vir[0] = mo * inv_dt * dot(dv0, x0 - com);
    vir[1] = mh * inv_dt * dot(dv1, x1 - com);
    vir[2] = mh * inv_dt * dot(dv2, x2 - com);
  }
}

__global__ void k_settle_vel(const uint4 *__restrict__ atoms, const float2 *__restrict__ mass,
                             const float4 *__restrict__ posq, float4 *__restrict__ vel,
                             const DBox *__restrict__ box, float dt, float *__restrict__ virial,
                             uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const DBox bx = *box;
  const uint4 at = atoms[g];
  float4 w0 = vel[at.x], w1 = vel[at.y], w2 = vel[at.z];
  float vir[3] = {0.f, 0.f, 0.f};
  settle_vel_core(posq[at.x], posq[at.y], posq[at.z], w0, w1, w2, mass[g].x, mass[g].y, bx,
                  virial ? dt : 0.0f, vir);
  vel[at.x] = w0;
  vel[at.y] = w1;
  vel[at.z] = w2;
  if (virial && dt > 0.0f) {
    virial[at.x] += vir[0];
    virial[at.y] += vir[1];
    virial[at.z] += vir[2];
  }
}

// The whole Langevin head of a step for a system whose every atom is in a
// SETTLE water, one thread per water with every value in registers: the
// kick of its three atoms, the velocity projection, drift / O / drift with
// the wrap, and the position reset with its virial -- the same arithmetic
// per atom as k_lang_kick, k_settle_vel (dt = 0), k_lang_drift_ou and
// k_settle_pos in turn.  The block that finishes last (a completion
// counter, no waiting) advances the Langevin draw counter, which every
// thread read first.
__global__ void __launch_bounds__(128) k_lang_settle_head(
    const uint4 *__restrict__ atoms, const float4 *__restrict__ geom,
    const float2 *__restrict__ mass, float4 *__restrict__ posq, float4 *__restrict__ vel,
    int4 *__restrict__ image, float4 *__restrict__ prev, const float4 *__restrict__ force,
    const DBox *__restrict__ box, float dt, float a, float kt, uint32_t s_lo, uint32_t s_hi,
    uint64_t *__restrict__ step_ptr, uint32_t *__restrict__ done, float *__restrict__ virial,
    uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t step = *step_ptr;
  if (g < ng) {
    const DBox bx = *box;
    const uint4 at = atoms[g];
    const uint32_t id[3] = {at.x, at.y, at.z};
    const float mo = mass[g].x, mh = mass[g].y;
    float4 Q[3], V[3], P[3];
    int4 M[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      V[k] = vel[id[k]];
      hb_lang_kick(V[k], force[id[k]], dt);
      P[k] = posq[id[k]];
    }
    float vir[3] = {0.f, 0.f, 0.f};
    settle_vel_core(P[0], P[1], P[2], V[0], V[1], V[2], mo, mh, bx, 0.0f, vir);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      Q[k] = P[k];
      M[k] = image[id[k]];
      hb_lang_drift_ou(Q[k], V[k], M[k], dt, a, kt, s_lo, s_hi, step, id[k], bx);
      prev[id[k]] = P[k];
      image[id[k]] = M[k];
    }
    settle_pos_core(P[0], P[1], P[2], Q, V, geom[g], mo, mh, bx, dt, vir);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      posq[id[k]] = Q[k];
      vel[id[k]] = V[k];
      if (virial) virial[id[k]] = vir[k];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(done, 1u) == gridDim.x - 1u) {
      *step_ptr = step + 1ull;
      *done = 0u;
    }
  }
}

#define SHAKE_MAX_ATOMS 8
#define SHAKE_MAX_CONS 12

// Per-constraint inputs of the learned warm start (8 features), the first
// Gauss-Seidel multiplier lam1 = sigma / (2 mu s.g) and the scale that
// turns a multiplier difference into sigma units: ls = 2 mu s.g / d^2 * 1e3.
// The network predicts (lam - lam1) * ls from the features; lam0 = lam1 +
// prediction / ls warm-starts the sweeps.  Features: 1e3 sigma/d^2,
// 1e3 (s.g/d^2 - 1), 1e3 (|g|^2/d^2 - 1), the first-order change of sigma
// from the coupled constraints' first updates (1e3, in units of d^2), the
// summed coupling strength, coupled count / 3, im_i / mu, 1e6 (sigma/d^2)^2.
#define SHAKE_NF 8

__device__ void shake_features(uint32_t nc, const uint32_t *ci, const uint32_t *cj,
                               const double (*xc)[3], const double (*gdir)[3], const double *tgt,
                               const double *im, float *feat, double *lam1, double *lsc) {
  double sg[SHAKE_MAX_CONS], sig[SHAKE_MAX_CONS], mu[SHAKE_MAX_CONS];
  for (uint32_t k = 0; k < nc; ++k) {
    const uint32_t i = ci[k], j = cj[k];
    double sx = xc[i][0] - xc[j][0], sy = xc[i][1] - xc[j][1], sz = xc[i][2] - xc[j][2];
    sg[k] = sx * gdir[k][0] + sy * gdir[k][1] + sz * gdir[k][2];
    sig[k] = sx * sx + sy * sy + sz * sz - tgt[k];
    mu[k] = im[i] + im[j];
  }
  for (uint32_t k = 0; k < nc; ++k) {
    const uint32_t i = ci[k], j = cj[k];
    const double d2 = tgt[k];
    const double sx = xc[i][0] - xc[j][0], sy = xc[i][1] - xc[j][1], sz = xc[i][2] - xc[j][2];
    const double g2 = gdir[k][0] * gdir[k][0] + gdir[k][1] * gdir[k][1] + gdir[k][2] * gdir[k][2];
    double cpl = 0.0, strength = 0.0;
    int cnt = 0;
    for (uint32_t l = 0; l < nc; ++l) {
      if (l == k) continue;
      const uint32_t il = ci[l], jl = cj[l];
      uint32_t a;
      double ek, el;
      if (il == i || il == j) {
        a = il;
        el = 1.0;
      } else if (jl == i || jl == j) {
        a = jl;
        el = -1.0;
      } else {
        continue;
      }
      ek = (a == i) ? 1.0 : -1.0;
      const double skgl = sx * gdir[l][0] + sy * gdir[l][1] + sz * gdir[l][2];
      const double w = (sg[l] != 0.0 && mu[l] != 0.0) ? -el * ek * (im[a] / mu[l]) * skgl / sg[l] : 0.0;
      cpl += w * sig[l];
      strength += fabs(w);
      ++cnt;
    }
    const double l1 = (sg[k] != 0.0 && mu[k] != 0.0) ? sig[k] / (2.0 * mu[k] * sg[k]) : 0.0;
    lam1[k] = l1;
    lsc[k] = 2.0 * mu[k] * sg[k] / d2 * 1e3;
    float *f = feat + (size_t)k * SHAKE_NF;
    f[0] = (float)(1e3 * sig[k] / d2);
    f[1] = (float)(1e3 * (sg[k] / d2 - 1.0));
    f[2] = (float)(1e3 * (g2 / d2 - 1.0));
    f[3] = (float)(1e3 * cpl / d2);
    f[4] = (float)strength;
    f[5] = (float)cnt / 3.0f;
    f[6] = (float)(mu[k] > 0.0 ? im[i] / mu[k] : 0.0);
    f[7] = (float)(1e6 * (sig[k] / d2) * (sig[k] / d2));
  }
}

// Gauss-Seidel SHAKE on one group per thread (FP64).  rel: tolerance
// relative to d^2 instead of absolute.  Optional: lam0 / lam1 / lsc warm
// start from a predicted multiplier correction (pred), features out
// (feat, lam1_out, lsc_out, computed before any update), converged total
// multipliers out (lam_out), sweep statistics (stats[0] group-sweeps,
// stats[1] groups), features_only (compute features, move nothing).
__global__ void k_shake_pos(const uint32_t *__restrict__ aoff, const uint32_t *__restrict__ atoms,
                            const uint32_t *__restrict__ coff, const uint2 *__restrict__ pairs,
                            const double *__restrict__ d2, float4 *__restrict__ posq,
                            float4 *__restrict__ vel, const float4 *__restrict__ prev,
                            const DBox *__restrict__ box, float dt, double tol, int rel,
                            int max_iter, float *__restrict__ virial, uint32_t *__restrict__ iters,
                            unsigned long long *__restrict__ stats, const float *__restrict__ pred,
                            float *__restrict__ feat, double *__restrict__ lam1_io,
                            double *__restrict__ lsc_io, double *__restrict__ lam_out,
                            int features_only, uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t it_used = 0;
  if (g < ng) {
    const DBox bx = *box;
    const uint32_t a0 = aoff[g], na = aoff[g + 1] - a0;
    const uint32_t c0 = coff[g], nc = coff[g + 1] - c0;
    double xr[SHAKE_MAX_ATOMS][3], xu[SHAKE_MAX_ATOMS][3], xc[SHAKE_MAX_ATOMS][3];
    double im[SHAKE_MAX_ATOMS], ms[SHAKE_MAX_ATOMS];
    const float4 r0 = prev[atoms[a0]], u0 = posq[atoms[a0]];
    for (uint32_t a = 0; a < na; ++a) {
      const uint32_t id = atoms[a0 + a];
      const float4 r = prev[id], u = posq[id];
      const float w = vel[id].w;
      im[a] = (double)w;
      ms[a] = w > 0.0f ? 1.0 / (double)w : 0.0;
      V3 dr = mi(v3(r.x - r0.x, r.y - r0.y, r.z - r0.z), bx);
      V3 du = mi(v3(u.x - u0.x, u.y - u0.y, u.z - u0.z), bx);
      xr[a][0] = dr.x; xr[a][1] = dr.y; xr[a][2] = dr.z;
      xu[a][0] = du.x; xu[a][1] = du.y; xu[a][2] = du.z;
      for (int d = 0; d < 3; ++d) xc[a][d] = xu[a][d];
    }
    double gdir[SHAKE_MAX_CONS][3];
    uint32_t ci[SHAKE_MAX_CONS], cj[SHAKE_MAX_CONS];
    double tgt[SHAKE_MAX_CONS], lam_tot[SHAKE_MAX_CONS];
    for (uint32_t k = 0; k < nc; ++k) {
      const uint2 pr = pairs[c0 + k];
      ci[k] = pr.x;
      cj[k] = pr.y;
      tgt[k] = d2[c0 + k];
      lam_tot[k] = 0.0;
      for (int d = 0; d < 3; ++d) gdir[k][d] = xr[pr.x][d] - xr[pr.y][d];
    }
    if (feat) {
      shake_features(nc, ci, cj, xc, gdir, tgt, im, feat + (size_t)c0 * SHAKE_NF, lam1_io + c0,
                     lsc_io + c0);
    }
    if (!features_only) {
      if (pred) {
        // warm start: every constraint's predicted multiplier applied at once
        for (uint32_t k = 0; k < nc; ++k) {
          const double ls = lsc_io[c0 + k];
          const double l0 = lam1_io[c0 + k] + (ls != 0.0 ? (double)pred[c0 + k] / ls : 0.0);
          if (!(fabs(l0) < 1e30)) continue;
          const uint32_t i = ci[k], j = cj[k];
          for (int d = 0; d < 3; ++d) {
            xc[i][d] -= l0 * im[i] * gdir[k][d];
            xc[j][d] += l0 * im[j] * gdir[k][d];
          }
          lam_tot[k] += l0;
        }
      }
      int it = 0;
      for (; it < max_iter; ++it) {
        bool conv = true;
        for (uint32_t k = 0; k < nc; ++k) {
          const uint32_t i = ci[k], j = cj[k];
          const double dx = xc[i][0] - xc[j][0], dy = xc[i][1] - xc[j][1], dz = xc[i][2] - xc[j][2];
          const double sigma = dx * dx + dy * dy + dz * dz - tgt[k];
          const double tk = rel ? tol * tgt[k] : tol;
          if (fabs(sigma) > tk) {
            conv = false;
            const double den = 2.0 * (dx * gdir[k][0] + dy * gdir[k][1] + dz * gdir[k][2]) * (im[i] + im[j]);
            if (den == 0.0) continue;
            const double lam = sigma / den;
            lam_tot[k] += lam;
            for (int d = 0; d < 3; ++d) {
              xc[i][d] -= lam * im[i] * gdir[k][d];
              xc[j][d] += lam * im[j] * gdir[k][d];
            }
          }
        }
        if (conv) break;
      }
      it_used = (uint32_t)it;
      if (iters) atomicMax(iters, (uint32_t)it);
      if (lam_out)
        for (uint32_t k = 0; k < nc; ++k) lam_out[c0 + k] = lam_tot[k];
      double tm = 0.0, com[3] = {0, 0, 0};
      for (uint32_t a = 0; a < na; ++a) {
        tm += ms[a];
        for (int d = 0; d < 3; ++d) com[d] += ms[a] * xc[a][d];
      }
      for (int d = 0; d < 3; ++d) com[d] = tm > 0.0 ? com[d] / tm : 0.0;
      const double inv_dt = dt != 0.0f ? 1.0 / (double)dt : 0.0;
      for (uint32_t a = 0; a < na; ++a) {
        const uint32_t id = atoms[a0 + a];
        float4 q = posq[id];
        float4 v = vel[id];
        double wv = 0.0;
        double del[3];
        for (int d = 0; d < 3; ++d) {
          del[d] = xc[a][d] - xu[a][d];
          wv += del[d] * (xc[a][d] - com[d]);
        }
        q.x += (float)del[0];
        q.y += (float)del[1];
        q.z += (float)del[2];
        v.x += (float)(del[0] * inv_dt);
        v.y += (float)(del[1] * inv_dt);
        v.z += (float)(del[2] * inv_dt);
        posq[id] = q;
        vel[id] = v;
        if (virial) virial[id] = (float)(ms[a] * inv_dt * inv_dt * wv);
      }
    }
  }
  if (stats && !features_only) {
    // group-sweeps and groups of this call, one atomic per warp
    unsigned long long s0 = it_used, s1 = g < ng ? 1ull : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, o);
      s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, o);
    }
    if ((threadIdx.x & 31u) == 0u && s1) {
      atomicAdd(&stats[0], s0);
      atomicAdd(&stats[1], s1);
    }
  }
}

// Position-only projection (the minimizer's apply_position_projection_only,
// settle_positions_no_velocity kernels/settle.cu:519-584 and
// shake_positions_no_velocity kernels/shake.cu:558-697): Gauss-Seidel
// sweeps with gradient directions taken at the current off-manifold
// positions, FP64, |r^2 - d^2| below tol (absolute, or relative to d^2),
// at most max_iter sweeps; no velocity change, no virial.  skip (optional):
// a device flag that turns the launch into a no-op.
__device__ void project_group(uint32_t nc, const uint32_t *ci, const uint32_t *cj,
                              const double *tgt, const double *im, double (*xc)[3], double tol,
                              int rel, int max_iter) {
  double g[SHAKE_MAX_CONS][3];
  for (uint32_t k = 0; k < nc; ++k)
    for (int d = 0; d < 3; ++d) g[k][d] = xc[ci[k]][d] - xc[cj[k]][d];
  for (int it = 0; it < max_iter; ++it) {
    bool conv = true;
    for (uint32_t k = 0; k < nc; ++k) {
      const uint32_t i = ci[k], j = cj[k];
      const double dx = xc[i][0] - xc[j][0], dy = xc[i][1] - xc[j][1], dz = xc[i][2] - xc[j][2];
      const double sigma = dx * dx + dy * dy + dz * dz - tgt[k];
      if (fabs(sigma) > (rel ? tol * tgt[k] : tol)) {
        conv = false;
        const double den = 2.0 * (dx * g[k][0] + dy * g[k][1] + dz * g[k][2]) * (im[i] + im[j]);
        if (den == 0.0) continue;
        const double lam = sigma / den;
        for (int d = 0; d < 3; ++d) {
          xc[i][d] -= lam * im[i] * g[k][d];
          xc[j][d] += lam * im[j] * g[k][d];
        }
      }
    }
    if (conv) break;
  }
}

__global__ void k_settle_project(const uint4 *__restrict__ at, const float4 *__restrict__ geom,
                                 const float2 *__restrict__ mass, float4 *__restrict__ posq,
                                 const DBox *__restrict__ box, double tol, int max_iter,
                                 const int *__restrict__ skip, uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng || (skip && *skip)) return;
  const DBox bx = *box;
  const uint4 a = at[g];
  const uint32_t id[3] = {a.x, a.y, a.z};
  const float4 gm = geom[g];
  const float2 m = mass[g];
  const double ra = gm.x, rb = gm.y, rc = gm.z;
  const double tgt[3] = {(ra + rb) * (ra + rb) + rc * rc, (ra + rb) * (ra + rb) + rc * rc,
                         4.0 * rc * rc};
  const double im[3] = {m.x > 0.f ? 1.0 / m.x : 0.0, m.y > 0.f ? 1.0 / m.y : 0.0,
                        m.y > 0.f ? 1.0 / m.y : 0.0};
  const uint32_t ci[3] = {0, 0, 1}, cj[3] = {1, 2, 2};
  const float4 p0 = posq[id[0]];
  double xc[SHAKE_MAX_ATOMS][3], xu[3][3];
  for (int q = 0; q < 3; ++q) {
    const float4 p = posq[id[q]];
    const V3 d = mi(v3(p.x - p0.x, p.y - p0.y, p.z - p0.z), bx);
    xu[q][0] = xc[q][0] = d.x;
    xu[q][1] = xc[q][1] = d.y;
    xu[q][2] = xc[q][2] = d.z;
  }
  project_group(3, ci, cj, tgt, im, xc, tol, 0, max_iter);
  for (int q = 0; q < 3; ++q) {
    float4 p = posq[id[q]];
    p.x += (float)(xc[q][0] - xu[q][0]);
    p.y += (float)(xc[q][1] - xu[q][1]);
    p.z += (float)(xc[q][2] - xu[q][2]);
    posq[id[q]] = p;
  }
}

__global__ void k_shake_project(const uint32_t *__restrict__ aoff, const uint32_t *__restrict__ atoms,
                                const uint32_t *__restrict__ coff, const uint2 *__restrict__ pairs,
                                const double *__restrict__ d2, float4 *__restrict__ posq,
                                const float4 *__restrict__ vel, const DBox *__restrict__ box,
                                double tol, int rel, int max_iter, const int *__restrict__ skip,
                                uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng || (skip && *skip)) return;
  const DBox bx = *box;
  const uint32_t a0 = aoff[g], na = aoff[g + 1] - a0;
  const uint32_t c0 = coff[g], nc = coff[g + 1] - c0;
  double xc[SHAKE_MAX_ATOMS][3], xu[SHAKE_MAX_ATOMS][3], im[SHAKE_MAX_ATOMS];
  const float4 p0 = posq[atoms[a0]];
  for (uint32_t a = 0; a < na; ++a) {
    const uint32_t id = atoms[a0 + a];
    const float4 p = posq[id];
    im[a] = (double)vel[id].w;
    const V3 d = mi(v3(p.x - p0.x, p.y - p0.y, p.z - p0.z), bx);
    xu[a][0] = xc[a][0] = d.x;
    xu[a][1] = xc[a][1] = d.y;
    xu[a][2] = xc[a][2] = d.z;
  }
  uint32_t ci[SHAKE_MAX_CONS], cj[SHAKE_MAX_CONS];
  double tgt[SHAKE_MAX_CONS];
  for (uint32_t k = 0; k < nc; ++k) {
    const uint2 pr = pairs[c0 + k];
    ci[k] = pr.x;
    cj[k] = pr.y;
    tgt[k] = d2[c0 + k];
  }
  project_group(nc, ci, cj, tgt, im, xc, tol, rel, max_iter);
  for (uint32_t a = 0; a < na; ++a) {
    const uint32_t id = atoms[a0 + a];
    float4 p = posq[id];
    p.x += (float)(xc[a][0] - xu[a][0]);
    p.y += (float)(xc[a][1] - xu[a][1]);
    p.z += (float)(xc[a][2] - xu[a][2]);
    posq[id] = p;
  }
}

__global__ void k_rattle_vel(const uint32_t *__restrict__ aoff, const uint32_t *__restrict__ atoms,
                             const uint32_t *__restrict__ coff, const uint2 *__restrict__ pairs,
                             const float4 *__restrict__ posq, float4 *__restrict__ vel,
                             const DBox *__restrict__ box, float dt, float *__restrict__ virial,
                             uint32_t ng) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const DBox bx = *box;
  const uint32_t a0 = aoff[g], na = aoff[g + 1] - a0;
  const uint32_t c0 = coff[g], nc = coff[g + 1] - c0;
  double x[SHAKE_MAX_ATOMS][3], v[SHAKE_MAX_ATOMS][3], dv[SHAKE_MAX_ATOMS][3];
  double im[SHAKE_MAX_ATOMS], ms[SHAKE_MAX_ATOMS];
  const float4 p0 = posq[atoms[a0]];
  for (uint32_t a = 0; a < na; ++a) {
    const uint32_t id = atoms[a0 + a];
    const float4 p = posq[id], w = vel[id];
    V3 d = mi(v3(p.x - p0.x, p.y - p0.y, p.z - p0.z), bx);
    x[a][0] = d.x; x[a][1] = d.y; x[a][2] = d.z;
    v[a][0] = w.x; v[a][1] = w.y; v[a][2] = w.z;
    dv[a][0] = dv[a][1] = dv[a][2] = 0.0;
    im[a] = (double)w.w;
    ms[a] = w.w > 0.0f ? 1.0 / (double)w.w : 0.0;
  }
  for (int it = 0; it < 256; ++it) {
    double worst = 0.0;
    for (uint32_t k = 0; k < nc; ++k) {
      const uint2 pr = pairs[c0 + k];
      const uint32_t i = pr.x, j = pr.y;
      double r[3], rv = 0.0, rr = 0.0;
      for (int d = 0; d < 3; ++d) {
        r[d] = x[i][d] - x[j][d];
        rv += (v[i][d] - v[j][d]) * r[d];
        rr += r[d] * r[d];
      }
      const double den = rr * (im[i] + im[j]);
      if (den == 0.0) continue;
      const double gk = -rv / den;
      worst = fmax(worst, fabs(rv) / sqrt(rr));
      for (int d = 0; d < 3; ++d) {
        v[i][d] += gk * im[i] * r[d];
        v[j][d] -= gk * im[j] * r[d];
        dv[i][d] += gk * im[i] * r[d];
        dv[j][d] -= gk * im[j] * r[d];
      }
    }
    if (worst < 1.0e-14) break;
  }
  double tm = 0.0, com[3] = {0, 0, 0};
  for (uint32_t a = 0; a < na; ++a) {
    tm += ms[a];
    for (int d = 0; d < 3; ++d) com[d] += ms[a] * x[a][d];
  }
  for (int d = 0; d < 3; ++d) com[d] = tm > 0.0 ? com[d] / tm : 0.0;
  for (uint32_t a = 0; a < na; ++a) {
    const uint32_t id = atoms[a0 + a];
    float4 w = vel[id];
    w.x = (float)v[a][0];
    w.y = (float)v[a][1];
    w.z = (float)v[a][2];
    vel[id] = w;
    if (virial && dt > 0.0f) {
      double wv = 0.0;
      for (int d = 0; d < 3; ++d) wv += dv[a][d] * (x[a][d] - com[d]);
      virial[id] += (float)(ms[a] / (double)dt * wv);
    }
  }
}

}  // namespace

int cons_positions(hb_constraints *c, double dt, cudaStream_t s) {
  hb_system *sys = c->sys;
  if (c->n_settle)
    k_settle_pos<<<hb_div_up(c->n_settle, 128), 128, 0, s>>>(
        c->d_settle_atoms, c->d_settle_geom, c->d_settle_mass, sys->d_posq, sys->d_vel,
        sys->d_pos_prev, sys->d_box, (float)dt, c->d_virial, c->n_settle);
  if (c->n_shake) {
    const unsigned gs = hb_div_up(c->n_shake, 64);
    const float *pred = nullptr;
    if (c->mlp) {
      // learned warm start: features, network, then the sweeps
      k_shake_pos<<<gs, 64, 0, s>>>(
          c->d_shake_aoff, c->d_shake_atoms, c->d_shake_coff, c->d_shake_pairs, c->d_shake_d2,
          sys->d_posq, sys->d_vel, sys->d_pos_prev, sys->d_box, (float)dt, c->shake_tol,
          c->shake_rel, (int)c->shake_max_iter, nullptr, nullptr, nullptr, nullptr, c->d_feat,
          c->d_lam1, c->d_lsc, nullptr, 1, c->n_shake);
      HB_TRY(mlp_infer(c->mlp, c->d_feat, c->n_shake_cons, c->d_pred, s));
      pred = c->d_pred;
    }
    const bool rec = c->record;
    k_shake_pos<<<gs, 64, 0, s>>>(
        c->d_shake_aoff, c->d_shake_atoms, c->d_shake_coff, c->d_shake_pairs, c->d_shake_d2,
        sys->d_posq, sys->d_vel, sys->d_pos_prev, sys->d_box, (float)dt, c->shake_tol,
        c->shake_rel, (int)c->shake_max_iter, c->d_virial, c->d_iters, c->d_stats, pred,
        (rec && !pred) ? c->d_feat : nullptr, c->d_lam1, c->d_lsc, rec ? c->d_lam : nullptr, 0,
        c->n_shake);
  }
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

bool cons_lang_head_fusable(const hb_constraints *c) {
  return c && c->fuse_head && c->n_shake == 0 && c->n_settle > 0 &&
         3ull * c->n_settle == c->sys->n;
}

int cons_lang_settle_head(hb_constraints *c, float dt, float a, float kt, uint32_t s_lo,
                          uint32_t s_hi, uint64_t *d_step, uint32_t *d_done, cudaStream_t s) {
  hb_system *sys = c->sys;
  k_lang_settle_head<<<hb_div_up(c->n_settle, 128), 128, 0, s>>>(
      c->d_settle_atoms, c->d_settle_geom, c->d_settle_mass, sys->d_posq, sys->d_vel,
      sys->d_image, sys->d_pos_prev, sys->d_force, sys->d_box, dt, a, kt, s_lo, s_hi, d_step,
      d_done, c->d_virial, c->n_settle);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int cons_project(hb_constraints *c, const int *skip, cudaStream_t s) {
  hb_system *sys = c->sys;
  // the reference's projection tolerance for SETTLE groups (SETTLE_TOL2,
  // kernels/settle.cu:105); SHAKE groups keep their configured tolerance
  if (c->n_settle)
    k_settle_project<<<hb_div_up(c->n_settle, 128), 128, 0, s>>>(
        c->d_settle_atoms, c->d_settle_geom, c->d_settle_mass, sys->d_posq, sys->d_box, 3.57e-6,
        32, skip, c->n_settle);
  if (c->n_shake)
    k_shake_project<<<hb_div_up(c->n_shake, 64), 64, 0, s>>>(
        c->d_shake_aoff, c->d_shake_atoms, c->d_shake_coff, c->d_shake_pairs, c->d_shake_d2,
        sys->d_posq, sys->d_vel, sys->d_box, c->shake_tol, c->shake_rel, (int)c->shake_max_iter,
        skip, c->n_shake);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int cons_velocities(hb_constraints *c, double dt, bool virial, cudaStream_t s) {
  hb_system *sys = c->sys;
  float *vir = virial ? c->d_virial : nullptr;
  if (c->n_settle)
    k_settle_vel<<<hb_div_up(c->n_settle, 128), 128, 0, s>>>(
        c->d_settle_atoms, c->d_settle_mass, sys->d_posq, sys->d_vel, sys->d_box, (float)dt, vir,
        c->n_settle);
  if (c->n_shake)
    k_rattle_vel<<<hb_div_up(c->n_shake, 64), 64, 0, s>>>(
        c->d_shake_aoff, c->d_shake_atoms, c->d_shake_coff, c->d_shake_pairs, sys->d_posq,
        sys->d_vel, sys->d_box, (float)dt, vir, c->n_shake);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}
