// hb_bonded.cu -- harmonic bonds, harmonic angles and periodic dihedrals.
//
// Physics of the reference's bonded slots: HarmonicPairFunctor
// (src/forces/harmonic_bond.rs:283-307), HarmonicAngleFunctor
// (src/forces/angle.rs:260-313) and PeriodicDihedralFunctor
// (src/forces/dihedral.rs:383-467), single precision with minimum-image
// displacements.  The reference writes per-term force slots and reduces
// them per atom through a CSR in a second kernel (kernels/morse.cu:14-61
// and its angle/dihedral analogues) to stay deterministic; here one thread
// per term adds its forces straight into the int64 fixed-point accumulators
// the pair kernel uses (integer addition is order-independent, so the sums
// are the same run to run), and the combine kernel that already converts
// those accumulators picks them up.  One launch covers all three kinds.
// Per-atom energy and virial shares split each term equally over its atoms.
#include <cmath>
#include <vector>

#include "hb_internal.cuh"

namespace {

__device__ __forceinline__ long long fixq(float v) { return __float2ll_rn(v * HB_FP_SCALE); }

__device__ __forceinline__ void add_force(unsigned long long *fp, size_t np, uint32_t slot,
                                          float fx, float fy, float fz) {
  atomicAdd(&fp[slot], (unsigned long long)fixq(fx));
  atomicAdd(&fp[np + slot], (unsigned long long)fixq(fy));
  atomicAdd(&fp[2 * np + slot], (unsigned long long)fixq(fz));
}

__device__ __forceinline__ void add_ev(unsigned long long *fp, size_t np, uint32_t slot, float e,
                                       float w) {
  atomicAdd(&fp[3 * np + slot], (unsigned long long)fixq(e));
  atomicAdd(&fp[4 * np + slot], (unsigned long long)fixq(w));
}

__device__ __forceinline__ float3 disp(const float4 *posq, uint32_t a, uint32_t b, const DBox &bx) {
  const float4 pa = posq[a], pb = posq[b];
  float dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
  hb_min_image(dx, dy, dz, bx);
  return make_float3(dx, dy, dz);
}

__device__ __forceinline__ float dot3(const float3 &a, const float3 &b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}

template <bool EV>
__global__ void k_bonded(const float4 *__restrict__ posq, const uint32_t *__restrict__ slot_of,
                         const DBox *__restrict__ box, const uint2 *__restrict__ bond_atoms,
                         const float2 *__restrict__ bond_par, uint32_t nb,
                         const uint4 *__restrict__ angle_atoms,
                         const float2 *__restrict__ angle_par, uint32_t na,
                         const uint4 *__restrict__ dih_atoms, const float4 *__restrict__ dih_par,
                         uint32_t nd, unsigned long long *__restrict__ fp, size_t np,
                         unsigned long long *__restrict__ acc) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const DBox bx = *box;
  float u = 0.0f, w = 0.0f;
  if (t < nb) {
    // U = k/2 (r - r0)^2, F_i = -k (r - r0) / r d, d = r_i - r_j
    const uint2 at = bond_atoms[t];
    const float2 kp = bond_par[t];
    const float3 d = disp(posq, at.x, at.y, bx);
    const float r2 = dot3(d, d);
    const float r = sqrtf(r2);
    if (r >= 1.0e-7f) {
      const float dr = r - kp.y;
      const float fmag = -kp.x * dr / r;
      const uint32_t si = slot_of[at.x], sj = slot_of[at.y];
      add_force(fp, np, si, fmag * d.x, fmag * d.y, fmag * d.z);
      add_force(fp, np, sj, -fmag * d.x, -fmag * d.y, -fmag * d.z);
      if (EV) {
        u = 0.5f * kp.x * dr * dr;
        w = fmag * r2;
        add_ev(fp, np, si, 0.5f * u, 0.5f * w);
        add_ev(fp, np, sj, 0.5f * u, 0.5f * w);
      }
    }
  } else if (t < nb + na) {
    // U = k/2 (theta - theta0)^2, theta at the vertex j
    const uint32_t q = t - nb;
    const uint4 at = angle_atoms[q];
    const float2 kp = angle_par[q];
    const float3 a = disp(posq, at.x, at.y, bx);  // r_i - r_j
    const float3 c = disp(posq, at.z, at.y, bx);  // r_k - r_j
    const float a2 = dot3(a, a), c2 = dot3(c, c);
    if (a2 > 0.0f && c2 > 0.0f) {
      const float la = sqrtf(a2), lc = sqrtf(c2);
      const float inv_ac = 1.0f / (la * lc);
      const float dt = dot3(a, c);
      const float cs = fminf(1.0f, fmaxf(-1.0f, dt * inv_ac));
      const float sn = sqrtf(fmaxf(1.0f - cs * cs, 0.0f));
      if (sn >= 1.0e-7f) {
        const float th = atan2f(la * lc * sn, dt);
        const float dth = th - kp.y;
        const float g = -kp.x * dth / sn;
        const float ia2 = 1.0f / a2, ic2 = 1.0f / c2;
        const float3 fi = make_float3(g * (cs * ia2 * a.x - inv_ac * c.x),
                                      g * (cs * ia2 * a.y - inv_ac * c.y),
                                      g * (cs * ia2 * a.z - inv_ac * c.z));
        const float3 fk = make_float3(g * (cs * ic2 * c.x - inv_ac * a.x),
                                      g * (cs * ic2 * c.y - inv_ac * a.y),
                                      g * (cs * ic2 * c.z - inv_ac * a.z));
        const uint32_t si = slot_of[at.x], sj = slot_of[at.y], sk = slot_of[at.z];
        add_force(fp, np, si, fi.x, fi.y, fi.z);
        add_force(fp, np, sk, fk.x, fk.y, fk.z);
        add_force(fp, np, sj, -fi.x - fk.x, -fi.y - fk.y, -fi.z - fk.z);
        if (EV) {
          u = 0.5f * kp.x * dth * dth;
          w = dot3(a, fi) + dot3(c, fk);
          const float third = 1.0f / 3.0f;
          add_ev(fp, np, si, third * u, third * w);
          add_ev(fp, np, sj, third * u, third * w);
          add_ev(fp, np, sk, third * u, third * w);
        }
      }
    }
  } else if (t < nb + na + nd) {
    // U = k (1 + cos(n phi - phi0)); b1 = r_i - r_j, b2 = r_k - r_j,
    // b3 = r_k - r_l, m = b1 x b2, n = b2 x b3
    const uint32_t q = t - nb - na;
    const uint4 at = dih_atoms[q];
    const float4 kp = dih_par[q];
    const float3 b1 = disp(posq, at.x, at.y, bx);
    const float3 b2 = disp(posq, at.z, at.y, bx);
    const float3 b3 = disp(posq, at.z, at.w, bx);
    const float3 m = make_float3(b1.y * b2.z - b1.z * b2.y, b1.z * b2.x - b1.x * b2.z,
                                 b1.x * b2.y - b1.y * b2.x);
    const float3 n = make_float3(b2.y * b3.z - b2.z * b3.y, b2.z * b3.x - b2.x * b3.z,
                                 b2.x * b3.y - b2.y * b3.x);
    const float m2 = dot3(m, m), n2 = dot3(n, n), b22 = dot3(b2, b2);
    if (m2 >= 1.0e-14f && n2 >= 1.0e-14f && b22 >= 1.0e-14f) {
      const float lb2 = sqrtf(b22);
      const float phi = atan2f(lb2 * dot3(b1, n), dot3(m, n));
      const float del = kp.z * phi - kp.y;
      float sd, cd;
      sincosf(del, &sd, &cd);
      const float fphi = kp.x * kp.z * sd;
      const float ci = fphi * lb2 / m2, cl = -fphi * lb2 / n2;
      const float3 fi = make_float3(ci * m.x, ci * m.y, ci * m.z);
      const float3 fl = make_float3(cl * n.x, cl * n.y, cl * n.z);
      const float ib = 1.0f / b22;
      const float s = dot3(b1, b2) * ib, tt = dot3(b3, b2) * ib;
      const float3 fj = make_float3((s - 1.0f) * fi.x - tt * fl.x, (s - 1.0f) * fi.y - tt * fl.y,
                                    (s - 1.0f) * fi.z - tt * fl.z);
      const float3 fk = make_float3(-s * fi.x + (tt - 1.0f) * fl.x, -s * fi.y + (tt - 1.0f) * fl.y,
                                    -s * fi.z + (tt - 1.0f) * fl.z);
      const uint32_t si = slot_of[at.x], sj = slot_of[at.y], sk = slot_of[at.z],
                     sl = slot_of[at.w];
      add_force(fp, np, si, fi.x, fi.y, fi.z);
      add_force(fp, np, sj, fj.x, fj.y, fj.z);
      add_force(fp, np, sk, fk.x, fk.y, fk.z);
      add_force(fp, np, sl, fl.x, fl.y, fl.z);
      if (EV) {
        u = kp.x * (1.0f + cd);
        const float3 bl = make_float3(b2.x - b3.x, b2.y - b3.y, b2.z - b3.z);
        w = dot3(b1, fi) + dot3(b2, fk) + dot3(bl, fl);
        const float q4 = 0.25f;
        add_ev(fp, np, si, q4 * u, q4 * w);
        add_ev(fp, np, sj, q4 * u, q4 * w);
        add_ev(fp, np, sk, q4 * u, q4 * w);
        add_ev(fp, np, sl, q4 * u, q4 * w);
      }
    }
  }
  if (EV) {
    // bonded energy total, one integer reduction per warp
    long long v = fixq(u);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31u) == 0u && v != 0) atomicAdd(&acc[3], (unsigned long long)v);
  }
}

}  // namespace

int bonded_free(hb_forcefield *ff) {
  cudaFree(ff->d_bond_atoms);
  cudaFree(ff->d_bond_par);
  cudaFree(ff->d_angle_atoms);
  cudaFree(ff->d_angle_par);
  cudaFree(ff->d_dih_atoms);
  cudaFree(ff->d_dih_par);
  return HB_OK;
}

int bonded_setup(hb_forcefield *ff, const hb_forcefield_desc *d) {
  const uint32_t n = ff->sys->n;
  ff->n_bonds = d->n_bonds;
  ff->n_angles = d->n_angles;
  ff->n_dihedrals = d->n_dihedrals;
  if (d->n_bonds) {
    HB_REQUIRE(d->bond_atoms && d->bond_k && d->bond_r0, HB_ERR_INVALID_ARGUMENT, "bond arrays");
    std::vector<uint2> at(d->n_bonds);
    std::vector<float2> par(d->n_bonds);
    for (uint32_t q = 0; q < d->n_bonds; ++q) {
      const uint32_t i = d->bond_atoms[2 * q], j = d->bond_atoms[2 * q + 1];
      HB_REQUIRE(i < n && j < n && i != j, HB_ERR_INVALID_ARGUMENT, "bond atom out of range");
      HB_REQUIRE(std::isfinite(d->bond_k[q]) && std::isfinite(d->bond_r0[q]), HB_ERR_NOT_FINITE,
                 "bond parameters must be finite");
      at[q] = make_uint2(i, j);
      par[q] = make_float2((float)d->bond_k[q], (float)d->bond_r0[q]);
    }
    HB_CUDA(cudaMalloc(&ff->d_bond_atoms, sizeof(uint2) * at.size()));
    HB_CUDA(cudaMalloc(&ff->d_bond_par, sizeof(float2) * par.size()));
    HB_CUDA(cudaMemcpy(ff->d_bond_atoms, at.data(), sizeof(uint2) * at.size(), cudaMemcpyHostToDevice));
    HB_CUDA(cudaMemcpy(ff->d_bond_par, par.data(), sizeof(float2) * par.size(), cudaMemcpyHostToDevice));
  }
  if (d->n_angles) {
    HB_REQUIRE(d->angle_atoms && d->angle_k && d->angle_theta0, HB_ERR_INVALID_ARGUMENT,
               "angle arrays");
    std::vector<uint4> at(d->n_angles);
    std::vector<float2> par(d->n_angles);
    for (uint32_t q = 0; q < d->n_angles; ++q) {
      const uint32_t *a = d->angle_atoms + 3 * q;
      HB_REQUIRE(a[0] < n && a[1] < n && a[2] < n && a[0] != a[1] && a[1] != a[2] && a[0] != a[2],
                 HB_ERR_INVALID_ARGUMENT, "angle atom out of range");
      HB_REQUIRE(std::isfinite(d->angle_k[q]) && std::isfinite(d->angle_theta0[q]),
                 HB_ERR_NOT_FINITE, "angle parameters must be finite");
      at[q] = make_uint4(a[0], a[1], a[2], 0u);
      par[q] = make_float2((float)d->angle_k[q], (float)d->angle_theta0[q]);
    }
    HB_CUDA(cudaMalloc(&ff->d_angle_atoms, sizeof(uint4) * at.size()));
    HB_CUDA(cudaMalloc(&ff->d_angle_par, sizeof(float2) * par.size()));
    HB_CUDA(cudaMemcpy(ff->d_angle_atoms, at.data(), sizeof(uint4) * at.size(), cudaMemcpyHostToDevice));
    HB_CUDA(cudaMemcpy(ff->d_angle_par, par.data(), sizeof(float2) * par.size(), cudaMemcpyHostToDevice));
  }
  if (d->n_dihedrals) {
    HB_REQUIRE(d->dihedral_atoms && d->dihedral_k && d->dihedral_phi0 && d->dihedral_n,
               HB_ERR_INVALID_ARGUMENT, "dihedral arrays");
    std::vector<uint4> at(d->n_dihedrals);
    std::vector<float4> par(d->n_dihedrals);
    for (uint32_t q = 0; q < d->n_dihedrals; ++q) {
      const uint32_t *a = d->dihedral_atoms + 4 * q;
      HB_REQUIRE(a[0] < n && a[1] < n && a[2] < n && a[3] < n, HB_ERR_INVALID_ARGUMENT,
                 "dihedral atom out of range");
      HB_REQUIRE(std::isfinite(d->dihedral_k[q]) && std::isfinite(d->dihedral_phi0[q]),
                 HB_ERR_NOT_FINITE, "dihedral parameters must be finite");
      at[q] = make_uint4(a[0], a[1], a[2], a[3]);
      par[q] = make_float4((float)d->dihedral_k[q], (float)d->dihedral_phi0[q],
                           (float)d->dihedral_n[q], 0.0f);
    }
    HB_CUDA(cudaMalloc(&ff->d_dih_atoms, sizeof(uint4) * at.size()));
    HB_CUDA(cudaMalloc(&ff->d_dih_par, sizeof(float4) * par.size()));
    HB_CUDA(cudaMemcpy(ff->d_dih_atoms, at.data(), sizeof(uint4) * at.size(), cudaMemcpyHostToDevice));
    HB_CUDA(cudaMemcpy(ff->d_dih_par, par.data(), sizeof(float4) * par.size(), cudaMemcpyHostToDevice));
  }
  return HB_OK;
}

int bonded_launch(hb_forcefield *ff, bool ev, cudaStream_t s) {
  const uint32_t total = ff->n_bonds + ff->n_angles + ff->n_dihedrals;
  if (total == 0) return HB_OK;
  hb_system *sys = ff->sys;
  const unsigned grid = hb_div_up(total, 128);
  if (ev)
    k_bonded<true><<<grid, 128, 0, s>>>(sys->d_posq, ff->d_inv_perm, sys->d_box, ff->d_bond_atoms,
                                        ff->d_bond_par, ff->n_bonds, ff->d_angle_atoms,
                                        ff->d_angle_par, ff->n_angles, ff->d_dih_atoms,
                                        ff->d_dih_par, ff->n_dihedrals, ff->d_fp, ff->n_pad,
                                        ff->d_acc);
  else
    k_bonded<false><<<grid, 128, 0, s>>>(sys->d_posq, ff->d_inv_perm, sys->d_box, ff->d_bond_atoms,
                                         ff->d_bond_par, ff->n_bonds, ff->d_angle_atoms,
                                         ff->d_angle_par, ff->n_angles, ff->d_dih_atoms,
                                         ff->d_dih_par, ff->n_dihedrals, ff->d_fp, ff->n_pad,
                                         ff->d_acc);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}
