// hb_spme.cu -- SPME reciprocal space: charge spread, 3-D FFT with the
// influence-function convolution fused into the middle pass, force gather.
//
// Physics follows the reference (src/forces/spme.rs:228-503, :815-822;
// kernels/spme_recip.cu:34-402; kernels/spme_spread_gather.cuh:36-334):
// cardinal B-splines of order p on the fractional grid u = (s + 1/2) n,
// grid points floor(u) - d with weight M_p(d + t); the influence function
// G(k) = (1/V)(4 pi / K^2) exp(-K^2 / 4 alpha^2) |b_a b_b b_c|^2 with
// Essmann's near-zero averaging of the b-factors; tinfoil k = 0; energy
// 1/2 sum_k G |rho_hat|^2, virial 1/2 sum_k G (1 - K^2 / 2 alpha^2)
// |rho_hat|^2; per-atom energy share 1/2 q phi - alpha / sqrt(pi) q^2;
// uniform per-atom virial share W_recip / N.
//
// Device pipeline (own design):
//   spread   : p threads per atom (sorted, spatially coherent order), one
//              per c stencil offset, each adding its p^2 contributions to
//              an int64 grid with scale 2^32 (order-independent,
//              byte-identical repeat runs);
//   fft_c    : per row, int64 -> f32, clears the int64 grid for the next
//              step, length-n_c transform, keeps n_c / 2 + 1 modes;
//   fft_b    : batches of 16 lines along b, transform in shared memory;
//   fft_a    : batches along a: forward transform, multiply by G computed
//              on the fly (no influence buffers, so a box change needs no
//              refresh pass), FP64 energy / virial partials, inverse
//              transform -- the convolution costs no extra grid pass;
//   ifft_b, ifft_c (Hermitian extension, real part) -> V;
//   gather   : p^3 reads of V per atom, force, energy share; for p = 4 and
//              8 one thread per c offset (runs of consecutive reads, sums
//              met by shuffles), else one thread per atom.
// The line passes are Stockham autosort transforms with radix 8, 4, 2, 3,
// 5, 7 butterflies, twiddles from an FP64-built table, lines held in shared
// memory with a padded stride.  For 64 x 64 and 128 x 128 (a, b) planes
// the c pass writes kc-major planes instead, and one whole-plane pass per
// kc replaces fft_b, fft_a and ifft_b: both forward transforms, the
// influence function and both inverse transforms run in place on the plane
// in shared memory (radix-16 and radix-8 stages).  Deterministic by
// construction.
#include <cmath>
#include <vector>

#include "hb_internal.cuh"

namespace {

struct FftPlan {
  int n;
  int nst;
  int r[16];
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// p-point DFT of v (forward: exp(-2 pi i qr / p)), p in {2, 3, 4, 5, 7, 8};
// the twiddle constants are cos / sin of 2 pi k / p.
template <int P, bool INV>
__device__ __forceinline__ void butterfly(float2 *v) {
  if constexpr (P == 8) {
    // two 4-point DFTs of the even and odd elements, the odd ones turned by
    // w^k (w = exp(-+2 pi i / 8)), then X_k = E_k + w^k O_k, X_{k+4} = E_k - w^k O_k
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    butterfly<4, INV>(e);
    butterfly<4, INV>(o);
    const float h = 0.70710678118654752f;
    const float2 o1 = o[1], o2 = o[2], o3 = o[3];
    if (INV) {
      o[1] = make_float2((o1.x - o1.y) * h, (o1.x + o1.y) * h);
      o[2] = make_float2(-o2.y, o2.x);
      o[3] = make_float2((-o3.x - o3.y) * h, (o3.x - o3.y) * h);
    } else {
      o[1] = make_float2((o1.x + o1.y) * h, (o1.y - o1.x) * h);
      o[2] = make_float2(o2.y, -o2.x);
      o[3] = make_float2((o3.y - o3.x) * h, (-o3.x - o3.y) * h);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = make_float2(e[k].x + o[k].x, e[k].y + o[k].y);
      v[k + 4] = make_float2(e[k].x - o[k].x, e[k].y - o[k].y);
    }
  } else if constexpr (P == 16) {
    // 4 x 4: 4-point DFTs of the elements n2, n2 + 4, n2 + 8, n2 + 12, turned
    // by w^(n2 k1) (w = exp(-+2 pi i / 16)), then 4-point DFTs across n2:
    // X[k1 + 4 k2]; the twiddles are cos / sin of multiples of pi / 8
    float2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      float2 t[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
      butterfly<4, INV>(t);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
    }
    constexpr float c16[10] = {1.0f, 0.92387953251128674f, 0.70710678118654752f,
                               0.38268343236508977f, 0.0f, -0.38268343236508977f,
                               -0.70710678118654752f, -0.92387953251128674f, -1.0f,
                               -0.92387953251128674f};
    constexpr float s16[10] = {0.0f, 0.38268343236508977f, 0.70710678118654752f,
                               0.92387953251128674f, 1.0f, 0.92387953251128674f,
                               0.70710678118654752f, 0.38268343236508977f, 0.0f,
                               -0.38268343236508977f};
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
      for (int k1 = 1; k1 < 4; ++k1) {
        const int e = n2 * k1;
        const float2 w = make_float2(c16[e], INV ? s16[e] : -s16[e]);
        a[n2][k1] = cmul(a[n2][k1], w);
      }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      butterfly<4, INV>(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
    }
  } else if constexpr (P == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if constexpr (P == 4) {
    const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
    const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
    const float2 a2 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
    const float2 a3 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
    // forward: X1 = a1 - i a3, X3 = a1 + i a3 (inverse swaps the sign)
    const float2 ia3 = INV ? make_float2(-a3.y, a3.x) : make_float2(a3.y, -a3.x);
    v[0] = make_float2(a0.x + a2.x, a0.y + a2.y);
    v[2] = make_float2(a0.x - a2.x, a0.y - a2.y);
    v[1] = make_float2(a1.x + ia3.x, a1.y + ia3.y);
    v[3] = make_float2(a1.x - ia3.x, a1.y - ia3.y);
  } else {
    constexpr float c3[3] = {1.0f, -0.5f, -0.5f};
    constexpr float s3[3] = {0.0f, 0.86602540378443865f, -0.86602540378443865f};
    constexpr float c5[5] = {1.0f, 0.30901699437494742f, -0.80901699437494742f,
                             -0.80901699437494742f, 0.30901699437494742f};
    constexpr float s5[5] = {0.0f, 0.95105651629515357f, 0.58778525229247313f,
                             -0.58778525229247313f, -0.95105651629515357f};
    constexpr float c7[7] = {1.0f, 0.62348980185873353f, -0.22252093395631440f,
                             -0.90096886790241913f, -0.90096886790241913f,
                             -0.22252093395631440f, 0.62348980185873353f};
    constexpr float s7[7] = {0.0f, 0.78183148246802981f, 0.97492791218182361f,
                             0.43388373911755812f, -0.43388373911755812f,
                             -0.97492791218182361f, -0.78183148246802981f};
    const float *cs = P == 3 ? c3 : (P == 5 ? c5 : c7);
    const float *sn = P == 3 ? s3 : (P == 5 ? s5 : s7);
    float2 o[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      float2 acc = v[0];
#pragma unroll
      for (int q = 1; q < P; ++q) {
        const int e = (q * r) % P;
        const float c = cs[e], sgn = INV ? sn[e] : -sn[e];
        acc.x += v[q].x * c - v[q].y * sgn;
        acc.y += v[q].x * sgn + v[q].y * c;
      }
      o[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < P; ++r) v[r] = o[r];
  }
}

// One Stockham radix-P stage over L lines (line-major, stride n + 1):
// butterfly j of a line reads elements j + q m, twiddles them by
// w^(q (j mod Ns)), and writes (j / Ns) Ns P + (j mod Ns) + q Ns.
template <int P, bool INV>
__device__ __forceinline__ void stage_dyn(const float2 *A, float2 *B, const float2 *tw, int n,
                                          int L, int Ns) {
  const int S = n + 1, m = n / P, tstep = n / (Ns * P);
  for (int idx = threadIdx.x; idx < m * L; idx += blockDim.x) {
    const int l = idx / m, j = idx - l * m;
    const int k = j % Ns;
    const float2 *src = A + l * S;
    float2 v[P];
#pragma unroll
    for (int q = 0; q < P; ++q) v[q] = src[j + q * m];
    if (Ns > 1) {
#pragma unroll
      for (int q = 1; q < P; ++q) {
        const float2 w = tw[q * k * tstep];
        v[q] = INV ? cmulc(v[q], w) : cmul(v[q], w);
      }
    }
    butterfly<P, INV>(v);
    float2 *dst = B + l * S;
    const int base = (j / Ns) * Ns * P + k;
#pragma unroll
    for (int q = 0; q < P; ++q) dst[base + q * Ns] = v[q];
  }
}

// Runtime-planned transform of L lines of length n (fallback for sizes
// without a compile-time specialisation).  Returns the result buffer.
template <bool INV>
__device__ float2 *fft_lines(float2 *A, float2 *B, const float2 *__restrict__ tw, int n,
                             int L, const FftPlan &pl) {
  int Ns = 1;
  for (int st = 0; st < pl.nst; ++st) {
    const int p = pl.r[st];
    switch (p) {
      case 2: stage_dyn<2, INV>(A, B, tw, n, L, Ns); break;
      case 3: stage_dyn<3, INV>(A, B, tw, n, L, Ns); break;
      case 4: stage_dyn<4, INV>(A, B, tw, n, L, Ns); break;
      case 5: stage_dyn<5, INV>(A, B, tw, n, L, Ns); break;
      default: stage_dyn<7, INV>(A, B, tw, n, L, Ns); break;
    }
    __syncthreads();
    float2 *t = A;
    A = B;
    B = t;
    Ns *= p;
  }
  return A;
}

// ---- compile-time transforms: radix order 8, 4, 2, 3, 5, 7 (fewer shared-
// memory stages than the runtime plans of make_plan, which start at 4) ----
__host__ __device__ constexpr int radix_first(int n) {
  return n % 8 == 0 ? 8
                    : (n % 4 == 0 ? 4 : (n % 2 == 0 ? 2 : (n % 3 == 0 ? 3 : (n % 5 == 0 ? 5 : 7))));
}
__host__ __device__ constexpr int stage_radix(int n, int s) {
  int p = radix_first(n);
  while (s > 0) {
    n /= p;
    p = radix_first(n);
    --s;
  }
  return p;
}
__host__ __device__ constexpr int n_stages(int n) {
  int c = 0;
  while (n > 1) {
    n /= radix_first(n);
    ++c;
  }
  return c;
}
__host__ __device__ constexpr int lines_of(int n) { return 2048 / n > 16 ? 16 : (2048 / n < 2 ? 2 : 2048 / n); }
constexpr int FFT_THREADS = 256;

template <int N, int L, bool INV, int S, int NS>
__device__ __forceinline__ float2 *fft_stages(float2 *A, float2 *B, const float2 *__restrict__ tw) {
  if constexpr (S == n_stages(N)) {
    return A;
  } else {
    constexpr int P = stage_radix(N, S), M = N / P, TSTEP = N / (NS * P), STR = N + 1;
    for (int idx = threadIdx.x; idx < M * L; idx += FFT_THREADS) {
      const int l = idx / M, j = idx % M;
      const int k = j % NS;
      const float2 *src = A + l * STR;
      float2 v[P];
#pragma unroll
      for (int q = 0; q < P; ++q) v[q] = src[j + q * M];
      if constexpr (NS > 1) {
#pragma unroll
        for (int q = 1; q < P; ++q) {
          const float2 w = tw[q * k * TSTEP];
          v[q] = INV ? cmulc(v[q], w) : cmul(v[q], w);
        }
      }
      butterfly<P, INV>(v);
      float2 *dst = B + l * STR;
      const int base = (j / NS) * NS * P + k;
#pragma unroll
      for (int q = 0; q < P; ++q) dst[base + q * NS] = v[q];
    }
    __syncthreads();
    return fft_stages<N, L, INV, S + 1, NS * P>(B, A, tw);
  }
}

// N > 0: compile-time transform of lines_of(N) lines; N == 0: runtime plan
template <int N, bool INV>
__device__ __forceinline__ float2 *fft_run(float2 *A, float2 *B, const float2 *__restrict__ tw,
                                           int n, int L, const FftPlan &pl) {
  if constexpr (N == 0) {
    return fft_lines<INV>(A, B, tw, n, L, pl);
  } else {
    return fft_stages<N, lines_of(N), INV, 0, 1>(A, B, tw);
  }
}

// B-spline weights w[d] = M_P(d + t), d = 0..P-1, and optionally their
// derivatives, by the Cox-de Boor recursion raised one order at a time.
template <int P, bool DERIV>
__device__ __forceinline__ void bspline(float t, float *w, float *dw) {
  if constexpr (P == 4) {
    // the cubic case in closed form (the recursion below, multiplied out):
    // w = (t^3, 1 + 3t + 3t^2 - 3t^3, 4 - 6t^2 + 3t^3, (1 - t)^3) / 6,
    // dw = (t^2, 1 + 2t - 3t^2, 3t^2 - 4t, -(1 - t)^2) / 2
    const float t2 = t * t, t3 = t2 * t, s = 1.0f - t, s2 = s * s;
    w[0] = t3 * (1.0f / 6.0f);
    w[1] = fmaf(0.5f, (t + t2) - t3, 1.0f / 6.0f);
    w[2] = fmaf(0.5f, t3, (2.0f / 3.0f) - t2);
    w[3] = s2 * s * (1.0f / 6.0f);
    if constexpr (DERIV) {
      dw[0] = 0.5f * t2;
      dw[1] = fmaf(-1.5f, t2, 0.5f + t);
      dw[2] = fmaf(1.5f, t2, -2.0f * t);
      dw[3] = -0.5f * s2;
    }
    return;
  }
  float c[P];
  c[0] = 1.0f;
#pragma unroll
  for (int d = 1; d < P; ++d) c[d] = 0.0f;
#pragma unroll
  for (int k = 2; k <= P; ++k) {
    if (DERIV && k == P) {
#pragma unroll
      for (int d = 0; d < P; ++d) dw[d] = (d < P - 1 ? c[d] : 0.0f) - (d >= 1 ? c[d - 1] : 0.0f);
    }
    const float inv = 1.0f / (float)(k - 1);
#pragma unroll
    for (int d = k - 1; d >= 0; --d) {
      float a = (d <= k - 2) ? (t + (float)d) * c[d] : 0.0f;
      float b = (d >= 1) ? ((float)k - t - (float)d) * c[d - 1] : 0.0f;
      c[d] = (a + b) * inv;
    }
  }
#pragma unroll
  for (int d = 0; d < P; ++d) w[d] = c[d];
}

__device__ __forceinline__ void grid_setup(float x, float y, float z, const DBox &b, int na,
                                           int nb, int nc, float t[3], int g0[3]) {
  int ka, kb, kc;
  hb_wrap(x, y, z, ka, kb, kc, b);
  float s[3];
  hb_frac(x, y, z, b, s[0], s[1], s[2]);
  const int n[3] = {na, nb, nc};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float u = (s[d] + 0.5f) * (float)n[d];
    float f = floorf(u);
    t[d] = u - f;
    // s lies in [-1/2, 1/2] up to rounding after the wrap, so fi is in
    // [-1, n]: one conditional step gives the residue mod n; positions far
    // outside any cell (a system blowing up) take the full residue, so the
    // index stays inside the grid whatever the input
    int fi = (int)f;
    if (fi >= n[d]) fi -= n[d];
    else if (fi < 0) fi += n[d];
    if ((unsigned)fi >= (unsigned)n[d]) {
      fi %= n[d];
      if (fi < 0) fi += n[d];
    }
    g0[d] = fi;
  }
}

// P threads per atom, one per c stencil offset, each adding the P^2 points
// of its (a, b) stencil: the P threads of one atom differ only in c, so one
// atomic instruction of a warp writes runs of P consecutive grid words (few
// L2 sectors) instead of 32 scattered ones
template <int P>
__global__ void k_spread(const float4 *__restrict__ tile_posq, const DBox *__restrict__ box,
                         int na, int nb, int nc, unsigned long long *__restrict__ rho,
                         uint32_t n) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t k = g / P;
  const int dc = (int)(g - k * P);
  if (k >= n) return;
  const float4 p = tile_posq[k];
  if (p.w == 0.0f) return;
  const DBox b = *box;
  float t[3];
  int g0[3];
  grid_setup(p.x, p.y, p.z, b, na, nb, nc, t, g0);
  float wa[P], wb[P], wc[P];
  bspline<P, false>(t[0], wa, nullptr);
  bspline<P, false>(t[1], wb, nullptr);
  bspline<P, false>(t[2], wc, nullptr);
  int gc = g0[2] - dc;
  if (gc < 0) gc += nc;
  float wdc = 0.0f;
#pragma unroll
  for (int d = 0; d < P; ++d)
    if (d == dc) wdc = wc[d];
#pragma unroll
  for (int da = 0; da < P; ++da) {
    int ga = g0[0] - da;
    if (ga < 0) ga += na;
    const float qa = p.w * wa[da];
#pragma unroll
    for (int db = 0; db < P; ++db) {
      int gb = g0[1] - db;
      if (gb < 0) gb += nb;
      const float qab = qa * wb[db];
      const long long v = __float2ll_rn(qab * wdc * HB_RHO_SCALE);
      if (v != 0) atomicAdd(&rho[((size_t)ga * nb + gb) * nc + gc], (unsigned long long)v);
    }
  }
}

// forward transform along c, one CTA per L rows; clears the int64 grid.
// The half spectrum goes out row-major ([row][kc], KCM = false) or as
// kc-major planes ([kc][row], KCM = true) for the whole-plane pass.
template <int N, bool KCM = false>
__global__ void __launch_bounds__(256) k_fft_c_fwd(unsigned long long *__restrict__ rho,
                                                   float2 *__restrict__ grid,
                                                   const float2 *__restrict__ tw_g, FftPlan pl,
                                                   int nrows, int nch, int L_rt) {
  extern __shared__ float2 sm[];
  const int n = N ? N : pl.n, S = n + 1;
  const int L = N ? lines_of(N) : L_rt;
  float2 *tw = sm;
  float2 *A = sm + n;
  float2 *B = A + L * S;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  const int row0 = blockIdx.x * L;
  const int nr = min(L, nrows - row0);
  if constexpr (N > 0) {
    // every load of the thread first, then the clearing stores: interleaved
    // with stores to the same array the loads would run one at a time
    constexpr int LN = lines_of(N) * N, IT = (LN + 255) / 256;
    unsigned long long *base = rho + (size_t)row0 * N;
    long long v[IT];
#pragma unroll
    for (int q = 0; q < IT; ++q) {
      const int idx = (int)threadIdx.x + q * 256;
      v[q] = (idx < LN && idx / N < nr) ? (long long)base[idx] : 0ll;
    }
#pragma unroll
    for (int q = 0; q < IT; ++q) {
      const int idx = (int)threadIdx.x + q * 256;
      if (idx < LN) {
        const int r = idx / N, c = idx - r * N;
        if (r < nr) base[idx] = 0ull;
        A[r * S + c] = make_float2((float)v[q] * (1.0f / HB_RHO_SCALE), 0.0f);
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
      const int r = idx / n, c = idx - (idx / n) * n;
      float v = 0.0f;
      if (r < nr) {
        const size_t gi = (size_t)(row0 + r) * n + c;
        v = (float)(long long)rho[gi] * (1.0f / HB_RHO_SCALE);
        rho[gi] = 0ull;
      }
      A[r * S + c] = make_float2(v, 0.0f);
    }
  }
  __syncthreads();
  float2 *R = fft_run<N, false>(A, B, tw, n, L, pl);
  if constexpr (KCM) {
    for (int idx = threadIdx.x; idx < L * nch; idx += blockDim.x) {
      const int r = idx % L, c = idx / L;
      if (r < nr) grid[(size_t)c * nrows + row0 + r] = R[r * S + c];
    }
  } else {
    for (int idx = threadIdx.x; idx < L * nch; idx += blockDim.x) {
      const int r = idx / nch, c = idx - (idx / nch) * nch;
      if (r < nr) grid[(size_t)(row0 + r) * nch + c] = R[r * S + c];
    }
  }
}

// transform along b for L consecutive kc of one a-plane
template <int N, bool INV>
__global__ void __launch_bounds__(256) k_fft_b(float2 *__restrict__ grid,
                                               const float2 *__restrict__ tw_g, FftPlan pl,
                                               int nb_rt, int nch, int L_rt) {
  extern __shared__ float2 sm[];
  const int n = N ? N : pl.n, S = n + 1;
  const int nb = n;
  const int L = N ? lines_of(N) : L_rt;
  (void)nb_rt;
  float2 *tw = sm;
  float2 *A = sm + n;
  float2 *B = A + L * S;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  const int nchunk = (nch + L - 1) / L;
  const int a = blockIdx.x / nchunk;
  const int kc0 = (blockIdx.x - a * nchunk) * L;
  for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
    const int l = idx % L, bp = idx / L;
    const int kc = kc0 + l;
    A[l * S + bp] = kc < nch ? grid[((size_t)a * nb + bp) * nch + kc] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2 *R = fft_run<N, INV>(A, B, tw, n, L, pl);
  for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
    const int l = idx % L, bp = idx / L;
    const int kc = kc0 + l;
    if (kc < nch) grid[((size_t)a * nb + bp) * nch + kc] = R[l * S + bp];
  }
}

// transform along a, influence multiply with FP64 energy / virial
// partials, inverse transform along a
template <int N>
__global__ void __launch_bounds__(256) k_fft_a_conv(float2 *__restrict__ grid,
                                                    const float2 *__restrict__ tw_g, FftPlan pl,
                                                    int na_rt, int nb, int nc, int nch, int L_rt,
                                                    const DBox *__restrict__ box,
                                                    const float *__restrict__ bfac, float alpha,
                                                    double *__restrict__ part) {
  extern __shared__ float2 sm[];
  __shared__ double red_e[256], red_w[256];
  const int n = N ? N : pl.n, S = n + 1;
  const int na = n;
  const int L = N ? lines_of(N) : L_rt;
  (void)na_rt;
  float2 *tw = sm;
  float2 *A = sm + n;
  float2 *B = A + L * S;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  const int nchunk = (nch + L - 1) / L;
  const int bq = blockIdx.x / nchunk;
  const int kc0 = (blockIdx.x - bq * nchunk) * L;
  for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
    const int l = idx % L, ap = idx / L;
    const int kc = kc0 + l;
    A[l * S + ap] = kc < nch ? grid[((size_t)ap * nb + bq) * nch + kc] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2 *R = fft_run<N, false>(A, B, tw, n, L, pl);
  float2 *O = (R == A) ? B : A;
  const DBox bx = *box;
  const float ilx = bx.ilx, ily = bx.ily, ilz = bx.ilz;
  const float bax = ilx, bay = -bx.xy * ilx * ily, baz = (bx.xy * bx.yz - bx.xz * bx.ly) * ilx * ily * ilz;
  const float bby = ily, bbz = -bx.yz * ily * ilz, bcz = ilz;
  const float two_pi = 6.283185307179586f;
  const float inv_vol = ilx * ily * ilz;
  const float inv4a2 = 1.0f / (4.0f * alpha * alpha);
  const float inv2a2 = 1.0f / (2.0f * alpha * alpha);
  const float mb = (bq <= nb / 2) ? (float)bq : (float)(bq - nb);
  const float bfb = bfac[na + bq];
  double e_acc = 0.0, w_acc = 0.0;
  for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
    const int l = idx / n, ka = idx - (idx / n) * n;
    const int kc = kc0 + l;
    float2 X = R[l * S + ka];
    float G = 0.0f, vf = 0.0f;
    if (kc < nch) {
      const float ma = (ka <= na / 2) ? (float)ka : (float)(ka - na);
      const float mc = (float)kc;
      const float kx = two_pi * (ma * bax);
      const float ky = two_pi * (ma * bay + mb * bby);
      const float kz = two_pi * (ma * baz + mb * bbz + mc * bcz);
      const float k2 = kx * kx + ky * ky + kz * kz;
      if (k2 > 0.0f) {
        G = inv_vol * (12.566370614359172f / k2) * expf(-k2 * inv4a2) * bfac[ka] * bfb *
            bfac[na + nb + kc];
        vf = G * (1.0f - k2 * inv2a2);
      }
      const double hw = (kc == 0 || ((nc & 1) == 0 && 2 * kc == nc)) ? 1.0 : 2.0;
      const double x2 = (double)X.x * X.x + (double)X.y * X.y;
      e_acc += hw * (double)G * x2;
      w_acc += hw * (double)vf * x2;
    }
    R[l * S + ka] = make_float2(G * X.x, G * X.y);
  }
  red_e[threadIdx.x] = e_acc;
  red_w[threadIdx.x] = w_acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      red_e[threadIdx.x] += red_e[threadIdx.x + st];
      red_w[threadIdx.x] += red_w[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = red_e[0];
    part[2 * blockIdx.x + 1] = red_w[0];
  }
  float2 *R2 = fft_run<N, true>(R, O, tw, n, L, pl);
  for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
    const int l = idx % L, ap = idx / L;
    const int kc = kc0 + l;
    if (kc < nch) grid[((size_t)ap * nb + bq) * nch + kc] = R2[l * S + ap];
  }
}

// inverse transform along c with Hermitian extension; writes V (real).
// KCM: the half spectrum is stored as kc-major planes.
template <int N, bool KCM = false>
__global__ void __launch_bounds__(256) k_fft_c_inv(const float2 *__restrict__ grid,
                                                   float *__restrict__ v,
                                                   const float2 *__restrict__ tw_g, FftPlan pl,
                                                   int nrows, int nch, int L_rt) {
  extern __shared__ float2 sm[];
  const int n = N ? N : pl.n, S = n + 1;
  const int L = N ? lines_of(N) : L_rt;
  float2 *tw = sm;
  float2 *A = sm + n;
  float2 *B = A + L * S;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  const int row0 = blockIdx.x * L;
  const int nr = min(L, nrows - row0);
  if constexpr (KCM) {
    for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
      const int r = idx % L, c = idx / L;
      float2 x = make_float2(0.f, 0.f);
      if (r < nr) {
        if (c < nch) {
          x = grid[(size_t)c * nrows + row0 + r];
        } else {
          float2 y = grid[(size_t)(n - c) * nrows + row0 + r];
          x = make_float2(y.x, -y.y);
        }
      }
      A[r * S + c] = x;
    }
  } else {
    for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
      const int r = idx / n, c = idx - (idx / n) * n;
      float2 x = make_float2(0.f, 0.f);
      if (r < nr) {
        if (c < nch) {
          x = grid[(size_t)(row0 + r) * nch + c];
        } else {
          float2 y = grid[(size_t)(row0 + r) * nch + (n - c)];
          x = make_float2(y.x, -y.y);
        }
      }
      A[r * S + c] = x;
    }
  }
  __syncthreads();
  float2 *R = fft_run<N, true>(A, B, tw, n, L, pl);
  for (int idx = threadIdx.x; idx < L * n; idx += blockDim.x) {
    const int r = idx / n, c = idx - (idx / n) * n;
    if (r < nr) v[(size_t)(row0 + r) * n + c] = R[r * S + c].x;
  }
}

// ---------------------------------------------------------------------
// Whole-plane pass: one CTA per kc plane of the kc-major half spectrum,
// the plane (na x nb complex, padded stride nb + 1) held in shared memory.
// Forward transforms along b and along a run in place as decimation in
// frequency (output in digit-reversed order), the influence function
// multiplies each mode at its digit-reversed position, and the inverse
// transforms run in place as decimation in time (digit-reversed input,
// natural output): no reordering pass and no ping-pong buffer, so a 128 x
// 128 plane fits one CTA.  Replaces the b, a + convolution and inverse b
// passes (two grid round trips fewer).
// ---------------------------------------------------------------------
constexpr int PLANE_THREADS = 512;

// the whole-plane pass's stages: a radix-16 first stage where the rest
// still splits into radix-8 or smaller stages (128 = 16 x 8), else the
// line passes' order (8, 4, 2, 3, 5, 7)
__host__ __device__ constexpr int plane_radix_first(int n) {
  return (n % 16 == 0 && n >= 128) ? 16 : radix_first(n);
}
__host__ __device__ constexpr int plane_radix(int n, int s) {
  int p = plane_radix_first(n);
  while (s > 0) {
    n /= p;
    p = plane_radix_first(n);
    --s;
  }
  return p;
}
__host__ __device__ constexpr int plane_stages(int n) {
  int c = 0;
  while (n > 1) {
    n /= plane_radix_first(n);
    ++c;
  }
  return c;
}

// product of the radices of stages [0, s)
__host__ __device__ constexpr int radix_prod(int n, int s) {
  int p = 1;
  for (int k = 0; k < s; ++k) p *= plane_radix(n, k);
  return p;
}

// One in-place stage STG over LINES lines of length N (line and element
// strides LS and ES in float2).  Forward (decimation in frequency): butterfly on
// elements j + q h of each block of length m, then twiddles W_m^(r j);
// inverse (decimation in time): conjugate twiddles, then the inverse
// butterfly.  The inverse stage undoes the forward one up to the factor p.
template <int N, int STG, bool INV, int LINES, int LS, int ES>
__device__ __forceinline__ void plane_stage(float2 *P, const float2 *tw) {
  constexpr int p = plane_radix(N, STG);
  constexpr int m = N / radix_prod(N, STG);
  constexpr int h = m / p;
  constexpr int NBF = N / p;  // butterflies per line
  for (int w = threadIdx.x; w < LINES * NBF; w += PLANE_THREADS) {
    const int line = w % LINES, beta = w / LINES;
    const int blk = beta / h, j = beta - blk * h;
    float2 *x = P + line * LS + (blk * m + j) * ES;
    float2 v[p];
#pragma unroll
    for (int q = 0; q < p; ++q) v[q] = x[q * h * ES];
    if constexpr (!INV) {
      butterfly<p, false>(v);
#pragma unroll
      for (int r = 1; r < p; ++r) v[r] = cmul(v[r], tw[(N / m) * r * j]);
    } else {
#pragma unroll
      for (int r = 1; r < p; ++r) v[r] = cmulc(v[r], tw[(N / m) * r * j]);
      butterfly<p, true>(v);
    }
#pragma unroll
    for (int q = 0; q < p; ++q) x[q * h * ES] = v[q];
  }
}

template <int N, int STG, int LINES, int LS, int ES>
__device__ __forceinline__ void plane_dif(float2 *P, const float2 *tw) {
  if constexpr (STG < plane_stages(N)) {
    plane_stage<N, STG, false, LINES, LS, ES>(P, tw);
    __syncthreads();
    plane_dif<N, STG + 1, LINES, LS, ES>(P, tw);
  }
}

template <int N, int STG, int LINES, int LS, int ES>
__device__ __forceinline__ void plane_dit(float2 *P, const float2 *tw) {
  if constexpr (STG >= 0) {
    plane_stage<N, STG, true, LINES, LS, ES>(P, tw);
    __syncthreads();
    plane_dit<N, STG - 1, LINES, LS, ES>(P, tw);
  }
}

// frequency index held at position pos after the forward stages: pos has
// digit r_s at weight N / (p_0 ... p_s), the frequency has it at weight
// p_0 ... p_(s-1)
template <int N>
__device__ __forceinline__ int plane_freq(int pos) {
  int k = 0;
#pragma unroll
  for (int s = 0; s < plane_stages(N); ++s) {
    const int p = plane_radix(N, s);
    const int h = N / (radix_prod(N, s) * p);
    k += ((pos / h) % p) * radix_prod(N, s);
  }
  return k;
}

__host__ __device__ constexpr size_t plane_smem(int na, int nb) {
  return sizeof(float2) * ((size_t)na * (nb + 1) + na + nb);
}

// EV: also the FP64 energy / virial partials of the plane (steps that
// report energies or pressure); without, the influence function alone
template <int NA, int NB, bool EV>
__global__ void __launch_bounds__(PLANE_THREADS) k_fft_plane(
    float2 *__restrict__ grid, const float2 *__restrict__ tw_g, int nc,
    const DBox *__restrict__ box, const float *__restrict__ bfac, float alpha,
    double *__restrict__ part) {
  extern __shared__ float2 smp[];
  __shared__ double red_e[PLANE_THREADS / 32], red_w[PLANE_THREADS / 32];
  constexpr int S = NB + 1;
  float2 *P = smp;
  float2 *twa = P + NA * S;
  float2 *twb = twa + NA;
  const int kc = blockIdx.x;
  for (int i = threadIdx.x; i < NA; i += PLANE_THREADS) twa[i] = tw_g[i];
  for (int i = threadIdx.x; i < NB; i += PLANE_THREADS) twb[i] = tw_g[NA + i];
  float2 *g = grid + (size_t)kc * NA * NB;
  for (int idx = threadIdx.x; idx < NA * NB; idx += PLANE_THREADS) {
    const int a = idx / NB, b = idx - a * NB;
    P[a * S + b] = g[idx];
  }
  __syncthreads();
  plane_dif<NB, 0, NA, S, 1>(P, twb);  // along b: the NA rows
  plane_dif<NA, 0, NB, 1, S>(P, twa);  // along a: the NB columns

  // influence function at each mode, FP64 energy / virial partials
  const DBox bx = *box;
  const float ilx = bx.ilx, ily = bx.ily, ilz = bx.ilz;
  const float bax = ilx, bay = -bx.xy * ilx * ily, baz = (bx.xy * bx.yz - bx.xz * bx.ly) * ilx * ily * ilz;
  const float bby = ily, bbz = -bx.yz * ily * ilz, bcz = ilz;
  const float two_pi = 6.283185307179586f;
  const float inv_vol = ilx * ily * ilz;
  const float inv4a2 = 1.0f / (4.0f * alpha * alpha);
  const float inv2a2 = 1.0f / (2.0f * alpha * alpha);
  const float mc = (float)kc;
  const float bfc = bfac[NA + NB + kc];
  const double hw = (kc == 0 || ((nc & 1) == 0 && 2 * kc == nc)) ? 1.0 : 2.0;
  double e_acc = 0.0, w_acc = 0.0;
  for (int idx = threadIdx.x; idx < NA * NB; idx += PLANE_THREADS) {
    const int pa = idx / NB, pb = idx - pa * NB;
    const int ka = plane_freq<NA>(pa), kb = plane_freq<NB>(pb);
    const float ma = (ka <= NA / 2) ? (float)ka : (float)(ka - NA);
    const float mb = (kb <= NB / 2) ? (float)kb : (float)(kb - NB);
    const float kx = two_pi * (ma * bax);
    const float ky = two_pi * (ma * bay + mb * bby);
    const float kz = two_pi * (ma * baz + mb * bbz + mc * bcz);
    const float k2 = kx * kx + ky * ky + kz * kz;
    float G = 0.0f, vf = 0.0f;
    if (k2 > 0.0f) {
      G = inv_vol * (12.566370614359172f / k2) * expf(-k2 * inv4a2) * bfac[ka] * bfac[NA + kb] * bfc;
      if constexpr (EV) vf = G * (1.0f - k2 * inv2a2);
    }
    float2 &X = P[pa * S + pb];
    if constexpr (EV) {
      const double x2 = (double)X.x * X.x + (double)X.y * X.y;
      e_acc += hw * (double)G * x2;
      w_acc += hw * (double)vf * x2;
    }
    X = make_float2(G * X.x, G * X.y);
  }
  if constexpr (EV) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      e_acc += __shfl_xor_sync(0xFFFFFFFFu, e_acc, o);
      w_acc += __shfl_xor_sync(0xFFFFFFFFu, w_acc, o);
    }
    if ((threadIdx.x & 31u) == 0u) {
      red_e[threadIdx.x >> 5] = e_acc;
      red_w[threadIdx.x >> 5] = w_acc;
    }
  }
  __syncthreads();
  if (EV && threadIdx.x == 0) {
    double e = 0.0, w = 0.0;
    for (int k = 0; k < PLANE_THREADS / 32; ++k) {
      e += red_e[k];
      w += red_w[k];
    }
    part[2 * kc] = e;
    part[2 * kc + 1] = w;
  }
  plane_dit<NA, plane_stages(NA) - 1, NB, 1, S>(P, twa);
  plane_dit<NB, plane_stages(NB) - 1, NA, S, 1>(P, twb);
  for (int idx = threadIdx.x; idx < NA * NB; idx += PLANE_THREADS) {
    const int a = idx / NB, b = idx - a * NB;
    g[idx] = P[a * S + b];
  }
}

template <int P>
__global__ void k_gather(const float4 *__restrict__ tile_posq, const float *__restrict__ V,
                         const DBox *__restrict__ box, int na, int nb, int nc, float self_pref,
                         float4 *__restrict__ out, uint32_t n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float4 p = tile_posq[k];
  const DBox b = *box;
  float t[3];
  int g0[3];
  grid_setup(p.x, p.y, p.z, b, na, nb, nc, t, g0);
  float wa[P], wb[P], wc[P], dwa[P], dwb[P], dwc[P];
  bspline<P, true>(t[0], wa, dwa);
  bspline<P, true>(t[1], wb, dwb);
  bspline<P, true>(t[2], wc, dwc);
  int gc[P];
#pragma unroll
  for (int d = 0; d < P; ++d) {
    int x = g0[2] - d;
    gc[d] = x < 0 ? x + nc : x;
  }
  float phi = 0.f, ga = 0.f, gb = 0.f, gcc = 0.f;
#pragma unroll
  for (int da = 0; da < P; ++da) {
    int ia = g0[0] - da;
    if (ia < 0) ia += na;
#pragma unroll
    for (int db = 0; db < P; ++db) {
      int ib = g0[1] - db;
      if (ib < 0) ib += nb;
      const float *row = V + ((size_t)ia * nb + ib) * nc;
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int dc = 0; dc < P; ++dc) {
        const float v = __ldg(row + gc[dc]);
        s0 += v * wc[dc];
        s1 += v * dwc[dc];
      }
      phi += wa[da] * wb[db] * s0;
      ga += dwa[da] * wb[db] * s0;
      gb += wa[da] * dwb[db] * s0;
      gcc += wa[da] * wb[db] * s1;
    }
  }
  ga *= (float)na;
  gb *= (float)nb;
  gcc *= (float)nc;
  // rows of H^{-T} (spme_spread_gather.cuh:128-148)
  const float bax = b.ilx, bay = -b.xy * b.ilx * b.ily,
              baz = (b.xy * b.yz - b.xz * b.ly) * b.ilx * b.ily * b.ilz;
  const float bby = b.ily, bbz = -b.yz * b.ily * b.ilz, bcz = b.ilz;
  const float q = p.w;
  float4 o;
  o.x = -q * (ga * bax);
  o.y = -q * (ga * bay + gb * bby);
  o.z = -q * (ga * baz + gb * bbz + gcc * bcz);
  o.w = 0.5f * q * phi - self_pref * q * q;
  out[k] = o;
}

// Gather with P threads per atom (P a power of two), one per c stencil
// offset: the P threads of an atom read runs of P consecutive potential
// words (few L1 sectors per load instruction instead of 32 scattered ones),
// and their partial sums meet by shuffles within the aligned group of P
// lanes
template <int P>
__global__ void k_gather_c(const float4 *__restrict__ tile_posq, const float *__restrict__ V,
                           const DBox *__restrict__ box, int na, int nb, int nc, float self_pref,
                           float4 *__restrict__ out, uint32_t n) {
  static_assert(P == 4 || P == 8, "lane groups must tile the warp");
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t k = g / P;
  const int dc = (int)(g % P);
  const bool valid = k < n;
  // lanes past the end follow the last atom so that every lane of the warp
  // takes part in the shuffles; they write nothing
  const float4 p = tile_posq[valid ? k : n - 1];
  const DBox b = *box;
  float t[3];
  int g0[3];
  grid_setup(p.x, p.y, p.z, b, na, nb, nc, t, g0);
  float wa[P], wb[P], wc[P], dwa[P], dwb[P], dwc[P];
  bspline<P, true>(t[0], wa, dwa);
  bspline<P, true>(t[1], wb, dwb);
  bspline<P, true>(t[2], wc, dwc);
  int ic = g0[2] - dc;
  if (ic < 0) ic += nc;
  float A = 0.f, B = 0.f, C = 0.f;
#pragma unroll
  for (int da = 0; da < P; ++da) {
    int ia = g0[0] - da;
    if (ia < 0) ia += na;
#pragma unroll
    for (int db = 0; db < P; ++db) {
      int ib = g0[1] - db;
      if (ib < 0) ib += nb;
      const float v = __ldg(V + ((size_t)ia * nb + ib) * nc + ic);
      A += wa[da] * wb[db] * v;
      B += dwa[da] * wb[db] * v;
      C += wa[da] * dwb[db] * v;
    }
  }
  float wdc = 0.f, dwdc = 0.f;
#pragma unroll
  for (int d = 0; d < P; ++d)
    if (d == dc) {
      wdc = wc[d];
      dwdc = dwc[d];
    }
  float phi = wdc * A, ga = wdc * B, gb = wdc * C, gcc = dwdc * A;
#pragma unroll
  for (int o = P / 2; o > 0; o >>= 1) {
    phi += __shfl_xor_sync(0xFFFFFFFFu, phi, o);
    ga += __shfl_xor_sync(0xFFFFFFFFu, ga, o);
    gb += __shfl_xor_sync(0xFFFFFFFFu, gb, o);
    gcc += __shfl_xor_sync(0xFFFFFFFFu, gcc, o);
  }
  if (!valid || dc != 0) return;
  ga *= (float)na;
  gb *= (float)nb;
  gcc *= (float)nc;
  // rows of H^{-T} (spme_spread_gather.cuh:128-148)
  const float bax = b.ilx, bay = -b.xy * b.ilx * b.ily,
              baz = (b.xy * b.yz - b.xz * b.ly) * b.ilx * b.ily * b.ilz;
  const float bby = b.ily, bbz = -b.yz * b.ily * b.ilz, bcz = b.ilz;
  const float q = p.w;
  float4 o;
  o.x = -q * (ga * bax);
  o.y = -q * (ga * bay + gb * bby);
  o.z = -q * (ga * baz + gb * bbz + gcc * bcz);
  o.w = 0.5f * q * phi - self_pref * q * q;
  out[k] = o;
}

__global__ void k_spme_sums(const double *__restrict__ part, int n_part,
                            double *__restrict__ sums) {
  __shared__ double se[256], sw[256];
  double e = 0.0, w = 0.0;
  for (int i = threadIdx.x; i < n_part; i += 256) {
    e += part[2 * i];
    w += part[2 * i + 1];
  }
  se[threadIdx.x] = e;
  sw[threadIdx.x] = w;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      se[threadIdx.x] += se[threadIdx.x + st];
      sw[threadIdx.x] += sw[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[0] = 0.5 * se[0];
    sums[1] = 0.5 * sw[0];
  }
}

bool make_plan(int n, FftPlan &pl) {
  pl.n = n;
  pl.nst = 0;
  int m = n;
  while (m % 4 == 0 && m > 4 && pl.nst < 16) {
    pl.r[pl.nst++] = 4;
    m /= 4;
  }
  const int primes[5] = {4, 2, 3, 5, 7};
  for (int pi = 0; pi < 5; ++pi) {
    while (m % primes[pi] == 0 && pl.nst < 16) {
      pl.r[pl.nst++] = primes[pi];
      m /= primes[pi];
    }
  }
  return m == 1;
}

int lines_per_cta(int n) {
  int L = 2048 / n;
  if (L > 16) L = 16;
  if (L < 2) L = 2;
  return L;
}

// host restatement of the b-factors (src/forces/spme.rs:524-585)
double bspline_host(int p, double x) {
  double v[16];
  for (int i = 0; i < p; ++i) {
    double xi = x - i;
    v[i] = (xi >= 0.0 && xi < 1.0) ? 1.0 : 0.0;
  }
  for (int k = 2; k <= p; ++k)
    for (int i = 0; i <= p - k; ++i) {
      double xi = x - i;
      v[i] = (xi * v[i] + ((double)k - xi) * v[i + 1]) / (double)(k - 1);
    }
  return v[0];
}

void b_factors(int n, int p, std::vector<float> &out) {
  std::vector<double> mod(n);
  for (int k = 0; k < n; ++k) {
    double th = 2.0 * M_PI * k / n, re = 0.0, im = 0.0;
    for (int j = 0; j < p - 1; ++j) {
      double m = bspline_host(p, (double)(j + 1));
      re += m * std::cos(th * j);
      im += m * std::sin(th * j);
    }
    mod[k] = re * re + im * im;
  }
  for (int k = 0; k < n; ++k)
    if (mod[k] < 1.0e-7) mod[k] = 0.5 * (mod[(k + n - 1) % n] + mod[(k + 1) % n]);
  for (int k = 0; k < n; ++k) out.push_back(mod[k] > 0.0 ? (float)(1.0 / mod[k]) : 0.0f);
}

void twiddles(int n, std::vector<float2> &out) {
  for (int t = 0; t < n; ++t) {
    double a = -2.0 * M_PI * (double)t / (double)n;
    out.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
  }
}

size_t fft_smem(int n, int L) { return sizeof(float2) * ((size_t)n + 2 * (size_t)L * (n + 1)); }

#define HB_FFT_SIZES(X) \
  X(16) X(20) X(24) X(25) X(27) X(30) X(32) X(36) X(40) X(45) X(48) X(50) X(54) X(60) X(64) \
  X(80) X(96) X(128) X(160) X(192) X(256)

struct SpmeLaunch {
  int na, nb, nc, nch, La, Lb, Lc;
  FftPlan pa, pb, pc;
};

SpmeLaunch spme_plan(int na, int nb, int nc) {
  SpmeLaunch q;
  q.na = na;
  q.nb = nb;
  q.nc = nc;
  q.nch = nc / 2 + 1;
  q.La = lines_per_cta(na);
  q.Lb = lines_per_cta(nb);
  q.Lc = lines_per_cta(nc);
  make_plan(na, q.pa);
  make_plan(nb, q.pb);
  make_plan(nc, q.pc);
  return q;
}

// planes handled by the whole-plane pass: square, and small enough for one
// CTA's shared memory (128 x 129 complex = 132 KB)
bool plane_supported(int na, int nb) { return na == nb && (na == 64 || na == 128); }

// once per size, outside any stream capture: the 128 x 128 plane needs more
// than the default 48 KB of dynamic shared memory
int plane_prepare(int na) {
  if (na == 128) {
    HB_CUDA(cudaFuncSetAttribute(k_fft_plane<128, 128, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane_smem(128, 128)));
    HB_CUDA(cudaFuncSetAttribute(k_fft_plane<128, 128, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane_smem(128, 128)));
  } else {
    HB_CUDA(cudaFuncSetAttribute(k_fft_plane<64, 64, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane_smem(64, 64)));
    HB_CUDA(cudaFuncSetAttribute(k_fft_plane<64, 64, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plane_smem(64, 64)));
  }
  return HB_OK;
}

// the transform passes of one step.  Row layout: c forward (+ int64 -> f32
// and clearing), b forward, a forward + influence + a inverse, b inverse,
// c inverse -> V.  Plane layout (plane = true, sizes with plane_supported):
// c forward into kc-major planes, the whole-plane pass, c inverse.
void fft_passes(const SpmeLaunch &q, unsigned long long *rho, float2 *grid, float *v,
                const float2 *tw, const DBox *box, const float *bfac, float alpha, double *part,
                cudaStream_t s, bool plane, bool ev = true) {
  const int nrows = q.na * q.nb;
  const float2 *twa = tw, *twb = tw + q.na, *twc = tw + q.na + q.nb;
  const int gc = hb_div_up(nrows, q.Lc);
  const int gb = q.na * ((q.nch + q.Lb - 1) / q.Lb);
  const int ga = q.nb * ((q.nch + q.La - 1) / q.La);
  const size_t sc = fft_smem(q.nc, q.Lc), sb = fft_smem(q.nb, q.Lb), sa = fft_smem(q.na, q.La);
  if (plane) {
    switch (q.nc) {
#define HB_C(NN) case NN: k_fft_c_fwd<NN, true><<<gc, 256, sc, s>>>(rho, grid, twc, q.pc, nrows, q.nch, q.Lc); break;
      HB_FFT_SIZES(HB_C)
#undef HB_C
      default: k_fft_c_fwd<0, true><<<gc, 256, sc, s>>>(rho, grid, twc, q.pc, nrows, q.nch, q.Lc);
    }
    const size_t sp = plane_smem(q.na, q.nb);
    if (q.na == 128) {
      if (ev) k_fft_plane<128, 128, true><<<q.nch, PLANE_THREADS, sp, s>>>(grid, tw, q.nc, box, bfac, alpha, part);
      else k_fft_plane<128, 128, false><<<q.nch, PLANE_THREADS, sp, s>>>(grid, tw, q.nc, box, bfac, alpha, part);
    } else {
      if (ev) k_fft_plane<64, 64, true><<<q.nch, PLANE_THREADS, sp, s>>>(grid, tw, q.nc, box, bfac, alpha, part);
      else k_fft_plane<64, 64, false><<<q.nch, PLANE_THREADS, sp, s>>>(grid, tw, q.nc, box, bfac, alpha, part);
    }
    switch (q.nc) {
#define HB_C(NN) case NN: k_fft_c_inv<NN, true><<<gc, 256, sc, s>>>(grid, v, twc, q.pc, nrows, q.nch, q.Lc); break;
      HB_FFT_SIZES(HB_C)
#undef HB_C
      default: k_fft_c_inv<0, true><<<gc, 256, sc, s>>>(grid, v, twc, q.pc, nrows, q.nch, q.Lc);
    }
    return;
  }
  switch (q.nc) {
#define HB_C(NN) case NN: k_fft_c_fwd<NN><<<gc, 256, sc, s>>>(rho, grid, twc, q.pc, nrows, q.nch, q.Lc); break;
    HB_FFT_SIZES(HB_C)
#undef HB_C
    default: k_fft_c_fwd<0><<<gc, 256, sc, s>>>(rho, grid, twc, q.pc, nrows, q.nch, q.Lc);
  }
  switch (q.nb) {
#define HB_B(NN) case NN: k_fft_b<NN, false><<<gb, 256, sb, s>>>(grid, twb, q.pb, q.nb, q.nch, q.Lb); break;
    HB_FFT_SIZES(HB_B)
#undef HB_B
    default: k_fft_b<0, false><<<gb, 256, sb, s>>>(grid, twb, q.pb, q.nb, q.nch, q.Lb);
  }
  switch (q.na) {
#define HB_A(NN) case NN: k_fft_a_conv<NN><<<ga, 256, sa, s>>>(grid, twa, q.pa, q.na, q.nb, q.nc, q.nch, q.La, box, bfac, alpha, part); break;
    HB_FFT_SIZES(HB_A)
#undef HB_A
    default: k_fft_a_conv<0><<<ga, 256, sa, s>>>(grid, twa, q.pa, q.na, q.nb, q.nc, q.nch, q.La, box, bfac, alpha, part);
  }
  switch (q.nb) {
#define HB_B(NN) case NN: k_fft_b<NN, true><<<gb, 256, sb, s>>>(grid, twb, q.pb, q.nb, q.nch, q.Lb); break;
    HB_FFT_SIZES(HB_B)
#undef HB_B
    default: k_fft_b<0, true><<<gb, 256, sb, s>>>(grid, twb, q.pb, q.nb, q.nch, q.Lb);
  }
  switch (q.nc) {
#define HB_C(NN) case NN: k_fft_c_inv<NN><<<gc, 256, sc, s>>>(grid, v, twc, q.pc, nrows, q.nch, q.Lc); break;
    HB_FFT_SIZES(HB_C)
#undef HB_C
    default: k_fft_c_inv<0><<<gc, 256, sc, s>>>(grid, v, twc, q.pc, nrows, q.nch, q.Lc);
  }
}

}  // namespace

// energy / virial partials written per step: one per kc plane (plane form)
// or one per a-pass CTA (line form)
int spme_n_part(const SpmeState &S) {
  const int La = lines_per_cta(S.na);
  return S.use_plane ? S.nch : S.nb * ((S.nch + La - 1) / La);
}

int spme_set_form(hb_forcefield *ff, int param, int value) {
  SpmeState &S = ff->spme;
  HB_REQUIRE(value == 0 || value == 1, HB_ERR_INVALID_ARGUMENT, "form switch is 0 or 1");
  if (!S.on) return HB_OK;
  if (param == HB_LAUNCH_FFT_PLANE) {
    const int use = (value && plane_supported(S.na, S.nb)) ? 1 : 0;
    if (use && !S.use_plane) HB_TRY(plane_prepare(S.na));
    S.use_plane = use;
    S.n_part = spme_n_part(S);
  } else {
    S.gather_c = value;
  }
  return HB_OK;
}

int spme_setup(hb_forcefield *ff, const hb_forcefield_desc *d) {
  SpmeState &S = ff->spme;
  S.on = 1;
  S.na = (int)d->grid[0];
  S.nb = (int)d->grid[1];
  S.nc = (int)d->grid[2];
  S.nch = S.nc / 2 + 1;
  S.order = (int)d->spline_order;
  S.alpha = (float)d->alpha;
  S.self_pref = (float)(d->alpha / std::sqrt(M_PI));
  FftPlan p;
  for (int ax = 0; ax < 3; ++ax) {
    int n = (int)d->grid[ax];
    if (n < 2 * S.order)
      return hb_fail(HB_ERR_INVALID_GRID, "SPME grid[" + std::string(1, "abc"[ax]) + "] = " +
                                              std::to_string(n) + " is less than 2 * spline_order = " +
                                              std::to_string(2 * S.order));
    if (!make_plan(n, p) || n > 1024)
      return hb_fail(HB_ERR_INVALID_GRID, "SPME grid sizes must factor into 2, 3, 5, 7 and be <= 1024");
  }
  const size_t m = (size_t)S.na * S.nb * S.nc;
  const size_t mc = (size_t)S.na * S.nb * S.nch;
  HB_CUDA(cudaMalloc(&S.d_rho_fixed, sizeof(unsigned long long) * m));
  HB_CUDA(cudaMemset(S.d_rho_fixed, 0, sizeof(unsigned long long) * m));
  HB_CUDA(cudaMalloc(&S.d_grid, sizeof(float2) * mc));
  HB_CUDA(cudaMalloc(&S.d_v, sizeof(float) * m));
  std::vector<float> bf;
  b_factors(S.na, S.order, bf);
  b_factors(S.nb, S.order, bf);
  b_factors(S.nc, S.order, bf);
  HB_CUDA(cudaMalloc(&S.d_bfac, sizeof(float) * bf.size()));
  HB_CUDA(cudaMemcpy(S.d_bfac, bf.data(), sizeof(float) * bf.size(), cudaMemcpyHostToDevice));
  std::vector<float2> tw;
  twiddles(S.na, tw);
  twiddles(S.nb, tw);
  twiddles(S.nc, tw);
  HB_CUDA(cudaMalloc(&S.d_tw, sizeof(float2) * tw.size()));
  HB_CUDA(cudaMemcpy(S.d_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice));
  S.use_plane = plane_supported(S.na, S.nb) ? 1 : 0;
  if (S.use_plane) HB_TRY(plane_prepare(S.na));
  S.n_part = spme_n_part(S);
  // room for the partials of either transform form (HB_LAUNCH_FFT_PLANE)
  const int La = lines_per_cta(S.na);
  const int max_part = std::max(S.nch, S.nb * ((S.nch + La - 1) / La));
  HB_CUDA(cudaMalloc(&S.d_part, sizeof(double) * 2 * max_part));
  HB_CUDA(cudaMalloc(&S.d_sums, sizeof(double) * 2));
  HB_CUDA(cudaMemset(S.d_sums, 0, sizeof(double) * 2));
  HB_CUDA(cudaMalloc(&S.d_recip, sizeof(float4) * std::max(ff->n_pad, 32u)));
  HB_CUDA(cudaMemset(S.d_recip, 0, sizeof(float4) * std::max(ff->n_pad, 32u)));
  return HB_OK;
}

int spme_free(hb_forcefield *ff) {
  SpmeState &S = ff->spme;
  cudaFree(S.d_rho_fixed);
  cudaFree(S.d_grid);
  cudaFree(S.d_v);
  cudaFree(S.d_bfac);
  cudaFree(S.d_tw);
  cudaFree(S.d_part);
  cudaFree(S.d_sums);
  cudaFree(S.d_recip);
  return HB_OK;
}

int spme_launch(hb_forcefield *ff, bool ev, cudaStream_t s) {
  SpmeState &S = ff->spme;
  if (!S.on) return HB_OK;
  hb_system *sys = ff->sys;
  const uint32_t n = sys->n;
  const int na = S.na, nb = S.nb, nc = S.nc;
  if (n > 0) {
    // small blocks (128-thread spread, 64-thread gather): they fit in the SM
    // room the persistent pair kernel leaves, so the chain overlaps it
    const uint64_t th = (uint64_t)n * S.order;
    switch (S.order) {
      case 4: k_spread<4><<<hb_div_up(th, 128), 128, 0, s>>>(ff->d_tile_posq, sys->d_box, na, nb, nc, S.d_rho_fixed, n); break;
      case 5: k_spread<5><<<hb_div_up(th, 128), 128, 0, s>>>(ff->d_tile_posq, sys->d_box, na, nb, nc, S.d_rho_fixed, n); break;
      case 6: k_spread<6><<<hb_div_up(th, 128), 128, 0, s>>>(ff->d_tile_posq, sys->d_box, na, nb, nc, S.d_rho_fixed, n); break;
      case 7: k_spread<7><<<hb_div_up(th, 128), 128, 0, s>>>(ff->d_tile_posq, sys->d_box, na, nb, nc, S.d_rho_fixed, n); break;
      case 8: k_spread<8><<<hb_div_up(th, 128), 128, 0, s>>>(ff->d_tile_posq, sys->d_box, na, nb, nc, S.d_rho_fixed, n); break;
      default: return hb_fail(HB_ERR_INVALID_ARGUMENT, "spline order must be 4..8");
    }
  }
  fft_passes(spme_plan(na, nb, nc), S.d_rho_fixed, S.d_grid, S.d_v, S.d_tw, sys->d_box, S.d_bfac,
             S.alpha, S.d_part, s, S.use_plane != 0, ev);
  if (n > 0) {
    switch (S.order) {
      case 4:
        if (S.gather_c) k_gather_c<4><<<hb_div_up((uint64_t)n * 4u, 128), 128, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n);
        else k_gather<4><<<hb_div_up(n, 64), 64, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n);
        break;
      case 5: k_gather<5><<<hb_div_up(n, 64), 64, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n); break;
      case 6: k_gather<6><<<hb_div_up(n, 64), 64, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n); break;
      case 7: k_gather<7><<<hb_div_up(n, 64), 64, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n); break;
      case 8:
        if (S.gather_c) k_gather_c<8><<<hb_div_up((uint64_t)n * 8u, 128), 128, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n);
        else k_gather<8><<<hb_div_up(n, 64), 64, 0, s>>>(ff->d_tile_posq, S.d_v, sys->d_box, na, nb, nc, S.self_pref, S.d_recip, n);
        break;
    }
  }
  if (ev) k_spme_sums<<<1, 256, 0, s>>>(S.d_part, S.n_part, S.d_sums);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

// ---------------------------------------------------------------------
// Allocation-free SPME reciprocal evaluation (hb_spme_recip_noalloc).
//
// For callers that must not allocate device memory -- a host process whose
// device memory is owned by another allocator (a framework's caching pool,
// a fixed-budget serving process), where cudaMalloc would take memory that
// allocator counts on and cudaMalloc / cudaFree would stall the device --
// this entry point runs the same spread / FFT / convolution / gather
// kernels as the force field on grids of at most HB_NOALLOC_MAX_POINTS
// points, with all scratch in one file-scope device array.  Every GPU that
// loads the library holds that array until the process exits.  The array's
// device address is looked up once per device (primary context) and cached.
// ---------------------------------------------------------------------
#include <mutex>

#define HB_NOALLOC_MAX_DIM 64           // grid points per axis
#define HB_NOALLOC_MAX_POINTS 32768     // grid points in total (e.g. 32^3)
#define HB_NOALLOC_MAX_PART 2048        // energy / virial partial slots

namespace {

// byte offsets of the scratch regions (each 256-byte aligned)
constexpr size_t kNaRho = 0;                                                  // int64 grid
constexpr size_t kNaGrid = kNaRho + 8u * HB_NOALLOC_MAX_POINTS;               // complex grid
constexpr size_t kNaV = kNaGrid + 8u * HB_NOALLOC_MAX_POINTS;                 // real potential
constexpr size_t kNaBfac = kNaV + 4u * HB_NOALLOC_MAX_POINTS;                 // b-factors
constexpr size_t kNaTw = kNaBfac + 4u * 3u * HB_NOALLOC_MAX_DIM + 256u;       // twiddles
constexpr size_t kNaPart = kNaTw + 8u * 3u * HB_NOALLOC_MAX_DIM + 256u;       // partials
constexpr size_t kNaSums = kNaPart + 16u * HB_NOALLOC_MAX_PART;               // E, W
constexpr size_t kNaBox = kNaSums + 256u;                                     // DBox
constexpr size_t kNaBytes = kNaBox + 256u;

// The scratch of hb_spme_recip_noalloc.  In host code this name is only a
// host-side stand-in for the symbol; its device address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[64] = {nullptr};

// host b-factors on the stack (same restatement as b_factors above)
void b_factors_fixed(int n, int p, float *out) {
  double mod[HB_NOALLOC_MAX_DIM];
  for (int k = 0; k < n; ++k) {
    double th = 2.0 * M_PI * k / n, re = 0.0, im = 0.0;
    for (int j = 0; j < p - 1; ++j) {
      double m = bspline_host(p, (double)(j + 1));
      re += m * std::cos(th * j);
      im += m * std::sin(th * j);
    }
    mod[k] = re * re + im * im;
  }
  for (int k = 0; k < n; ++k)
    if (mod[k] < 1.0e-7) mod[k] = 0.5 * (mod[(k + n - 1) % n] + mod[(k + 1) % n]);
  for (int k = 0; k < n; ++k) out[k] = mod[k] > 0.0 ? (float)(1.0 / mod[k]) : 0.0f;
}

}  // namespace

extern "C" int hb_spme_recip_noalloc(const float *posq, uint32_t n, const double box[6],
                                     const uint32_t grid[3], uint32_t order, double alpha,
                                     float *out, double *energy, void *stream) {
  if (!box || !grid || (n > 0 && (!posq || !out)))
    return hb_fail(HB_ERR_INVALID_ARGUMENT, "null argument");
  if (order < 4 || order > 8) return hb_fail(HB_ERR_INVALID_ARGUMENT, "spline order must be 4..8");
  if (!(std::isfinite(alpha) && alpha > 0.0)) return hb_fail(HB_ERR_INVALID_ARGUMENT, "alpha must be > 0");
  for (int d = 0; d < 6; ++d)
    if (!std::isfinite(box[d])) return hb_fail(HB_ERR_NOT_FINITE, "box must be finite");
  if (!(box[0] > 0.0 && box[1] > 0.0 && box[2] > 0.0))
    return hb_fail(HB_ERR_INVALID_ARGUMENT, "box diagonal must be positive");
  const int na = (int)grid[0], nb = (int)grid[1], nc = (int)grid[2];
  FftPlan pa, pb, pc;
  for (int d = 0; d < 3; ++d) {
    const int g = (int)grid[d];
    if (g < 2 * (int)order)
      return hb_fail(HB_ERR_INVALID_GRID, "grid[" + std::to_string(d) + "] = " + std::to_string(g) +
                                              " is less than 2 * spline_order");
    if (g > HB_NOALLOC_MAX_DIM)
      return hb_fail(HB_ERR_INVALID_GRID, "allocation-free SPME supports at most " +
                                              std::to_string(HB_NOALLOC_MAX_DIM) + " points per axis");
  }
  if ((uint64_t)na * nb * nc > HB_NOALLOC_MAX_POINTS)
    return hb_fail(HB_ERR_INVALID_GRID, "allocation-free SPME supports at most " +
                                            std::to_string(HB_NOALLOC_MAX_POINTS) + " grid points");
  if (!make_plan(na, pa) || !make_plan(nb, pb) || !make_plan(nc, pc))
    return hb_fail(HB_ERR_INVALID_GRID, "SPME grid sizes must factor into 2, 3, 5, 7");
  const int nch = nc / 2 + 1;
  const int La = lines_per_cta(na), Lb = lines_per_cta(nb), Lc = lines_per_cta(nc);
  const int n_part = nb * ((nch + La - 1) / La);
  if (n_part > HB_NOALLOC_MAX_PART) return hb_fail(HB_ERR_INVALID_GRID, "grid too large");

  // once per device: the device address of the scratch array
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return hb_fail(HB_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  unsigned char *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return hb_fail(HB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_ptr[dev] = p;
    }
    base = (unsigned char *)g_noalloc_ptr[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long *rho = (unsigned long long *)(base + kNaRho);
  float2 *cgrid = (float2 *)(base + kNaGrid);
  float *v = (float *)(base + kNaV);
  float *bfac = (float *)(base + kNaBfac);
  float2 *tw = (float2 *)(base + kNaTw);
  double *part = (double *)(base + kNaPart);
  double *sums = (double *)(base + kNaSums);
  DBox *dbox = (DBox *)(base + kNaBox);

  // per-call constants (host stack -> scratch); the array keeps the last
  // call's contents, so everything the kernels read is written here
  float h_bfac[3 * HB_NOALLOC_MAX_DIM];
  float2 h_tw[3 * HB_NOALLOC_MAX_DIM];
  b_factors_fixed(na, (int)order, h_bfac);
  b_factors_fixed(nb, (int)order, h_bfac + na);
  b_factors_fixed(nc, (int)order, h_bfac + na + nb);
  int off = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const int g = (int)grid[ax];
    for (int t = 0; t < g; ++t) {
      double a = -2.0 * M_PI * (double)t / (double)g;
      h_tw[off + t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    off += g;
  }
  DBox h_box;
  h_box.lx = (float)box[0];
  h_box.ly = (float)box[1];
  h_box.lz = (float)box[2];
  h_box.xy = (float)box[3];
  h_box.xz = (float)box[4];
  h_box.yz = (float)box[5];
  h_box.ilx = (float)(1.0 / box[0]);
  h_box.ily = (float)(1.0 / box[1]);
  h_box.ilz = (float)(1.0 / box[2]);
  h_box.ortho = (box[3] == 0.0 && box[4] == 0.0 && box[5] == 0.0) ? 1 : 0;
  HB_CUDA(cudaMemcpyAsync(bfac, h_bfac, sizeof(float) * (na + nb + nc), cudaMemcpyHostToDevice, s));
  HB_CUDA(cudaMemcpyAsync(tw, h_tw, sizeof(float2) * (na + nb + nc), cudaMemcpyHostToDevice, s));
  HB_CUDA(cudaMemcpyAsync(dbox, &h_box, sizeof(DBox), cudaMemcpyHostToDevice, s));
  // the charge grid must start at zero
  HB_CUDA(cudaMemsetAsync(rho, 0, sizeof(unsigned long long) * (size_t)na * nb * nc, s));

  const float4 *pq = (const float4 *)posq;
  float4 *o = (float4 *)out;
  const float self_pref = (float)(alpha / std::sqrt(M_PI));
  if (n > 0) {
    const uint64_t th = (uint64_t)n * order;
    switch (order) {
      case 4: k_spread<4><<<hb_div_up(th, 256), 256, 0, s>>>(pq, dbox, na, nb, nc, rho, n); break;
      case 5: k_spread<5><<<hb_div_up(th, 256), 256, 0, s>>>(pq, dbox, na, nb, nc, rho, n); break;
      case 6: k_spread<6><<<hb_div_up(th, 256), 256, 0, s>>>(pq, dbox, na, nb, nc, rho, n); break;
      case 7: k_spread<7><<<hb_div_up(th, 256), 256, 0, s>>>(pq, dbox, na, nb, nc, rho, n); break;
      default: k_spread<8><<<hb_div_up(th, 256), 256, 0, s>>>(pq, dbox, na, nb, nc, rho, n); break;
    }
  }
  fft_passes(spme_plan(na, nb, nc), rho, cgrid, v, tw, dbox, bfac, (float)alpha, part, s, false);
  if (n > 0) {
    switch (order) {
      case 4: k_gather<4><<<hb_div_up(n, 128), 128, 0, s>>>(pq, v, dbox, na, nb, nc, self_pref, o, n); break;
      case 5: k_gather<5><<<hb_div_up(n, 128), 128, 0, s>>>(pq, v, dbox, na, nb, nc, self_pref, o, n); break;
      case 6: k_gather<6><<<hb_div_up(n, 128), 128, 0, s>>>(pq, v, dbox, na, nb, nc, self_pref, o, n); break;
      case 7: k_gather<7><<<hb_div_up(n, 128), 128, 0, s>>>(pq, v, dbox, na, nb, nc, self_pref, o, n); break;
      default: k_gather<8><<<hb_div_up(n, 128), 128, 0, s>>>(pq, v, dbox, na, nb, nc, self_pref, o, n); break;
    }
  }
  k_spme_sums<<<1, 256, 0, s>>>(part, n_part, sums);
  HB_CUDA(cudaGetLastError());
  if (energy) {
    double h_sums[2];
    HB_CUDA(cudaMemcpyAsync(h_sums, sums, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    *energy = h_sums[0];
  }
  return HB_OK;
}
