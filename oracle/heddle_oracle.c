/*
 * heddle_oracle.c -- FP64 CPU restatement of HeddleMD's per-timestep
 * force-and-constraint path (TEST INFRASTRUCTURE: the checker, never the
 * product).  Every function cites the reference file:line it restates;
 * paths are relative to the HeddleMD project root.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 * -ffp-contract=off matters: the f32 neighbour rule below must round after
 * every operation.
 */
#include "heddle_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.14159265358979323846

/* ------------------------------------------------------------------ */
/* periodic boundaries: kernels/pbc.cuh:18-93                          */
/* ------------------------------------------------------------------ */

static inline void cart_to_frac(const or_box *b, double x, double y, double z,
                                double *sa, double *sb, double *sc) {
  /* back-substitution z -> y -> x (kernels/pbc.cuh:18-27) */
  *sc = z / b->lz;
  *sb = (y - *sc * b->yz) / b->ly;
  *sa = (x - *sb * b->xy - *sc * b->xz) / b->lx;
}

void or_min_image(const or_box *b, double *dx, double *dy, double *dz) {
  /* kernels/pbc.cuh:30-43 */
  double sa, sb, sc;
  cart_to_frac(b, *dx, *dy, *dz, &sa, &sb, &sc);
  double ka = floor(sa + 0.5), kb = floor(sb + 0.5), kc = floor(sc + 0.5);
  *dx -= ka * b->lx + kb * b->xy + kc * b->xz;
  *dy -= kb * b->ly + kc * b->yz;
  *dz -= kc * b->lz;
}

void or_wrap_with_image(const or_box *b, double *x, double *y, double *z,
                        int *ka, int *kb, int *kc) {
  /* kernels/pbc.cuh:73-91 */
  double sa, sb, sc;
  cart_to_frac(b, *x, *y, *z, &sa, &sb, &sc);
  double fa = floor(sa + 0.5), fb = floor(sb + 0.5), fc = floor(sc + 0.5);
  *x -= fa * b->lx + fb * b->xy + fc * b->xz;
  *y -= fb * b->ly + fc * b->yz;
  *z -= fc * b->lz;
  *ka = (int)fa;
  *kb = (int)fb;
  *kc = (int)fc;
}

/* perpendicular widths of the lattice (src/pbc.rs perpendicular_widths) */
static void perp_widths(const or_box *b, double w[3]) {
  double a[3] = {b->lx, 0.0, 0.0};
  double bb[3] = {b->xy, b->ly, 0.0};
  double c[3] = {b->xz, b->yz, b->lz};
  double vol = b->lx * b->ly * b->lz;
  double bc[3] = {bb[1] * c[2] - bb[2] * c[1], bb[2] * c[0] - bb[0] * c[2],
                  bb[0] * c[1] - bb[1] * c[0]};
  double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2],
                  c[0] * a[1] - c[1] * a[0]};
  double ab[3] = {a[1] * bb[2] - a[2] * bb[1], a[2] * bb[0] - a[0] * bb[2],
                  a[0] * bb[1] - a[1] * bb[0]};
  w[0] = vol / sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
  w[1] = vol / sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]);
  w[2] = vol / sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
}

/* ------------------------------------------------------------------ */
/* cell list used to enumerate candidate pairs (FP64, with margin)     */
/* ------------------------------------------------------------------ */

typedef struct {
  int nc[3];
  int brute;       /* 1: fewer than 3 cells on some axis -> all pairs */
  int32_t *head;   /* CSR offsets per cell (ncell + 1) */
  int32_t *atoms;  /* atom ids grouped by cell, ascending id within cell */
  int32_t *cell_of;
} or_cells;

static void cells_build(or_cells *cl, int32_t n, const double *pos,
                        const or_box *b, double rcut) {
  double w[3];
  perp_widths(b, w);
  cl->brute = 0;
  for (int d = 0; d < 3; ++d) {
    cl->nc[d] = (int)floor(w[d] / rcut);
    if (cl->nc[d] < 3) cl->brute = 1;
  }
  cl->head = NULL;
  cl->atoms = NULL;
  cl->cell_of = NULL;
  if (cl->brute) return;
  int ncell = cl->nc[0] * cl->nc[1] * cl->nc[2];
  cl->head = (int32_t *)calloc((size_t)ncell + 1, sizeof(int32_t));
  cl->atoms = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  cl->cell_of = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  for (int32_t i = 0; i < n; ++i) {
    double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double sa, sb, sc;
    cart_to_frac(b, x, y, z, &sa, &sb, &sc);
    sa -= floor(sa);
    sb -= floor(sb);
    sc -= floor(sc);
    int ia = (int)(sa * cl->nc[0]), ib = (int)(sb * cl->nc[1]),
        ic = (int)(sc * cl->nc[2]);
    if (ia >= cl->nc[0]) ia = cl->nc[0] - 1;
    if (ib >= cl->nc[1]) ib = cl->nc[1] - 1;
    if (ic >= cl->nc[2]) ic = cl->nc[2] - 1;
    if (ia < 0) ia = 0;
    if (ib < 0) ib = 0;
    if (ic < 0) ic = 0;
    int c = (ia * cl->nc[1] + ib) * cl->nc[2] + ic;
    cl->cell_of[i] = c;
    cl->head[c + 1]++;
  }
  for (int c = 0; c < ncell; ++c) cl->head[c + 1] += cl->head[c];
  int32_t *cur = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncell);
  memcpy(cur, cl->head, sizeof(int32_t) * (size_t)ncell);
  for (int32_t i = 0; i < n; ++i) cl->atoms[cur[cl->cell_of[i]]++] = i;
  free(cur);
}

static void cells_free(or_cells *cl) {
  free(cl->head);
  free(cl->atoms);
  free(cl->cell_of);
}

/* Visit candidate partners j != i of atom i (both orders are visited over
 * all i).  Calls cb for each candidate; order is deterministic. */
#define OR_FOR_CANDIDATES(cl, n, i, J, ...)                                  \
  do {                                                                        \
    if ((cl)->brute) {                                                        \
      for (int32_t J = 0; J < (n); ++J) {                                     \
        if (J == (i)) continue;                                               \
        __VA_ARGS__                                                           \
      }                                                                       \
    } else {                                                                  \
      int c_ = (cl)->cell_of[i];                                              \
      int ic_ = c_ % (cl)->nc[2];                                             \
      int ib_ = (c_ / (cl)->nc[2]) % (cl)->nc[1];                             \
      int ia_ = c_ / ((cl)->nc[2] * (cl)->nc[1]);                             \
      for (int da_ = -1; da_ <= 1; ++da_)                                     \
        for (int db_ = -1; db_ <= 1; ++db_)                                   \
          for (int dc_ = -1; dc_ <= 1; ++dc_) {                               \
            int a_ = (ia_ + da_ + (cl)->nc[0]) % (cl)->nc[0];                 \
            int b_ = (ib_ + db_ + (cl)->nc[1]) % (cl)->nc[1];                 \
            int cc_ = (ic_ + dc_ + (cl)->nc[2]) % (cl)->nc[2];                \
            int nb_ = (a_ * (cl)->nc[1] + b_) * (cl)->nc[2] + cc_;            \
            for (int32_t k_ = (cl)->head[nb_]; k_ < (cl)->head[nb_ + 1];      \
                 ++k_) {                                                      \
              int32_t J = (cl)->atoms[k_];                                    \
              if (J == (i)) continue;                                         \
              __VA_ARGS__                                                     \
            }                                                                 \
          }                                                                   \
    }                                                                         \
  } while (0)

/* ------------------------------------------------------------------ */
/* neighbour set, f32 rule (kernels/neighbor.cu:509-529 membership)    */
/* ------------------------------------------------------------------ */

static inline float f32_min_image_r2(float dx, float dy, float dz,
                                     const float *b) {
  /* same operation order as kernels/pbc.cuh:18-43 evaluated in float with
   * one rounding per operation (no FMA: compiled -ffp-contract=off) */
  float sc = dz / b[2];
  float sb = (dy - sc * b[5]) / b[1];
  float sa = (dx - sb * b[3] - sc * b[4]) / b[0];
  float ka = floorf(sa + 0.5f);
  float kb = floorf(sb + 0.5f);
  float kc = floorf(sc + 0.5f);
  dx -= ka * b[0] + kb * b[3] + kc * b[4];
  dy -= kb * b[1] + kc * b[5];
  dz -= kc * b[2];
  return dx * dx + dy * dy + dz * dz;
}

static int cmp_pair(const void *a, const void *b) {
  const uint32_t *x = (const uint32_t *)a, *y = (const uint32_t *)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
  return 0;
}

/* f32 squared minimum-image distance of given pairs (i, j) by the rule
 * above, for checking another list's pairs against the exact cut. */
void or_pair_r2_f32(int64_t n_pairs, const uint32_t *pairs, const float *xyz,
                    const float *box6, float *out_r2) {
  for (int64_t k = 0; k < n_pairs; ++k) {
    uint32_t i = pairs[2 * k], j = pairs[2 * k + 1];
    float dx = xyz[3 * i] - xyz[3 * j];
    float dy = xyz[3 * i + 1] - xyz[3 * j + 1];
    float dz = xyz[3 * i + 2] - xyz[3 * j + 2];
    out_r2[k] = f32_min_image_r2(dx, dy, dz, box6);
  }
}

int64_t or_neighbor_pairs_f32(int32_t n, const float *xyz, const float *box6,
                              float r_search, uint32_t *out_pairs,
                              int64_t cap) {
  or_box b = {box6[0], box6[1], box6[2], box6[3], box6[4], box6[5]};
  double *pos = (double *)calloc(3 * (size_t)(n > 0 ? n : 1), sizeof(double));
  for (int64_t k = 0; k < 3 * (int64_t)n; ++k) pos[k] = (double)xyz[k];
  or_cells cl;
  /* f64 candidate radius with a margin so the f32 test decides alone */
  cells_build(&cl, n, pos, &b, (double)r_search * (1.0 + 1e-4) + 1e-6);
  float rs2 = r_search * r_search;
  int64_t cnt = 0, capn = 1024;
  uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)capn);
  for (int32_t i = 0; i < n; ++i) {
    OR_FOR_CANDIDATES(&cl, n, i, j, {
      if (j > i) {
        float dx = xyz[3 * i] - xyz[3 * j];
        float dy = xyz[3 * i + 1] - xyz[3 * j + 1];
        float dz = xyz[3 * i + 2] - xyz[3 * j + 2];
        float r2 = f32_min_image_r2(dx, dy, dz, box6);
        if (r2 <= rs2) {
          if (cnt == capn) {
            capn *= 2;
            buf = (uint32_t *)realloc(buf, sizeof(uint32_t) * 2 * (size_t)capn);
          }
          buf[2 * cnt] = (uint32_t)i;
          buf[2 * cnt + 1] = (uint32_t)j;
          cnt++;
        }
      }
    });
  }
  qsort(buf, (size_t)cnt, 2 * sizeof(uint32_t), cmp_pair);
  /* remove duplicates that a brute-force small box cannot create but a
   * 3-cell periodic stencil could (same neighbour cell reached twice) */
  int64_t w = 0;
  for (int64_t k = 0; k < cnt; ++k) {
    if (w > 0 && buf[2 * (w - 1)] == buf[2 * k] &&
        buf[2 * (w - 1) + 1] == buf[2 * k + 1])
      continue;
    buf[2 * w] = buf[2 * k];
    buf[2 * w + 1] = buf[2 * k + 1];
    w++;
  }
  int64_t ncopy = w < cap ? w : cap;
  if (out_pairs && ncopy > 0)
    memcpy(out_pairs, buf, sizeof(uint32_t) * 2 * (size_t)ncopy);
  free(buf);
  cells_free(&cl);
  free(pos);
  return w;
}

/* ------------------------------------------------------------------ */
/* pair terms                                                          */
/* ------------------------------------------------------------------ */

static double excl_scale(const or_ff *ff, int32_t i, int32_t j,
                         int coulomb) {
  /* per-pair scale lookup, jit_composed.rs:1448-1460 */
  if (!ff->excl_off) return 1.0;
  for (int32_t m = ff->excl_off[i]; m < ff->excl_off[i + 1]; ++m) {
    if (ff->excl_partner[m] == j)
      return coulomb ? ff->excl_coul_scale[m] : ff->excl_lj_scale[m];
  }
  return 1.0;
}

/* LJ with optional CHARMM-style switch: src/forces/lj.rs:261-283 */
static void lj_pair(double r2, double sigma, double eps, double cut,
                    double rsw, double *factor, double *energy) {
  double inv_r2 = 1.0 / r2;
  double s2 = sigma * sigma * inv_r2;
  double s6 = s2 * s2 * s2;
  double s12 = s6 * s6;
  double f = 24.0 * eps * inv_r2 * (2.0 * s12 - s6);
  double e = 4.0 * eps * (s12 - s6);
  double rs2 = rsw * rsw, rc2 = cut * cut;
  double delta = rc2 - rs2;
  if (delta > 0.0 && r2 > rs2) {
    double tau = (r2 - rs2) / delta;
    double omt = 1.0 - tau;
    double s = omt * omt * (1.0 + 2.0 * tau);
    double chain = 12.0 * tau * omt / delta;
    f = s * f + chain * e;
    e = s * e;
  }
  *factor = f;
  *energy = e;
}

/* Abramowitz & Stegun 7.1.26 (the f32 form of src/forces/spme.rs:742-751) */
static double erfc_as(double x) {
  double t = 1.0 / (1.0 + 0.3275911 * x);
  double poly = 0.254829592 +
                (-0.284496736 +
                 (1.421413741 + (-1.453152027 + 1.061405429 * t) * t) * t) *
                    t;
  return poly * t * exp(-x * x);
}

/* erfc-screened Coulomb: src/forces/spme.rs:730-759 */
static void coul_pair(double r2, double qq, double alpha, int poly,
                      double *factor, double *energy) {
  double r = sqrt(r2);
  double ar = alpha * r;
  double g = exp(-ar * ar);
  double ec = poly ? erfc_as(ar) : erfc(ar);
  *energy = qq * ec / r;
  *factor = qq / r2 * (ec / r + 2.0 * alpha / sqrt(OR_PI) * g);
}

/* ------------------------------------------------------------------ */
/* FFT (mixed radix, recursive; used by the SPME restatement)          */
/* ------------------------------------------------------------------ */

static int smallest_factor(int n) {
  if (n % 4 == 0) return 4;
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

static void fft_rec(int n, const double complex *in, int istride,
                    double complex *out, const double complex *tw,
                    int twstride, int ntop) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = smallest_factor(n);
  int m = n / p;
  for (int r = 0; r < p; ++r)
    fft_rec(m, in + (size_t)r * istride, istride * p, out + (size_t)r * m, tw,
            twstride * p, ntop);
  double complex t[64];
  double complex *tt = p <= 64 ? t : (double complex *)malloc(sizeof(double complex) * p);
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < p; ++r) tt[r] = out[(size_t)r * m + k];
    for (int q = 0; q < p; ++q) {
      double complex s = 0.0;
      int kk = k + q * m;
      for (int r = 0; r < p; ++r) {
        long e = ((long)r * kk) % n;
        s += tt[r] * tw[(size_t)e * twstride];
      }
      out[kk] = s;
    }
  }
  if (tt != t) free(tt);
  (void)ntop;
}

/* in-place 1-D transform of x[0..n), sign -1 forward, +1 inverse, no
 * normalisation (the cuFFT R2C / C2R convention of src/gpu/cufft.rs) */
static void fft1d(int n, double complex *x, int sign, double complex *scratch,
                  const double complex *tw) {
  fft_rec(n, x, 1, scratch, tw, 1, n);
  memcpy(x, scratch, sizeof(double complex) * (size_t)n);
  (void)sign;
}

static double complex *twiddles(int n, int sign) {
  double complex *tw = (double complex *)malloc(sizeof(double complex) * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double a = 2.0 * OR_PI * (double)k / (double)n;
    tw[k] = cos(a) + I * (sign * sin(a));
  }
  return tw;
}

/* 3-D transform of a full complex grid [na][nb][nc] along every axis */
static void fft3d(double complex *g, const int grid[3], int sign) {
  int na = grid[0], nb = grid[1], nc = grid[2];
  double complex *twa = twiddles(na, sign), *twb = twiddles(nb, sign),
                 *twc = twiddles(nc, sign);
  int nmax = na > nb ? (na > nc ? na : nc) : (nb > nc ? nb : nc);
  /* axis c (contiguous) */
#pragma omp parallel
  {
    double complex *line = (double complex *)malloc(sizeof(double complex) * (size_t)nmax);
    double complex *scr = (double complex *)malloc(sizeof(double complex) * (size_t)nmax);
#pragma omp for schedule(static)
    for (int ab = 0; ab < na * nb; ++ab) {
      double complex *p = g + (size_t)ab * nc;
      memcpy(line, p, sizeof(double complex) * (size_t)nc);
      fft1d(nc, line, sign, scr, twc);
      memcpy(p, line, sizeof(double complex) * (size_t)nc);
    }
#pragma omp for schedule(static)
    for (int ac = 0; ac < na * nc; ++ac) {
      int a = ac / nc, c = ac % nc;
      for (int bq = 0; bq < nb; ++bq) line[bq] = g[((size_t)a * nb + bq) * nc + c];
      fft1d(nb, line, sign, scr, twb);
      for (int bq = 0; bq < nb; ++bq) g[((size_t)a * nb + bq) * nc + c] = line[bq];
    }
#pragma omp for schedule(static)
    for (int bc = 0; bc < nb * nc; ++bc) {
      int bq = bc / nc, c = bc % nc;
      for (int a = 0; a < na; ++a) line[a] = g[((size_t)a * nb + bq) * nc + c];
      fft1d(na, line, sign, scr, twa);
      for (int a = 0; a < na; ++a) g[((size_t)a * nb + bq) * nc + c] = line[a];
    }
    free(line);
    free(scr);
  }
  free(twa);
  free(twb);
  free(twc);
}

/* ------------------------------------------------------------------ */
/* SPME: kernels/spme_spread_gather.cuh:36-334, kernels/spme_recip.cu   */
/* ------------------------------------------------------------------ */

/* Cardinal B-spline M_p(x) by the Cox-de Boor recursion
 * (kernels/spme_spread_gather.cuh:36-53, src/forces/spme.rs:588-609). */
static double bspline_m(int p, double x) {
  double v[16];
  for (int i = 0; i < p; ++i) {
    double xi = x - i;
    v[i] = (xi >= 0.0 && xi < 1.0) ? 1.0 : 0.0;
  }
  for (int k = 2; k <= p; ++k) {
    for (int i = 0; i <= p - k; ++i) {
      double xi = x - i;
      v[i] = (xi * v[i] + ((double)k - xi) * v[i + 1]) / (double)(k - 1);
    }
  }
  return v[0];
}

/* weights w[d] = M_p(d + t) and derivatives dw[d] = M_{p-1}(d+t) -
 * M_{p-1}(d+t-1), d = 0..p-1 (spme_spread_gather.cuh:58-86) */
void or_bspline_weights(int order, double t, double *w, double *dw) {
  for (int d = 0; d < order; ++d) {
    double x = (double)d + t;
    w[d] = bspline_m(order, x);
    if (dw) dw[d] = bspline_m(order - 1, x) - bspline_m(order - 1, x - 1.0);
  }
}

/* |b(k)|^2 with Essmann near-zero averaging: src/forces/spme.rs:524-585 */
void or_b_factors(int n, int order, double *out) {
  double *mod = (double *)malloc(sizeof(double) * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double th = 2.0 * OR_PI * (double)k / (double)n;
    double re = 0.0, im = 0.0;
    for (int j = 0; j < order - 1; ++j) {
      double m = bspline_m(order, (double)(j + 1));
      re += m * cos(th * j);
      im += m * sin(th * j);
    }
    mod[k] = re * re + im * im;
  }
  for (int k = 0; k < n; ++k) {
    if (mod[k] < 1.0e-7) mod[k] = 0.5 * (mod[(k + n - 1) % n] + mod[(k + 1) % n]);
  }
  for (int k = 0; k < n; ++k) out[k] = mod[k] > 0.0 ? 1.0 / mod[k] : 0.0;
  free(mod);
}

/* per-atom grid setup (spme_spread_gather.cuh:90-126) */
static void spme_setup(const or_box *b, const int grid[3], double x, double y,
                       double z, double t[3], int g0[3]) {
  int ka, kb, kc;
  or_wrap_with_image(b, &x, &y, &z, &ka, &kb, &kc);
  double s[3];
  cart_to_frac(b, x, y, z, &s[0], &s[1], &s[2]);
  for (int d = 0; d < 3; ++d) {
    double u = (s[d] + 0.5) * grid[d];
    double f = floor(u);
    t[d] = u - f;
    long fl = (long)f;
    g0[d] = (int)(((fl % grid[d]) + grid[d]) % grid[d]);
  }
}

void or_spme_spread(int32_t n, const double *pos, const double *q,
                    const or_box *b, const int grid[3], int order,
                    double *rho) {
  size_t m = (size_t)grid[0] * grid[1] * grid[2];
  memset(rho, 0, sizeof(double) * m);
  for (int32_t i = 0; i < n; ++i) {
    if (q[i] == 0.0) continue;
    double t[3];
    int g0[3];
    spme_setup(b, grid, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], t, g0);
    double wa[16], wb[16], wc[16];
    or_bspline_weights(order, t[0], wa, NULL);
    or_bspline_weights(order, t[1], wb, NULL);
    or_bspline_weights(order, t[2], wc, NULL);
    for (int da = 0; da < order; ++da) {
      int ga = (g0[0] - da + grid[0]) % grid[0];
      for (int db = 0; db < order; ++db) {
        int gb = (g0[1] - db + grid[1]) % grid[1];
        for (int dc = 0; dc < order; ++dc) {
          int gc = (g0[2] - dc + grid[2]) % grid[2];
          rho[((size_t)ga * grid[1] + gb) * grid[2] + gc] +=
              q[i] * wa[da] * wb[db] * wc[dc];
        }
      }
    }
  }
}

/* rows of H^{-T} (spme_spread_gather.cuh:128-148) */
static void recip_rows(const or_box *b, double ba[3], double bb[3],
                       double bc[3]) {
  double ilx = 1.0 / b->lx, ily = 1.0 / b->ly, ilz = 1.0 / b->lz;
  ba[0] = ilx;
  ba[1] = -b->xy * ilx * ily;
  ba[2] = (b->xy * b->yz - b->xz * b->ly) * ilx * ily * ilz;
  bb[0] = 0.0;
  bb[1] = ily;
  bb[2] = -b->yz * ily * ilz;
  bc[0] = 0.0;
  bc[1] = 0.0;
  bc[2] = ilz;
}

/* Reciprocal part: E_recip, W_recip, per-atom force / energy / virial
 * shares.  Influence function kernels/spme_recip.cu:34-114; multiply and
 * virial :296-342; gather spme_spread_gather.cuh:227-334. */
static void spme_recip(int32_t n, const double *pos, const double *q,
                       const or_box *b, const or_ff *ff, double *F, double *E,
                       double *W, double *terms) {
  const int *grid = ff->grid;
  int p = ff->order;
  size_t m = (size_t)grid[0] * grid[1] * grid[2];
  double *rho = (double *)malloc(sizeof(double) * m);
  or_spme_spread(n, pos, q, b, grid, p, rho);
  double complex *g = (double complex *)malloc(sizeof(double complex) * m);
  for (size_t k = 0; k < m; ++k) g[k] = rho[k];
  fft3d(g, grid, -1);
  double *bfa = (double *)malloc(sizeof(double) * grid[0]);
  double *bfb = (double *)malloc(sizeof(double) * grid[1]);
  double *bfc = (double *)malloc(sizeof(double) * grid[2]);
  or_b_factors(grid[0], p, bfa);
  or_b_factors(grid[1], p, bfb);
  or_b_factors(grid[2], p, bfc);
  double ba[3], bb[3], bc[3];
  recip_rows(b, ba, bb, bc);
  double vol = b->lx * b->ly * b->lz;
  double alpha = ff->alpha;
  double e_sum = 0.0, w_sum = 0.0;
#pragma omp parallel for reduction(+ : e_sum, w_sum) schedule(static)
  for (int ka = 0; ka < grid[0]; ++ka) {
    double ma = ka <= grid[0] / 2 ? ka : ka - grid[0];
    for (int kb = 0; kb < grid[1]; ++kb) {
      double mb = kb <= grid[1] / 2 ? kb : kb - grid[1];
      for (int kc = 0; kc < grid[2]; ++kc) {
        double mc = kc <= grid[2] / 2 ? kc : kc - grid[2];
        size_t idx = ((size_t)ka * grid[1] + kb) * grid[2] + kc;
        double kx = 2.0 * OR_PI * (ma * ba[0] + mb * bb[0] + mc * bc[0]);
        double ky = 2.0 * OR_PI * (ma * ba[1] + mb * bb[1] + mc * bc[1]);
        double kz = 2.0 * OR_PI * (ma * ba[2] + mb * bb[2] + mc * bc[2]);
        double k2 = kx * kx + ky * ky + kz * kz;
        double G = 0.0, vf = 0.0;
        if (k2 != 0.0) {
          G = (1.0 / vol) * (4.0 * OR_PI / k2) * exp(-k2 / (4.0 * alpha * alpha)) *
              bfa[ka] * bfb[kb] * bfc[kc];
          vf = G * (1.0 - k2 / (2.0 * alpha * alpha));
        }
        double r2 = creal(g[idx]) * creal(g[idx]) + cimag(g[idx]) * cimag(g[idx]);
        e_sum += G * r2;
        w_sum += vf * r2;
        g[idx] *= G;
      }
    }
  }
  fft3d(g, grid, +1);
  double e_recip = 0.5 * e_sum, w_recip = 0.5 * w_sum;
  double self_pref = alpha / sqrt(OR_PI);
  double e_self = 0.0;
  for (int32_t i = 0; i < n; ++i) e_self += self_pref * q[i] * q[i];
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i) {
    double t[3];
    int g0[3];
    spme_setup(b, grid, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], t, g0);
    double wa[16], wb[16], wc[16], dwa[16], dwb[16], dwc[16];
    or_bspline_weights(p, t[0], wa, dwa);
    or_bspline_weights(p, t[1], wb, dwb);
    or_bspline_weights(p, t[2], wc, dwc);
    double phi = 0.0, ga = 0.0, gb = 0.0, gc = 0.0;
    for (int da = 0; da < p; ++da) {
      int ia = (g0[0] - da + grid[0]) % grid[0];
      for (int db = 0; db < p; ++db) {
        int ib = (g0[1] - db + grid[1]) % grid[1];
        for (int dc = 0; dc < p; ++dc) {
          int ic = (g0[2] - dc + grid[2]) % grid[2];
          double v = creal(g[((size_t)ia * grid[1] + ib) * grid[2] + ic]);
          phi += v * wa[da] * wb[db] * wc[dc];
          ga += v * dwa[da] * wb[db] * wc[dc];
          gb += v * wa[da] * dwb[db] * wc[dc];
          gc += v * wa[da] * wb[db] * dwc[dc];
        }
      }
    }
    ga *= grid[0];
    gb *= grid[1];
    gc *= grid[2];
    F[3 * i + 0] += -q[i] * (ga * ba[0] + gb * bb[0] + gc * bc[0]);
    F[3 * i + 1] += -q[i] * (ga * ba[1] + gb * bb[1] + gc * bc[1]);
    F[3 * i + 2] += -q[i] * (ga * ba[2] + gb * bb[2] + gc * bc[2]);
    E[i] += 0.5 * q[i] * phi - self_pref * q[i] * q[i];
    W[i] += n > 0 ? w_recip / (double)n : 0.0;
  }
  terms[OR_E_RECIP] += e_recip;
  terms[OR_E_SELF] += e_self;
  terms[OR_W_RECIP] += w_recip;
  free(rho);
  free(g);
  free(bfa);
  free(bfb);
  free(bfc);
}

double or_ewald_recip_energy(int32_t n, const double *pos, const double *q,
                             const or_box *b, double alpha, int m_max) {
  /* tests/spme_pipeline.rs:46-83 (orthorhombic) */
  double vol = b->lx * b->ly * b->lz;
  double total = 0.0;
  for (int ma = -m_max; ma <= m_max; ++ma)
    for (int mb = -m_max; mb <= m_max; ++mb)
      for (int mc = -m_max; mc <= m_max; ++mc) {
        if (ma == 0 && mb == 0 && mc == 0) continue;
        double kx = 2.0 * OR_PI * ma / b->lx, ky = 2.0 * OR_PI * mb / b->ly,
               kz = 2.0 * OR_PI * mc / b->lz;
        double k2 = kx * kx + ky * ky + kz * kz;
        double re = 0.0, im = 0.0;
        for (int32_t i = 0; i < n; ++i) {
          double ph = kx * pos[3 * i] + ky * pos[3 * i + 1] + kz * pos[3 * i + 2];
          re += q[i] * cos(ph);
          im -= q[i] * sin(ph);
        }
        total += (4.0 * OR_PI / k2) * exp(-k2 / (4.0 * alpha * alpha)) *
                 (re * re + im * im);
      }
  return total / (2.0 * vol);
}

/* ------------------------------------------------------------------ */
/* total force field                                                   */
/* ------------------------------------------------------------------ */

/* ---- bonded terms in FP64 (src/forces/harmonic_bond.rs:283-307,
 * src/forces/angle.rs:260-313, src/forces/dihedral.rs:383-467); per-atom
 * energy / virial shares split equally over each term's atoms ---- */
static void mi_disp(const double *pos, int a, int b, const or_box *box, double d[3]) {
  d[0] = pos[3 * a] - pos[3 * b];
  d[1] = pos[3 * a + 1] - pos[3 * b + 1];
  d[2] = pos[3 * a + 2] - pos[3 * b + 2];
  or_min_image(box, &d[0], &d[1], &d[2]);
}
static double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static void cross3(const double *a, const double *b, double *o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

static void bonded_terms(const double *pos, const or_box *box, const or_ff *ff, double *F,
                         double *E, double *W, double *terms) {
  double e_b = 0.0, w_b = 0.0;
  for (int32_t q = 0; q < ff->n_bonds; ++q) {
    const int i = ff->bond_atoms[2 * q], j = ff->bond_atoms[2 * q + 1];
    double d[3];
    mi_disp(pos, i, j, box, d);
    const double r2 = dot3(d, d), r = sqrt(r2);
    if (r < 1e-7) continue;
    const double dr = r - ff->bond_r0[q];
    const double fmag = -ff->bond_k[q] * dr / r;
    const double u = 0.5 * ff->bond_k[q] * dr * dr, w = fmag * r2;
    for (int x = 0; x < 3; ++x) {
      F[3 * i + x] += fmag * d[x];
      F[3 * j + x] -= fmag * d[x];
    }
    E[i] += 0.5 * u; E[j] += 0.5 * u;
    W[i] += 0.5 * w; W[j] += 0.5 * w;
    e_b += u;
    w_b += w;
  }
  for (int32_t q = 0; q < ff->n_angles; ++q) {
    const int i = ff->angle_atoms[3 * q], j = ff->angle_atoms[3 * q + 1],
              k = ff->angle_atoms[3 * q + 2];
    double a[3], c[3];
    mi_disp(pos, i, j, box, a);
    mi_disp(pos, k, j, box, c);
    const double a2 = dot3(a, a), c2 = dot3(c, c);
    if (a2 == 0.0 || c2 == 0.0) continue;
    const double la = sqrt(a2), lc = sqrt(c2), dt = dot3(a, c);
    double cs = dt / (la * lc);
    if (cs > 1.0) cs = 1.0;
    if (cs < -1.0) cs = -1.0;
    const double sn = sqrt(fmax(1.0 - cs * cs, 0.0));
    if (sn < 1e-7) continue;
    const double th = atan2(la * lc * sn, dt), dth = th - ff->angle_theta0[q];
    const double g = -ff->angle_k[q] * dth / sn;
    double fi[3], fk[3];
    for (int x = 0; x < 3; ++x) {
      fi[x] = g * (cs / a2 * a[x] - c[x] / (la * lc));
      fk[x] = g * (cs / c2 * c[x] - a[x] / (la * lc));
      F[3 * i + x] += fi[x];
      F[3 * k + x] += fk[x];
      F[3 * j + x] -= fi[x] + fk[x];
    }
    const double u = 0.5 * ff->angle_k[q] * dth * dth, w = dot3(a, fi) + dot3(c, fk);
    E[i] += u / 3; E[j] += u / 3; E[k] += u / 3;
    W[i] += w / 3; W[j] += w / 3; W[k] += w / 3;
    e_b += u;
    w_b += w;
  }
  for (int32_t q = 0; q < ff->n_dihedrals; ++q) {
    const int *at = ff->dihedral_atoms + 4 * q;
    double b1[3], b2[3], b3[3], m[3], nn[3];
    mi_disp(pos, at[0], at[1], box, b1);
    mi_disp(pos, at[2], at[1], box, b2);
    mi_disp(pos, at[2], at[3], box, b3);
    cross3(b1, b2, m);
    cross3(b2, b3, nn);
    const double m2 = dot3(m, m), n2 = dot3(nn, nn), b22 = dot3(b2, b2);
    if (m2 < 1e-14 || n2 < 1e-14 || b22 < 1e-14) continue;
    const double lb2 = sqrt(b22);
    const double phi = atan2(lb2 * dot3(b1, nn), dot3(m, nn));
    const double mult = (double)ff->dihedral_n[q];
    const double del = mult * phi - ff->dihedral_phi0[q];
    const double fphi = ff->dihedral_k[q] * mult * sin(del);
    const double ci = fphi * lb2 / m2, cl = -fphi * lb2 / n2;
    const double s = dot3(b1, b2) / b22, t = dot3(b3, b2) / b22;
    double fi[3], fj[3], fk[3], fl[3], bl[3];
    for (int x = 0; x < 3; ++x) {
      fi[x] = ci * m[x];
      fl[x] = cl * nn[x];
      fj[x] = (s - 1.0) * fi[x] - t * fl[x];
      fk[x] = -s * fi[x] + (t - 1.0) * fl[x];
      bl[x] = b2[x] - b3[x];
      F[3 * at[0] + x] += fi[x];
      F[3 * at[1] + x] += fj[x];
      F[3 * at[2] + x] += fk[x];
      F[3 * at[3] + x] += fl[x];
    }
    const double u = ff->dihedral_k[q] * (1.0 + cos(del));
    const double w = dot3(b1, fi) + dot3(b2, fk) + dot3(bl, fl);
    for (int a = 0; a < 4; ++a) {
      E[at[a]] += 0.25 * u;
      W[at[a]] += 0.25 * w;
    }
    e_b += u;
    w_b += w;
  }
  terms[OR_E_BONDED] = e_b;
  terms[OR_W_PAIR] += w_b;
}

int or_forces(int32_t n, const double *pos, const double *q,
              const int32_t *type, const or_box *box, const or_ff *ff,
              double *F, double *E, double *W, double *terms, int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
  for (int k = 0; k < OR_N_TERMS; ++k) terms[k] = 0.0;
  memset(F, 0, sizeof(double) * 3 * (size_t)n);
  memset(E, 0, sizeof(double) * (size_t)n);
  memset(W, 0, sizeof(double) * (size_t)n);
  double rmax = 0.0;
  if (ff->lj_on) {
    for (int k = 0; k < ff->n_types * ff->n_types; ++k)
      if (ff->lj_cutoff[k] > rmax) rmax = ff->lj_cutoff[k];
  }
  if (ff->coul_on && ff->r_cut_coul > rmax) rmax = ff->r_cut_coul;
  if (ff->recip_on) {
    for (int d = 0; d < 3; ++d)
      if (ff->grid[d] < 2 * ff->order) return -2; /* src/forces/spme.rs:238-251 */
  }
  double e_lj = 0.0, e_c = 0.0, w_p = 0.0, near = 0.0;
  if (rmax > 0.0 && n > 1) {
    or_cells cl;
    cells_build(&cl, n, pos, box, rmax * (1.0 + 1e-9));
#pragma omp parallel for reduction(+ : e_lj, e_c, w_p, near) schedule(dynamic, 64)
    for (int32_t i = 0; i < n; ++i) {
      double fx = 0, fy = 0, fz = 0, ei = 0, wi = 0;
      OR_FOR_CANDIDATES(&cl, n, i, j, {
        double dx = pos[3 * i] - pos[3 * j];
        double dy = pos[3 * i + 1] - pos[3 * j + 1];
        double dz = pos[3 * i + 2] - pos[3 * j + 2];
        or_min_image(box, &dx, &dy, &dz);
        double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= rmax * rmax && r2 > 0.0) {
          double fac = 0.0, en = 0.0;
          if (ff->lj_on) {
            int p = type[i] * ff->n_types + type[j];
            double cut = ff->lj_cutoff[p];
            if (fabs(sqrt(r2) - cut) < 1e-6 * cut) near += 0.5;
            if (r2 <= cut * cut && ff->lj_epsilon[p] != 0.0) {
              double s = excl_scale(ff, i, j, 0);
              if (s != 0.0) {
                double f1, e1;
                lj_pair(r2, ff->lj_sigma[p], ff->lj_epsilon[p], cut,
                        ff->lj_switch[p], &f1, &e1);
                fac += s * f1;
                en += s * e1;
                e_lj += 0.5 * s * e1;
              }
            }
          }
          if (ff->coul_on && q[i] != 0.0 && q[j] != 0.0) {
            double cut = ff->r_cut_coul;
            if (fabs(sqrt(r2) - cut) < 1e-6 * cut) near += 0.5;
            if (r2 <= cut * cut) {
              double s = excl_scale(ff, i, j, 1);
              if (s != 0.0) {
                double f1, e1;
                coul_pair(r2, q[i] * q[j], ff->alpha, ff->coul_poly_erfc, &f1,
                          &e1);
                fac += s * f1;
                en += s * e1;
                e_c += 0.5 * s * e1;
              }
            }
          }
          fx += fac * dx;
          fy += fac * dy;
          fz += fac * dz;
          ei += 0.5 * en;
          wi += 0.5 * fac * r2;
        }
      });
      F[3 * i] = fx;
      F[3 * i + 1] = fy;
      F[3 * i + 2] = fz;
      E[i] = ei;
      W[i] = wi;
      w_p += wi;
    }
    cells_free(&cl);
  }
  terms[OR_E_LJ] = e_lj;
  terms[OR_E_COUL_REAL] = e_c;
  terms[OR_W_PAIR] = w_p;
  terms[OR_N_PAIRS_NEAR_CUT] = near;
  bonded_terms(pos, box, ff, F, E, W, terms);
  if (ff->recip_on && n > 0) spme_recip(n, pos, q, box, ff, F, E, W, terms);
  return 0;
}

/* ------------------------------------------------------------------ */
/* constraints: kernels/settle.cu:145-510, kernels/shake.cu:108-556     */
/* ------------------------------------------------------------------ */

int or_constrain_positions(int32_t n_groups, const int32_t *group_off,
                           const int32_t *group_atoms, const int32_t *con_off,
                           const int32_t *con_i, const int32_t *con_j,
                           const double *con_d2, const double *mass,
                           const or_box *box, const double *ref_pos,
                           double *pos, double *vel, double dt,
                           double *vir_slot, double tol, int max_iter) {
  int worst = 0;
  for (int32_t g = 0; g < n_groups; ++g) {
    int a0 = group_off[g], na = group_off[g + 1] - a0;
    double x0[16][3], xu[16][3], xc[16][3], im[16], mm[16];
    for (int a = 0; a < na; ++a) {
      int id = group_atoms[a0 + a];
      mm[a] = mass[id];
      im[a] = mass[id] > 0.0 ? 1.0 / mass[id] : 0.0;
      for (int d = 0; d < 3; ++d) {
        x0[a][d] = ref_pos[3 * id + d];
        xu[a][d] = pos[3 * id + d];
      }
      if (a > 0) {
        /* bring every atom into atom 0's image (kernels/shake.cu:222-227) */
        double dx = x0[a][0] - x0[0][0], dy = x0[a][1] - x0[0][1],
               dz = x0[a][2] - x0[0][2];
        or_min_image(box, &dx, &dy, &dz);
        x0[a][0] = x0[0][0] + dx;
        x0[a][1] = x0[0][1] + dy;
        x0[a][2] = x0[0][2] + dz;
        dx = xu[a][0] - xu[0][0];
        dy = xu[a][1] - xu[0][1];
        dz = xu[a][2] - xu[0][2];
        or_min_image(box, &dx, &dy, &dz);
        xu[a][0] = xu[0][0] + dx;
        xu[a][1] = xu[0][1] + dy;
        xu[a][2] = xu[0][2] + dz;
      }
      for (int d = 0; d < 3; ++d) xc[a][d] = xu[a][d];
    }
    int c0 = con_off[g], nc = con_off[g + 1] - c0;
    double gdir[32][3];
    for (int k = 0; k < nc; ++k) {
      int li = con_i[c0 + k], lj = con_j[c0 + k];
      for (int d = 0; d < 3; ++d) gdir[k][d] = x0[li][d] - x0[lj][d];
    }
    int it, used = -1;
    for (it = 0; it < max_iter; ++it) {
      int conv = 1;
      for (int k = 0; k < nc; ++k) {
        int li = con_i[c0 + k], lj = con_j[c0 + k];
        double dx = xc[li][0] - xc[lj][0], dy = xc[li][1] - xc[lj][1],
               dz = xc[li][2] - xc[lj][2];
        double sigma = dx * dx + dy * dy + dz * dz - con_d2[c0 + k];
        if (fabs(sigma) > tol * con_d2[c0 + k]) {
          conv = 0;
          double ddot = dx * gdir[k][0] + dy * gdir[k][1] + dz * gdir[k][2];
          double denom = 2.0 * ddot * (im[li] + im[lj]);
          if (denom == 0.0) continue;
          double lam = sigma / denom;
          for (int d = 0; d < 3; ++d) {
            xc[li][d] -= lam * im[li] * gdir[k][d];
            xc[lj][d] += lam * im[lj] * gdir[k][d];
          }
        }
      }
      if (conv) {
        used = it;
        break;
      }
    }
    if (used < 0) worst = -1;
    else if (worst >= 0 && used > worst) worst = used;
    double tm = 0.0, com[3] = {0, 0, 0};
    for (int a = 0; a < na; ++a) {
      tm += mm[a];
      for (int d = 0; d < 3; ++d) com[d] += mm[a] * xc[a][d];
    }
    for (int d = 0; d < 3; ++d) com[d] = tm > 0.0 ? com[d] / tm : 0.0;
    for (int a = 0; a < na; ++a) {
      int id = group_atoms[a0 + a];
      double v = 0.0;
      for (int d = 0; d < 3; ++d) {
        double delta = xc[a][d] - xu[a][d];
        pos[3 * id + d] += delta;
        if (dt != 0.0) vel[3 * id + d] += delta / dt;
        v += delta * (xc[a][d] - com[d]);
      }
      if (vir_slot) vir_slot[a0 + a] = dt != 0.0 ? mm[a] / (dt * dt) * v : 0.0;
    }
  }
  return worst;
}

static int solve_dense(int n, double *A, double *b) {
  /* Gaussian elimination with partial pivoting, A n x n row-major */
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (fabs(A[r * n + c]) > fabs(A[piv * n + c])) piv = r;
    if (A[piv * n + c] == 0.0) return -1;
    if (piv != c) {
      for (int k = 0; k < n; ++k) {
        double t = A[c * n + k];
        A[c * n + k] = A[piv * n + k];
        A[piv * n + k] = t;
      }
      double t = b[c];
      b[c] = b[piv];
      b[piv] = t;
    }
    for (int r = c + 1; r < n; ++r) {
      double f = A[r * n + c] / A[c * n + c];
      for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int c = n - 1; c >= 0; --c) {
    double s = b[c];
    for (int k = c + 1; k < n; ++k) s -= A[c * n + k] * b[k];
    b[c] = s / A[c * n + c];
  }
  return 0;
}

int or_constrain_velocities(int32_t n_groups, const int32_t *group_off,
                            const int32_t *group_atoms, const int32_t *con_off,
                            const int32_t *con_i, const int32_t *con_j,
                            const double *mass, const or_box *box,
                            const double *pos, double *vel, double dt,
                            double *vir_slot) {
  int bad = 0;
  for (int32_t g = 0; g < n_groups; ++g) {
    int a0 = group_off[g], na = group_off[g + 1] - a0;
    int c0 = con_off[g], nc = con_off[g + 1] - c0;
    double x[16][3], v[16][3], im[16], mm[16];
    for (int a = 0; a < na; ++a) {
      int id = group_atoms[a0 + a];
      mm[a] = mass[id];
      im[a] = mass[id] > 0.0 ? 1.0 / mass[id] : 0.0;
      for (int d = 0; d < 3; ++d) {
        x[a][d] = pos[3 * id + d];
        v[a][d] = vel[3 * id + d];
      }
      if (a > 0) {
        double dx = x[a][0] - x[0][0], dy = x[a][1] - x[0][1],
               dz = x[a][2] - x[0][2];
        or_min_image(box, &dx, &dy, &dz);
        x[a][0] = x[0][0] + dx;
        x[a][1] = x[0][1] + dy;
        x[a][2] = x[0][2] + dz;
      }
    }
    double r[32][3], A[32 * 32], rhs[32];
    for (int k = 0; k < nc; ++k) {
      int li = con_i[c0 + k], lj = con_j[c0 + k];
      double bk = 0.0;
      for (int d = 0; d < 3; ++d) {
        r[k][d] = x[li][d] - x[lj][d];
        bk += (v[li][d] - v[lj][d]) * r[k][d];
      }
      rhs[k] = -bk;
    }
    for (int k = 0; k < nc; ++k) {
      int ik = con_i[c0 + k], jk = con_j[c0 + k];
      for (int l = 0; l < nc; ++l) {
        int il = con_i[c0 + l], jl = con_j[c0 + l];
        double c = ((ik == il) - (ik == jl)) * im[ik] - ((jk == il) - (jk == jl)) * im[jk];
        double dot = r[k][0] * r[l][0] + r[k][1] * r[l][1] + r[k][2] * r[l][2];
        A[k * nc + l] = c * dot;
      }
    }
    if (nc > 0 && solve_dense(nc, A, rhs) != 0) {
      bad = -1;
      continue;
    }
    double dv[16][3];
    memset(dv, 0, sizeof(dv));
    for (int k = 0; k < nc; ++k) {
      int li = con_i[c0 + k], lj = con_j[c0 + k];
      for (int d = 0; d < 3; ++d) {
        dv[li][d] += rhs[k] * r[k][d] * im[li];
        dv[lj][d] -= rhs[k] * r[k][d] * im[lj];
      }
    }
    double tm = 0.0, com[3] = {0, 0, 0};
    for (int a = 0; a < na; ++a) {
      tm += mm[a];
      for (int d = 0; d < 3; ++d) com[d] += mm[a] * x[a][d];
    }
    for (int d = 0; d < 3; ++d) com[d] = tm > 0.0 ? com[d] / tm : 0.0;
    for (int a = 0; a < na; ++a) {
      int id = group_atoms[a0 + a];
      double wv = 0.0;
      for (int d = 0; d < 3; ++d) {
        vel[3 * id + d] += dv[a][d];
        wv += dv[a][d] * (x[a][d] - com[d]);
      }
      if (vir_slot && dt > 0.0) vir_slot[a0 + a] += mm[a] / dt * wv;
    }
  }
  return bad;
}

/* ------------------------------------------------------------------ */
/* Philox-4x32-10 (kernels/philox.cuh; Salmon et al., SC'11)           */
/* ------------------------------------------------------------------ */

void or_philox4x32_10(uint32_t key_lo, uint32_t key_hi, const uint32_t ctr[4],
                      uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key_lo, k1 = key_hi;
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)c0 * 0xD2511F53u;
    uint64_t p1 = (uint64_t)c2 * 0xCD9E8D57u;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0;
    c1 = n1;
    c2 = n2;
    c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

double or_philox_gaussian(uint32_t seed_lo, uint32_t seed_hi, uint32_t step_lo,
                          uint32_t step_hi, uint32_t particle, uint32_t axis) {
  /* Box-Muller cosine branch on ((u + 0.5) * 2^-32), kernels/philox.cuh:135-150 */
  uint32_t ctr[4] = {step_lo, step_hi, particle, axis}, o[4];
  or_philox4x32_10(seed_lo, seed_hi, ctr, o);
  double u1 = ((double)o[0] + 0.5) * (1.0 / 4294967296.0);
  double u2 = ((double)o[1] + 0.5) * (1.0 / 4294967296.0);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * OR_PI * u2);
}

/* ------------------------------------------------------------------ */
/* MD driver for the timed CPU baseline                                */
/* ------------------------------------------------------------------ */

int or_md_run(int32_t n, double *pos, double *vel, const double *mass,
              const double *q, const int32_t *type, const or_box *box,
              const or_ff *ff, int32_t n_groups, const int32_t *group_off,
              const int32_t *group_atoms, const int32_t *con_off,
              const int32_t *con_i, const int32_t *con_j, const double *con_d2,
              int integrator, double dt, double friction, double kt,
              uint64_t seed, uint64_t step0, int n_steps, double *F,
              int n_threads) {
  double *E = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *W = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *ref = (double *)malloc(sizeof(double) * 3 * (size_t)(n > 0 ? n : 1));
  double terms[OR_N_TERMS];
  int rc = or_forces(n, pos, q, type, box, ff, F, E, W, terms, n_threads);
  if (rc != 0) goto done;
  for (int s = 0; s < n_steps; ++s) {
    uint64_t step = step0 + (uint64_t)s;
    if (integrator == 0) {
      /* velocity Verlet with the reference's hook order
       * (src/integrator/mod.rs:344-429, src/runner.rs:2611-2686) */
      memcpy(ref, pos, sizeof(double) * 3 * (size_t)n);
#pragma omp parallel for schedule(static)
      for (int32_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
          vel[3 * i + d] += 0.5 * dt * F[3 * i + d] / mass[i];
          pos[3 * i + d] += dt * vel[3 * i + d];
        }
      if (n_groups > 0)
        or_constrain_positions(n_groups, group_off, group_atoms, con_off, con_i,
                               con_j, con_d2, mass, box, ref, pos, vel, dt,
                               NULL, 1e-12, 1000);
      rc = or_forces(n, pos, q, type, box, ff, F, E, W, terms, n_threads);
      if (rc != 0) goto done;
      if (n_groups > 0)
        or_constrain_velocities(n_groups, group_off, group_atoms, con_off,
                                con_i, con_j, mass, box, pos, vel, dt, NULL);
#pragma omp parallel for schedule(static)
      for (int32_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) vel[3 * i + d] += 0.5 * dt * F[3 * i + d] / mass[i];
    } else {
      /* Langevin, middle scheme: kick, project velocities, half drift, OU,
       * half drift, project positions, force */
      double a = exp(-friction * dt);
#pragma omp parallel for schedule(static)
      for (int32_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) vel[3 * i + d] += dt * F[3 * i + d] / mass[i];
      if (n_groups > 0)
        or_constrain_velocities(n_groups, group_off, group_atoms, con_off,
                                con_i, con_j, mass, box, pos, vel, 0.0, NULL);
      memcpy(ref, pos, sizeof(double) * 3 * (size_t)n);
#pragma omp parallel for schedule(static)
      for (int32_t i = 0; i < n; ++i) {
        double sig = sqrt((1.0 - a * a) * kt / mass[i]);
        for (int d = 0; d < 3; ++d) {
          pos[3 * i + d] += 0.5 * dt * vel[3 * i + d];
          double xi = or_philox_gaussian((uint32_t)seed, (uint32_t)(seed >> 32),
                                         (uint32_t)step, (uint32_t)(step >> 32),
                                         (uint32_t)i, (uint32_t)d);
          vel[3 * i + d] = a * vel[3 * i + d] + sig * xi;
          pos[3 * i + d] += 0.5 * dt * vel[3 * i + d];
        }
      }
      if (n_groups > 0)
        or_constrain_positions(n_groups, group_off, group_atoms, con_off, con_i,
                               con_j, con_d2, mass, box, ref, pos, vel, dt,
                               NULL, 1e-12, 1000);
      rc = or_forces(n, pos, q, type, box, ff, F, E, W, terms, n_threads);
      if (rc != 0) goto done;
    }
  }
done:
  free(E);
  free(W);
  free(ref);
  return rc;
}

/* ---------------------------------------------------------------------
 * Monte-Carlo barostat centre-of-mass scaling
 * (kernels/mc_barostat.cu:19-74; the molecule is translated as its
 * contiguous image, see the header)
 * ------------------------------------------------------------------- */
void or_mc_scale_com(int32_t n_mol, const int32_t *off, const int32_t *atoms,
                     const double *mass, const or_box *box_old, const or_box *box_new,
                     double scale, double *pos, int32_t *img) {
  for (int32_t m = 0; m < n_mol; ++m) {
    const int32_t lo = off[m], hi = off[m + 1];
    if (hi <= lo) continue;
    const int32_t r = atoms[lo];
    const double rx = pos[3 * r], ry = pos[3 * r + 1], rz = pos[3 * r + 2];
    double mt = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    for (int32_t k = lo; k < hi; ++k) {
      const int32_t a = atoms[k];
      double dx = pos[3 * a] - rx, dy = pos[3 * a + 1] - ry, dz = pos[3 * a + 2] - rz;
      or_min_image(box_old, &dx, &dy, &dz);
      cx += mass[a] * dx;
      cy += mass[a] * dy;
      cz += mass[a] * dz;
      mt += mass[a];
    }
    const double f = scale - 1.0;
    const double sx = f * (rx + cx / mt), sy = f * (ry + cy / mt), sz = f * (rz + cz / mt);
    for (int32_t k = lo; k < hi; ++k) {
      const int32_t a = atoms[k];
      const double ox = pos[3 * a] - rx, oy = pos[3 * a + 1] - ry, oz = pos[3 * a + 2] - rz;
      double dx = ox, dy = oy, dz = oz;
      or_min_image(box_old, &dx, &dy, &dz);
      /* lattice counts of the minimum-image shift (ox - dx = K L) */
      double sa, sb, sc;
      cart_to_frac(box_old, ox - dx, oy - dy, oz - dz, &sa, &sb, &sc);
      double x = rx + dx + sx, y = ry + dy + sy, z = rz + dz + sz;
      int wa, wb, wc;
      or_wrap_with_image(box_new, &x, &y, &z, &wa, &wb, &wc);
      pos[3 * a] = x;
      pos[3 * a + 1] = y;
      pos[3 * a + 2] = z;
      img[3 * a] += (int32_t)lrint(sa) + wa;
      img[3 * a + 1] += (int32_t)lrint(sb) + wb;
      img[3 * a + 2] += (int32_t)lrint(sc) + wc;
    }
  }
}
