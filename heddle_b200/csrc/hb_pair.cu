// hb_pair.cu -- Lennard-Jones + erfc-screened real-space Coulomb pair
// kernel over the packed neighbour list.
//
// Physics follows the reference's composed pair kernel
// (src/forces/jit_composed.rs:1490-1831) with the LJ functor
// (src/forces/lj.rs:237-283, optional CHARMM switch) and the SPME real-space
// functor (src/forces/spme.rs:730-759, erfc by the Abramowitz-Stegun 7.1.26
// polynomial in single precision), per-fragment cutoffs, exclusion scales
// applied per fragment, energy and virial split 1/2 per atom.
//
// Structure (own design): persistent warps take (i-tile, chunk of entries)
// work items.  Per entry a distance pass over the 32 x 32 slot pairs leaves a
// hit mask per i-lane, one warp scan places the hits in a lane-major queue,
// and the math pass gives every lane a run of that queue (k_pair4, every
// fast step, with or without energies).  Pair forces are summed as integers
// (int32 shared sums folded into int64 fixed point at 2^40), so forces do
// not depend on entry order or on scheduling and repeat runs are
// byte-identical.  Exclusions arrive as a 32-bit mask per (entry, i-lane)
// built with the list, so an ordinary pair costs no exclusion lookup.  Tiles
// that satisfy the single-periodic-copy condition shift i and j positions
// against the tile centre once per entry and skip the per-pair minimum
// image.  The exact-pair form (k_pair2<.., EXACT>) converts every pair force
// to int64 fixed point and takes each pair's own minimum image, so forces
// are functions of the positions alone (the lossless integrator needs that).
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "hb_internal.cuh"

namespace {

struct PairParams {
  int n_types;
  int lj_on, coul_on;
  float rc2_max;
  float coul_rc2;
  float alpha;
  float c2a;  // 2 alpha / sqrt(pi)
  uint32_t n, n_tiles;
  uint32_t slab;
};

// one system of the multi-system pair launch: its lists, positions,
// accumulators and cell, and its first work item in the launch's item space
struct PairMember {
  const float4 *tile_posq;
  const int *tile_type;
  const float4 *center;
  const uint32_t *tile_nent;
  const uint32_t *entry_j;
  const uint32_t *entry_excl;
  const DBox *box;
  unsigned long long *fp;
  uint32_t n, n_tiles, slab, chunks, item0, pad[3];
};

__device__ __forceinline__ void shift_to(float &x, float &y, float &z, const float4 &c,
                                         const DBox &b) {
  float dx = x - c.x, dy = y - c.y, dz = z - c.z;
  x -= b.lx * rintf(dx * b.ilx);
  y -= b.ly * rintf(dy * b.ily);
  z -= b.lz * rintf(dz * b.ilz);
}

__device__ __forceinline__ long long to_fixed(float v) {
  return __float2ll_rn(v * HB_FP_SCALE);
}

__device__ __forceinline__ void red_add(unsigned long long *p, long long v) {
  if (v != 0) atomicAdd(p, (unsigned long long)v);
}

// ---------------------------------------------------------------------
// Balanced form (every step; with EV also per-atom energy and virial).
// One lane per i-atom of the tile.  Per entry: (1) a distance pass over the
// 32 j-slots (broadcast shared loads; two slots per packed FP32x2 step in
// single-periodic-copy tiles) leaves each
// lane's mask of the j-slots whose pair is inside the cutoff (bit j), with
// exclusions and padding slots masked out; (2) one
// warp scan of the mask counts places every lane's pairs contiguously in a
// per-warp queue (pairs with a Lennard-Jones term first); (3) the math pass
// gives each lane a run of the queue, so all lanes stay busy whatever the
// spatial imbalance.  Forces are int32 fixed point (scale 2^30, integer
// sums: order-independent, so the result is the same run to run): the
// i-side sums of a lane's run, which touches few i-atoms, stay in registers
// and are added to shared memory once per atom; the j-side sums go to
// shared memory by atomics, into one of two copies per slot.  Both are
// folded into int64 once per entry.  A pair force component above 0.06
// hartree/bohr takes the exact global int64 path instead, so the int32
// sums cannot wrap (32 pairs x 0.06 x 2^30 < 2^31).  With EV the energy and
// virial halves of each pair go to shared int32 sums at scale 2^28 (guard
// 0.25 hartree), and the LJ energy total is summed per lane in int64.
// ---------------------------------------------------------------------
#define P4_WARPS 4
#define P4_SHIFT 10               // 2^40 / 2^30
#define P4_SCALE 1073741824.0f    // 2^30
#define P4_FMAX 0.06f
#define P4_ESHIFT 12              // 2^40 / 2^28
#define P4_ESCALE 268435456.0f    // 2^28
#define P4_EMAX 0.25f

struct P4Warp {
  float4 ipos[32];
  float4 jpos[32];
  float4 jxy2[16];  // j-slots 2k, 2k + 1 negated: (-x, -x', -y, -y') for the packed distance pass
  float2 jz2[16];   // (-z, -z')
  int itype[32];
  int jtype[32];
  uint32_t oi[32];
  uint32_t oj[32];
  uint32_t xm[32];
  uint32_t jslot[32];
  int fi[3][32];
  int fj[3][80];  // two copies per j-slot, [j] and [48 + j], 16 banks apart
  uint16_t pairs[1024];
};

template <bool EV, bool SCALED, bool SWITCH, bool MULTI>
__global__ void __launch_bounds__(P4_WARPS * 32, MULTI ? 6 : 8)
    k_pair4(const float4 *__restrict__ a_tile_posq, const int *__restrict__ a_tile_type,
            const float4 *__restrict__ a_center, const uint32_t *__restrict__ a_tile_nent,
            const uint32_t *__restrict__ a_entry_j, const uint32_t *__restrict__ a_entry_excl,
            const DBox *__restrict__ a_box, const float4 *__restrict__ lj_table,
            const float *__restrict__ lj_invd, PairParams a_P, unsigned long long *__restrict__ a_fp,
            const uint32_t *__restrict__ sorted_ids, const uint32_t *__restrict__ eoff,
            const uint32_t *__restrict__ epart, const float2 *__restrict__ escale,
            uint32_t *__restrict__ work, uint32_t a_chunks, uint32_t chunk, uint32_t quota,
            unsigned long long *__restrict__ e_lj_total, const PairMember *__restrict__ members,
            uint32_t n_members, uint32_t n_items_all) {
  static_assert(!(MULTI && (EV || SCALED)), "the multi-system form is force-only, unscaled");
  const PairParams &P0 = a_P;
  extern __shared__ float4 sm_lj4[];
  __shared__ P4Warp smw4[P4_WARPS];
  __shared__ uint32_t sm_ljtypes[32];  // per i-type: j-types with a Lennard-Jones term
  // with energies: per warp int32 fixed-point (2^28) energy / virial halves
  // of the i-atoms [0, 32) and [32, 64) and of the j-atoms [64, 96) and
  // [96, 128); a half above 0.25 hartree takes the int64 path, so the int32
  // sums cannot wrap (32 pairs x 0.25 x 2^28 < 2^31)
  __shared__ int sm_ev[EV ? P4_WARPS * 128 : 1];
  // multi-system form: the members' first work items, for the per-item
  // member search (members beyond the table search global memory)
  constexpr uint32_t MT = 128u;
  __shared__ uint32_t sm_item0[MULTI ? MT : 1];
  if constexpr (MULTI) {
    for (uint32_t k = threadIdx.x; k < MT && k < n_members; k += blockDim.x) sm_item0[k] = members[k].item0;
  }
  const int nt2 = P0.n_types * P0.n_types;
  float *sm_ljd4 = reinterpret_cast<float *>(sm_lj4 + nt2);
  for (int k = threadIdx.x; k < nt2; k += blockDim.x) {
    sm_lj4[k] = lj_table[k];
    sm_ljd4[k] = lj_invd[k];
  }
  const bool few_types = P0.n_types <= 32;
  if (few_types && (int)threadIdx.x < P0.n_types) {
    uint32_t bits = 0u;
    for (int q = 0; q < P0.n_types; ++q)
      if (lj_table[threadIdx.x * P0.n_types + q].y != 0.0f) bits |= 1u << q;
    sm_ljtypes[threadIdx.x] = bits;
  }
  __syncthreads();
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  P4Warp &S = smw4[w];
  int *Ev = sm_ev + (EV ? w * 128u : 0u);
  long long elj_fix = 0;  // LJ energy of this lane's pairs (fixed point)
  const DBox b0 = *a_box;
  const uint32_t n_items = MULTI ? n_items_all : a_P.n_tiles * a_chunks;

  // warps take (tile, chunk of entries) items from a counter, at most
  // `quota` each: a finite quota retires blocks as they finish, so the
  // concurrent reciprocal-space kernels (a higher-priority stream) get SM
  // room between pair blocks instead of only what persistent blocks leave
  for (uint32_t taken = 0; taken < quota; ++taken) {
    uint32_t g = 0u;
    if (lane == 0) g = atomicAdd(work, 1u);
    g = __shfl_sync(0xFFFFFFFFu, g, 0);
    if (g >= n_items) break;
    // the system this item belongs to: the kernel's own arguments, or (the
    // multi-system form) the member whose item range holds g
    const float4 *__restrict__ tile_posq = a_tile_posq;
    const int *__restrict__ tile_type = a_tile_type;
    const float4 *__restrict__ center = a_center;
    const uint32_t *__restrict__ tile_nent = a_tile_nent;
    const uint32_t *__restrict__ entry_j = a_entry_j;
    const uint32_t *__restrict__ entry_excl = a_entry_excl;
    unsigned long long *__restrict__ fp = a_fp;
    PairParams P = a_P;
    uint32_t chunks = a_chunks;
    DBox b = b0;
    if constexpr (MULTI) {
      uint32_t lo = 0u, hi = n_members;  // largest m with members[m].item0 <= g
      while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((mid < MT ? sm_item0[mid] : members[mid].item0) <= g) lo = mid;
        else hi = mid;
      }
      const PairMember &M = members[lo];
      g -= M.item0;
      tile_posq = M.tile_posq;
      tile_type = M.tile_type;
      center = M.center;
      tile_nent = M.tile_nent;
      entry_j = M.entry_j;
      entry_excl = M.entry_excl;
      fp = M.fp;
      P.n = M.n;
      P.n_tiles = M.n_tiles;
      P.slab = M.slab;
      chunks = M.chunks;
      b = *M.box;
    }
    const size_t np_all = (size_t)P.n_tiles * 32u;
    const uint32_t I = g / chunks, ch = g - I * chunks;
    const uint32_t tile_e0 = I * P.slab;
    const uint32_t tile_e1 = tile_e0 + min(tile_nent[I], P.slab);
    const uint32_t e0 = tile_e0 + ch * chunk;
    if (e0 >= tile_e1) continue;
    const uint32_t e1 = min(e0 + chunk, tile_e1);
    const float4 c = center[I];
    const bool spc = ((int)c.w & 1) != 0;
    const uint32_t si = I * 32u + lane;
    const bool ivalid = si < P.n;
    float4 pi = tile_posq[si];
    if (ivalid) {
      if (spc) shift_to(pi.x, pi.y, pi.z, c, b);
    } else {
      pi = make_float4(-1.0e18f, -1.0e18f, -1.0e18f, 0.0f);
    }
    __syncwarp();
    S.ipos[lane] = pi;
    const int ti = ivalid ? tile_type[si] : 0;
    S.itype[lane] = ti * P.n_types;
    // j-types with a Lennard-Jones term against this lane's i-atom
    const uint32_t lj_types = few_types ? sm_ljtypes[ti] : 0u;
    if (SCALED) S.oi[lane] = ivalid ? sorted_ids[si] : HB_SENTINEL;
    long long ax = 0, ay = 0, az = 0, ae = 0, aw = 0;
    const bool has_self = P.n - I * 32u >= 2u;

    // software pipeline over the entries: the next entry's j-slots and
    // exclusion masks are requested at the top of an entry and its j
    // positions gathered right after the distance pass, so each entry's
    // dependent global loads are in flight while the previous entry computes
    const float4 far = make_float4(1.0e18f, 1.0e18f, 1.0e18f, 0.0f);
    uint32_t sj_n = entry_j[(uint64_t)e0 * 32u + lane];
    uint32_t xm_n = entry_excl[(uint64_t)e0 * 32u + lane];
    float4 pj_n = far;
    int tj_n = 0;
    if (sj_n != HB_SENTINEL) {
      pj_n = tile_posq[sj_n];
      tj_n = tile_type[sj_n];
    }

    for (uint32_t e = e0; e < e1; ++e) {
      const bool self = has_self && (e == tile_e0);
      const uint32_t sj = sj_n, xm = xm_n;
      const bool jvalid = sj != HB_SENTINEL;
      float4 pj = pj_n;
      const int tj = tj_n;
      if (jvalid && spc) shift_to(pj.x, pj.y, pj.z, c, b);
      const bool more = e + 1u < e1;
      if (more) {
        sj_n = entry_j[(uint64_t)(e + 1u) * 32u + lane];
        xm_n = entry_excl[(uint64_t)(e + 1u) * 32u + lane];
      }
      __syncwarp();
      S.jpos[lane] = pj;
      {
        float *jn = reinterpret_cast<float *>(&S.jxy2[lane >> 1]);
        jn[lane & 1u] = -pj.x;
        jn[2u + (lane & 1u)] = -pj.y;
        reinterpret_cast<float *>(&S.jz2[lane >> 1])[lane & 1u] = -pj.z;
      }
      S.jtype[lane] = tj;
      S.jslot[lane] = self ? si : sj;
      if (SCALED) S.oj[lane] = jvalid ? sorted_ids[sj] : HB_SENTINEL;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        S.fi[q][lane] = 0;
        S.fj[q][lane] = 0;
        S.fj[q][48 + lane] = 0;
      }
      if (EV) {
#pragma unroll
        for (int q = 0; q < 4; ++q) Ev[32 * q + lane] = 0;
      }
      __syncwarp();

      // (1) distance pass: lane L tests its i-atom against the 32 j-slots in
      // turn, each j position one broadcast shared load (one wavefront), so
      // bit j of the mask is the pair (L, j); in the self entry only j > L
      // counts (each pair once).  The tile's single-periodic-copy flag is
      // uniform over the warp, so each form is its own code path (no
      // per-pair minimum-image instructions where the shift already placed
      // the atoms)
      uint32_t m = 0u;
      auto dist_pass = [&](auto sp) {
        constexpr bool SP = decltype(sp)::value;
        if constexpr (SP) {
          // two j-slots per step in the packed FP32x2 pipe (FADD2 / FMUL2 /
          // FFMA2): pi - q is pi + (-q) exactly, each lane of a packed op
          // rounds like the scalar op
          const float2 px = make_float2(pi.x, pi.x), py = make_float2(pi.y, pi.y),
                       pz = make_float2(pi.z, pi.z);
          const float2 nrc = make_float2(-P.rc2_max, -P.rc2_max);
#pragma unroll
          for (uint32_t k = 0; k < 16u; ++k) {
            const float4 a = S.jxy2[k];
            const float2 dx = __fadd2_rn(px, make_float2(a.x, a.y));
            const float2 dy = __fadd2_rn(py, make_float2(a.z, a.w));
            const float2 dz = __fadd2_rn(pz, S.jz2[k]);
            float2 r2 = __fmul2_rn(dx, dx);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            // r2 < rc2 exactly when r2 - rc2 is negative (the difference of
            // two distinct finite floats is never zero): its sign bits are
            // the two mask bits
            const float2 d = __fadd2_rn(r2, nrc);
            m |= ((__float_as_uint(d.x) >> 31) | ((__float_as_uint(d.y) >> 30) & 2u)) << (2u * k);
          }
        } else {
#pragma unroll 4
          for (uint32_t t = 0; t < 32u; ++t) {
            const float4 q = S.jpos[t];
            float dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
            hb_min_image(dx, dy, dz, b);
            const float r2 = dx * dx + dy * dy + dz * dz;
            m |= (r2 < P.rc2_max ? 1u : 0u) << t;
          }
        }
        if (self) m &= lane == 31u ? 0u : (0xFFFFFFFFu << (lane + 1u));
      };
      if (spc) dist_pass(std::true_type{});
      else dist_pass(std::false_type{});
      // the next entry's j positions (its slots have arrived meanwhile)
      if (more) {
        pj_n = far;
        tj_n = 0;
        if (sj_n != HB_SENTINEL) {
          pj_n = tile_posq[sj_n];
          tj_n = tile_type[sj_n];
        }
      }
      // padding slots take part in no pair, whatever their placeholder
      // coordinates give under the minimum image
      const uint32_t jv_mask = __ballot_sync(0xFFFFFFFFu, jvalid);
      m &= ivalid ? jv_mask : 0u;
      // the list stores each lane's exclusion bits in rotation order (bit t:
      // j-slot (L + t) mod 32); rotating left by L gives j order
      const uint32_t xm_j = __funnelshift_l(xm, xm, lane);
      if (SCALED) S.xm[lane] = xm_j;  // read by the math pass (scaled exclusions)
      else m &= ~xm_j;

      // (2) lane-major queues of (i-lane, j-slot): each lane writes its
      // pairs with a Lennard-Jones term to [0, n_lj) and its Coulomb-only
      // pairs to [n_lj, n_lj + n_c) at offsets from one warp scan of the
      // packed counts; the LJ arithmetic runs only over the first range
      uint32_t lj_rot = 0xFFFFFFFFu;
      if (!P.lj_on) {
        lj_rot = 0u;
      } else if (few_types) {
        uint32_t lj_j = 0u;
        for (int q = 0; q < P.n_types; ++q) {
          const uint32_t bal_t = __ballot_sync(0xFFFFFFFFu, tj == q && jvalid);
          if ((lj_types >> q) & 1u) lj_j |= bal_t;
        }
        lj_rot = lj_j;  // bit j <-> j-slot j
      }
      uint32_t mq = m & lj_rot;
      uint32_t mc = P.coul_on ? (m & ~lj_rot) : 0u;
      const uint32_t cnt = ((uint32_t)__popc(mq) << 16) | (uint32_t)__popc(mc);
      uint32_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
      }
      const uint32_t tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
      const uint32_t n_lj = tot >> 16, n_c = tot & 0xFFFFu;
      {
        const uint32_t ex = incl - cnt;
        uint32_t pos = ex >> 16;
        while (mq != 0u) {
          const uint32_t t = (uint32_t)__ffs(mq) - 1u;
          mq &= mq - 1u;
          S.pairs[pos++] = (uint16_t)((lane << 8) | t);
        }
        pos = n_lj + (ex & 0xFFFFu);
        while (mc != 0u) {
          const uint32_t t = (uint32_t)__ffs(mc) - 1u;
          mc &= mc - 1u;
          S.pairs[pos++] = (uint16_t)((lane << 8) | t);
        }
      }
      __syncwarp();

      // (3) math over each range: in round `it` lane L takes pair
      // L * rounds + it, so a lane's pairs are a run of the queue that spans
      // few i-lanes: their i-side sums stay in registers and reach shared
      // memory once per i-atom.  The j-side sums go to one of two copies
      // (by lane parity), which halves the same-slot atomics of a round.
      // One code path per periodic form and per range.
      const uint32_t jo = (lane & 1u) * 48u;
      auto math_pass = [&](auto sp, auto ljc, uint32_t q0, uint32_t cnt_r) {
        constexpr bool SP = decltype(sp)::value, LJQ = decltype(ljc)::value;
        const uint32_t rounds = (cnt_r + 31u) >> 5;
        uint32_t ci = 32u;  // i-lane of the running sums (32: none)
        int sx = 0, sy = 0, sz = 0;
        for (uint32_t it = 0; it < rounds; ++it) {
          const uint32_t kk = lane * rounds + it;
          if (kk < cnt_r) {
            const uint32_t pr = S.pairs[q0 + kk];
            const uint32_t i = pr >> 8, j = pr & 255u;
            const float4 a = S.ipos[i], q = S.jpos[j];
            float dx = a.x - q.x, dy = a.y - q.y, dz = a.z - q.z;
            if constexpr (!SP) hb_min_image(dx, dy, dz, b);
            const float r2 = dx * dx + dy * dy + dz * dz;
            float s_lj = 1.0f, s_c = 1.0f;
            if (SCALED && ((S.xm[i] >> j) & 1u)) {
              s_lj = 0.0f;
              s_c = 0.0f;
              const uint32_t oi = S.oi[i], oj = S.oj[j];
              for (uint32_t z = eoff[oj]; z < eoff[oj + 1]; ++z) {
                if (epart[z] == oi) {
                  const float2 sc = escale[z];
                  s_lj = sc.x;
                  s_c = sc.y;
                  break;
                }
              }
            }
            const float inv_r = rsqrtf(r2);
            const float inv_r2 = inv_r * inv_r;
            float fac = 0.0f, en = 0.0f;
            if constexpr (LJQ) {
              const int tp = S.itype[i] + S.jtype[j];
              const float4 L = sm_lj4[tp];
              if (r2 <= L.z && L.y != 0.0f && s_lj != 0.0f) {
                const float sr2 = L.x * inv_r2;
                const float sr6 = sr2 * sr2 * sr2;
                const float sr12 = sr6 * sr6;
                float f = L.y * inv_r2 * (2.0f * sr12 - sr6);
                float u = (L.y * (1.0f / 6.0f)) * (sr12 - sr6);
                if (SWITCH && r2 > L.w) {
                  const float inv_d = sm_ljd4[tp];
                  const float tau = (r2 - L.w) * inv_d;
                  const float omt = 1.0f - tau;
                  const float sw = omt * omt * (1.0f + 2.0f * tau);
                  const float chain = 12.0f * tau * omt * inv_d;
                  f = sw * f + chain * u;
                  u = sw * u;
                }
                fac += s_lj * f;
                if (EV) {
                  en += s_lj * u;
                  elj_fix += to_fixed(s_lj * u);
                }
              }
            }
            if (P.coul_on && r2 <= P.coul_rc2 && s_c != 0.0f) {
              const float r = r2 * inv_r;
              const float ar = P.alpha * r;
              const float gg = __expf(-ar * ar);
              const float tt = __fdividef(1.0f, 1.0f + 0.3275911f * ar);
              const float poly =
                  0.254829592f +
                  (-0.284496736f + (1.421413741f + (-1.453152027f + 1.061405429f * tt) * tt) * tt) * tt;
              // erfc(ar) / r + c2a exp(-a^2 r^2) = gg (poly tt / r + c2a)
              const float pt = poly * tt;
              fac += s_c * a.w * q.w * inv_r2 * (gg * fmaf(pt, inv_r, P.c2a));
              if (EV) en += s_c * a.w * q.w * (pt * gg) * inv_r;
            }
            // the pair force in units of 2^-30 (an exact power-of-two scale,
            // so the rounding is that of fac * d)
            const float fs = fac * P4_SCALE;
            const float fx = fs * dx, fy = fs * dy, fz = fs * dz;
            if (EV) {
              // half of the pair's energy and virial to each atom (integer sums:
              // order-independent)
              const float he = 0.5f * en, hw = 0.5f * fac * r2;
              if (fabsf(he) <= P4_EMAX && fabsf(hw) <= P4_EMAX) {
                const int ie = __float2int_rn(he * P4_ESCALE), iw = __float2int_rn(hw * P4_ESCALE);
                atomicAdd(&Ev[i], ie);
                atomicAdd(&Ev[32 + i], iw);
                atomicAdd(&Ev[64 + j], ie);
                atomicAdd(&Ev[96 + j], iw);
              } else {
                const uint32_t ti_slot = I * 32u + i, tj_slot = S.jslot[j];
                red_add(&fp[3 * np_all + ti_slot], to_fixed(he));
                red_add(&fp[4 * np_all + ti_slot], to_fixed(hw));
                red_add(&fp[3 * np_all + tj_slot], to_fixed(he));
                red_add(&fp[4 * np_all + tj_slot], to_fixed(hw));
              }
            }
            constexpr float FLIM = P4_FMAX * P4_SCALE;
            if (fabsf(fx) <= FLIM && fabsf(fy) <= FLIM && fabsf(fz) <= FLIM) {
              const int ix = __float2int_rn(fx), iy = __float2int_rn(fy), iz = __float2int_rn(fz);
              atomicAdd(&S.fj[0][jo + j], -ix);
              atomicAdd(&S.fj[1][jo + j], -iy);
              atomicAdd(&S.fj[2][jo + j], -iz);
              // an i-atom has at most 32 pairs in an entry, so the running
              // sums stay below 32 x 0.06 x 2^30 < 2^31 like the shared ones
              if (i != ci) {
                if (ci < 32u) {
                  atomicAdd(&S.fi[0][ci], sx);
                  atomicAdd(&S.fi[1][ci], sy);
                  atomicAdd(&S.fi[2][ci], sz);
                }
                ci = i;
                sx = sy = sz = 0;
              }
              sx += ix;
              sy += iy;
              sz += iz;
            } else {
              // rare: the exact int64 path for both atoms
              const uint32_t ti_slot = I * 32u + i, tj_slot = S.jslot[j];
              const long long lx = __float2ll_rn(fx * (HB_FP_SCALE / P4_SCALE)),
                              ly = __float2ll_rn(fy * (HB_FP_SCALE / P4_SCALE)),
                              lz = __float2ll_rn(fz * (HB_FP_SCALE / P4_SCALE));
              red_add(&fp[0 * np_all + ti_slot], lx);
              red_add(&fp[1 * np_all + ti_slot], ly);
              red_add(&fp[2 * np_all + ti_slot], lz);
              red_add(&fp[0 * np_all + tj_slot], -lx);
              red_add(&fp[1 * np_all + tj_slot], -ly);
              red_add(&fp[2 * np_all + tj_slot], -lz);
            }
          }
        }
        if (ci < 32u) {
          atomicAdd(&S.fi[0][ci], sx);
          atomicAdd(&S.fi[1][ci], sy);
          atomicAdd(&S.fi[2][ci], sz);
        }
      };
      // Pairs of single-periodic-copy tiles on force-only steps (every pair
      // of a water box): two pairs of a lane's run per step in the packed
      // FP32x2 pipe (FADD2 / FMUL2 / FFMA2), the transcendentals and the
      // integer sums per pair as in math_pass.  LJQ: the range with a
      // Lennard-Jones term (unswitched kernels), then the Coulomb term where
      // the force field has one; otherwise the Coulomb-only range
      auto math_pass_2 = [&](auto ljc, uint32_t q0, uint32_t cnt_r) {
        constexpr bool LJQ = decltype(ljc)::value;
        const uint32_t rounds = (((cnt_r + 31u) >> 5) + 1u) & ~1u;  // even: pairs of pairs
        uint32_t ci = 32u;
        int sx = 0, sy = 0, sz = 0;
        constexpr float FLIM = P4_FMAX * P4_SCALE;
        auto accum = [&](uint32_t i, uint32_t j, float fx, float fy, float fz) {
          if (fabsf(fx) <= FLIM && fabsf(fy) <= FLIM && fabsf(fz) <= FLIM) {
            const int ix = __float2int_rn(fx), iy = __float2int_rn(fy), iz = __float2int_rn(fz);
            atomicAdd(&S.fj[0][jo + j], -ix);
            atomicAdd(&S.fj[1][jo + j], -iy);
            atomicAdd(&S.fj[2][jo + j], -iz);
            if (i != ci) {
              if (ci < 32u) {
                atomicAdd(&S.fi[0][ci], sx);
                atomicAdd(&S.fi[1][ci], sy);
                atomicAdd(&S.fi[2][ci], sz);
              }
              ci = i;
              sx = sy = sz = 0;
            }
            sx += ix;
            sy += iy;
            sz += iz;
          } else {
            const uint32_t ti_slot = I * 32u + i, tj_slot = S.jslot[j];
            const long long lx = __float2ll_rn(fx * (HB_FP_SCALE / P4_SCALE)),
                            ly = __float2ll_rn(fy * (HB_FP_SCALE / P4_SCALE)),
                            lz = __float2ll_rn(fz * (HB_FP_SCALE / P4_SCALE));
            red_add(&fp[0 * np_all + ti_slot], lx);
            red_add(&fp[1 * np_all + ti_slot], ly);
            red_add(&fp[2 * np_all + ti_slot], lz);
            red_add(&fp[0 * np_all + tj_slot], -lx);
            red_add(&fp[1 * np_all + tj_slot], -ly);
            red_add(&fp[2 * np_all + tj_slot], -lz);
          }
        };
        const float2 alpha2 = make_float2(P.alpha, P.alpha), one2 = make_float2(1.0f, 1.0f),
                     c2a2 = make_float2(P.c2a, P.c2a), sc2 = make_float2(P4_SCALE, P4_SCALE);
        // the i-atom of a lane's run changes rarely: its position stays in
        // registers and is reloaded only when the i-lane changes
        uint32_t pi_idx = 32u;
        float4 pi_c = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t it = 0; it < rounds; it += 2u) {
          const uint32_t ka = lane * rounds + it;
          if (ka < cnt_r) {
            const bool vb = ka + 1u < cnt_r;
            const uint32_t pa = S.pairs[q0 + ka], pb = vb ? S.pairs[q0 + ka + 1u] : pa;
            const uint32_t ia = pa >> 8, ja = pa & 255u, ib = pb >> 8, jb = pb & 255u;
            if (ia != pi_idx) {
              pi_c = S.ipos[ia];
              pi_idx = ia;
            }
            const float4 a = pi_c;
            float4 a2 = pi_c;
            if (ib != ia) {
              a2 = S.ipos[ib];
              pi_c = a2;
              pi_idx = ib;
            }
            const float4 qa = S.jpos[ja], qb = S.jpos[jb];
            const float2 dx = __fadd2_rn(make_float2(a.x, a2.x), make_float2(-qa.x, -qb.x));
            const float2 dy = __fadd2_rn(make_float2(a.y, a2.y), make_float2(-qa.y, -qb.y));
            const float2 dz = __fadd2_rn(make_float2(a.z, a2.z), make_float2(-qa.z, -qb.z));
            float2 r2 = __fmul2_rn(dx, dx);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            const float2 inv_r = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
            const float2 inv_r2 = __fmul2_rn(inv_r, inv_r);
            float2 fac = make_float2(0.0f, 0.0f);
            if constexpr (LJQ) {
              const int tpa = S.itype[ia] + S.jtype[ja], tpb = S.itype[ib] + S.jtype[jb];
              const float4 La = sm_lj4[tpa], Lb = sm_lj4[tpb];
              const float2 eps = make_float2(La.y, Lb.y);
              const float2 sr2 = __fmul2_rn(make_float2(La.x, Lb.x), inv_r2);
              const float2 sr6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
              const float2 sr12 = __fmul2_rn(sr6, sr6);
              const float2 nsr6 = make_float2(-sr6.x, -sr6.y);
              float2 f = __fmul2_rn(__fmul2_rn(eps, inv_r2),
                                    __ffma2_rn(make_float2(2.0f, 2.0f), sr12, nsr6));
              if (SWITCH && (r2.x > La.w || r2.y > Lb.w)) {
                const float2 u = __fmul2_rn(__fmul2_rn(eps, make_float2(1.0f / 6.0f, 1.0f / 6.0f)),
                                            __fadd2_rn(sr12, nsr6));
                const float2 inv_d = make_float2(sm_ljd4[tpa], sm_ljd4[tpb]);
                const float2 tau = __fmul2_rn(__fadd2_rn(r2, make_float2(-La.w, -Lb.w)), inv_d);
                const float2 omt = __fadd2_rn(one2, make_float2(-tau.x, -tau.y));
                const float2 sw = __fmul2_rn(__fmul2_rn(omt, omt),
                                             __ffma2_rn(make_float2(2.0f, 2.0f), tau, one2));
                const float2 chain =
                    __fmul2_rn(__fmul2_rn(__fmul2_rn(make_float2(12.0f, 12.0f), tau), omt), inv_d);
                const float2 fsw = __ffma2_rn(sw, f, __fmul2_rn(chain, u));
                if (r2.x > La.w) f.x = fsw.x;
                if (r2.y > Lb.w) f.y = fsw.y;
              }
              if (r2.x <= La.z && La.y != 0.0f) fac.x = f.x;
              if (r2.y <= Lb.z && Lb.y != 0.0f) fac.y = f.y;
            }
            if (!LJQ || P.coul_on) {
              const float2 r = __fmul2_rn(r2, inv_r);
              const float2 ar = __fmul2_rn(alpha2, r);
              const float2 ea = __fmul2_rn(make_float2(-ar.x, -ar.y), ar);
              const float2 gg = make_float2(__expf(ea.x), __expf(ea.y));
              const float2 den = __ffma2_rn(make_float2(0.3275911f, 0.3275911f), ar, one2);
              const float2 tt = make_float2(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y));
              float2 poly = __ffma2_rn(make_float2(1.061405429f, 1.061405429f), tt,
                                       make_float2(-1.453152027f, -1.453152027f));
              poly = __ffma2_rn(poly, tt, make_float2(1.421413741f, 1.421413741f));
              poly = __ffma2_rn(poly, tt, make_float2(-0.284496736f, -0.284496736f));
              poly = __ffma2_rn(poly, tt, make_float2(0.254829592f, 0.254829592f));
              const float2 pt = __fmul2_rn(poly, tt);
              const float2 wv = __fmul2_rn(gg, __ffma2_rn(pt, inv_r, c2a2));
              const float2 qq = __fmul2_rn(make_float2(a.w, a2.w), make_float2(qa.w, qb.w));
              float2 fc = __fmul2_rn(__fmul2_rn(qq, inv_r2), wv);
              if (!(r2.x <= P.coul_rc2)) fc.x = 0.0f;
              if (!(r2.y <= P.coul_rc2)) fc.y = 0.0f;
              if constexpr (LJQ) fac = __fadd2_rn(fac, fc);
              else fac = fc;
            }
            const float2 fs = __fmul2_rn(fac, sc2);
            const float2 fx = __fmul2_rn(fs, dx), fy = __fmul2_rn(fs, dy), fz = __fmul2_rn(fs, dz);
            accum(ia, ja, fx.x, fy.x, fz.x);
            if (vb) accum(ib, jb, fx.y, fy.y, fz.y);
          }
        }
        if (ci < 32u) {
          atomicAdd(&S.fi[0][ci], sx);
          atomicAdd(&S.fi[1][ci], sy);
          atomicAdd(&S.fi[2][ci], sz);
        }
      };
      if (spc && !EV && !SCALED) {
        // the switched Lennard-Jones range stays scalar: packed, its live
        // values exceed the 64-register budget of this kernel
        if constexpr (SWITCH) math_pass(std::true_type{}, std::true_type{}, 0u, n_lj);
        else math_pass_2(std::true_type{}, 0u, n_lj);
        math_pass_2(std::false_type{}, n_lj, n_c);
      } else if (spc) {
        math_pass(std::true_type{}, std::true_type{}, 0u, n_lj);
        math_pass(std::true_type{}, std::false_type{}, n_lj, n_c);
      } else {
        math_pass(std::false_type{}, std::true_type{}, 0u, n_lj);
        math_pass(std::false_type{}, std::false_type{}, n_lj, n_c);
      }
      __syncwarp();
      ax += (long long)S.fi[0][lane] << P4_SHIFT;
      ay += (long long)S.fi[1][lane] << P4_SHIFT;
      az += (long long)S.fi[2][lane] << P4_SHIFT;
      const long long jx = ((long long)S.fj[0][lane] + S.fj[0][48 + lane]) << P4_SHIFT;
      const long long jy = ((long long)S.fj[1][lane] + S.fj[1][48 + lane]) << P4_SHIFT;
      const long long jz = ((long long)S.fj[2][lane] + S.fj[2][48 + lane]) << P4_SHIFT;
      if (self) {
        ax += jx;
        ay += jy;
        az += jz;
      } else if (jvalid) {
        red_add(&fp[0 * np_all + sj], jx);
        red_add(&fp[1 * np_all + sj], jy);
        red_add(&fp[2 * np_all + sj], jz);
      }
      if (EV) {
        ae += (long long)Ev[lane] << P4_ESHIFT;
        aw += (long long)Ev[32 + lane] << P4_ESHIFT;
        const long long je = (long long)Ev[64 + lane] << P4_ESHIFT;
        const long long jw = (long long)Ev[96 + lane] << P4_ESHIFT;
        if (self) {
          ae += je;
          aw += jw;
        } else if (jvalid) {
          red_add(&fp[3 * np_all + sj], je);
          red_add(&fp[4 * np_all + sj], jw);
        }
      }
    }
    if (ivalid) {
      red_add(&fp[0 * np_all + si], ax);
      red_add(&fp[1 * np_all + si], ay);
      red_add(&fp[2 * np_all + si], az);
      if (EV) {
        red_add(&fp[3 * np_all + si], ae);
        red_add(&fp[4 * np_all + si], aw);
      }
    }
  }
  if (EV) {
    // LJ energy total for the scalar split: one integer reduction per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) elj_fix += __shfl_xor_sync(0xFFFFFFFFu, elj_fix, o);
    if (lane == 0) red_add(e_lj_total, elj_fix);
  }
}

template <bool EV, bool SCALED, bool SWITCH>
int launch4_t(hb_forcefield *ff, cudaStream_t s, const PairParams &P) {
  size_t smem = (sizeof(float4) + sizeof(float)) * (size_t)P.n_types * P.n_types;
  const uint32_t chunk = (uint32_t)ff->pair_chunk;  // entries per work item
  const uint32_t chunks = hb_div_up(P.slab, chunk);
  const uint32_t items = P.n_tiles * chunks;
  // persistent (quota 0): pair_blocks_per_sm blocks of 4 warps per SM (at
  // most 8 fit), or fewer for small systems; with a quota of q items per
  // warp, enough blocks that every item is taken
  uint32_t grid, quota = 0xFFFFFFFFu;
  if (ff->pair_quota > 0) {
    quota = (uint32_t)ff->pair_quota;
    grid = hb_div_up(items, P4_WARPS * quota);
  } else {
    grid = std::min<uint32_t>((uint32_t)ff->sys->ctx->n_sm * (uint32_t)ff->pair_blocks_per_sm,
                              hb_div_up(items, P4_WARPS));
  }
  k_pair4<EV, SCALED, SWITCH, false><<<std::max(grid, 1u), P4_WARPS * 32, smem, s>>>(
      ff->d_tile_posq, ff->d_tile_type, ff->d_tile_center, ff->d_tile_nent, ff->d_entry_j,
      ff->d_entry_excl, ff->sys->d_box, ff->d_lj, ff->d_lj_invd, P, ff->d_fp, ff->d_sorted_ids,
      ff->d_excl_off, ff->d_excl_partner, ff->d_excl_scale, ff->d_work, chunks, chunk, quota,
      ff->d_acc, nullptr, 0u, 0u);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

// ---------------------------------------------------------------------
// Compacted form.  Per entry: (1) a distance pass, one lane per i-atom over
// the 32 rotations, leaves a 32-bit mask of rotations whose pair is within
// the cutoff; (2) the active pairs are listed in shared memory slot-major
// (every lane's first active pair, then every lane's second, ...) so that
// consecutive pairs belong to different i-atoms; (3) a math pass evaluates
// only listed pairs with all 32 lanes busy, and adds the pair force to the
// i and j accumulators in shared memory as int64 fixed point (atomic,
// order-independent, so repeat runs stay byte-identical).
// ---------------------------------------------------------------------
#define P2_WARPS 4

struct P2Warp {
  float4 ipos[32];
  float4 jpos[32];
  int itype[32];
  int jtype[32];
  uint32_t oi[32];
  uint32_t oj[32];
  uint32_t xm[32];
  unsigned long long fi[5][32];
  unsigned long long fj[5][32];
  uint16_t pairs[1024];
};

// EXACT: no single-periodic-copy shift (its rounding depends on the tile
// the pair was packed into); every pair takes the minimum image of pi - pj,
// so each pair force is a function of the two positions alone.
template <bool EV, bool SCALED, bool SWITCH, bool EXACT>
__global__ void __launch_bounds__(P2_WARPS * 32)
    k_pair2(const float4 *__restrict__ tile_posq, const int *__restrict__ tile_type,
            const float4 *__restrict__ center, const uint32_t *__restrict__ tile_nent,
            const uint32_t *__restrict__ entry_j, const uint32_t *__restrict__ entry_excl,
            const DBox *__restrict__ box, const float4 *__restrict__ lj_table, PairParams P,
            unsigned long long *__restrict__ fp, unsigned long long *__restrict__ e_lj_total,
            const uint32_t *__restrict__ sorted_ids, const uint32_t *__restrict__ eoff,
            const uint32_t *__restrict__ epart, const float2 *__restrict__ escale) {
  extern __shared__ float4 sm_lj2[];
  __shared__ P2Warp smw[P2_WARPS];
  const int nt2 = P.n_types * P.n_types;
  for (int k = threadIdx.x; k < nt2; k += blockDim.x) sm_lj2[k] = lj_table[k];
  __syncthreads();
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t I = blockIdx.x * P2_WARPS + w;
  if (I >= P.n_tiles) return;
  P2Warp &S = smw[w];
  constexpr int NC = EV ? 5 : 3;
  const DBox b = *box;
  const float4 c = center[I];
  const bool spc = !EXACT && ((int)c.w & 1) != 0;
  const uint32_t si = I * 32u + lane;
  const bool ivalid = si < P.n;
  float4 pi = tile_posq[si];
  if (ivalid) {
    if (spc) shift_to(pi.x, pi.y, pi.z, c, b);
  } else {
    pi = make_float4(-1.0e18f, -1.0e18f, -1.0e18f, 0.0f);
  }
  S.ipos[lane] = pi;
  S.itype[lane] = ivalid ? tile_type[si] : 0;
  if (SCALED) S.oi[lane] = ivalid ? sorted_ids[si] : HB_SENTINEL;
#pragma unroll
  for (int q = 0; q < NC; ++q) S.fi[q][lane] = 0ull;
  float elj = 0.0f;
  const uint32_t e0 = I * P.slab;
  const uint32_t e1 = e0 + min(tile_nent[I], P.slab);
  const bool has_self = P.n - I * 32u >= 2u;
  const uint32_t lt = (1u << lane) - 1u;

  for (uint32_t e = e0; e < e1; ++e) {
    const bool self = has_self && (e == e0);
    const uint32_t sj = entry_j[(uint64_t)e * 32u + lane];
    const uint32_t xm = entry_excl[(uint64_t)e * 32u + lane];
    const bool jvalid = sj != HB_SENTINEL;
    float4 pj;
    if (jvalid) {
      pj = tile_posq[sj];
      if (spc) shift_to(pj.x, pj.y, pj.z, c, b);
    } else {
      pj = make_float4(1.0e18f, 1.0e18f, 1.0e18f, 0.0f);
    }
    S.jpos[lane] = pj;
    S.jtype[lane] = jvalid ? tile_type[sj] : 0;
    if (SCALED) {
      S.oj[lane] = jvalid ? sorted_ids[sj] : HB_SENTINEL;
      S.xm[lane] = xm;
    }
#pragma unroll
    for (int q = 0; q < NC; ++q) S.fj[q][lane] = 0ull;
    __syncwarp();

    // (1) distance pass
    uint32_t mask = 0u;
    const int t0 = self ? 1 : 0, t1 = self ? 16 : 31;
    for (int t = t0; t <= t1; ++t) {
      const float4 q = S.jpos[(lane + t) & 31u];
      float dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
      if (!spc) hb_min_image(dx, dy, dz, b);
      const float r2 = dx * dx + dy * dy + dz * dz;
      bool act = r2 < P.rc2_max && (SCALED || !((xm >> t) & 1u));
      if (self && t == 16 && lane >= 16u) act = false;
      mask |= (act ? 1u : 0u) << t;
    }
    // padding slots take part in no pair, whatever their placeholder
    // coordinates give under the minimum image
    {
      const uint32_t jv_mask = __ballot_sync(0xFFFFFFFFu, jvalid);
      mask &= ivalid ? __funnelshift_r(jv_mask, jv_mask, lane) : 0u;
    }
    // (2) slot-major pair list
    const uint32_t maxcnt = __reduce_max_sync(0xFFFFFFFFu, (uint32_t)__popc(mask));
    uint32_t np = 0, m = mask;
    for (uint32_t slot = 0; slot < maxcnt; ++slot) {
      const bool has = m != 0u;
      const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
      if (has) {
        const uint32_t t = (uint32_t)__ffs(m) - 1u;
        m &= m - 1u;
        S.pairs[np + __popc(bal & lt)] = (uint16_t)((lane << 8) | t);
      }
      np += __popc(bal);
    }
    __syncwarp();
    // (3) math pass over the listed pairs
    for (uint32_t k = lane; k < np; k += 32u) {
      const uint32_t pr = S.pairs[k];
      const uint32_t i = pr >> 8, t = pr & 255u, j = (i + t) & 31u;
      const float4 a = S.ipos[i], q = S.jpos[j];
      float dx = a.x - q.x, dy = a.y - q.y, dz = a.z - q.z;
      if (!spc) hb_min_image(dx, dy, dz, b);
      const float r2 = dx * dx + dy * dy + dz * dz;
      float s_lj = 1.0f, s_c = 1.0f;
      if (SCALED && ((S.xm[i] >> t) & 1u)) {
        s_lj = 0.0f;
        s_c = 0.0f;
        const uint32_t oi = S.oi[i], oj = S.oj[j];
        for (uint32_t z = eoff[oj]; z < eoff[oj + 1]; ++z) {
          if (epart[z] == oi) {
            const float2 sc = escale[z];
            s_lj = sc.x;
            s_c = sc.y;
            break;
          }
        }
      }
      const float inv_r = rsqrtf(r2);
      const float inv_r2 = inv_r * inv_r;
      float fac = 0.0f, en = 0.0f;
      if (P.lj_on) {
        const float4 L = sm_lj2[S.itype[i] * P.n_types + S.jtype[j]];
        if (r2 <= L.z && L.y != 0.0f && s_lj != 0.0f) {
          const float sr2 = L.x * inv_r2;
          const float sr6 = sr2 * sr2 * sr2;
          const float sr12 = sr6 * sr6;
          float f = L.y * inv_r2 * (2.0f * sr12 - sr6);
          float u = (L.y * (1.0f / 6.0f)) * (sr12 - sr6);
          if (SWITCH && r2 > L.w && L.z > L.w) {
            const float inv_d = 1.0f / (L.z - L.w);
            const float tau = (r2 - L.w) * inv_d;
            const float omt = 1.0f - tau;
            const float sw = omt * omt * (1.0f + 2.0f * tau);
            const float chain = 12.0f * tau * omt * inv_d;
            f = sw * f + chain * u;
            u = sw * u;
          }
          fac += s_lj * f;
          if (EV) {
            en += s_lj * u;
            elj += s_lj * u;
          }
        }
      }
      if (P.coul_on && r2 <= P.coul_rc2 && s_c != 0.0f) {
        const float r = r2 * inv_r;
        const float ar = P.alpha * r;
        const float g = __expf(-ar * ar);
        const float tt = __fdividef(1.0f, 1.0f + 0.3275911f * ar);
        const float poly =
            0.254829592f +
            (-0.284496736f + (1.421413741f + (-1.453152027f + 1.061405429f * tt) * tt) * tt) * tt;
        const float erfc_ar = poly * tt * g;
        const float qq = a.w * q.w;
        fac += s_c * qq * inv_r2 * (erfc_ar * inv_r + P.c2a * g);
        if (EV) en += s_c * qq * erfc_ar * inv_r;
      }
      const long long fx = to_fixed(fac * dx), fy = to_fixed(fac * dy), fz = to_fixed(fac * dz);
      atomicAdd(&S.fi[0][i], (unsigned long long)fx);
      atomicAdd(&S.fi[1][i], (unsigned long long)fy);
      atomicAdd(&S.fi[2][i], (unsigned long long)fz);
      atomicAdd(&S.fj[0][j], (unsigned long long)(-fx));
      atomicAdd(&S.fj[1][j], (unsigned long long)(-fy));
      atomicAdd(&S.fj[2][j], (unsigned long long)(-fz));
      if (EV) {
        const long long he = to_fixed(0.5f * en), hw = to_fixed(0.5f * fac * r2);
        atomicAdd(&S.fi[3][i], (unsigned long long)he);
        atomicAdd(&S.fi[4][i], (unsigned long long)hw);
        atomicAdd(&S.fj[3][j], (unsigned long long)he);
        atomicAdd(&S.fj[4][j], (unsigned long long)hw);
      }
    }
    __syncwarp();
    if (self) {
#pragma unroll
      for (int q = 0; q < NC; ++q) S.fi[q][lane] += S.fj[q][lane];
    } else if (jvalid) {
      const size_t np_all = (size_t)P.n_tiles * 32u;
#pragma unroll
      for (int q = 0; q < NC; ++q) red_add(&fp[q * np_all + sj], (long long)S.fj[q][lane]);
    }
    __syncwarp();
  }
  if (ivalid) {
    const size_t np_all = (size_t)P.n_tiles * 32u;
#pragma unroll
    for (int q = 0; q < NC; ++q) red_add(&fp[q * np_all + si], (long long)S.fi[q][lane]);
  }
  if (EV) {
    long long v = to_fixed(elj);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) red_add(e_lj_total, v);
  }
}

template <bool EV, bool SCALED, bool SWITCH, bool EXACT>
int launch2_t(hb_forcefield *ff, cudaStream_t s, const PairParams &P) {
  size_t smem = sizeof(float4) * (size_t)P.n_types * P.n_types;
  k_pair2<EV, SCALED, SWITCH, EXACT><<<hb_div_up(P.n_tiles, P2_WARPS), P2_WARPS * 32, smem, s>>>(
      ff->d_tile_posq, ff->d_tile_type, ff->d_tile_center, ff->d_tile_nent, ff->d_entry_j,
      ff->d_entry_excl, ff->sys->d_box, ff->d_lj, P, ff->d_fp, ff->d_acc, ff->d_sorted_ids,
      ff->d_excl_off, ff->d_excl_partner, ff->d_excl_scale);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

}  // namespace

int pair_launch(hb_forcefield *ff, bool ev, cudaStream_t s) {
  if (ff->sys->n < 2 || ff->n_tiles == 0) return HB_OK;
  if (!ff->lj_on && !ff->coul_on) return HB_OK;
  PairParams P;
  P.n_types = (int)ff->n_types;
  P.lj_on = ff->lj_on;
  P.coul_on = ff->coul_on;
  P.rc2_max = ff->rc_max * ff->rc_max;
  P.coul_rc2 = ff->coul_rc2;
  P.alpha = ff->alpha;
  P.c2a = 2.0f * ff->alpha / 1.7724538509055160273f;
  P.n = ff->sys->n;
  P.n_tiles = ff->n_tiles;
  P.slab = ff->slab;
  const bool sc = ff->excl_scaled != 0, sw = ff->any_switch != 0;
  if (ff->exact_pairs) {
    if (ev) {
      if (sc) return sw ? launch2_t<true, true, true, true>(ff, s, P) : launch2_t<true, true, false, true>(ff, s, P);
      return sw ? launch2_t<true, false, true, true>(ff, s, P) : launch2_t<true, false, false, true>(ff, s, P);
    }
    if (sc) return sw ? launch2_t<false, true, true, true>(ff, s, P) : launch2_t<false, true, false, true>(ff, s, P);
    return sw ? launch2_t<false, false, true, true>(ff, s, P) : launch2_t<false, false, false, true>(ff, s, P);
  }
  if (ev) {
    if (sc) return sw ? launch4_t<true, true, true>(ff, s, P) : launch4_t<true, true, false>(ff, s, P);
    return sw ? launch4_t<true, false, true>(ff, s, P) : launch4_t<true, false, false>(ff, s, P);
  }
  if (sc) return sw ? launch4_t<false, true, true>(ff, s, P) : launch4_t<false, true, false>(ff, s, P);
  return sw ? launch4_t<false, false, true>(ff, s, P) : launch4_t<false, false, false>(ff, s, P);
}

// ---------------------------------------------------------------------
// Multi-system pair launch (replica batches): one persistent k_pair4 over
// the work items of every member, each item finding its member by a binary
// search of the members' first items.  Members must share the pair physics
// (types, tables, cut-offs, Ewald alpha, switch) and take the force-only,
// unscaled, tile-shifted form; their own lists, positions, cells and
// accumulators stay where they are.
// ---------------------------------------------------------------------
size_t pair_member_bytes() { return sizeof(PairMember); }

bool pair_batchable(hb_forcefield *const *ffs, uint32_t n) {
  if (n == 0) return false;
  const hb_forcefield *a = ffs[0];
  for (uint32_t k = 0; k < n; ++k) {
    const hb_forcefield *f = ffs[k];
    if (f->exact_pairs || f->excl_scaled || f->n_tiles == 0 || f->sys->n < 2) return false;
    if (f->lj_on != a->lj_on || f->coul_on != a->coul_on || f->any_switch != a->any_switch ||
        f->n_types != a->n_types || f->rc_max != a->rc_max || f->coul_rc2 != a->coul_rc2 ||
        f->alpha != a->alpha)
      return false;
    // the switch factors (lj_invd) follow from these tables
    if (f->h_lj.size() != a->h_lj.size()) return false;
    if (std::memcmp(f->h_lj.data(), a->h_lj.data(), sizeof(float4) * a->h_lj.size()) != 0) return false;
  }
  return a->lj_on || a->coul_on;
}

// the member table (host-built, copied synchronously: call outside capture)
int pair_batch_table(hb_forcefield *const *ffs, uint32_t n, void *d_table, uint32_t *items_total) {
  std::vector<PairMember> t(n);
  uint32_t item0 = 0;
  const uint32_t chunk = (uint32_t)ffs[0]->pair_chunk;
  for (uint32_t k = 0; k < n; ++k) {
    hb_forcefield *f = ffs[k];
    PairMember &m = t[k];
    std::memset(&m, 0, sizeof(m));
    m.tile_posq = f->d_tile_posq;
    m.tile_type = f->d_tile_type;
    m.center = f->d_tile_center;
    m.tile_nent = f->d_tile_nent;
    m.entry_j = f->d_entry_j;
    m.entry_excl = f->d_entry_excl;
    m.box = f->sys->d_box;
    m.fp = f->d_fp;
    m.n = f->sys->n;
    m.n_tiles = f->n_tiles;
    m.slab = f->slab;
    m.chunks = hb_div_up(f->slab, chunk);
    m.item0 = item0;
    item0 += m.n_tiles * m.chunks;
  }
  HB_CUDA(cudaMemcpy(d_table, t.data(), sizeof(PairMember) * n, cudaMemcpyHostToDevice));
  *items_total = item0;
  return HB_OK;
}

int pair_launch_batch(hb_forcefield *const *ffs, uint32_t n, const void *d_table,
                      uint32_t items_total, uint32_t *d_work, cudaStream_t s) {
  const hb_forcefield *a = ffs[0];
  PairParams P;
  std::memset(&P, 0, sizeof(P));
  P.n_types = (int)a->n_types;
  P.lj_on = a->lj_on;
  P.coul_on = a->coul_on;
  P.rc2_max = a->rc_max * a->rc_max;
  P.coul_rc2 = a->coul_rc2;
  P.alpha = a->alpha;
  P.c2a = 2.0f * a->alpha / 1.7724538509055160273f;
  size_t smem = (sizeof(float4) + sizeof(float)) * (size_t)P.n_types * P.n_types;
  const uint32_t grid = std::min<uint32_t>(
      (uint32_t)a->sys->ctx->n_sm * (uint32_t)a->pair_blocks_per_sm, hb_div_up(items_total, P4_WARPS));
  HB_CUDA(cudaMemsetAsync(d_work, 0, sizeof(uint32_t), s));
  const PairMember *tab = static_cast<const PairMember *>(d_table);
  if (a->any_switch)
    k_pair4<false, false, true, true><<<std::max(grid, 1u), P4_WARPS * 32, smem, s>>>(
        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, a->sys->d_box, a->d_lj, a->d_lj_invd, P,
        nullptr, nullptr, nullptr, nullptr, nullptr, d_work, 1u, (uint32_t)a->pair_chunk, 0xFFFFFFFFu,
        nullptr, tab, n, items_total);
  else
    k_pair4<false, false, false, true><<<std::max(grid, 1u), P4_WARPS * 32, smem, s>>>(
        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, a->sys->d_box, a->d_lj, a->d_lj_invd, P,
        nullptr, nullptr, nullptr, nullptr, nullptr, d_work, 1u, (uint32_t)a->pair_chunk, 0xFFFFFFFFu,
        nullptr, tab, n, items_total);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}
