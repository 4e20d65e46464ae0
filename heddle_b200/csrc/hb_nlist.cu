// hb_nlist.cu -- packed neighbour list for the B200 force path.
//
// Replaces the reference's cell list + packed-neighbour construction
// (kernels/neighbor.cu:95-724, src/forces/neighbor_list.rs:945-1354) with a
// design of its own:
//   * atoms are counting-sorted into a 2^k-per-axis voxel grid walked in
//     Hilbert order, ties broken by atom id, so every 32 consecutive sorted
//     atoms form a compact tile and the order is deterministic (a Hilbert
//     walk never jumps between voxels, so its runs are more compact than
//     Morton runs: on liquid water about 10% fewer atoms lie within
//     r_search of a tile, which is 10% less pair-kernel work);
//   * all per-step force work runs in this sorted-slot space (positions are
//     gathered once per step, forces are scattered back once);
//   * one block per i-tile sweeps j-tiles J > I through an AABB prune, keeps
//     every j-atom within r_search of any i-atom, and deals them round-robin
//     into entries of 32 together with a 32-bit exclusion mask per j-atom
//     (bit m: the pair with i-atom m is in the exclusion list), so the pair
//     kernel never scans exclusion lists for ordinary pairs;
//   * the self tile is entry 0 of each i-tile and is evaluated with a half
//     rotation (each unordered pair once);
//   * entries live in a fixed-size slab per i-tile (sized from a counting
//     pass at the first build), so a rebuild is one pass and the layout is
//     identical run to run;
//   * a j-atom is refined against the 32 i-atoms only when it lies within
//     r_search of the i-tile's box (one test prunes most far atoms);
//   * every rebuild kernel is gated on the device status word, so a rebuild
//     is decided on the device each step with no host read.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "hb_internal.cuh"

namespace {

__device__ __forceinline__ bool gate_off(const uint32_t *gate) {
  return gate != nullptr && ((*(volatile const uint32_t *)gate) & HB_ST_DISPLACED) == 0u;
}

// ---- bulk-copy staging of candidate tiles (cp.async.bulk, TMA engine) ----
__device__ __forceinline__ uint32_t nl_smem(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void nl_mbar_init(uint64_t *m) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(nl_smem(m)) : "memory");
}

// one 16-byte-aligned tile of 32 float4 (512 B) from global memory into
// shared memory; completion (bytes) is signalled on the mbarrier
__device__ __forceinline__ void nl_bulk_tile(void *dst, const void *src, uint64_t *m, bool issue) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], 512;" ::"r"(nl_smem(m)) : "memory");
  if (issue)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 512, [%2];" ::"r"(
            nl_smem(dst)),
        "l"(src), "r"(nl_smem(m))
        : "memory");
}

// bounded wait for phase `ph` of the mbarrier: false when `polls` tries
// (each may suspend briefly) run out
__device__ __forceinline__ bool nl_mbar_wait(uint64_t *m, uint32_t ph, uint32_t polls) {
  for (uint32_t i = 0; i < polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(nl_smem(m)), "r"(ph)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Index of voxel (x, y, z) along the 3-D Hilbert curve of order `bits`,
// by J. Skilling's transpose method ("Programming the Hilbert curve", AIP
// Conf. Proc. 707, 2004): undo the excess rotations level by level, Gray
// encode, then interleave the transposed bits (x most significant).
__device__ __forceinline__ uint32_t hilbert_key(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t X[3] = {x, y, z};
  for (uint32_t q = 1u << (bits - 1); q > 1u; q >>= 1) {
    const uint32_t p = q - 1u;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & q) {
        X[0] ^= p;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & p;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  uint32_t t = 0u;
  for (uint32_t q = 1u << (bits - 1); q > 1u; q >>= 1)
    if (X[2] & q) t ^= q - 1u;
  X[0] ^= t;
  X[1] ^= t;
  X[2] ^= t;
  uint32_t h = 0u;
  for (int b = bits - 1; b >= 0; --b)
    h = (h << 3) | (((X[0] >> b) & 1u) << 2) | (((X[1] >> b) & 1u) << 1) | ((X[2] >> b) & 1u);
  return h;
}

__global__ void k_vox_hist(const uint32_t *gate, const float4 *__restrict__ posq,
                           const DBox *__restrict__ box, int nv_log2,
                           uint32_t *__restrict__ key, uint32_t *__restrict__ count,
                           uint32_t n) {
  if (gate_off(gate)) return;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DBox b = *box;
  float4 p = posq[i];
  float sa, sb, sc;
  hb_frac(p.x, p.y, p.z, b, sa, sb, sc);
  const int nv = 1 << nv_log2;
  int v[3];
  float s[3] = {sa, sb, sc};
  for (int d = 0; d < 3; ++d) {
    float u = s[d] + 0.5f;
    u -= floorf(u);
    int c = (int)(u * (float)nv);
    v[d] = c < 0 ? 0 : (c >= nv ? nv - 1 : c);
  }
  const uint32_t k = hilbert_key((uint32_t)v[0], (uint32_t)v[1], (uint32_t)v[2], nv_log2);
  key[i] = k;
  atomicAdd(&count[k], 1u);
}

// ---- three-phase exclusive scan (integer, deterministic) ----
__global__ void __launch_bounds__(1024) k_scan_block(const uint32_t *gate, const uint32_t *in,
                                                     uint32_t *out, uint32_t *bsum,
                                                     uint32_t len) {
  if (gate_off(gate)) return;
  __shared__ uint32_t ws[32];
  uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t i = blockIdx.x * 1024u + threadIdx.x;
  uint32_t v = i < len ? in[i] : 0u;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if ((int)lane >= o) x += y;
  }
  if (lane == 31u) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if ((int)lane >= o) w += y;
    }
    ws[lane] = w;
  }
  __syncthreads();
  if (warp > 0) x += ws[warp - 1];
  if (i < len) out[i] = x - v;
  if (threadIdx.x == 1023u) bsum[blockIdx.x] = x;
}

__global__ void __launch_bounds__(1024) k_scan_top(const uint32_t *gate, uint32_t *bsum,
                                                   uint32_t nb) {
  if (gate_off(gate)) return;
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0u;
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += 1024u) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < nb ? bsum[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if ((int)lane >= o) x += y;
    }
    if (lane == 31u) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = ws[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
        if ((int)lane >= o) w += y;
      }
      ws[lane] = w;
    }
    __syncthreads();
    if (warp > 0) x += ws[warp - 1];
    uint32_t c = carry;
    if (i < nb) bsum[i] = c + x - v;
    __syncthreads();
    if (threadIdx.x == 1023u) carry = c + x;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(1024) k_scan_add(const uint32_t *gate, uint32_t *out,
                                                   const uint32_t *bsum, uint32_t len) {
  if (gate_off(gate)) return;
  uint32_t i = blockIdx.x * 1024u + threadIdx.x;
  if (i < len && blockIdx.x > 0) out[i] += bsum[blockIdx.x];
}

// Scatter atoms to their voxel ranges.  atomicSub on the histogram hands
// out slots (in an arbitrary order) and leaves the histogram at zero for
// the next rebuild; k_vox_sort then orders each voxel by atom id.
__global__ void k_vox_scatter(const uint32_t *gate, const uint32_t *__restrict__ key,
                              const uint32_t *__restrict__ off, uint32_t *count,
                              uint32_t *__restrict__ sorted_ids, uint32_t n) {
  if (gate_off(gate)) return;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = key[i];
  uint32_t slot = atomicSub(&count[k], 1u) - 1u;
  sorted_ids[off[k] + slot] = i;
}

__global__ void k_vox_sort(const uint32_t *gate, const uint32_t *__restrict__ off,
                           uint32_t *sorted_ids, uint32_t n_vox) {
  if (gate_off(gate)) return;
  uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_vox) return;
  uint32_t s = off[v], e = off[v + 1];
  for (uint32_t k = s + 1; k < e; ++k) {
    uint32_t key = sorted_ids[k];
    int p = (int)k - 1;
    while (p >= (int)s && sorted_ids[p] > key) {
      sorted_ids[p + 1] = sorted_ids[p];
      --p;
    }
    sorted_ids[p + 1] = key;
  }
}

// Fill the sorted-slot views and the displacement reference.
__global__ void k_tile_fill(const uint32_t *gate, uint32_t *sorted_ids,
                            const float4 *__restrict__ posq, const int4 *__restrict__ image,
                            uint32_t *__restrict__ inv_perm, float4 *__restrict__ tile_posq,
                            int *__restrict__ tile_type, float4 *__restrict__ ref_pos,
                            uint32_t n, uint32_t n_pad) {
  if (gate_off(gate)) return;
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_pad) return;
  if (k < n) {
    uint32_t id = sorted_ids[k];
    inv_perm[id] = k;
    float4 p = posq[id];
    tile_posq[k] = p;
    tile_type[k] = image[id].w;
    ref_pos[id] = p;
  } else {
    sorted_ids[k] = HB_SENTINEL;
    tile_posq[k] = make_float4(1.0e18f, 1.0e18f, 1.0e18f, 0.0f);
    tile_type[k] = 0;
  }
}

// Per-tile axis-aligned box (one warp per tile).  centre.w = 1 when the
// single-periodic-copy shortcut is valid for the tile until the next
// rebuild: half + r_skin / 2 + rc_max <= L / 2 on every axis of an
// orthorhombic box (the condition of jit_composed.rs:1577-1607 with the
// skin margin added, because atoms drift between rebuilds).
__global__ void k_tile_bbox(const uint32_t *gate, const float4 *__restrict__ tile_posq,
                            const DBox *__restrict__ box, float rc_max, float r_skin,
                            float4 *__restrict__ center, float4 *__restrict__ half, uint32_t n,
                            uint32_t n_tiles) {
  if (gate_off(gate)) return;
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31u;
  if (warp >= n_tiles) return;
  uint32_t k = warp * 32u + lane;
  bool valid = k < n;
  float4 p = tile_posq[k];
  float lo[3] = {valid ? p.x : 3.0e38f, valid ? p.y : 3.0e38f, valid ? p.z : 3.0e38f};
  float hi[3] = {valid ? p.x : -3.0e38f, valid ? p.y : -3.0e38f, valid ? p.z : -3.0e38f};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xFFFFFFFFu, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xFFFFFFFFu, hi[d], o));
    }
  }
  if (lane == 0) {
    DBox b = *box;
    float c[3], h[3];
    for (int d = 0; d < 3; ++d) {
      c[d] = 0.5f * (lo[d] + hi[d]);
      h[d] = 0.5f * (hi[d] - lo[d]);
    }
    // the margin also covers a cell scaled by up to HB_BOX_SLACK before the
    // next rebuild (atoms move by up to that fraction of the half width)
    float m = 0.5f * r_skin + rc_max;
    const float hw = 0.5f - HB_BOX_SLACK;
    bool spc = b.ortho && (h[0] + m <= hw * b.lx) && (h[1] + m <= hw * b.ly) &&
               (h[2] + m <= hw * b.lz);
    // bit 0: single periodic copy; bit 1: per-axis minimum-image box tests
    // are exact (orthorhombic cell)
    const int flags = (spc ? 1 : 0) | (b.ortho ? 2 : 0);
    center[warp] = make_float4(c[0], c[1], c[2], (float)flags);
    half[warp] = make_float4(h[0], h[1], h[2], 0.0f);
  }
}

// Exclusion mask of one j-atom against the 32 slots of i-tile I.
__device__ __forceinline__ uint32_t excl_mask(uint32_t sj, uint32_t I,
                                              const uint32_t *__restrict__ sorted_ids,
                                              const uint32_t *__restrict__ inv_perm,
                                              const uint32_t *__restrict__ eoff,
                                              const uint32_t *__restrict__ epart) {
  if (eoff == nullptr || sj == HB_SENTINEL) return 0u;
  uint32_t oj = sorted_ids[sj];
  uint32_t m = 0u;
  uint32_t lo = I * 32u;
  for (uint32_t q = eoff[oj]; q < eoff[oj + 1]; ++q) {
    uint32_t sp = inv_perm[epart[q]];
    if (sp >= lo && sp < lo + 32u) m |= 1u << (sp - lo);
  }
  return m;
}

#define NLT_WARPS 8
#define NLT_SWEEP 4  // 32-tile groups per warp and block step of the candidate sweep

// k-th set bit (0-based) of a 32-bit mask
// (k < popc(m)), by a binary search on the popcounts of low halves
__device__ __forceinline__ uint32_t select_bit(uint32_t m, uint32_t k) {
  uint32_t pos = 0u;
#pragma unroll
  for (uint32_t w = 16u; w > 0u; w >>= 1) {
    const uint32_t c = (uint32_t)__popc(m & ((1u << w) - 1u));
    if (k >= c) {
      k -= c;
      m >>= w;
      pos += w;
    }
  }
  return pos;
}

// Packed-entry construction, one 256-thread block per i-tile I:
//  1. the block sweeps j-tiles J > I in order, keeping those whose box lies
//     within r_search of I's box (candidate list in shared memory);
//  2. each warp takes candidates and computes a 32-bit hit mask: bit l is
//     set when j-atom l of the candidate lies within r_search of any i-atom.
//     Far from the r_search boundary a j-atom shifted once to the image
//     nearest I's centre decides with plain differences; inside a 1e-4
//     relative band the exact single-precision rule decides.  With the
//     single shift, only the j-atoms within r_search of one of the i-tile's
//     8-atom sub-tile boxes are refined, one at a time, with the lanes as
//     i-atoms and one vote per j-atom;
//  3. a prefix sum of the masks' popcounts fixes where every hit goes;
//  4. the warps write the entries (self tile first) into I's slab, each
//     with the exclusion masks of its 32 j-atoms.
// WRITE = false only counts entries and candidates (first-build sizing).
template <bool WRITE>
__global__ void __launch_bounds__(NLT_WARPS * 32, 4)
    k_nl_tile(const uint32_t *gate, const float4 *__restrict__ tile_posq,
              const float4 *__restrict__ center, const float4 *__restrict__ half,
              const DBox *__restrict__ box, float rs2, float rb, float band_lo, float band_hi,
              uint32_t n, uint32_t n_tiles, uint32_t maxc, uint32_t *__restrict__ tile_nent,
              uint32_t slab, uint32_t *__restrict__ entry_j, uint32_t *__restrict__ entry_excl,
              uint32_t *__restrict__ status, uint32_t *__restrict__ counters,
              const uint32_t *__restrict__ sorted_ids, const uint32_t *__restrict__ inv_perm,
              const uint32_t *__restrict__ eoff, const uint32_t *__restrict__ epart,
              uint32_t polls, uint32_t issue) {
  if (gate_off(gate)) return;
  extern __shared__ uint32_t sm_nl[];
  uint32_t *cand = sm_nl;             // [maxc] candidate j-tiles
  uint32_t *hmask = sm_nl + maxc;     // [maxc] hit masks
  uint32_t *pre = hmask + maxc;       // [maxc + 1] exclusive prefix of hits
  __shared__ uint32_t s_cnt[NLT_WARPS];
  __shared__ uint32_t s_ncand;
  __shared__ float4 s_jsh[NLT_WARPS][32], s_jor[NLT_WARPS][32];  // a candidate's j-atoms: shifted, as stored
  // per warp, two candidate tiles in flight: bulk copies (TMA engine) fill
  // one buffer while the warp refines the other
  __shared__ __align__(128) float4 s_jt[NLT_WARPS][2][32];
  __shared__ __align__(8) uint64_t s_mbar[NLT_WARPS][2];
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t I = blockIdx.x;
  const DBox b = *box;
  const float4 ci = center[I], hi = half[I];
  const bool ortho = ((int)ci.w & 2) != 0;
  const float rb2 = rb * rb;
  // corner distance^2 below which a sub-tile's atoms all lie inside the
  // plain-hit band (a relative margin far above the rounding of the boxes
  // and of the distances)
  const float acc2 = band_lo * (1.0f - 1.0e-5f);
  if (threadIdx.x == 0) s_ncand = 0u;
  __syncthreads();

  // 1. ordered candidate sweep, NLT_SWEEP x 32 tiles per warp per block
  // step (warp w takes the w-th run of them, its lanes one 32-tile group
  // after another, so the list stays in tile order)
  auto box_near = [&](uint32_t J) {
    if (J >= n_tiles) return false;
    if (!ortho) return true;
    const float4 cj = center[J], hj = half[J];
    float dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
    hb_min_image(dx, dy, dz, b);
    const float ex = fmaxf(fabsf(dx) - (hi.x + hj.x), 0.0f);
    const float ey = fmaxf(fabsf(dy) - (hi.y + hj.y), 0.0f);
    const float ez = fmaxf(fabsf(dz) - (hi.z + hj.z), 0.0f);
    return ex * ex + ey * ey + ez * ez <= rb2;
  };
  for (uint32_t base = I + 1u; base < n_tiles; base += 32u * NLT_SWEEP * NLT_WARPS) {
    const uint32_t J0 = base + w * 32u * NLT_SWEEP + lane;
    uint32_t bal[NLT_SWEEP];
    uint32_t tot = 0u;
#pragma unroll
    for (int q = 0; q < NLT_SWEEP; ++q) {
      bal[q] = __ballot_sync(0xFFFFFFFFu, box_near(J0 + 32u * q));
      tot += __popc(bal[q]);
    }
    if (lane == 0) s_cnt[w] = tot;
    __syncthreads();
    uint32_t off = s_ncand;
    for (uint32_t k = 0; k < w; ++k) off += s_cnt[k];
    const uint32_t below = (1u << lane) - 1u;
#pragma unroll
    for (int q = 0; q < NLT_SWEEP; ++q) {
      if ((bal[q] >> lane) & 1u) {
        const uint32_t pos = off + __popc(bal[q] & below);
        if (pos < maxc) cand[pos] = J0 + 32u * q;
      }
      off += __popc(bal[q]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = s_ncand;
      for (uint32_t k = 0; k < NLT_WARPS; ++k) t += s_cnt[k];
      s_ncand = t;
    }
    __syncthreads();
  }
  const uint32_t ncand_all = s_ncand;
  const uint32_t ncand = ncand_all < maxc ? ncand_all : maxc;

  // 2. hit masks; i-atoms stay in registers and are broadcast by shuffles
  const uint32_t ki = I * 32u + lane;
  const float4 pim = tile_posq[ki];
  const uint32_t ivalid = __ballot_sync(0xFFFFFFFFu, ki < n);
  const bool shift_ok = ortho && (hi.x + rb <= 0.5f * b.lx) && (hi.y + rb <= 0.5f * b.ly) &&
                        (hi.z + rb <= 0.5f * b.lz);
  // With the single shift, the tile's four 8-atom sub-tiles (lanes 8q..8q+7)
  // get their own boxes: a j-atom is refined only against the atoms of the
  // sub-tiles whose box lies within r_search (plus the rounding margin), so
  // a j-atom near one corner of the tile costs 8 or 16 tests instead of 32.
  // Every pair within r_search lies in the box of its i-atom's sub-tile, so
  // the hits are those of the full refinement.
  float sc[4][3], sh[4][3];
  if (shift_ok) {
    const bool iv = ki < n;
    float lo3[3] = {iv ? pim.x : 3.0e38f, iv ? pim.y : 3.0e38f, iv ? pim.z : 3.0e38f};
    float hi3[3] = {iv ? pim.x : -3.0e38f, iv ? pim.y : -3.0e38f, iv ? pim.z : -3.0e38f};
#pragma unroll
    for (int o = 1; o < 8; o <<= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo3[d] = fminf(lo3[d], __shfl_xor_sync(0xFFFFFFFFu, lo3[d], o));
        hi3[d] = fmaxf(hi3[d], __shfl_xor_sync(0xFFFFFFFFu, hi3[d], o));
      }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float l = __shfl_sync(0xFFFFFFFFu, lo3[d], 8 * q);
        const float h = __shfl_sync(0xFFFFFFFFu, hi3[d], 8 * q);
        sc[q][d] = 0.5f * (l + h);
        sh[q][d] = h >= l ? 0.5f * (h - l) : -1.0f;  // empty sub-tile: never near
      }
  }
  // candidate tiles are staged by bulk copies one candidate ahead; a wait
  // that runs out sets HB_ST_DEVICE_TIMEOUT (the host returns
  // HB_ERR_DEVICE_TIMEOUT), drains the copies still in flight and stops
  if (lane == 0) {
    nl_mbar_init(&s_mbar[w][0]);
    nl_mbar_init(&s_mbar[w][1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (w < ncand) nl_bulk_tile(s_jt[w][0], tile_posq + (size_t)cand[w] * 32u, &s_mbar[w][0], issue != 0);
  }
  __syncwarp();
  uint32_t ph0 = 0u, ph1 = 0u, k_it = 0u;
  bool timed_out = false;
  for (uint32_t c = w; c < ncand; c += NLT_WARPS, ++k_it) {
    const uint32_t buf = k_it & 1u;
    const uint32_t cn = c + NLT_WARPS;
    if (lane == 0 && cn < ncand) {
      // the other buffer was last read in the previous candidate (all lanes
      // passed the __syncwarp at its end): order those reads before the
      // async-proxy write
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      nl_bulk_tile(s_jt[w][buf ^ 1u], tile_posq + (size_t)cand[cn] * 32u, &s_mbar[w][buf ^ 1u], issue != 0);
    }
    const bool ok = nl_mbar_wait(&s_mbar[w][buf], buf ? ph1 : ph0, polls);
    if (!__all_sync(0xFFFFFFFFu, ok)) {
      timed_out = true;
      break;
    }
    if (buf) ph1 ^= 1u;
    else ph0 ^= 1u;
    const uint32_t kj = cand[c] * 32u + lane;
    const bool jvalid = kj < n;
    const float4 pj = s_jt[w][buf][lane];
    float sx = pj.x, sy = pj.y, sz = pj.z;
    if (shift_ok) {
      sx -= b.lx * rintf((sx - ci.x) * b.ilx);
      sy -= b.ly * rintf((sy - ci.y) * b.ily);
      sz -= b.lz * rintf((sz - ci.z) * b.ilz);
    }
    if (shift_ok) {
      uint32_t qm = 0u;
      bool inside = false;
      if (jvalid) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float ax = fabsf(sx - sc[q][0]), ay = fabsf(sy - sc[q][1]),
                      az = fabsf(sz - sc[q][2]);
          const float ex = fmaxf(ax - sh[q][0], 0.0f);
          const float ey = fmaxf(ay - sh[q][1], 0.0f);
          const float ez = fmaxf(az - sh[q][2], 0.0f);
          if (sh[q][0] >= 0.0f && ex * ex + ey * ey + ez * ez <= rb2) qm |= 1u << q;
          // the box's farthest corner well inside the band: every i-atom of
          // the (non-empty) sub-tile is, so the vote would find a plain hit
          const float fx = ax + sh[q][0], fy = ay + sh[q][1], fz = az + sh[q][2];
          if (sh[q][0] >= 0.0f && fx * fx + fy * fy + fz * fz < acc2) inside = true;
        }
      }
      // the j-atoms near a sub-tile box are refined one at a time with the
      // lanes as i-atoms: each lane tests its own i-atom against the
      // broadcast j-atom and one vote decides (padding i-slots sit at 1e18
      // and never hit); the exact rule runs only when some pair falls in
      // the band.  The j-atoms found inside a sub-tile's reach above need
      // no vote.
      const uint32_t sure = __ballot_sync(0xFFFFFFFFu, inside);
      uint32_t rem = __ballot_sync(0xFFFFFFFFu, qm != 0u && !inside);
      s_jsh[w][lane] = make_float4(sx, sy, sz, 0.0f);
      s_jor[w][lane] = pj;
      __syncwarp();
      // two near j-atoms per step in the packed FP32x2 pipe (plain
      // distances only decide far from the band, so their rounding is free)
      uint32_t hm = sure;
      const float2 px2 = make_float2(pim.x, pim.x), py2 = make_float2(pim.y, pim.y),
                   pz2 = make_float2(pim.z, pim.z);
      auto vote = [&](uint32_t jl, float r2) {
        bool hit = __any_sync(0xFFFFFFFFu, r2 < band_lo);
        const bool inb = r2 >= band_lo && r2 <= band_hi;
        if (!hit && __any_sync(0xFFFFFFFFu, inb)) {
          const float4 qo = s_jor[w][jl];
          const bool ex = inb && hb_exact_r2(pim.x - qo.x, pim.y - qo.y, pim.z - qo.z, b) <= rs2;
          hit = __any_sync(0xFFFFFFFFu, ex);
        }
        if (hit) hm |= 1u << jl;
      };
      while (rem != 0u) {
        const uint32_t ja = (uint32_t)__ffs(rem) - 1u;
        rem &= rem - 1u;
        const bool two = rem != 0u;
        const uint32_t jb = two ? (uint32_t)__ffs(rem) - 1u : ja;
        rem &= rem - 1u;
        const float4 qa = s_jsh[w][ja], qb = s_jsh[w][jb];
        const float2 dx = __fadd2_rn(px2, make_float2(-qa.x, -qb.x));
        const float2 dy = __fadd2_rn(py2, make_float2(-qa.y, -qb.y));
        const float2 dz = __fadd2_rn(pz2, make_float2(-qa.z, -qb.z));
        float2 r2 = __fmul2_rn(dx, dx);
        r2 = __ffma2_rn(dy, dy, r2);
        r2 = __ffma2_rn(dz, dz, r2);
        vote(ja, r2.x);
        if (two) vote(jb, r2.y);
      }
      __syncwarp();
      if (lane == 0) hmask[c] = hm;
      continue;
    }
    bool near = jvalid;
    if (near && ortho) {
      float dx = sx - ci.x, dy = sy - ci.y, dz = sz - ci.z;
      hb_min_image(dx, dy, dz, b);
      const float ex = fmaxf(fabsf(dx) - hi.x, 0.0f);
      const float ey = fmaxf(fabsf(dy) - hi.y, 0.0f);
      const float ez = fmaxf(fabsf(dz) - hi.z, 0.0f);
      near = ex * ex + ey * ey + ez * ez <= rb2;
    }
    bool hit = false;
    uint32_t open = __ballot_sync(0xFFFFFFFFu, near);
    for (uint32_t m = 0; m < 32u && open != 0u; ++m) {
      const float xi = __shfl_sync(0xFFFFFFFFu, pim.x, m);
      const float yi = __shfl_sync(0xFFFFFFFFu, pim.y, m);
      const float zi = __shfl_sync(0xFFFFFFFFu, pim.z, m);
      if (near && !hit && ((ivalid >> m) & 1u)) {
        float dx = xi - sx, dy = yi - sy, dz = zi - sz;
        hb_min_image(dx, dy, dz, b);
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < band_lo) {
          hit = true;
        } else if (r2 <= band_hi && hb_exact_r2(xi - pj.x, yi - pj.y, zi - pj.z, b) <= rs2) {
          hit = true;
        }
      }
      open = __ballot_sync(0xFFFFFFFFu, near && !hit);
    }
    const uint32_t hm = __ballot_sync(0xFFFFFFFFu, hit);
    if (lane == 0) hmask[c] = hm;
    __syncwarp();
  }
  if (timed_out) {
    // the copies still in flight land before the block's shared memory is
    // released: one more bounded wait on each buffer's pending phase
    if (lane == 0) {
      atomicOr(status, HB_ST_DEVICE_TIMEOUT);
      nl_mbar_wait(&s_mbar[w][0], ph0, polls);
      nl_mbar_wait(&s_mbar[w][1], ph1, polls);
    }
  }
  __syncthreads();
  if (__syncthreads_or(timed_out ? 1 : 0)) return;

  // 3. exclusive prefix of the hit counts (one warp)
  if (w == 0) {
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < ncand; c0 += 32u) {
      const uint32_t c = c0 + lane;
      const uint32_t v = c < ncand ? __popc(hmask[c]) : 0u;
      uint32_t x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if ((int)lane >= o) x += y;
      }
      if (c < ncand) pre[c] = carry + x - v;
      carry += __shfl_sync(0xFFFFFFFFu, x, 31);
    }
    if (lane == 0) pre[ncand] = carry;
  }
  __syncthreads();
  const uint32_t H = pre[ncand];
  const uint32_t has_self = (n - I * 32u >= 2u) ? 1u : 0u;
  const uint32_t nent = has_self + (H + 31u) / 32u;

  // 4. entries.  Hits are dealt round-robin over the tile's entries (hit h
  // goes to entry h mod E, lane h / E), so every entry samples the whole
  // shell of candidates around the i-tile and the pairs inside the cutoff
  // spread evenly over the i-lanes instead of piling onto the lanes nearest
  // one spatial cluster of j-atoms.
  if (WRITE) {
    const uint32_t E = (H + 31u) / 32u;
    for (uint32_t e = w; e < nent && e < slab; e += NLT_WARPS) {
      uint32_t sj = HB_SENTINEL;
      if (has_self && e == 0) {
        if (ki < n) sj = ki;
      } else {
        const uint32_t h = (e - has_self) + lane * E;
        if (h < H) {
          uint32_t lo = 0, hiidx = ncand;  // largest c with pre[c] <= h
          while (hiidx - lo > 1u) {
            const uint32_t mid = (lo + hiidx) >> 1;
            if (pre[mid] <= h) lo = mid;
            else hiidx = mid;
          }
          sj = cand[lo] * 32u + select_bit(hmask[lo], h - pre[lo]);
        }
      }
      const uint64_t slot = ((uint64_t)I * slab + e) * 32u + lane;
      entry_j[slot] = sj;
      // stored in the i-lane's rotation order: bit t of lane l's word says
      // whether i-atom l and the j-atom of lane (l + t) mod 32 are excluded
      const uint32_t jm = excl_mask(sj, I, sorted_ids, inv_perm, eoff, epart);
      uint32_t im = 0u;
      if (__any_sync(0xFFFFFFFFu, jm != 0u)) {
        for (uint32_t t = 0; t < 32u; ++t) {
          const uint32_t m = __shfl_sync(0xFFFFFFFFu, jm, (lane + t) & 31u);
          im |= ((m >> lane) & 1u) << t;
        }
      }
      entry_excl[slot] = im;
    }
  }
  if (threadIdx.x == 0) {
    tile_nent[I] = nent;
    atomicMax(&counters[3], ncand_all);
    if (WRITE) {
      atomicAdd(&counters[2], nent);
      if (nent > slab || ncand_all > maxc) atomicOr(status, HB_ST_ENTRY_OVERFLOW);
      else if (4u * nent > 3u * slab) atomicOr(status, HB_ST_ENTRY_HIGHWATER);
    }
  }
}

// Last kernel of a rebuild: counters, and clearing of the displacement bit
// (which gates every kernel of the rebuild).
__global__ void k_nl_finish(const uint32_t *gate, uint32_t *status, uint32_t *counters,
                            const DBox *__restrict__ box, DBox *__restrict__ ref_box) {
  if (gate_off(gate)) return;
  *ref_box = *box;
  *status &= ~HB_ST_DISPLACED;
  counters[0] += 1u;
  counters[1] = counters[2];
  counters[2] = 0u;
}

// The list built at reference positions x0 in cell L0 holds every pair
// within r_c while each atom stays within r_skin / 2 of x0.  A barostat
// scales the cell (and the positions about the origin): for an isotropic
// scaling L = mu L0 with |mu - 1| <= HB_BOX_SLACK the test is against the
// scaled reference mu x0, and a pair within r_c now was within
// (r_c + 2 d) / mu of its reference separation, so the bound on each
// atom's displacement d becomes min(r_skin, mu (r_c + r_skin) - r_c) / 2.
// Any other change of the cell (a shear, a larger scaling, set_box to a new
// shape) invalidates the list.
__global__ void k_disp_check(const float4 *__restrict__ posq, const float4 *__restrict__ ref,
                             const DBox *__restrict__ box, const DBox *__restrict__ ref_box,
                             float r_skin, float rc_max, uint32_t *status, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const DBox a = *box, r = *ref_box;
  const float mu = a.lx / r.lx;  // r.lx = 0 before the first build: not finite
  const float tol = 1.0e-6f * a.lx;
  const bool iso = isfinite(mu) && fabsf(mu - 1.0f) <= HB_BOX_SLACK &&
                   fabsf(a.ly - mu * r.ly) <= tol && fabsf(a.lz - mu * r.lz) <= tol &&
                   fabsf(a.xy - mu * r.xy) <= tol && fabsf(a.xz - mu * r.xz) <= tol &&
                   fabsf(a.yz - mu * r.yz) <= tol;
  float thr = 0.5f * r_skin;
  if (mu < 1.0f) thr = fminf(thr, 0.5f * (mu * (rc_max + r_skin) - rc_max));
  bool moved = i == 0u && (!iso || !(thr > 0.0f));
  if (i < n && iso) {
    const float4 p = posq[i], q = ref[i];
    float dx = p.x - mu * q.x, dy = p.y - mu * q.y, dz = p.z - mu * q.z;
    hb_min_image(dx, dy, dz, a);
    moved = moved || dx * dx + dy * dy + dz * dz > thr * thr;
  }
  // one atomic per warp at most
  if (__any_sync(0xFFFFFFFFu, moved) && (threadIdx.x & 31u) == 0u) atomicOr(status, HB_ST_DISPLACED);
}

__global__ void k_gather_pos(const uint32_t *__restrict__ sorted_ids,
                             const float4 *__restrict__ posq, float4 *__restrict__ tile_posq,
                             uint32_t n) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) tile_posq[k] = posq[sorted_ids[k]];
}

int scan_exclusive(const uint32_t *gate, const uint32_t *in, uint32_t *out, uint32_t *tmp,
                   uint32_t len, cudaStream_t s) {
  uint32_t nb = hb_div_up(len, 1024);
  k_scan_block<<<nb, 1024, 0, s>>>(gate, in, out, tmp, len);
  k_scan_top<<<1, 1024, 0, s>>>(gate, tmp, nb);
  k_scan_add<<<nb, 1024, 0, s>>>(gate, out, tmp, len);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

}  // namespace

int nl_setup(hb_forcefield *ff) {
  hb_system *sys = ff->sys;
  const uint32_t n = sys->n;
  ff->n_tiles = hb_div_up(n, 32);
  ff->n_pad = ff->n_tiles * 32u;
  // voxel grid: the smallest power of two per axis with nv^3 >= n
  int l2 = 2;
  while ((1u << (3 * l2)) < n && l2 < 9) ++l2;
  ff->nv_log2 = l2;
  const uint32_t n_vox = 1u << (3 * l2);
  const uint32_t n_pad = ff->n_pad ? ff->n_pad : 32u;
  HB_CUDA(cudaMalloc(&ff->d_vox_key, sizeof(uint32_t) * std::max(n, 1u)));
  HB_CUDA(cudaMalloc(&ff->d_vox_count, sizeof(uint32_t) * (n_vox + 1)));
  HB_CUDA(cudaMemset(ff->d_vox_count, 0, sizeof(uint32_t) * (n_vox + 1)));
  HB_CUDA(cudaMalloc(&ff->d_vox_off, sizeof(uint32_t) * (n_vox + 1)));
  uint32_t scan_len = std::max(n_vox + 1, ff->n_tiles + 1);
  HB_CUDA(cudaMalloc(&ff->d_scan_tmp, sizeof(uint32_t) * (hb_div_up(scan_len, 1024) + 1)));
  HB_CUDA(cudaMalloc(&ff->d_sorted_ids, sizeof(uint32_t) * n_pad));
  HB_CUDA(cudaMalloc(&ff->d_inv_perm, sizeof(uint32_t) * std::max(n, 1u)));
  HB_CUDA(cudaMalloc(&ff->d_tile_posq, sizeof(float4) * n_pad));
  HB_CUDA(cudaMalloc(&ff->d_tile_type, sizeof(int) * n_pad));
  HB_CUDA(cudaMalloc(&ff->d_tile_center, sizeof(float4) * std::max(ff->n_tiles, 1u)));
  HB_CUDA(cudaMalloc(&ff->d_tile_half, sizeof(float4) * std::max(ff->n_tiles, 1u)));
  HB_CUDA(cudaMalloc(&ff->d_tile_nent, sizeof(uint32_t) * (ff->n_tiles + 1)));
  HB_CUDA(cudaMemset(ff->d_tile_nent, 0, sizeof(uint32_t) * (ff->n_tiles + 1)));
  HB_CUDA(cudaMalloc(&ff->d_ref_pos, sizeof(float4) * std::max(n, 1u)));
  HB_CUDA(cudaMalloc(&ff->d_ref_box, sizeof(DBox)));
  HB_CUDA(cudaMemset(ff->d_ref_box, 0, sizeof(DBox)));
  HB_CUDA(cudaMalloc(&ff->d_status, sizeof(uint32_t)));
  HB_CUDA(cudaMemset(ff->d_status, 0, sizeof(uint32_t)));
  HB_CUDA(cudaMalloc(&ff->d_counters, sizeof(uint32_t) * 4));
  HB_CUDA(cudaMalloc(&ff->d_work, sizeof(uint32_t)));
  HB_CUDA(cudaMemset(ff->d_work, 0, sizeof(uint32_t)));
  HB_CUDA(cudaMemset(ff->d_counters, 0, sizeof(uint32_t) * 4));
  HB_CUDA(cudaMallocHost(&ff->h_status, sizeof(uint32_t) * 8));
  HB_CUDA(cudaMalloc(&ff->d_fp, sizeof(unsigned long long) * 5 * n_pad));
  HB_CUDA(cudaMemset(ff->d_fp, 0, sizeof(unsigned long long) * 5 * n_pad));
  return HB_OK;
}

int nl_free(hb_forcefield *ff) {
  cudaFree(ff->d_vox_key);
  cudaFree(ff->d_vox_count);
  cudaFree(ff->d_vox_off);
  cudaFree(ff->d_scan_tmp);
  cudaFree(ff->d_sorted_ids);
  cudaFree(ff->d_inv_perm);
  cudaFree(ff->d_tile_posq);
  cudaFree(ff->d_tile_type);
  cudaFree(ff->d_tile_center);
  cudaFree(ff->d_tile_half);
  cudaFree(ff->d_tile_nent);
  cudaFree(ff->d_entry_j);
  cudaFree(ff->d_entry_excl);
  cudaFree(ff->d_ref_pos);
  cudaFree(ff->d_work);
  cudaFree(ff->d_ref_box);
  cudaFree(ff->d_status);
  cudaFree(ff->d_counters);
  cudaFreeHost(ff->h_status);
  cudaFree(ff->d_fp);
  return HB_OK;
}

// The rebuild sequence: voxel sort, sorted-slot views and tile boxes
// (sort), then either the counting pass of the first build (count_only)
// or the single fill pass plus the finishing kernel.
static int nl_launch(hb_forcefield *ff, const uint32_t *gate, cudaStream_t s, bool sort,
                     bool count_only) {
  hb_system *sys = ff->sys;
  const uint32_t n = sys->n;
  const uint32_t n_vox = 1u << (3 * ff->nv_log2);
  const float rs = ff->r_search;
  const float rs2 = rs * rs;
  // box-prune radius with a margin so rounding never drops a pair, and the
  // relative band inside which the exact rule decides
  const float rb = rs * (1.0f + 1.0e-4f) + 1.0e-4f;
  const float band_lo = rs2 * (1.0f - 1.0e-4f), band_hi = rs2 * (1.0f + 1.0e-4f);
  const size_t smem = sizeof(uint32_t) * (3u * ff->maxc + 1u);
  if (sort) {
    k_vox_hist<<<hb_div_up(n, 256), 256, 0, s>>>(gate, sys->d_posq, sys->d_box, ff->nv_log2,
                                                  ff->d_vox_key, ff->d_vox_count, n);
    HB_TRY(scan_exclusive(gate, ff->d_vox_count, ff->d_vox_off, ff->d_scan_tmp, n_vox + 1, s));
    k_vox_scatter<<<hb_div_up(n, 256), 256, 0, s>>>(gate, ff->d_vox_key, ff->d_vox_off,
                                                     ff->d_vox_count, ff->d_sorted_ids, n);
    k_vox_sort<<<hb_div_up(n_vox, 256), 256, 0, s>>>(gate, ff->d_vox_off, ff->d_sorted_ids, n_vox);
    k_tile_fill<<<hb_div_up(ff->n_pad, 256), 256, 0, s>>>(
        gate, ff->d_sorted_ids, sys->d_posq, sys->d_image, ff->d_inv_perm, ff->d_tile_posq,
        ff->d_tile_type, ff->d_ref_pos, n, ff->n_pad);
    k_tile_bbox<<<hb_div_up((uint64_t)ff->n_tiles * 32u, 128), 128, 0, s>>>(
        gate, ff->d_tile_posq, sys->d_box, ff->rc_max, ff->r_skin, ff->d_tile_center,
        ff->d_tile_half, n, ff->n_tiles);
  }
  if (count_only) {
    k_nl_tile<false><<<ff->n_tiles, NLT_WARPS * 32, smem, s>>>(
        gate, ff->d_tile_posq, ff->d_tile_center, ff->d_tile_half, sys->d_box, rs2, rb, band_lo,
        band_hi, n, ff->n_tiles, ff->maxc, ff->d_tile_nent, 0u, nullptr, nullptr, ff->d_status,
        ff->d_counters, ff->d_sorted_ids, ff->d_inv_perm, ff->d_excl_off, ff->d_excl_partner,
        ff->nl_polls, ff->nl_issue);
  } else {
    k_nl_tile<true><<<ff->n_tiles, NLT_WARPS * 32, smem, s>>>(
        gate, ff->d_tile_posq, ff->d_tile_center, ff->d_tile_half, sys->d_box, rs2, rb, band_lo,
        band_hi, n, ff->n_tiles, ff->maxc, ff->d_tile_nent, ff->slab, ff->d_entry_j,
        ff->d_entry_excl, ff->d_status, ff->d_counters, ff->d_sorted_ids, ff->d_inv_perm,
        ff->d_excl_off, ff->d_excl_partner, ff->nl_polls, ff->nl_issue);
    k_nl_finish<<<1, 1, 0, s>>>(gate, ff->d_status, ff->d_counters, sys->d_box, ff->d_ref_box);
  }
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

// kernels launched by one rebuild: voxel histogram, three scan kernels,
// scatter, voxel sort, tile fill, tile boxes, tile build, finish
int nl_kernel_count() { return 10; }

int nl_rebuild(hb_forcefield *ff, bool gated, cudaStream_t s) {
  if (ff->sys->n == 0) return HB_OK;
  const uint32_t *gate = gated ? ff->d_status : nullptr;
  if (!gated) {
    // an explicit rebuild: raise the displacement bit so k_nl_finish clears it
    uint32_t one = HB_ST_DISPLACED;
    HB_CUDA(cudaMemcpyAsync(ff->d_status, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    HB_CUDA(cudaStreamSynchronize(s));
  }
  return nl_launch(ff, gate, s, true, false);
}

// First build: counting pass, slab size = 1.5 x the largest tile count + 4,
// then the fill pass.  Host-synchronous; runs at force-field creation and
// when the host grows the slabs after a high-water signal.
int nl_first_build(hb_forcefield *ff) {
  hb_system *sys = ff->sys;
  if (sys->n == 0) {
    ff->built = true;
    return HB_OK;
  }
  cudaStream_t s = sys->ctx->stream;
  uint32_t one = HB_ST_DISPLACED;
  HB_CUDA(cudaMemcpyAsync(ff->d_status, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  for (int attempt = 0; attempt < 4; ++attempt) {
    HB_CUDA(cudaMemsetAsync(ff->d_counters + 3, 0, sizeof(uint32_t), s));
    HB_TRY(nl_launch(ff, nullptr, s, attempt == 0, true));
    uint32_t mc = 0;
    HB_CUDA(cudaMemcpyAsync(&mc, ff->d_counters + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    const uint32_t want_c = mc + mc / 2 + 64;
    if (mc <= ff->maxc && ff->maxc >= want_c) break;
    ff->maxc = std::max(want_c, ff->maxc);
    ff->layout_gen++;
    HB_CUDA(cudaFuncSetAttribute(k_nl_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(uint32_t) * (3u * ff->maxc + 1u))));
    HB_CUDA(cudaFuncSetAttribute(k_nl_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(uint32_t) * (3u * ff->maxc + 1u))));
  }
  std::vector<uint32_t> nent(ff->n_tiles);
  HB_CUDA(cudaMemcpyAsync(nent.data(), ff->d_tile_nent, sizeof(uint32_t) * ff->n_tiles,
                          cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  uint32_t mx = 0;
  for (uint32_t v : nent) mx = std::max(mx, v);
  const uint32_t want = mx + mx / 2 + 4;
  if (want > ff->slab) {
    if (ff->slab) ff->reallocations++;
    cudaFree(ff->d_entry_j);
    cudaFree(ff->d_entry_excl);
    ff->d_entry_j = nullptr;
    ff->d_entry_excl = nullptr;
    const size_t cap = (size_t)ff->n_tiles * want;
    HB_CUDA(cudaMalloc(&ff->d_entry_j, sizeof(uint32_t) * 32 * cap));
    HB_CUDA(cudaMalloc(&ff->d_entry_excl, sizeof(uint32_t) * 32 * cap));
    ff->slab = want;
    ff->entry_cap = cap;
    ff->layout_gen++;
  }
  HB_TRY(nl_launch(ff, nullptr, s, false, false));
  uint32_t st = 0;
  HB_CUDA(cudaMemcpyAsync(&st, ff->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  if (st & HB_ST_ENTRY_OVERFLOW) return hb_fail(HB_ERR_NL_OVERFLOW, "slab sizing failed");
  st &= ~(HB_ST_ENTRY_HIGHWATER | HB_ST_ENTRY_OVERFLOW);
  HB_CUDA(cudaMemcpyAsync(ff->d_status, &st, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  HB_CUDA(cudaStreamSynchronize(s));
  ff->built = true;
  return HB_OK;
}

// Slabs of a caller-chosen size (capacity tests, and recovery after an
// overflow): reallocate the entry buffers, clear the capacity bits and
// rebuild at once into the new slabs.  The fill pass writes at most `slab`
// entries per tile and raises the overflow bit when a tile has more, so a
// slab that is too small halts the force field (HB_ERR_NL_OVERFLOW from the
// caller's status check) without writing past the buffers.
int nl_set_slab(hb_forcefield *ff, uint32_t slab) {
  hb_system *sys = ff->sys;
  if (sys->n == 0) return HB_OK;
  cudaStream_t s = sys->ctx->stream;
  HB_CUDA(cudaStreamSynchronize(s));
  cudaFree(ff->d_entry_j);
  cudaFree(ff->d_entry_excl);
  ff->d_entry_j = nullptr;
  ff->d_entry_excl = nullptr;
  const size_t cap = (size_t)ff->n_tiles * slab;
  HB_CUDA(cudaMalloc(&ff->d_entry_j, sizeof(uint32_t) * 32 * cap));
  HB_CUDA(cudaMalloc(&ff->d_entry_excl, sizeof(uint32_t) * 32 * cap));
  ff->slab = slab;
  ff->entry_cap = cap;
  ff->reallocations++;
  ff->layout_gen++;
  uint32_t st = 0;
  HB_CUDA(cudaMemcpyAsync(&st, ff->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  st &= ~(HB_ST_ENTRY_HIGHWATER | HB_ST_ENTRY_OVERFLOW);
  HB_CUDA(cudaMemcpyAsync(ff->d_status, &st, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  return nl_rebuild(ff, false, s);
}

namespace {
__global__ void k_set_rebuild_condition(cudaGraphConditionalHandle h, const uint32_t *status) {
  cudaGraphSetConditional(h, ((*status) & HB_ST_DISPLACED) ? 1u : 0u);
}
}  // namespace

// Inside a stream capture: the rebuild becomes an IF node of the graph
// being captured, taken when the displacement bit is set.  The body (the
// ungated rebuild sequence) is captured on the context's side stream.
int nl_rebuild_conditional(hb_forcefield *ff, cudaStream_t s) {
  if (ff->sys->n == 0) return HB_OK;
  cudaStreamCaptureStatus st;
  cudaGraph_t g;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  HB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  if (st != cudaStreamCaptureStatusActive)
    return hb_fail(HB_ERR_INVALID_ARGUMENT, "conditional rebuild needs an active capture");
  cudaGraphConditionalHandle h;
  HB_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  k_set_rebuild_condition<<<1, 1, 0, s>>>(h, ff->d_status);
  HB_CUDA(cudaGetLastError());
  HB_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  HB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaStream_t side = ff->sys->ctx->stream3;
  HB_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
  int rc = nl_launch(ff, nullptr, side, true, false);
  cudaGraph_t out;
  cudaError_t ce = cudaStreamEndCapture(side, &out);
  if (rc != HB_OK) return rc;
  if (ce != cudaSuccess) return hb_fail(HB_ERR_CUDA, std::string("rebuild body capture: ") + cudaGetErrorString(ce));
  HB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return HB_OK;
}

int nl_displacement_check(hb_forcefield *ff, cudaStream_t s) {
  hb_system *sys = ff->sys;
  if (sys->n == 0) return HB_OK;
  k_disp_check<<<hb_div_up(sys->n, 256), 256, 0, s>>>(sys->d_posq, ff->d_ref_pos, sys->d_box,
                                                       ff->d_ref_box, ff->r_skin, ff->rc_max,
                                                       ff->d_status, sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

int nl_gather_positions(hb_forcefield *ff, cudaStream_t s) {
  hb_system *sys = ff->sys;
  if (sys->n == 0) return HB_OK;
  k_gather_pos<<<hb_div_up(sys->n, 256), 256, 0, s>>>(ff->d_sorted_ids, sys->d_posq,
                                                       ff->d_tile_posq, sys->n);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

// Host decode of the packed list (the pair_snapshot analogue): every pair
// held by an entry whose exact single-precision distance is within
// r_search, as canonical (min id, max id), plus a duplicate count.
static float host_exact_r2(float dx, float dy, float dz, const float b[6]) {
  volatile float sc = dz / b[2];
  volatile float sb = (dy - sc * b[5]) / b[1];
  volatile float t1 = sb * b[3];
  volatile float t2 = sc * b[4];
  volatile float t3 = dx - t1;
  volatile float sa = (t3 - t2) / b[0];
  float ka = std::floor(sa + 0.5f), kb = std::floor(sb + 0.5f), kc = std::floor(sc + 0.5f);
  volatile float u1 = ka * b[0];
  volatile float u2 = kb * b[3];
  volatile float u3 = kc * b[4];
  volatile float u4 = u1 + u2;
  volatile float u5 = u4 + u3;
  volatile float ddx = dx - u5;
  volatile float v1 = kb * b[1];
  volatile float v2 = kc * b[5];
  volatile float v3 = v1 + v2;
  volatile float ddy = dy - v3;
  volatile float w1 = kc * b[2];
  volatile float ddz = dz - w1;
  volatile float q1 = ddx * ddx;
  volatile float q2 = ddy * ddy;
  volatile float q3 = ddz * ddz;
  volatile float q4 = q1 + q2;
  volatile float q5 = q4 + q3;
  return q5;
}

int nl_pairs(hb_forcefield *ff, std::vector<uint32_t> &pairs, uint64_t &dups) {
  hb_system *sys = ff->sys;
  cudaStream_t s = sys->ctx->stream;
  HB_CUDA(cudaStreamSynchronize(s));
  HB_CUDA(cudaStreamSynchronize(sys->ctx->stream2));
  const uint32_t n = sys->n;
  pairs.clear();
  dups = 0;
  if (n == 0) return HB_OK;
  std::vector<uint32_t> nent(ff->n_tiles), ids(ff->n_pad);
  std::vector<float4> pos(ff->n_pad);
  HB_CUDA(cudaMemcpy(nent.data(), ff->d_tile_nent, sizeof(uint32_t) * ff->n_tiles,
                     cudaMemcpyDeviceToHost));
  HB_CUDA(cudaMemcpy(ids.data(), ff->d_sorted_ids, sizeof(uint32_t) * ff->n_pad,
                     cudaMemcpyDeviceToHost));
  HB_CUDA(cudaMemcpy(pos.data(), ff->d_tile_posq, sizeof(float4) * ff->n_pad,
                     cudaMemcpyDeviceToHost));
  std::vector<uint32_t> ej((size_t)ff->entry_cap * 32);
  if (ff->entry_cap)
    HB_CUDA(cudaMemcpy(ej.data(), ff->d_entry_j, sizeof(uint32_t) * 32 * ff->entry_cap,
                       cudaMemcpyDeviceToHost));
  HB_TRY(sys_refresh_box(sys));
  float b[6];
  for (int d = 0; d < 6; ++d) b[d] = (float)sys->box[d];
  const float rs2 = ff->r_search * ff->r_search;
  std::vector<uint64_t> keys;
  for (uint32_t I = 0; I < ff->n_tiles; ++I) {
    if (nent[I] > ff->slab) return hb_fail(HB_ERR_NL_OVERFLOW, "packed entries overflowed");
    const bool has_self = n - I * 32u >= 2u;
    for (uint32_t q = 0; q < nent[I]; ++q) {
      const uint64_t e = (uint64_t)I * ff->slab + q;
      const bool self = has_self && q == 0;
      for (uint32_t l = 0; l < 32; ++l) {
        uint32_t si = I * 32u + l;
        if (si >= n) continue;
        const uint32_t t0 = self ? 1u : 0u, t1 = self ? 16u : 31u;
        for (uint32_t t = t0; t <= t1; ++t) {
          if (self && t == 16u && l >= 16u) continue;
          uint32_t sj = ej[e * 32 + ((l + t) & 31u)];
          if (sj == HB_SENTINEL || sj >= n) continue;
          float4 a = pos[si], c = pos[sj];
          float r2 = host_exact_r2(a.x - c.x, a.y - c.y, a.z - c.z, b);
          if (r2 <= rs2) {
            uint32_t oi = ids[si], oj = ids[sj];
            uint32_t lo = std::min(oi, oj), hi = std::max(oi, oj);
            keys.push_back(((uint64_t)lo << 32) | hi);
          }
        }
      }
    }
  }
  std::sort(keys.begin(), keys.end());
  pairs.reserve(keys.size() * 2);
  for (size_t k = 0; k < keys.size(); ++k) {
    if (k > 0 && keys[k] == keys[k - 1]) {
      dups++;
      continue;
    }
    pairs.push_back((uint32_t)(keys[k] >> 32));
    pairs.push_back((uint32_t)(keys[k] & 0xFFFFFFFFu));
  }
  return HB_OK;
}
