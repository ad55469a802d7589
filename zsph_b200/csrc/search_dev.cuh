// Device code of the neighbour search shared by the search kernels
// (search.cu) and the batched form's persistent kernel (equations.cu): the
// hash, the ticket and scan helpers, the gather, and the bodies of the
// fused search's four stages, each written for one CTA (or one thread) so
// that a kernel can run one unit per CTA or loop over units.  Every CTA
// running these has kSearchBlock threads.
#pragma once
#include <climits>

#include "zsph_internal.cuh"

namespace zsph {
namespace {

constexpr int kHashItems = 4;             // particles per thread in the fused hash
constexpr int kScatterItems = 4;          // particles per thread in the fused scatter
constexpr unsigned kLookbackSpins = 1u << 20;  // bound on the one-pass scan's wait for a predecessor tile

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// floorf(a / c) with a correctly rounded division, for c > 0 and rc the
// correctly rounded 1 / c, without the division in the common case.
// q = a * rc is within 2^-23 |a / c| (relative) of a / c, and the rounded
// quotient within 2^-24: both lie within 2^-22 |q| of q.  When q is farther
// than 2^-20 |q| from every integer (and not tiny, where the bound would be
// absolute), q, a / c and its rounding share one floor.  Otherwise (q near a
// cell face, NaN, infinite) the division is taken as written.  The distance
// d is exact: q - floor(q) and floor(q) + 1 - q subtract numbers within a
// factor two of each other (or from zero).
__device__ __forceinline__ int floor_quot(float a, float c, float rc) {
  const float q = __fmul_rn(a, rc);
  const float f = floorf(q);
  const float d = fminf(__fsub_rn(q, f), __fsub_rn(__fadd_rn(f, 1.0f), q));
  if (d > fmaxf(fabsf(q) * 0x1p-20f, 0x1p-100f)) return (int)f;
  return (int)floorf(__fdiv_rn(a, c));
}

// Cell hash of one position, as hash.cu:12-15 computes it (IEEE subtract and
// divide, floorf, float->int conversion, int multiply-add); rc is
// __frcp_rn(p.grid_size) and the divisions go through floor_quot.
__device__ __forceinline__ int cell_hash(const zsph_gpu_param_t& p, float x, float y, float z, float rc) {
  const int hx = floor_quot(__fsub_rn(x, p.grid_xmin), p.grid_size, rc);
  const int hy = floor_quot(__fsub_rn(y, p.grid_ymin), p.grid_size, rc);
  const int hz = floor_quot(__fsub_rn(z, p.grid_zmin), p.grid_size, rc);
  return hz * p.grid_xdim * p.grid_ydim + hy * p.grid_xdim + hx;
}

// hash.cu:16-23: a particle outside the grid becomes type 100 at the grid
// origin with zero velocity and (rho0, 0); its key becomes 0.  Takes the
// particle's position (x, y, z) or, in the precision form, its packed cell
// (cpk), already loaded.  PLAIN: the single-scene FP32 form (no packed
// cells, no scene table), resolved at compile time.
template <bool PLAIN = false>
__device__ __forceinline__ int hash_and_kill_at(const KParams& kp, const zsph_ptc_t& s, int i, float x, float y,
                                                float z, int cpk, int* flags, float rc) {
  const zsph_gpu_param_t& p = kp.p;
  const bool c3 = !PLAIN && kp.c3o;
  int h;
  bool out;
  if (c3) {  // precision form: the cell is stored, the offset is local
    const int3 c = unpack_cell(cpk);
    out = c.x >= p.grid_xdim || c.y >= p.grid_ydim || c.z >= p.grid_zdim;
    h = (c.z * p.grid_ydim + c.y) * p.grid_xdim + c.x;
  } else {
    // batched form: the scene's cells start at grid_hash_min (0 for one scene)
    h = cell_hash(p, x, y, z, rc);
    out = h < 0 || h > p.grid_hash_max - p.grid_hash_min;
    h += p.grid_hash_min;
  }
  if (out) {
    s.type[i] = 100;
    if (c3) {  // the grid origin: cell (0, 0, 0), offset 0
      kp.c3o[i] = 0;
      s.pos[3 * i] = 0.0f;
      s.pos[3 * i + 1] = 0.0f;
      s.pos[3 * i + 2] = 0.0f;
    } else {
      s.pos[3 * i] = p.grid_xmin;
      s.pos[3 * i + 1] = p.grid_ymin;
      s.pos[3 * i + 2] = p.grid_zmin;
    }
    s.vel[3 * i] = 0.0f;
    s.vel[3 * i + 1] = 0.0f;
    s.vel[3 * i + 2] = 0.0f;
    s.rhop[2 * i] = p.rho0;
    s.rhop[2 * i + 1] = 0.0f;
    h = !PLAIN && kp.scenes ? p.grid_hash_min : 0;  // the scene's first cell (batched form)
    atomicOr(flags, ZSPH_FLAG_KILLED);
  }
  return h;
}

__device__ __forceinline__ int hash_and_kill(const KParams& kp, const zsph_ptc_t& s, int i, int* flags) {
  float x = 0.0f, y = 0.0f, z = 0.0f;
  int cpk = 0;
  if (kp.c3o) {
    cpk = kp.c3o[i];
  } else {
    x = s.pos[3 * i];
    y = s.pos[3 * i + 1];
    z = s.pos[3 * i + 2];
  }
  return hash_and_kill_at(kp, s, i, x, y, z, cpk, flags, __frcp_rn(kp.p.grid_size));
}

// One atomic per distinct key per warp; returns this lane's ticket (its
// arrival rank inside the key's cell).  Lanes of one warp that share a key
// get consecutive tickets in lane order.
__device__ __forceinline__ int warp_ticket(int* cnt, int key, unsigned active) {
  const unsigned peers = __match_any_sync(active, key);
  const int leader = __ffs(peers) - 1;
  const int rank = __popc(peers & lanemask_lt());
  int base = 0;
  if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&cnt[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + rank;
}

// Fused search, step 1: hash + kill + per-cell ticket, kHashItems particles
// per thread (i = tile base + k * kSearchBlock + thread, so each warp access
// stays coalesced).  All positions are loaded before any hash is formed and
// all ticket atomics are issued before any result is used, so a thread keeps
// kHashItems loads and atomics in flight.  Also prepares the one-pass scan:
// the largest key (misc[4]), a fresh tile counter (misc[5]), the next epoch
// (misc[6]) and an empty big-cell list (misc[3]).
// hash_count_body is one CTA's chunk `chunk` of the particles; k_hash_count
// runs one chunk per CTA, the batched form's persistent kernel loops over
// chunks (every thread of the CTA takes part).  PLAIN: kp_in has neither
// packed cells nor scenes, so the per-particle parameter lookup and those
// branches are left out at compile time (the same arithmetic).
template <bool PLAIN = false>
__device__ __forceinline__ void hash_count_body(const KParams& kp_in, const zsph_ptc_t& s, const Scratch& sc,
                                                int chunk) {
  __shared__ int s_max[kSearchBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = chunk * (kSearchBlock * kHashItems) + threadIdx.x;
  const int n = kp_in.n;
  if (chunk == 0 && threadIdx.x == 0) {
    sc.misc[3] = 0;
    sc.misc[5] = 0;
    sc.misc[6] = (int)((unsigned)sc.misc[6] + 1u);
  }
  float x[kHashItems], y[kHashItems], z[kHashItems];
  int cpk[kHashItems];
#pragma unroll
  for (int k = 0; k < kHashItems; ++k) {
    const int i = base + k * kSearchBlock;
    x[k] = y[k] = z[k] = 0.0f;
    cpk[k] = 0;
    if (i < n) {
      if (!PLAIN && kp_in.c3o) {
        cpk[k] = kp_in.c3o[i];
      } else {
        x[k] = s.pos[3 * i];
        y[k] = s.pos[3 * i + 1];
        z[k] = s.pos[3 * i + 2];
      }
    }
  }
  int h[kHashItems];
  int kmax = -1;
  const float rc0 = __frcp_rn(kp_in.p.grid_size);
#pragma unroll
  for (int k = 0; k < kHashItems; ++k) {
    const int i = base + k * kSearchBlock;
    h[k] = 0;
    if (i < n) {
      if constexpr (PLAIN) {
        h[k] = hash_and_kill_at<true>(kp_in, s, i, x[k], y[k], z[k], 0, sc.flags, rc0);
      } else {
        const KParams kp = kp_of_particle(kp_in, i);
        const float rc = kp_in.scenes ? __frcp_rn(kp.p.grid_size) : rc0;  // a scene's own cell size
        h[k] = hash_and_kill_at(kp, s, i, x[k], y[k], z[k], cpk[k], sc.flags, rc);
      }
      sc.key[i] = h[k];
      kmax = max(kmax, h[k]);
    }
  }
  // Tickets: one atomic per run of equal keys among a warp's consecutive
  // particles (the particles are nearly sorted by cell, so a warp holds a few
  // runs).  Lanes of a run get consecutive tickets in lane order; two runs of
  // one key draw separate ranges.  The ranking step restores stability.
  unsigned heads[kHashItems];
  int got[kHashItems];
#pragma unroll
  for (int k = 0; k < kHashItems; ++k) {
    const int i = base + k * kSearchBlock;
    const int prev = __shfl_up_sync(0xffffffffu, h[k], 1);
    // active lanes form a prefix of the warp; an inactive lane counts as a head
    const bool head = i >= n || lane == 0 || prev != h[k];
    heads[k] = __ballot_sync(0xffffffffu, head);
    got[k] = 0;
    if (i < n && head) {
      const unsigned after = heads[k] & ~((2u << lane) - 1u);  // heads above this lane (lane 31: none)
      const int next = after ? __ffs(after) - 1 : 32;
      got[k] = atomicAdd(&sc.cnt[h[k]], next - lane);
    }
  }
#pragma unroll
  for (int k = 0; k < kHashItems; ++k) {
    const int i = base + k * kSearchBlock;
    const int lead = 31 - __clz(heads[k] & ((2u << lane) - 1u));  // this lane's run head
    const int b = __shfl_sync(0xffffffffu, got[k], lead);
    if (i < n) sc.ticket[i] = b + lane - lead;
  }
  kmax = __reduce_max_sync(0xffffffffu, kmax);
  if (lane == 0) s_max[warp] = kmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    int m = -1;
#pragma unroll
    for (int w = 0; w < kSearchBlock / 32; ++w) m = max(m, s_max[w]);
    if (m >= 0) atomicMax(&sc.misc[4], m);
  }
}

// Block-wide exclusive scan of one int per thread (kSearchBlock threads).
__device__ __forceinline__ int block_exclusive_scan(int v, int* smem_warp, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kSearchBlock / 32 ? smem_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kSearchBlock / 32) smem_warp[lane] = w;
  }
  __syncthreads();
  total = smem_warp[kSearchBlock / 32 - 1];
  const int before = warp > 0 ? smem_warp[warp - 1] : 0;
  __syncthreads();
  return before + x - v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Fused search, step 2: one-pass scan of the per-cell counts with decoupled
// look-back, writing cell_lb, grid_start/grid_end in closed form and the
// big-cell list, and zeroing the counts (all but the last occupied cell's,
// which every tile reads; the scatter zeroes that one).
//
// A tile is kOneTile cells, kOneItems consecutive cells per thread, read and
// written with 16-byte vector accesses.  Tiles are claimed in launch order
// through an atomic counter (misc[5]), so every predecessor of a tile belongs
// to a CTA that is already running.  A tile publishes its aggregate at once,
// then its inclusive prefix after looking back; the status word of a tile is
// (tag << 32) | value with tag 2e+1 (aggregate) or 2e+2 (inclusive prefix)
// for this search's epoch e (misc[6]), so the words never need clearing.
// The look-back wait is bounded: a tile that gives up raises
// ZSPH_FLAG_TIMEOUT and carries on (the sort is then wrong, and flagged).
// The last occupied cell comes from the hash's atomic maximum (misc[4]).
constexpr int kOneItems = 16;
constexpr int kOneTile = kSearchBlock * kOneItems;

__device__ __forceinline__ void st4(int* p, int a, int b, int c, int d) {
  *reinterpret_cast<int4*>(p) = make_int4(a, b, c, d);
}


// scan_onepass_body: one CTA on tile `tile` (claimed by the caller through
// misc[5], in the order the tiles are claimed).
__device__ __forceinline__ void scan_onepass_body(const KParams& kp, const Scratch& sc, const zsph_tmp_t& t,
                                                  int tile) {
  __shared__ int sw[kSearchBlock / 32];
  __shared__ int s_excl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned epoch = (unsigned)sc.misc[6];
  const unsigned tag_agg = 2u * epoch + 1u, tag_inc = 2u * epoch + 2u;
  const int G = kp.G, n = kp.n;
  const int klast = sc.misc[4];
  const bool last_single = sc.cnt[klast] == 1;
  const int base = tile * kOneTile + threadIdx.x * kOneItems;
  const bool full = base + kOneItems <= G;  // 16-byte aligned: base is a multiple of 16 cells
  int v[kOneItems];
  if (full) {
#pragma unroll
    for (int q = 0; q < kOneItems / 4; ++q) {
      const int4 a = *reinterpret_cast<const int4*>(sc.cnt + base + 4 * q);
      v[4 * q] = a.x; v[4 * q + 1] = a.y; v[4 * q + 2] = a.z; v[4 * q + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kOneItems; ++k) v[k] = base + k < G ? sc.cnt[base + k] : 0;
  }
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kOneItems; ++k) sum += v[k];
  int total;
  const int ex = block_exclusive_scan(sum, sw, total);
  if (warp == 0) {
    unsigned long long* ts = sc.tile_state;
    int excl = 0;
    if (tile == 0) {
      if (lane == 0) st_relaxed_u64(ts, ((unsigned long long)tag_inc << 32) | (unsigned)total);
    } else {
      if (lane == 0) st_relaxed_u64(ts + tile, ((unsigned long long)tag_agg << 32) | (unsigned)total);
      int j = tile - 1;  // nearest predecessor not yet added
      unsigned spins = 0;
      for (;;) {
        const int idx = j - lane;
        unsigned long long w;
        for (;;) {
          w = idx >= 0 ? ld_relaxed_u64(ts + idx) : ((unsigned long long)tag_inc << 32);
          const unsigned tg = (unsigned)(w >> 32);
          if (__all_sync(0xffffffffu, tg == tag_agg || tg == tag_inc)) break;
          if (++spins >= kLookbackSpins) break;
          if (spins > 64) __nanosleep(32);
        }
        if (spins >= kLookbackSpins) {
          if (lane == 0) atomicOr(sc.flags, ZSPH_FLAG_TIMEOUT);
          break;
        }
        const unsigned inc = __ballot_sync(0xffffffffu, (unsigned)(w >> 32) == tag_inc);
        int val = (int)(unsigned)(w & 0xffffffffu);
        if (inc) {
          const int f = __ffs(inc) - 1;  // nearest tile holding an inclusive prefix
          if (lane > f) val = 0;
          excl += __reduce_add_sync(0xffffffffu, val);
          break;
        }
        excl += __reduce_add_sync(0xffffffffu, val);
        j -= 32;
      }
      if (lane == 0) st_relaxed_u64(ts + tile, ((unsigned long long)tag_inc << 32) | (unsigned)(excl + total));
    }
    if (lane == 0) s_excl = excl;
  }
  __syncthreads();
  int lb[kOneItems + 1];
  lb[0] = s_excl + ex;
#pragma unroll
  for (int k = 0; k < kOneItems; ++k) lb[k + 1] = lb[k] + v[k];
  // the stale-bounds rule touches only cells >= klast of a single last particle
  const bool plain = full && !(last_single && base + kOneItems > klast) && (klast < base || klast >= base + kOneItems);
  if (plain) {
#pragma unroll
    for (int q = 0; q < kOneItems / 4; ++q) {
      const int k = 4 * q;
      st4(sc.cell_lb + base + k, lb[k], lb[k + 1], lb[k + 2], lb[k + 3]);
      st4(t.grid_start + base + k, min(lb[k], n - 1), min(lb[k + 1], n - 1), min(lb[k + 2], n - 1),
          min(lb[k + 3], n - 1));
      st4(t.grid_end + base + k, min(lb[k + 1], n - 1), min(lb[k + 2], n - 1), min(lb[k + 3], n - 1),
          min(lb[k + 4], n - 1));
      st4(sc.cnt + base + k, 0, 0, 0, 0);
    }
  }
#pragma unroll
  for (int k = 0; k < kOneItems; ++k) {
    const int c = base + k;
    if (c < G) {
      if (!plain) {
        sc.cell_lb[c] = lb[k];
        if (!(last_single && c > klast)) t.grid_start[c] = min(lb[k], n - 1);
        if (!(last_single && c >= klast)) t.grid_end[c] = min(lb[k + 1], n - 1);
        if (v[k] != 0 && c != klast) sc.cnt[c] = 0;
      }
      if (v[k] > kBigSegment) {
        const int slot = atomicAdd(&sc.misc[3], 1);
        if (slot < kBigListCap) sc.big_list[slot] = c;
      }
      if (c == G - 1) sc.cell_lb[G] = lb[k + 1];
    }
  }
}

// Sorts v[0, n) ascending in place with one CTA: a bitonic network in
// which every comparator puts the minimum at the lower index, so virtual
// +inf padding beyond n never has to be stored.
template <class Ptr>
__device__ void cta_sort_segment(Ptr v, int n) {
  int P = 1;
  while (P < n) P <<= 1;
  for (int k = 2; k <= P; k <<= 1) {
    for (int idx = threadIdx.x; idx < P / 2; idx += blockDim.x) {
      const int half = k >> 1;
      const int blk = idx / half, off = idx % half;
      const int lo = blk * k + off, hi = blk * k + k - 1 - off;
      if (hi < n) {
        const int a = v[lo], b = v[hi];
        if (a > b) { v[lo] = b; v[hi] = a; }
      }
    }
    __syncthreads();
    for (int j = k >> 2; j >= 1; j >>= 1) {
      for (int idx = threadIdx.x; idx < P / 2; idx += blockDim.x) {
        const int blk = idx / j, off = idx % j;
        const int lo = blk * 2 * j + off, hi = lo + j;
        if (hi < n) {
          const int a = v[lo], b = v[hi];
          if (a > b) { v[lo] = b; v[hi] = a; }
        }
      }
      __syncthreads();
    }
  }
}

// scatter_body: one CTA's chunk of the scatter (also zeroes the last
// occupied cell's count and the largest key, at chunk 0).
__device__ __forceinline__ void scatter_body(const KParams& kp, const Scratch& sc, int chunk) {
  if (chunk == 0 && threadIdx.x == 0) {
    sc.cnt[sc.misc[4]] = 0;
    sc.misc[4] = 0;
  }
  const int base = chunk * (kSearchBlock * kScatterItems) + threadIdx.x;
  int key[kScatterItems], tk[kScatterItems];
#pragma unroll
  for (int k = 0; k < kScatterItems; ++k) {
    const int i = base + k * kSearchBlock;
    key[k] = i < kp.n ? sc.key[i] : 0;
    tk[k] = i < kp.n ? sc.ticket[i] : 0;
  }
#pragma unroll
  for (int k = 0; k < kScatterItems; ++k) {
    const int i = base + k * kSearchBlock;
    if (i < kp.n) sc.perm[sc.cell_lb[key[k]] + tk[k]] = i;
  }
}

// Final slot of the particle scattered to slot t: its rank by original
// position among the members of its cell.
// NC: read the members through the read-only (non-coherent) path, valid
// only when they were written by an earlier launch.
template <bool NC = true>
__device__ __forceinline__ int ranked_slot(const Scratch& sc, int t, int i, int c) {
  const int a = sc.cell_lb[c], b = sc.cell_lb[c + 1];
  if (b - a > kBigSegment) return t;  // pre-sorted (k_sort_big_cells or the scatter's last CTA)
  int r = 0;
  for (int k = a; k < b; ++k) r += ((NC ? __ldg(&sc.perm[k]) : sc.perm[k]) < i) ? 1 : 0;
  return a + r;
}

// Density with the sign bit marking a non-fluid particle (type != 1).
__device__ __forceinline__ float packed_rho(float rho, int type) {
  return type == 1 ? fabsf(rho) : -fabsf(rho);
}

__device__ __forceinline__ void gather_one(const zsph_ptc_t& o, const zsph_ptc_t& w, int src,
                                           int dst) {
  const float x = o.pos[3 * src], y = o.pos[3 * src + 1], z = o.pos[3 * src + 2];
  const float vx = o.vel[3 * src], vy = o.vel[3 * src + 1], vz = o.vel[3 * src + 2];
  const float2 rp = reinterpret_cast<const float2*>(o.rhop)[src];
  const float tx = o.tmp_pos[3 * src], ty = o.tmp_pos[3 * src + 1], tz = o.tmp_pos[3 * src + 2];
  const float ux = o.tmp_vel[3 * src], uy = o.tmp_vel[3 * src + 1], uz = o.tmp_vel[3 * src + 2];
  const float2 trp = reinterpret_cast<const float2*>(o.tmp_rhop)[src];
  const int ty_ = o.type[src];
  const int tb = o.table[src];
  w.pos[3 * dst] = x; w.pos[3 * dst + 1] = y; w.pos[3 * dst + 2] = z;
  w.vel[3 * dst] = vx; w.vel[3 * dst + 1] = vy; w.vel[3 * dst + 2] = vz;
  reinterpret_cast<float2*>(w.rhop)[dst] = rp;
  w.tmp_pos[3 * dst] = tx; w.tmp_pos[3 * dst + 1] = ty; w.tmp_pos[3 * dst + 2] = tz;
  w.tmp_vel[3 * dst] = ux; w.tmp_vel[3 * dst + 1] = uy; w.tmp_vel[3 * dst + 2] = uz;
  reinterpret_cast<float2*>(w.tmp_rhop)[dst] = trp;
  w.type[dst] = ty_;
  w.table[dst] = tb + src - dst;  // sort.cu:82
}

// One particle's record of the eight reference arrays (72 bytes).
struct PtcRec {
  float x, y, z, vx, vy, vz;
  float2 rp;
  float tx, ty, tz, ux, uy, uz;
  float2 trp;
  int type, table;
};

// The record in two halves: the current state (pos, vel, rhop, type,
// table) and the predictor's copies (tmp_pos, tmp_vel, tmp_rhop).
__device__ __forceinline__ void load_rec_state(const zsph_ptc_t& o, int src, PtcRec& r) {
  r.x = o.pos[3 * src]; r.y = o.pos[3 * src + 1]; r.z = o.pos[3 * src + 2];
  r.vx = o.vel[3 * src]; r.vy = o.vel[3 * src + 1]; r.vz = o.vel[3 * src + 2];
  r.rp = reinterpret_cast<const float2*>(o.rhop)[src];
  r.type = o.type[src];
  r.table = o.table[src];
}
__device__ __forceinline__ void load_rec_tmp(const zsph_ptc_t& o, int src, PtcRec& r) {
  r.tx = o.tmp_pos[3 * src]; r.ty = o.tmp_pos[3 * src + 1]; r.tz = o.tmp_pos[3 * src + 2];
  r.ux = o.tmp_vel[3 * src]; r.uy = o.tmp_vel[3 * src + 1]; r.uz = o.tmp_vel[3 * src + 2];
  r.trp = reinterpret_cast<const float2*>(o.tmp_rhop)[src];
}

__device__ __forceinline__ void store_rec(const zsph_ptc_t& w, const PtcRec& r, int src, int dst) {
  w.pos[3 * dst] = r.x; w.pos[3 * dst + 1] = r.y; w.pos[3 * dst + 2] = r.z;
  w.vel[3 * dst] = r.vx; w.vel[3 * dst + 1] = r.vy; w.vel[3 * dst + 2] = r.vz;
  reinterpret_cast<float2*>(w.rhop)[dst] = r.rp;
  w.tmp_pos[3 * dst] = r.tx; w.tmp_pos[3 * dst + 1] = r.ty; w.tmp_pos[3 * dst + 2] = r.tz;
  w.tmp_vel[3 * dst] = r.ux; w.tmp_vel[3 * dst + 1] = r.uy; w.tmp_vel[3 * dst + 2] = r.uz;
  reinterpret_cast<float2*>(w.tmp_rhop)[dst] = r.trp;
  w.type[dst] = r.type;
  w.table[dst] = r.table + src - dst;  // sort.cu:82
}


// Fused search, last step: rank, write sorted hash/index, gather the eight
// particle arrays (sort.cu:62-82).  The current-state half of the source
// record is loaded as soon as the source is known, before the rank (which
// needs the key, the cell's range and its members) is counted, so those
// loads overlap that dependent chain; the tmp half follows the rank.  That
// split fits 32 registers, so k_rank_gather keeps 64 warps per SM: loading
// the whole record first needs 40 registers (48 warps), and loading all of
// it after the rank leaves the rank's latency exposed (both measured
// slower).
// rank_gather_one: sorted slot `slot`.  NC: the members of the cell are read
// through the read-only path (only where the scatter ran in an earlier launch).
template <bool NC = true>
__device__ __forceinline__ void rank_gather_one(const KParams& kp, const Scratch& sc, const zsph_ptc_t& o,
                                                const zsph_ptc_t& w, const zsph_tmp_t& t, int slot) {
  const int i = sc.perm[slot];
  PtcRec r;
  load_rec_state(o, i, r);
  const int cpk = kp.c3o ? kp.c3o[i] : 0;
  const int c = sc.key[i];
  const int dst = ranked_slot<NC>(sc, slot, i, c);
  load_rec_tmp(o, i, r);
  t.index[dst] = i;
  t.hash[dst] = c;
  if (r.type == 1) sc.cfe[c] = sc.misc[6];  // a fluid particle in cell c in this search
  store_rec(w, r, i, dst);
  if (kp.c3o) kp.c3n[dst] = cpk;
}

}  // namespace
}  // namespace zsph
