// Neighbour search for sm_100a: cell hash, stable counting sort by cell,
// cell bounds and reorder.
//
// Reference path replaced (single_gpu_sph_src/):
//   lib/hash.cu:3-26     cuda_ptc_hash      -> k_hash (drop-in) / k_hash_count (fused)
//   lib/sort.cu:3-6      thrust::sort_by_key-> counting sort: count -> scan -> scatter -> rank
//   lib/sort.cu:8-84     cuda_sort_data     -> k_scan_onepass / k_scan_cells (bounds) + k_rank_gather (reorder)
//
// The reference sorts all 32 key bits with a generic radix sort.  Here the
// keys are cell ids in [0, G), so a counting sort needs one histogram, one
// scan over G cells and one scatter.  The scatter uses atomic tickets (one
// atomic per run of equal keys in a warp), which are not ordered across
// warps; stability (ties in prior position order, the reference's
// sort_by_key contract) is restored by ranking each particle among the
// members of its cell by original position.  Cells with more than
// kBigSegment members are first sorted in place by one CTA each.
//
// The fused search of a sub-step is four launches: k_hash_count (hash, kill,
// tickets, largest key), k_scan_onepass (decoupled look-back scan and cell
// bounds), k_scatter_fused (scatter; crowded cells pre-sorted by its last
// CTA) and k_rank_gather (rank and reorder).  The drop-in entry points
// (zsph_sort_index, zsph_sort_data and the allocation-free sort) use the
// two-kernel scan k_scan_reduce + k_scan_cells.  The cell bounds are written from the scanned
// offsets in closed form, including the reference's end-of-array rules
// (sort.cu:30-60): with lb(c) the number of particles whose key is below c,
//   grid_start[c] = min(lb(c),   N-1)
//   grid_end[c]   = min(lb(c+1), N-1)
// except that, when the last sorted particle is alone in its cell (key k),
// grid_end[c] for c >= k and grid_start[c] for c > k are left untouched.
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

// Cell hash of one position, exactly as hash.cu:12-15 computes it (IEEE
// subtract and divide, floorf, float->int conversion, int multiply-add).
__device__ __forceinline__ int cell_hash(const zsph_gpu_param_t& p, float x, float y, float z) {
  const int hx = (int)floorf(__fdiv_rn(__fsub_rn(x, p.grid_xmin), p.grid_size));
  const int hy = (int)floorf(__fdiv_rn(__fsub_rn(y, p.grid_ymin), p.grid_size));
  const int hz = (int)floorf(__fdiv_rn(__fsub_rn(z, p.grid_zmin), p.grid_size));
  return hz * p.grid_xdim * p.grid_ydim + hy * p.grid_xdim + hx;
}

// hash.cu:16-23: a particle outside the grid becomes type 100 at the grid
// origin with zero velocity and (rho0, 0); its key becomes 0.  Takes the
// particle's position (x, y, z) or, in the precision form, its packed cell
// (cpk), already loaded.
__device__ __forceinline__ int hash_and_kill_at(const KParams& kp, const zsph_ptc_t& s, int i, float x, float y,
                                                float z, int cpk, int* flags) {
  const zsph_gpu_param_t& p = kp.p;
  int h;
  bool out;
  if (kp.c3o) {  // precision form: the cell is stored, the offset is local
    const int3 c = unpack_cell(cpk);
    out = c.x >= p.grid_xdim || c.y >= p.grid_ydim || c.z >= p.grid_zdim;
    h = (c.z * p.grid_ydim + c.y) * p.grid_xdim + c.x;
  } else {
    // batched form: the scene's cells start at grid_hash_min (0 for one scene)
    h = cell_hash(p, x, y, z);
    out = h < 0 || h > p.grid_hash_max - p.grid_hash_min;
    h += p.grid_hash_min;
  }
  if (out) {
    s.type[i] = 100;
    if (kp.c3o) {  // the grid origin: cell (0, 0, 0), offset 0
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
    h = kp.scenes ? p.grid_hash_min : 0;  // the scene's first cell (batched form)
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
  return hash_and_kill_at(kp, s, i, x, y, z, cpk, flags);
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

// Drop-in cuda_ptc_hash: hash + identity index (hash.cu:3-26).
__global__ void __launch_bounds__(kSearchBlock) k_hash(KParams kp_in, zsph_ptc_t s, zsph_tmp_t t, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp_in.n) return;
  const KParams kp = kp_of_particle(kp_in, i);
  t.hash[i] = hash_and_kill(kp, s, i, flags);
  t.index[i] = i;
}

// Fused search, step 1: hash + kill + per-cell ticket, kHashItems particles
// per thread (i = tile base + k * kSearchBlock + thread, so each warp access
// stays coalesced).  All positions are loaded before any hash is formed and
// all ticket atomics are issued before any result is used, so a thread keeps
// kHashItems loads and atomics in flight.  Also prepares the one-pass scan:
// the largest key (misc[4]), a fresh tile counter (misc[5]), the next epoch
// (misc[6]) and an empty big-cell list (misc[3]).
__global__ void __launch_bounds__(kSearchBlock) k_hash_count(KParams kp_in, zsph_ptc_t s, Scratch sc) {
  __shared__ int s_max[kSearchBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = blockIdx.x * (kSearchBlock * kHashItems) + threadIdx.x;
  const int n = kp_in.n;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
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
      if (kp_in.c3o) {
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
#pragma unroll
  for (int k = 0; k < kHashItems; ++k) {
    const int i = base + k * kSearchBlock;
    h[k] = 0;
    if (i < n) {
      const KParams kp = kp_of_particle(kp_in, i);
      h[k] = hash_and_kill_at(kp, s, i, x[k], y[k], z[k], cpk[k], sc.flags);
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

// Drop-in sort_index, step 1: copy keys and carried values, count.
__global__ void __launch_bounds__(kSearchBlock) k_count_keys(KParams kp, zsph_tmp_t t, Scratch sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned active = __ballot_sync(0xffffffffu, i < kp.n);
  if (i >= kp.n) return;
  int h = t.hash[i];
  if (h < 0 || h >= kp.G) {
    atomicOr(sc.flags, ZSPH_FLAG_BAD_KEY);
    h = h < 0 ? 0 : kp.G - 1;
  }
  sc.key[i] = h;
  sc.val[i] = t.index[i];
  sc.ticket[i] = warp_ticket(sc.cnt, h, active);
}

// Drop-in sort_data, step 1: histogram of already-sorted keys.
__global__ void __launch_bounds__(kSearchBlock) k_count_sorted(KParams kp, zsph_tmp_t t, Scratch sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned active = __ballot_sync(0xffffffffu, i < kp.n);
  if (i >= kp.n) return;
  int h = t.hash[i];
  if (h < 0 || h >= kp.G) {
    atomicOr(sc.flags, ZSPH_FLAG_BAD_KEY);
    h = h < 0 ? 0 : kp.G - 1;
  }
  warp_ticket(sc.cnt, h, active);
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

// Scan step 1: per-tile count sums and last occupied cell; the last CTA to
// finish scans the tile sums into tile offsets and finds the last key.
__global__ void __launch_bounds__(kSearchBlock) k_scan_reduce(KParams kp, Scratch sc, int tiles) {
  __shared__ int sw[kSearchBlock / 32];
  __shared__ int s_last;
  __shared__ bool s_am_last;
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int sum = 0, last = -1;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int c = base + k;
    if (c < kp.G) {
      const int v = sc.cnt[c];
      sum += v;
      if (v > 0) last = c;
    }
  }
  if (threadIdx.x == 0) s_last = -1;
  int total;
  block_exclusive_scan(sum, sw, total);
  if (last >= 0) atomicMax(&s_last, last);
  __syncthreads();
  if (threadIdx.x == 0) {
    sc.tile_sum[blockIdx.x] = total;
    sc.tile_last[blockIdx.x] = s_last;
    __threadfence();
    const int done = atomicAdd(&sc.misc[0], 1);
    s_am_last = (done == tiles - 1);
  }
  __syncthreads();
  if (!s_am_last) return;
  __threadfence();
  // Last CTA: exclusive scan over the tile sums, in chunks of kSearchBlock.
  int carry = 0, klast = -1;
  for (int b0 = 0; b0 < tiles; b0 += kSearchBlock) {
    const int b = b0 + threadIdx.x;
    const int v = b < tiles ? ((volatile int*)sc.tile_sum)[b] : 0;
    const int tl = b < tiles ? ((volatile int*)sc.tile_last)[b] : -1;
    int chunk;
    const int ex = block_exclusive_scan(v, sw, chunk);
    if (b < tiles) sc.tile_off[b] = carry + ex;
    carry += chunk;
    if (tl > klast) klast = tl;
  }
  if (threadIdx.x == 0) s_last = -1;
  __syncthreads();
  atomicMax(&s_last, klast);
  __syncthreads();
  if (threadIdx.x == 0) {
    sc.misc[1] = s_last;
    sc.misc[2] = s_last >= 0 ? sc.cnt[s_last] : 0;
    sc.misc[3] = 0;  // big-cell list length
    sc.misc[0] = 0;  // ready for the next use
  }
}

// Scan step 2: cell offsets, grid_start/grid_end in closed form, count reset.
__global__ void __launch_bounds__(kSearchBlock) k_scan_cells(KParams kp, Scratch sc, zsph_tmp_t t, int bounds) {
  __shared__ int sw[kSearchBlock / 32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int c = base + k;
    v[k] = c < kp.G ? sc.cnt[c] : 0;
    sum += v[k];
  }
  int total;
  int lb = block_exclusive_scan(sum, sw, total) + sc.tile_off[blockIdx.x];
  const int n = kp.n, klast = sc.misc[1];
  const bool last_single = sc.misc[2] == 1;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int c = base + k;
    if (c < kp.G) {
      const int lb1 = lb + v[k];
      sc.cell_lb[c] = lb;
      if (bounds && !(last_single && c > klast)) t.grid_start[c] = min(lb, n - 1);
      if (bounds && !(last_single && c >= klast)) t.grid_end[c] = min(lb1, n - 1);
      if (v[k] != 0) sc.cnt[c] = 0;
      if (v[k] > kBigSegment) {
        const int slot = atomicAdd(&sc.misc[3], 1);
        if (slot < kBigListCap) sc.big_list[slot] = c;
      }
      if (c == kp.G - 1) sc.cell_lb[kp.G] = lb1;
      lb = lb1;
    }
  }
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

__global__ void __launch_bounds__(kSearchBlock) k_scan_onepass(KParams kp, Scratch sc, zsph_tmp_t t) {
  __shared__ int sw[kSearchBlock / 32];
  __shared__ int s_tile, s_excl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_tile = atomicAdd(&sc.misc[5], 1);
  __syncthreads();
  const int tile = s_tile;
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

// Scatter by ticket (unstable inside a cell until ranked).
__global__ void __launch_bounds__(kSearchBlock) k_scatter(KParams kp, Scratch sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  sc.perm[sc.cell_lb[sc.key[i]] + sc.ticket[i]] = i;
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

// Fused search, step 3: scatter by ticket, kScatterItems particles per
// thread.  Also zeroes the last occupied cell's count and the largest key
// left for the next search by the one-pass scan.  When the scan listed
// crowded cells (more than kBigSegment members), the last CTA to finish
// (counter misc[7]) pre-sorts their members, reading the other CTAs' scatter
// through volatile accesses after a fence; otherwise no CTA takes part in
// that protocol, and the common case costs no extra launch.
__global__ void __launch_bounds__(kSearchBlock) k_scatter_fused(KParams kp, Scratch sc) {
  __shared__ bool s_last;
  const bool crowded = sc.misc[3] != 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc.cnt[sc.misc[4]] = 0;
    sc.misc[4] = 0;
  }
  const int base = blockIdx.x * (kSearchBlock * kScatterItems) + threadIdx.x;
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
  if (!crowded) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&sc.misc[7], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) sc.misc[7] = 0;
  const int listed = sc.misc[3];
  volatile int* perm = sc.perm;
  if (listed <= kBigListCap) {
    for (int e = 0; e < listed; ++e) {
      const int c = sc.big_list[e];
      const int a = sc.cell_lb[c], b = sc.cell_lb[c + 1];
      cta_sort_segment(perm + a, b - a);
    }
  } else {
    for (int c = 0; c < kp.G; ++c) {
      const int a = sc.cell_lb[c], b = sc.cell_lb[c + 1];
      if (b - a > kBigSegment) cta_sort_segment(perm + a, b - a);
    }
  }
}

// Pre-sorts the members of crowded cells (more than kBigSegment particles).
// Uses the list built by the scan, or every cell if the list overflowed.
__global__ void __launch_bounds__(1024) k_sort_big_cells(KParams kp, Scratch sc) {
  const int listed = sc.misc[3];
  if (listed == 0) return;
  if (listed <= kBigListCap) {
    for (int e = blockIdx.x; e < listed; e += gridDim.x) {
      const int c = sc.big_list[e];
      const int a = sc.cell_lb[c], b = sc.cell_lb[c + 1];
      cta_sort_segment(sc.perm + a, b - a);
    }
  } else {
    for (int c = blockIdx.x; c < kp.G; c += gridDim.x) {
      const int a = sc.cell_lb[c], b = sc.cell_lb[c + 1];
      if (b - a > kBigSegment) cta_sort_segment(sc.perm + a, b - a);
    }
  }
}

// Final slot of the particle scattered to slot t: its rank by original
// position among the members of its cell.
__device__ __forceinline__ int ranked_slot(const Scratch& sc, int t, int i, int c) {
  const int a = sc.cell_lb[c], b = sc.cell_lb[c + 1];
  if (b - a > kBigSegment) return t;  // pre-sorted by k_sort_big_cells
  int r = 0;
  for (int k = a; k < b; ++k) r += (__ldg(&sc.perm[k]) < i) ? 1 : 0;
  return a + r;
}

// Density with the sign bit marking a non-fluid particle (type != 1).
__device__ __forceinline__ float packed_rho(float rho, int type) {
  return type == 1 ? fabsf(rho) : -fabsf(rho);
}

__device__ __forceinline__ void gather_one(const zsph_ptc_t& o, const zsph_ptc_t& w, const Shadow& sh, int src,
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
  st_rec(&sh.pr(dst), make_float4(x, y, z, packed_rho(rp.x, ty_)), make_float4(vx, vy, vz, rp.y));
}

// One particle's record of the eight reference arrays (72 bytes).
struct PtcRec {
  float x, y, z, vx, vy, vz;
  float2 rp;
  float tx, ty, tz, ux, uy, uz;
  float2 trp;
  int type, table;
};

__device__ __forceinline__ void load_rec(const zsph_ptc_t& o, int src, PtcRec& r) {
  r.x = o.pos[3 * src]; r.y = o.pos[3 * src + 1]; r.z = o.pos[3 * src + 2];
  r.vx = o.vel[3 * src]; r.vy = o.vel[3 * src + 1]; r.vz = o.vel[3 * src + 2];
  r.rp = reinterpret_cast<const float2*>(o.rhop)[src];
  r.tx = o.tmp_pos[3 * src]; r.ty = o.tmp_pos[3 * src + 1]; r.tz = o.tmp_pos[3 * src + 2];
  r.ux = o.tmp_vel[3 * src]; r.uy = o.tmp_vel[3 * src + 1]; r.uz = o.tmp_vel[3 * src + 2];
  r.trp = reinterpret_cast<const float2*>(o.tmp_rhop)[src];
  r.type = o.type[src];
  r.table = o.table[src];
}

__device__ __forceinline__ void store_rec(const zsph_ptc_t& w, const Shadow& sh, const PtcRec& r, int src, int dst) {
  w.pos[3 * dst] = r.x; w.pos[3 * dst + 1] = r.y; w.pos[3 * dst + 2] = r.z;
  w.vel[3 * dst] = r.vx; w.vel[3 * dst + 1] = r.vy; w.vel[3 * dst + 2] = r.vz;
  reinterpret_cast<float2*>(w.rhop)[dst] = r.rp;
  w.tmp_pos[3 * dst] = r.tx; w.tmp_pos[3 * dst + 1] = r.ty; w.tmp_pos[3 * dst + 2] = r.tz;
  w.tmp_vel[3 * dst] = r.ux; w.tmp_vel[3 * dst + 1] = r.uy; w.tmp_vel[3 * dst + 2] = r.uz;
  reinterpret_cast<float2*>(w.tmp_rhop)[dst] = r.trp;
  w.type[dst] = r.type;
  w.table[dst] = r.table + src - dst;  // sort.cu:82
  st_rec(&sh.pr(dst), make_float4(r.x, r.y, r.z, packed_rho(r.rp.x, r.type)),
         make_float4(r.vx, r.vy, r.vz, r.rp.y));
}

// Fused search, last step: rank, write sorted hash/index, gather the eight
// particle arrays (sort.cu:62-82) and the packed shadows.  The source record's
// loads are issued as soon as the source is known, before the rank (which
// needs the key, the cell's range and its members) is counted, so they
// overlap that dependent chain.
__global__ void __launch_bounds__(kSearchBlock) k_rank_gather(KParams kp, Scratch sc, zsph_ptc_t o, zsph_ptc_t w,
                                                              zsph_tmp_t t) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= kp.n) return;
  const int i = sc.perm[slot];
  PtcRec r;
  load_rec(o, i, r);
  const int cpk = kp.c3o ? kp.c3o[i] : 0;
  const int c = sc.key[i];
  const int dst = ranked_slot(sc, slot, i, c);
  t.index[dst] = i;
  t.hash[dst] = c;
  store_rec(w, sc.sh, r, i, dst);
  if (kp.c3o) kp.c3n[dst] = cpk;
}

// Drop-in sort_index, last step: sorted keys and carried values.
__global__ void __launch_bounds__(kSearchBlock) k_rank_values(KParams kp, Scratch sc, zsph_tmp_t t) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= kp.n) return;
  const int i = sc.perm[slot];
  const int c = sc.key[i];
  const int dst = ranked_slot(sc, slot, i, c);
  t.hash[dst] = c;
  t.index[dst] = sc.val[i];
}

// Drop-in sort_data reorder: new[t] = old[index[t]] (sort.cu:62-82).
__global__ void __launch_bounds__(kSearchBlock) k_gather_by_index(KParams kp, Scratch sc, zsph_ptc_t o,
                                                                  zsph_ptc_t w, zsph_tmp_t t) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= kp.n) return;
  gather_one(o, w, sc.sh, t.index[slot], slot);
}

// Exact per-cell particle ranges [cell_lb[c], cell_lb[c+1]) of an already
// sorted key array (drop-in pair entry points, whose caller sorted the
// particles; the fused search produces them in its scan).  Each particle
// that starts a new key fills the offsets of the cells since the previous key.
__global__ void __launch_bounds__(kSearchBlock) k_cell_lb(KParams kp, Scratch sc, zsph_tmp_t t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  const int k = min(max(t.hash[i], 0), kp.G - 1);
  const int kprev = i > 0 ? min(max(t.hash[i - 1], 0), kp.G - 1) : -1;
  for (int c = kprev + 1; c <= k; ++c) sc.cell_lb[c] = i;
  if (i == kp.n - 1)
    for (int c = max(k, kprev) + 1; c <= kp.G; ++c) sc.cell_lb[c] = kp.n;
}

// Packed shadows of an unsorted-by-us state (drop-in pair entry points).
__global__ void __launch_bounds__(kSearchBlock) k_pack(KParams kp, Shadow sh, zsph_ptc_t s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  const float2 rp = reinterpret_cast<const float2*>(s.rhop)[i];
  st_rec(&sh.pr(i), make_float4(s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2], packed_rho(rp.x, s.type[i])),
         make_float4(s.vel[3 * i], s.vel[3 * i + 1], s.vel[3 * i + 2], rp.y));
}

inline int blocks_for(int n, int b) { return (n + b - 1) / b; }

cudaError_t launch_scan(const KParams& kp, const Scratch& s, int tiles, const zsph_tmp_t& t, int bounds,
                        cudaStream_t st, Prof* pf = nullptr) {
  k_scan_reduce<<<tiles, kSearchBlock, 0, st>>>(kp, s, tiles);
  mark(pf, "scan_reduce", st);
  k_scan_cells<<<tiles, kSearchBlock, 0, st>>>(kp, s, t, bounds);
  mark(pf, "scan_cells", st);
  return cudaGetLastError();
}

constexpr int kBigSortCtas = 148;

}  // namespace

cudaError_t launch_hash(const KParams& kp, int* flags, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                        cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  k_hash<<<blocks_for(kp.n, kSearchBlock), kSearchBlock, 0, st>>>(kp, ptc, tmp, flags);
  return cudaGetLastError();
}

cudaError_t launch_sort_index(const KParams& kp, const Scratch& s, int tiles, const zsph_tmp_t& tmp,
                              cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  const int nb = blocks_for(kp.n, kSearchBlock);
  k_count_keys<<<nb, kSearchBlock, 0, st>>>(kp, tmp, s);
  // cell offsets only: cuda_sort_index leaves grid_start/grid_end alone
  cudaError_t e = launch_scan(kp, s, tiles, tmp, 0, st);
  if (e) return e;
  k_scatter<<<nb, kSearchBlock, 0, st>>>(kp, s);
  k_sort_big_cells<<<kBigSortCtas, 1024, 0, st>>>(kp, s);
  k_rank_values<<<nb, kSearchBlock, 0, st>>>(kp, s, tmp);
  return cudaGetLastError();
}

cudaError_t launch_sort_data(const KParams& kp, const Scratch& s, int tiles, const zsph_ptc_t& o,
                             const zsph_ptc_t& w, const zsph_tmp_t& tmp, cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  const int nb = blocks_for(kp.n, kSearchBlock);
  k_count_sorted<<<nb, kSearchBlock, 0, st>>>(kp, tmp, s);
  cudaError_t e = launch_scan(kp, s, tiles, tmp, 1, st);
  if (e) return e;
  k_gather_by_index<<<nb, kSearchBlock, 0, st>>>(kp, s, o, w, tmp);
  return cudaGetLastError();
}

cudaError_t launch_search(const KParams& kp, const Scratch& s, int tiles, const zsph_ptc_t& o, const zsph_ptc_t& w,
                          const zsph_tmp_t& tmp, cudaStream_t st, Prof* pf) {
  if (kp.n == 0) return cudaSuccess;
  k_hash_count<<<blocks_for(kp.n, kSearchBlock * kHashItems), kSearchBlock, 0, st>>>(kp, o, s);
  mark(pf, "hash_count", st);
  k_scan_onepass<<<(kp.G + kOneTile - 1) / kOneTile, kSearchBlock, 0, st>>>(kp, s, tmp);
  mark(pf, "scan", st);
  k_scatter_fused<<<blocks_for(kp.n, kSearchBlock * kScatterItems), kSearchBlock, 0, st>>>(kp, s);
  mark(pf, "scatter", st);
  k_rank_gather<<<blocks_for(kp.n, kSearchBlock), kSearchBlock, 0, st>>>(kp, s, o, w, tmp);
  mark(pf, "rank_gather", st);
  return cudaGetLastError();
}

cudaError_t launch_pack_shadows(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  k_pack<<<blocks_for(kp.n, kSearchBlock), kSearchBlock, 0, st>>>(kp, s.sh, ptc);
  return cudaGetLastError();
}

cudaError_t launch_pack(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& tmp,
                        cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  k_pack<<<blocks_for(kp.n, kSearchBlock), kSearchBlock, 0, st>>>(kp, s.sh, ptc);
  k_cell_lb<<<blocks_for(kp.n, kSearchBlock), kSearchBlock, 0, st>>>(kp, s, tmp);
  return cudaGetLastError();
}

}  // namespace zsph
