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

#include "search_dev.cuh"

namespace zsph {
namespace {

// device helpers and stage bodies: search_dev.cuh

// Drop-in cuda_ptc_hash: hash + identity index (hash.cu:3-26).
__global__ void __launch_bounds__(kSearchBlock) k_hash(KParams kp_in, zsph_ptc_t s, zsph_tmp_t t, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp_in.n) return;
  const KParams kp = kp_of_particle(kp_in, i);
  t.hash[i] = hash_and_kill(kp, s, i, flags);
  t.index[i] = i;
}

// PLAIN: the single-scene FP32 form (no packed cells, no scene table).
template <bool PLAIN>
__global__ void __launch_bounds__(kSearchBlock) k_hash_count(KParams kp_in, zsph_ptc_t s, Scratch sc) {
  pdl_wait();
  hash_count_body<PLAIN>(kp_in, s, sc, blockIdx.x);
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

__global__ void __launch_bounds__(kSearchBlock) k_scan_onepass(KParams kp, Scratch sc, zsph_tmp_t t) {
  __shared__ int s_tile;
  pdl_wait();
  if (threadIdx.x == 0) s_tile = atomicAdd(&sc.misc[5], 1);
  __syncthreads();
  scan_onepass_body(kp, sc, t, s_tile);
}

// Scatter by ticket (unstable inside a cell until ranked).
__global__ void __launch_bounds__(kSearchBlock) k_scatter(KParams kp, Scratch sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  sc.perm[sc.cell_lb[sc.key[i]] + sc.ticket[i]] = i;
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
  pdl_wait();
  const bool crowded = sc.misc[3] != 0;
  scatter_body(kp, sc, blockIdx.x);
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

// Fused search, last step: rank, write sorted hash/index, gather the eight
// particle arrays (sort.cu:62-82) (rank_gather_one).  The packed records of
// the sorted state are written by the list build, which reads each
// particle's arrays anyway.  Eight resident CTAs (32 registers, no spills).
__global__ void __launch_bounds__(kSearchBlock, 8) k_rank_gather(KParams kp, Scratch sc, zsph_ptc_t o, zsph_ptc_t w,
                                                                 zsph_tmp_t t) {
  pdl_wait();
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot == 0) sc.misc[kMiscFluidEpoch] = sc.misc[6];  // this search's cell stamps are valid
  if (slot >= kp.n) return;
  rank_gather_one(kp, sc, o, w, t, slot);
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
  if (slot == 0) sc.misc[kMiscFluidEpoch] = 0;  // no cell stamps for this sort: the wall pass takes every wall
  if (slot >= kp.n) return;
  gather_one(o, w, t.index[slot], slot);
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
  if (!ptc_aligned8(o) || !ptc_aligned8(w)) return cudaErrorMisalignedAddress;  // nothing launched
  // each kernel waits for its predecessor's completion first (pdl_wait), so
  // only the launches overlap the predecessors' drain
  const bool plain = !kp.c3o && !kp.scenes;
  cudaError_t e = launch_pdl(plain ? k_hash_count<true> : k_hash_count<false>,
                             blocks_for(kp.n, kSearchBlock * kHashItems), kSearchBlock, 0, st, kp, o, s);
  mark(pf, "hash_count", st);
  if (!e) e = launch_pdl(k_scan_onepass, (kp.G + kOneTile - 1) / kOneTile, kSearchBlock, 0, st, kp, s, tmp);
  mark(pf, "scan", st);
  if (!e) e = launch_pdl(k_scatter_fused, blocks_for(kp.n, kSearchBlock * kScatterItems), kSearchBlock, 0, st, kp, s);
  mark(pf, "scatter", st);
  if (!e) e = launch_pdl(k_rank_gather, blocks_for(kp.n, kSearchBlock), kSearchBlock, 0, st, kp, s, o, w, tmp);
  mark(pf, "rank_gather", st);
  return e ? e : cudaGetLastError();
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
