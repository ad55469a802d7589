// delta-SPH pair-interaction kernels for sm_100a.
//
// Reference path replaced (single_gpu_sph_src/):
//   equation/delta_ns.cu:5-177   cuda_boundary_ns  -> k_nblist_seq (lists) + k_walls (wall pressure) + k_boundary
//   equation/delta_ns.cu:179-267 cuda_govering_ns  -> k_governing (optionally fused with time_int.cu)
//   lib/time_int.cu:3-92         cuda_prediction / cuda_correction -> k_integrate or k_governing epilogue
//
// Design.  The reference re-scans every candidate of the cell stencil in each
// of its three neighbour loops per sub-step, one thread per particle, and
// every lane of a warp pays for the full pair arithmetic whenever any lane
// has a neighbour.  Here:
//  * The list build filters the candidates ONCE per sub-step (the governing
//    stencil is a superset of the boundary stencil).  k_nblist_seq gives
//    each warp 32 consecutive sorted particles, one per lane.  Candidates
//    are staged 64 at a time in shared memory and tested two per step with
//    packed f32x2 arithmetic; the hits are emitted in candidate order, so a
//    list is in the reference's visit order: stencil rows in (z, y) order,
//    inside a row the sorted particle range.  Entries are 16-bit,
//    row << 11 | offset inside the particle's row range, 128 per particle,
//    stored blocked by 32-particle groups (nb_vec) and read 8 per 16-byte load.
//  * k_boundary and k_governing walk their particle's list with one thread
//    per particle, all lanes converged, loading the next four neighbours'
//    packed data before doing their arithmetic: one 256-bit load of the
//    neighbour's 32-byte shadow record (position, density, velocity,
//    pressure), plus its grad(rho) in k_governing.  The walk is bound by the
//    L1 data pipe (the 32 lanes' k-th neighbours spread over ~12 lines), so
//    one wide request per neighbour costs fewer L1 wavefronts than two
//    16-byte ones.  k_boundary folds the
//    reference's second loop into its first walk.  The visit order is the
//    reference's, so the order-dependent recurrence on grad(rho).x
//    (delta_ns.cu:244-245) sees the same sequence.
//  * The pair arithmetic uses hardware reciprocal and square-root
//    approximations (MUFU, relative error ~1 ulp) in place of IEEE divisions;
//    results agree with the reference to FP32 rounding, not bitwise.
//
// Neighbour test: the reference's q = sqrtf(r2)/h <= 2 (delta_ns.cu:67-68),
// with r2 formed as fma(dz,dz,fma(dy,dy,dx*dx)).  IEEE sqrt and division
// are monotone, so the test holds exactly for r2 <= r2max, the largest float
// that passes it (found on the host with the same float operations): one
// compare gives the reference's neighbour set.
//
// Particle type: only "fluid (type 1)" vs "not fluid" enters the equations,
// so the packed shadow stores the density with the sign bit set for
// non-fluid particles (densities are non-negative).
//
// Wall densities: the reference writes them in place while neighbours read
// them (a race, delta_ns.cu:65,130,151).  Here k_walls extrapolates every
// wall's (rho, p) first and publishes it in the packed shadows; k_boundary
// reads neighbours' densities from the shadows (new wall values) and a
// wall's own old density from ptc.rhop, and writes the new wall values to
// ptc.rhop at the end, when no reader is left.
#include <cuda_bf16.h>

#include <climits>

#include "integrate.cuh"
#include "search_dev.cuh"
#include "zsph_internal.cuh"

namespace zsph {
namespace {

template <int GF> struct Stencil {
  static constexpr int W = 2 * GF + 1;  // rows per z-plane
  static constexpr int NR = W * W;      // governing rows (y = -GF..GF)
  __device__ static bool boundary_row(int r) { return (r % W) < 2 * GF; }  // y = -GF..GF-1
};

constexpr int kRowShift = 11;
constexpr int kOffMask = (1 << kRowShift) - 1;
constexpr uint8_t kOverflow = 255;
constexpr int kListVec = kMaxNb / 8;  // uint4 per particle list

// Lists are stored blocked by groups of 32 consecutive particles: entries
// 8b..8b+7 of particle i (one uint4) sit at uint4 index nb_vec(i, b), so the
// 32 lanes of a warp walking 32 consecutive particles read 512 contiguous
// bytes per list load, and the list build writes them the same way.
__device__ __forceinline__ size_t nb_vec(int i, int b) {
  return ((size_t)(i >> 5) * kListVec + (size_t)b) * 32 + (size_t)(i & 31);
}
// entry k of particle i's skin list (list transfer), blocked the same way
__device__ __forceinline__ size_t sk_idx(int i, int k) {
  return ((size_t)(i >> 5) * kSkinCap + (size_t)k) * 32 + (size_t)(i & 31);
}

__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrt_fast(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ bool fluid_of(float w) { return !signbit(w); }

__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// The reference's neighbour test q = sqrtf(rr2)/h <= 2 (delta_ns.cu:67-68):
// IEEE sqrt and division are monotone, so it holds exactly for rr2 <= r2max.
__device__ __forceinline__ bool interacts(const KParams& kp, float rr2) { return rr2 <= kp.r2max; }

// Range [s, e) of stencil row r of a particle in cell c (delta_ns.cu:39-46),
// clamped to the particle range so that bounds a caller left stale can never
// index outside the arrays (bounds the search writes are always inside).
template <int GF>
__device__ __forceinline__ void row_range(const KParams& kp, const zsph_tmp_t& t, int c, int r, int& s, int& e) {
  const zsph_gpu_param_t& p = kp.p;
  const int z = r / Stencil<GF>::W - GF, y = r % Stencil<GF>::W - GF;
  const int cell = c + z * kp.XY + y * p.grid_xdim;
  const int cs = cell - GF, ce = cell + GF;
  s = 0;
  e = 0;
  if (cs >= p.grid_hash_min && ce <= p.grid_hash_max) {
    s = max(t.grid_start[cs], 0);
    e = min(t.grid_end[ce], kp.n);
  }
}

template <int GF>
__device__ __forceinline__ void load_rows(const KParams& kp, const zsph_tmp_t& t, int c, int* rs, int* re) {
#pragma unroll
  for (int r = 0; r < Stencil<GF>::NR; ++r) {
    int s, e;
    row_range<GF>(kp, t, c, r, s, e);
    rs[r * kPairBlock] = s;
    re[r * kPairBlock] = e;
  }
}

// Walks particle i's neighbours in visit order.  List entries (row r,
// offset o) name the global particle rs[r] + o; what the arithmetic needs is
// fetched from index fb[r] + o (fb = rs for the global arrays, or the row's
// base in a shared-memory window), four neighbours ahead of their
// arithmetic; invalid slots fetch index fdummy.  Every caller builds the
// lists from the same cell bounds just before the walk, so o is inside the
// row; the fetch index is only clamped to fmax (the last particle, or the
// window's last slot), which keeps every access in bounds without a
// shared-memory load of the row end per entry.  Particles whose list
// overflowed re-filter their stencil rows directly (in the precision form
// with the candidates moved into the frame of the particle's cell ci).
template <bool PRECISE>
__device__ __forceinline__ float4 shadow_pr(const KParams& kp, const Scratch& s, int j, int3 ci);

template <int GF, bool BOUNDARY_ONLY, class Nb, bool PRECISE = false, class Fetch, class Use>
__device__ __forceinline__ void walk(const KParams& kp, const Scratch& s, int i, float4 pi, const int* rs,
                                     const int* re, const int* fb, int fdummy, int fmax, Fetch&& fetch,
                                     Use&& use, int3 ci = int3{0, 0, 0}) {
  const int cnt = s.nb_cnt[i];
  if (cnt != kOverflow) {
    const uint4* lst = reinterpret_cast<const uint4*>(s.nb);
    for (int k = 0; k < cnt; k += 8) {
      const uint4 v = lst[nb_vec(i, k >> 3)];
      const unsigned wv[4] = {v.x, v.y, v.z, v.w};
      int js[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const unsigned ent = (wv[e >> 1] >> ((e & 1) * 16)) & 0xffffu;
        const int r = (int)(ent >> kRowShift), off = (int)(ent & kOffMask);
        const bool ok = (k + e < cnt) && (!BOUNDARY_ONLY || Stencil<GF>::boundary_row(r));
        js[e] = ok ? min(fb[r * kPairBlock] + off, fmax) : -1;
      }
#pragma unroll
      for (int h = 0; h < 8; h += 4) {
        Nb nb[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) nb[e] = fetch(js[h + e] >= 0 ? js[h + e] : fdummy);
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (js[h + e] >= 0) use(nb[e]);
      }
    }
    return;
  }
  for (int r = 0; r < Stencil<GF>::NR; ++r) {
    if (BOUNDARY_ONLY && !Stencil<GF>::boundary_row(r)) continue;
    const int a = rs[r * kPairBlock], b = re[r * kPairBlock];
    for (int j = a; j < b; ++j) {
      if (j == i) continue;
      const float4 pj = shadow_pr<PRECISE>(kp, s, j, ci);
      if (interacts(kp, dist2(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z))) use(fetch(fb[r * kPairBlock] + (j - a)));
    }
  }
}

// ---- shared-memory neighbour windows staged with TMA bulk copies ---------

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// A CTA's window: for each staged stencil row r, the union [w0, w0+len) of
// its particles' candidate ranges, packed at offset woff in shared memory.
// Thread 0 issues one cp.async.bulk per row and array, completing on one
// mbarrier; every thread then waits with a bounded number of polls.
struct WinHdr {
  int w0[32], w1[32], woff[32], len[32];
  unsigned long long bar;
  int total, staged;
};

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ bool bar_try_wait(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

constexpr int kWaitPolls = 1 << 22;  // bounded wait on the window barrier (each poll suspends briefly)

// Computes the window of the CTA's particles over the rows selected by ROWS
// (ROWS(r) true), copies NARR packed arrays, whose elements are wid[a]
// float4s wide, into `win` (array a at win + cap * (wid[0] + .. + wid[a-1]))
// and rewrites fb (per-thread row bases) to shared indices.
// Returns false (and leaves fb = rs) when the window does not fit `cap`
// candidates or the copies did not complete in time.
template <int NR, int NARR, class RowSel>
__device__ bool stage_window(WinHdr& wh, float4* win, int cap, const float4* const (&src)[NARR],
                             const int (&wid)[NARR], bool act, const int* rs, const int* re, int* fb, int* flags, RowSel rows) {
  const int tid = threadIdx.x;
  if (tid < NR) {
    wh.w0[tid] = 0x7fffffff;
    wh.w1[tid] = -1;
  }
  __syncthreads();
  if (act) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int a = rs[r * kPairBlock], b = re[r * kPairBlock];
      if (rows(r) && a < b) {
        atomicMin(&wh.w0[r], a);
        atomicMax(&wh.w1[r], b);
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    int tot = 0;
    for (int r = 0; r < NR; ++r) {
      const int l = wh.w1[r] > wh.w0[r] ? wh.w1[r] - wh.w0[r] : 0;
      wh.len[r] = l;
      wh.woff[r] = tot;
      tot += l;
    }
    wh.total = tot;
    wh.staged = (tot > 0 && tot <= cap) ? 1 : 0;
    if (wh.staged) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&wh.bar)), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  __syncthreads();
  if (!wh.staged) return false;
  if (tid == 0) {
    int wsum = 0;
#pragma unroll
    for (int a = 0; a < NARR; ++a) wsum += wid[a];
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&wh.bar)),
                 "r"((uint32_t)(wh.total * wsum * 16))
                 : "memory");
    for (int r = 0; r < NR; ++r)
      if (wh.len[r] > 0) {
        int base = 0;
#pragma unroll
        for (int a = 0; a < NARR; ++a) {
          bulk_copy(win + (size_t)base * cap + (size_t)wh.woff[r] * wid[a], src[a] + (size_t)wh.w0[r] * wid[a],
                    (uint32_t)(wh.len[r] * wid[a] * 16), &wh.bar);
          base += wid[a];
        }
      }
  }
  if (act) {
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (rows(r)) fb[r * kPairBlock] = wh.woff[r] + (rs[r * kPairBlock] - wh.w0[r]);
  }
  int polls = 0;
  bool done = false;
  while (!(done = bar_try_wait(&wh.bar, 0)) && ++polls < kWaitPolls) {
  }
  if (!done) {  // never expected: report, let the copies land, use the global arrays
    atomicOr(flags, ZSPH_FLAG_TIMEOUT);
    polls = 0;
    while (!bar_try_wait(&wh.bar, 0) && ++polls < kWaitPolls) {
    }
  }
  return __syncthreads_and(done ? 1 : 0) != 0;
}


// Precision form: neighbour j's packed shadow moved into the frame of cell
// ci (positions are offsets from the own cell's corner; neighbouring cells
// differ by at most two in each coordinate, so k * gs is exact and the sum
// rounds once, at the scale of a few cells).
__device__ __forceinline__ float4 shifted(const KParams& kp, float4 pj, int cj, int3 ci) {
  const int3 c = unpack_cell(cj);
  const float gs = kp.p.grid_size;
  pj.x += (float)(c.x - ci.x) * gs;
  pj.y += (float)(c.y - ci.y) * gs;
  pj.z += (float)(c.z - ci.z) * gs;
  return pj;
}
template <bool PRECISE>
__device__ __forceinline__ float4 shadow_pr(const KParams& kp, const Scratch& s, int j, int3 ci) {
  const float4 pj = s.sh.pr(j);
  return PRECISE ? shifted(kp, pj, kp.c3n[j], ci) : pj;
}
// Neighbour j's whole record (one 256-bit load), positions as shadow_pr.
template <bool PRECISE>
__device__ __forceinline__ ShadowRec shadow_rec(const KParams& kp, const Scratch& s, int j, int3 ci) {
  ShadowRec r = s.sh.load(j);
  if (PRECISE) r.pr = shifted(kp, r.pr, kp.c3n[j], ci);
  return r;
}

// One fluid neighbour's term of a wall's (rho, p) extrapolation
// (delta_ns.cu:61-85): neighbour position pj, its (rho, p) rp.
__device__ __forceinline__ void wall_term_core(const KParams& kp, float4 pi, float4 pj, float2 rp, float& rsum,
                                               float& wsum) {
  const zsph_gpu_param_t& p = kp.p;
  const float dz = pi.z - pj.z;
  const float q = __fsqrt_rn(dist2(pi.x - pj.x, pi.y - pj.y, dz)) / p.h;
  const float aa = 1.0f - q / 2.0f;
  float w = aa * aa * aa;
  w = w * aa;
  w *= (2.0f * q + 1.0f) * p.adh;
  rsum += (rp.y - fabsf(rp.x) * ((0.0f - p.g) * dz)) * w;
  wsum += w;
}

// Wall pressure contribution of fluid neighbour j of wall particle i
// (delta_ns.cu:67-85), from j's packed record (one 256-bit load; the sign of
// its density marks a non-fluid particle).
template <bool PRECISE = false>
__device__ __forceinline__ void wall_term(const KParams& kp, const Scratch& s, float4 pi, int j, float& rsum,
                                          float& wsum, int3 ci = int3{0, 0, 0}) {
  const ShadowRec r = shadow_rec<PRECISE>(kp, s, j, ci);
  if (!fluid_of(r.pr.w)) return;
  wall_term_core(kp, pi, r.pr, make_float2(r.pr.w, r.vp.w), rsum, wsum);
}

// Particle j's position from the sorted arrays, in the precision form moved
// into the frame of cell ci (the list build reads the arrays: it writes the
// packed records itself).
template <bool PRECISE>
__device__ __forceinline__ float4 ptc_xyz(const KParams& kp, const zsph_ptc_t& ptc, int j, int3 ci) {
  const float4 p = make_float4(ptc.pos[3 * j], ptc.pos[3 * j + 1], ptc.pos[3 * j + 2], 0.0f);
  return PRECISE ? shifted(kp, p, kp.c3n[j], ci) : p;
}

// wall_term with the fluid neighbour's data from the sorted arrays
template <bool PRECISE = false>
__device__ __forceinline__ void wall_term_ptc(const KParams& kp, const zsph_ptc_t& ptc, float4 pi, int j,
                                              float& rsum, float& wsum, int3 ci = int3{0, 0, 0}) {
  if (ptc.type[j] != 1) return;
  wall_term_core(kp, pi, ptc_xyz<PRECISE>(kp, ptc, j, ci), reinterpret_cast<const float2*>(ptc.rhop)[j], rsum, wsum);
}

using u64 = unsigned long long;
// Packed FP32 pairs (sm_100 f32x2 instructions): each half is rounded
// exactly as the scalar operation, so r^2 keeps the reference's rounding.
__device__ __forceinline__ u64 pk2(float a, float b) {
  u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(u64 v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ u64 sub2(u64 a, u64 b) {
  u64 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
  u64 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
  u64 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// Whether a non-fluid particle in cell c can have a fluid neighbour in its
// boundary rows (grid factor 1): a kept row (row_range) with possibly stale
// bounds (sort.cu:30-60: a lone last particle in cell klast leaves the
// bounds of cells >= klast) or a cell stamped by this search's gather as
// holding a fluid particle.  False means the wall pass would sum nothing.
// Without valid stamps (the drop-in gather ran) the answer is true.
__device__ __forceinline__ bool walls_fluid_near(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, int c) {
  const int ep = s.misc[kMiscFluidEpoch];
  if (ep == 0) return true;
  const zsph_gpu_param_t& p = kp.p;
  const int n = kp.n, klast = t.hash[n - 1];
  const bool lone = n < 2 || klast != t.hash[n - 2];
  bool any = false;
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dy = -1; dy <= 0; ++dy) {  // the boundary rows, y = -1 and 0 (delta_ns.cu:37)
      const int cell = c + dz * kp.XY + dy * p.grid_xdim;
      const int cs = cell - 1, ce = cell + 1;
      if (cs < p.grid_hash_min || ce > p.grid_hash_max) continue;  // row_range drops it: no candidates
      any |= (lone && ce >= klast) || s.cfe[cs] == ep || s.cfe[cell] == ep || s.cfe[ce] == ep;
    }
  return any;
}

// The end of particle i's list build, once s.nb holds its finished list
// (cnt entries, or ovf): the particle's packed shadow record and list
// count, and, for a non-fluid particle that can have a fluid neighbour in
// its boundary rows (fluid_nb), its slot appended to s.wl for the wall pass
// (k_walls).  A non-fluid particle that cannot gets the wall pass's result
// for an empty sum here: p = 0, rho = rho0.  Every active lane of the warp
// calls it together.
template <int GF, bool PRECISE>
__device__ __forceinline__ void list_tail(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, int i, int cnt,
                                          bool ovf, float4 pi, float2 rp_self, bool fluid_nb) {
  float4 vp = make_float4(ptc.vel[3 * i], ptc.vel[3 * i + 1], ptc.vel[3 * i + 2], rp_self.y);
  float4 pr = pi;
  const bool nonfluid = !fluid_of(pi.w);
  if (nonfluid && !fluid_nb) {
    const float rsum = 0.0f;
    pr.w = -(rsum / kp.p.cs2 + kp.p.rho0);  // still non-fluid
    vp.w = rsum;
  }
  st_rec(&s.sh.pr(i), pr, vp);
  s.nb_cnt[i] = ovf ? kOverflow : (uint8_t)cnt;
  if (ovf) atomicOr(s.flags, ZSPH_FLAG_NB_OVERFLOW);  // rare: the walks re-filter this particle's rows
  const unsigned m = __activemask();
  const bool wall = nonfluid && fluid_nb;
  const unsigned wm = __ballot_sync(m, wall);
  if (wm) {  // one atomic per warp
    const int leader = __ffs(m) - 1;
    int base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&s.misc[kMiscWalls], __popc(wm));
    base = __shfl_sync(m, base, leader);
    const int slot = base + __popc(wm & lanemask_lt());
    if (wall && slot < kp.n) s.wl[slot] = i;
  }
}


constexpr int kCellWarps = 4;  // warps per CTA in the list build
// Builds the neighbour lists of 32 consecutive sorted particles per warp,
// one lane per particle (the plain form).  A cell holds about 18-24
// particles, so one warp per cell leaves lanes idle; here every lane has a
// particle.  The lanes of one cell are contiguous; a round takes up to kSegs
// cells (segments; usually all of the warp's two or three).  For each
// stencil row every segment's row range (delta_ns.cu:39-46) is staged, 64
// candidates at a time, in that segment's x/y/z arrays in shared memory, and
// every lane tests its own cell's range, two candidates per step with packed
// f32x2 arithmetic, in blocks of eight so a short row is not padded to 64.
// Testing the union of the segments' ranges instead (one set of arrays)
// costs 1.6x the candidate tests on the dam-break cases.  Hits come out in
// candidate order, so a list is in the reference's visit order, and its
// entries are offsets from the lane's row start.  Each lane emits the hits
// of a 16-candidate half block into its 32-entry ring in shared memory;
// after the half, the lanes write their completed 8-entry blocks together (a
// nearly converged loop) with 16-byte stores to the blocked list layout.
// Flushing at a lane's 8th entry inside the per-hit loop instead diverges:
// each flush then runs for 2-3 lanes.
//
// Precision form: candidates are moved into the frame of the lane's own
// cell (its position is the offset from that cell's corner, as in the pair
// kernels); every candidate lies within GF cells of it, so each shift k * gs
// is exact and one rounding forms every coordinate.
//
// The walls' (rho, p) come after, from the finished lists (k_walls).
constexpr int kRing = 32;  // list-build ring entries per lane (power of two)
constexpr int kSegs = 4;   // list build: cells whose lanes test their own rows concurrently
constexpr int kStage = 66; // list build: staged candidates per segment (64) plus two floats of padding
// warps per CTA of k_nblist_seq (the 5x5 stencil's row starts need more shared memory)
template <int GF> constexpr int kSeqWarps = GF == 1 ? kCellWarps : 2;

// At least 42 warps per SM (a register budget of 40-48 without spills in the
// plain form, 9.9 KB of shared memory per 2-warp CTA): the kernel is
// issue-bound and hides its staging loads with more resident warps.
//
// nblist_group is the work of one warp on group `group` (particles
// 32*group .. 32*group+31); k_nblist_seq runs one group per warp, the
// batched form's persistent kernel loops over groups.  The warp's staging
// arrays are slot `wid` of the CTA's CW slots.
template <int GF, int CW, bool BATCH, bool PRECISE, int SEGS = kSegs, bool SKIN = false>
__device__ __forceinline__ void nblist_group(const KParams& kp_arg, const Scratch& s, const zsph_ptc_t& ptc,
                                             const zsph_tmp_t& t, int group, int wid) {
  constexpr int NR = Stencil<GF>::NR;
  // per segment (cell) of a round: its 64 staged candidates' x, y and z; the
  // two floats of padding per array put the segments' arrays in different banks
  __shared__ __align__(16) float s_c[CW][SEGS][3][kStage];
  // per lane: a 32-entry ring (a partial 8-entry block plus one half block's
  // hits fit), padded to 80 bytes so that the lanes' rings spread over the banks
  __shared__ __align__(16) uint16_t s_ring[CW][32][kRing + 8];
  const int lane = threadIdx.x & 31;
  const int p0 = group * 32;
  if (p0 >= kp_arg.n) return;  // uniform per warp
  const int i = p0 + lane;
  const bool act = i < kp_arg.n;
  const int c = act ? t.hash[i] : INT_MAX;  // sorted: non-decreasing over the lanes
  // batched form: the scene of the lane's cell (scenes own disjoint cell ranges)
  const int scn = BATCH && act ? scene_of(kp_arg.scene_cbase, kp_arg.nscenes, c) : 0;
  // the lane's own position and packed density (its record is written at the end)
  const int iself = act ? i : p0;
  const float2 rp_self = reinterpret_cast<const float2*>(ptc.rhop)[iself];
  const float4 pi = make_float4(ptc.pos[3 * iself], ptc.pos[3 * iself + 1], ptc.pos[3 * iself + 2],
                                packed_rho(rp_self.x, ptc.type[iself]));
  // precision form: the lane's own cell (its position is the offset from that cell's corner)
  const int3 ci = PRECISE && act ? unpack_cell(kp_arg.c3n[i]) : int3{0, 0, 0};
  // the lane's scene (batched form): its cell's neighbour threshold and grid
  const KParams kp = BATCH ? scene_kp(kp_arg, scn) : kp_arg;
  const float r2max = kp.r2max;
  const u64 px = pk2(pi.x, pi.x), py = pk2(pi.y, pi.y), pz = pk2(pi.z, pi.z);
  uint16_t* ring = s_ring[wid][lane];
  uint4* nbv = reinterpret_cast<uint4*>(s.nb);
  int cnt = 0;   // entries emitted
  int done = 0;  // entries written to global memory (a multiple of 8)
  bool ovf = false;
  // SKIN (the list transfer's predictor): the candidates with
  // r2max < r^2 <= r2skin, in candidate order, into the skin list
  const float r2skin = kp.r2skin;
  int kc = 0;
  bool skovf = false;
  // writes the completed 8-entry blocks among the first min(cnt, kMaxNb) entries
  auto flush = [&]() {
    const int lim = min(cnt, kMaxNb);
    for (; done + 8 <= lim; done += 8)
      nbv[nb_vec(i, done >> 3)] = *reinterpret_cast<const uint4*>(ring + (done & (kRing - 1)));
  };
  // The lanes of one cell are contiguous (sorted particles).  A round takes
  // the next kSegs cells (segments): per stencil row each segment's range is
  // staged in its own arrays and every lane tests its own cell's range, so no
  // lane tests candidates outside its range.
  const int cprev = __shfl_up_sync(0xffffffffu, c, 1);
  const unsigned starts = __ballot_sync(0xffffffffu, act && (lane == 0 || c != cprev));
  unsigned todo = __ballot_sync(0xffffffffu, act);
  while (todo) {
    const unsigned sm = starts & todo;  // todo is a run of whole cells
    const int seg = ((todo >> lane) & 1u) ? __popc(sm & (0xffffffffu >> (31 - lane))) - 1 : SEGS;
    const bool inseg = seg < SEGS;
    todo &= ~__ballot_sync(0xffffffffu, inseg);
    const int nseg = min(__popc(sm), SEGS);
    const float* sx = s_c[wid][inseg ? seg : 0][0];  // y and z follow at kStage, 2 * kStage
    for (int r = 0; r < NR; ++r) {
      int sl = 0, el = 0;
      if (inseg) row_range<GF>(kp, t, c, r, sl, el);
      const int len = inseg ? max(el - sl, 0) : 0;
      const int L = __reduce_max_sync(0xffffffffu, len);
      for (int k0 = 0; k0 < L; k0 += 64) {
        __syncwarp();
        unsigned m = sm;
        for (int g = 0; g < nseg; ++g) {  // uniform: stage segment g's candidates k0 .. k0+63
          const int lead = __ffs(m) - 1;
          m &= m - 1;
          const int sg = __shfl_sync(0xffffffffu, sl, lead), lg = __shfl_sync(0xffffffffu, len, lead);
          // precision form: candidates move into the frame of the segment's cell
          int3 cg{0, 0, 0};
          if (PRECISE)
            cg = make_int3(__shfl_sync(0xffffffffu, ci.x, lead), __shfl_sync(0xffffffffu, ci.y, lead),
                           __shfl_sync(0xffffffffu, ci.z, lead));
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int o = k0 + 32 * h + lane;
            float4 q = make_float4(3e37f, 3e37f, 3e37f, 0.f);  // padding never passes the test
            if (o < lg) q = ptc_xyz<PRECISE>(kp, ptc, sg + o, cg);
            s_c[wid][g][0][32 * h + lane] = q.x;
            s_c[wid][g][1][32 * h + lane] = q.y;
            s_c[wid][g][2][32 * h + lane] = q.z;
          }
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int base = k0 + 32 * h;  // offset of the block in the lane's row range
          if (base >= L) break;          // uniform
          unsigned mh = 0u, mk = 0u;
#pragma unroll
          for (int blk = 0; blk < 4; ++blk) {
            if (base + 8 * blk >= L) break;  // uniform: the rest is padding
#pragma unroll
            for (int tt = 8 * blk; tt < 8 * blk + 8; tt += 2) {
              const u64 x2 = *reinterpret_cast<const u64*>(&sx[32 * h + tt]);
              const u64 y2 = *reinterpret_cast<const u64*>(&sx[kStage + 32 * h + tt]);
              const u64 z2 = *reinterpret_cast<const u64*>(&sx[2 * kStage + 32 * h + tt]);
              const u64 dx = sub2(px, x2), dy = sub2(py, y2), dz = sub2(pz, z2);
              const u64 d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
              float r0, r1;
              upk2(d2, r0, r1);
              if (r0 <= r2max) mh |= 1u << tt;
              if (r1 <= r2max) mh |= 2u << tt;
              if constexpr (SKIN) {
                if (r0 <= r2skin) mk |= 1u << tt;
                if (r1 <= r2skin) mk |= 2u << tt;
              }
            }
          }
          // keep the hits inside this lane's range (offsets < len), not itself
          const int hi = len - base;
          unsigned keep = hi <= 0 ? 0u : (hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u));
          const int self = i - sl - base;
          if (self >= 0 && self < 32) keep &= ~(1u << self);
          mh &= keep;
          if constexpr (SKIN) {
            mk &= keep & ~mh;
            while (mk) {
              const int bb = __ffs(mk) - 1;
              mk &= mk - 1;
              const int off = base + bb;
              if (kc < kSkinCap && off <= kOffMask)
                s.xf.sk[sk_idx(i, kc)] = (uint16_t)(((unsigned)r << kRowShift) | (unsigned)off);
              else
                skovf = true;
              ++kc;
            }
          }
          if (!mh) continue;
          const int off0 = base;
          if (cnt + __popc(mh) <= kMaxNb && off0 + 31 <= kOffMask) {
#pragma unroll
            for (int hb = 0; hb < 32; hb += 16) {  // one half block, then its flush
              const unsigned ent0 = ((unsigned)r << kRowShift) + (unsigned)(off0 + hb);
              unsigned part = (mh >> hb) & 0xffffu;
              while (part) {
                const int bb = __ffs(part) - 1;
                part &= part - 1;
                ring[cnt & (kRing - 1)] = (uint16_t)(ent0 + bb);
                ++cnt;
              }
              flush();
            }
          } else {
#pragma unroll
            for (int hb = 0; hb < 32; hb += 16) {
              unsigned part = (mh >> hb) & 0xffffu;
              while (part) {
                const int bb = __ffs(part) - 1;
                part &= part - 1;
                const int off = off0 + hb + bb;
                if (cnt < kMaxNb && off <= kOffMask && !ovf)
                  ring[cnt & (kRing - 1)] = (uint16_t)(((unsigned)r << kRowShift) | (unsigned)off);
                else
                  ovf = true;
                ++cnt;
              }
              flush();
            }
          }
        }
      }
    }
  }
  if (cnt > 254) ovf = true;
  if (act && !ovf && (cnt & 7)) nbv[nb_vec(i, cnt >> 3)] = *reinterpret_cast<const uint4*>(ring + (cnt & (kRing - 8)));
  if (SKIN && act) s.xf.sk_cnt[i] = skovf ? kOverflow : (uint8_t)kc;
  if (act) {
    const bool fluid_nb = GF != 1 || fluid_of(pi.w) || walls_fluid_near(kp, s, t, c);
    list_tail<GF, PRECISE>(kp, s, ptc, i, cnt, ovf, pi, rp_self, fluid_nb);
  }
}

template <int GF, int CW = kCellWarps, bool BATCH = false, bool PRECISE = false, int SEGS = kSegs,
          bool SKIN = false>
__global__ void __launch_bounds__(CW * 32, 42 / CW) k_nblist_seq(KParams kp_arg, Scratch s, zsph_ptc_t ptc,
                                                                   zsph_tmp_t t) {
  const int wid = threadIdx.x >> 5;
  nblist_group<GF, CW, BATCH, PRECISE, SEGS, SKIN>(kp_arg, s, ptc, t, blockIdx.x * CW + wid, wid);
}

// The list transfer's fallback: the full list build of the corrector, run
// only when the transfer's conditions failed this step (*s.xf.flag set);
// otherwise every CTA returns at once.
template <int CW, int SEGS>
__global__ void __launch_bounds__(CW * 32, 42 / CW) k_nblist_fallback(KParams kp, Scratch s, zsph_ptc_t ptc,
                                                                        zsph_tmp_t t) {
  if (*s.xf.flag == 0) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(s.xf.stats + 1, 1ull);
  const int wid = threadIdx.x >> 5;
  nblist_group<1, CW, false, false, SEGS>(kp, s, ptc, t, blockIdx.x * CW + wid, wid);
}

struct NbB1 {  // boundary loop 1
  float4 pr, vp;
};
struct NbB1C {  // boundary loop 1 on reused lists: also the neighbour's current y cell
  float4 pr, vp;
  int cy;
};

constexpr int kWinCapB = 1536;  // boundary window capacity (candidates), 3x3 stencil
constexpr int kWinCapG = 2048;  // governing window capacity (candidates), 3x3 stencil
constexpr int kHdrBytes = (int)((sizeof(WinHdr) + 15) / 16 * 16);

// Dynamic shared memory of a pair kernel: per-thread row starts and row ends
// (NR columns of kPairBlock); when windows are staged (narr > 0), also the
// fetch bases, the window header and, for the 3x3 stencil, the window of
// NARR packed arrays.  Without windows the rest of the layout is never
// touched, and leaving it out leaves more of the SM's SRAM to the L1 cache
// that serves the neighbour loads.
template <int GF> constexpr int pair_smem(int narr, int cap) {
  return narr == 0 ? 2 * Stencil<GF>::NR * kPairBlock * 4
                   : 3 * Stencil<GF>::NR * kPairBlock * 4 + kHdrBytes + (GF == 1 ? narr * cap * 16 : 0);
}

template <int GF> struct PairSmem {
  int *rs, *re, *fb;
  WinHdr* wh;
  float4* win;
  __device__ explicit PairSmem(unsigned char* dsm, int tid = threadIdx.x) {
    constexpr int NR = Stencil<GF>::NR;
    rs = reinterpret_cast<int*>(dsm) + tid;
    re = rs + NR * kPairBlock;
    fb = re + NR * kPairBlock;
    wh = reinterpret_cast<WinHdr*>(dsm + 3 * NR * kPairBlock * 4);
    win = reinterpret_cast<float4*>(dsm + 3 * NR * kPairBlock * 4 + kHdrBytes);
  }
};

// The walls' (rho, p) after the list build (delta_ns.cu:61-85, :116-131):
// non-fluid particle i extrapolates from the fluid neighbours of its
// boundary rows, summed in list order, and rewrites the (rho, p) of its
// packed record (its density stays negative, non-fluid).  The list build has
// written every record by then, so each neighbour costs one 256-bit load
// (four ahead of the arithmetic, as in the pair walks), and no fluid record
// read here is written.  A particle whose list overflowed re-filters its
// boundary rows.
template <int GF, bool PRECISE, bool BATCH>
__device__ __forceinline__ void walls_one(const KParams& kp_arg, const Scratch& s, const zsph_tmp_t& t, int i,
                                          const PairSmem<GF>& sm) {
  KParams kp_scene;  // batched form: the parameters of the particle's scene
  if constexpr (BATCH) kp_scene = kp_of_particle(kp_arg, i);
  const KParams& kp = BATCH ? kp_scene : kp_arg;
  const ShadowRec own = s.sh.load(i);
  const float4 pi = own.pr;
  const int3 ci = PRECISE ? unpack_cell(kp.c3n[i]) : int3{0, 0, 0};
  load_rows<GF>(kp, t, t.hash[i], sm.rs, sm.re);
  float rsum = 0.0f, wsum = 0.0f;
  walk<GF, true, NbB1, PRECISE>(
      kp, s, i, pi, sm.rs, sm.re, sm.rs, i, kp.n - 1,
      [&](int q) {
        const ShadowRec r = shadow_rec<PRECISE>(kp, s, q, ci);
        return NbB1{r.pr, r.vp};
      },
      [&](const NbB1& nb) {
        if (fluid_of(nb.pr.w)) wall_term_core(kp, pi, nb.pr, make_float2(nb.pr.w, nb.vp.w), rsum, wsum);
      },
      ci);
  const zsph_gpu_param_t& p = kp.p;
  if (fabsf(wsum) > 1e-8f) rsum = rsum / wsum; else rsum = 0.0f;
  if (rsum < 0.0f) rsum = 0.0f;
  float4 pr = own.pr, vp = own.vp;
  pr.w = -(rsum / p.cs2 + p.rho0);  // still non-fluid
  vp.w = rsum;
  st_rec(&s.sh.pr(i), pr, vp);
}

// The wall pass over the slots the list build listed in s.wl (grid-stride).
template <int GF, bool PRECISE = false, bool BATCH = false>
__global__ void __launch_bounds__(kPairBlock) k_walls(KParams kp, Scratch s, zsph_tmp_t t) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const PairSmem<GF> sm(dsm);
  const int nw = min(s.misc[kMiscWalls], kp.n);
  for (int q = blockIdx.x * kPairBlock + threadIdx.x; q < nw; q += gridDim.x * kPairBlock)
    walls_one<GF, PRECISE, BATCH>(kp, s, t, s.wl[q], sm);
}

// cuda_boundary_ns main part (delta_ns.cu:35-174): renormalisation matrix and
// div(v) over the boundary stencil, cofactor inverse, renormalised grad(rho).
// REUSE (learned form's corrector variants): the lists were built at an
// earlier state of the same sorted order, so every entry is tested again
// against the exact threshold at the current positions and skipped beyond it.
// boundary_one is the work of one thread on particle i (its row arrays in
// sm); `windows` (the kernel: every thread of the CTA together) allows the
// shared-memory windows when kp.stage_windows asks for them.
template <int GF, bool PRECISE, bool BATCH, bool REUSE>
__device__ __forceinline__ void boundary_one(const KParams& kp_arg, const Scratch& s, const zsph_ptc_t& ptc,
                                             const zsph_tmp_t& t, int i, const PairSmem<GF>& sm, bool windows) {
  KParams kp_scene;  // batched form: the parameters of the particle's scene
  if constexpr (BATCH) kp_scene = kp_of_particle(kp_arg, i);
  const KParams& kp = BATCH ? kp_scene : kp_arg;
  const bool act = i < kp.n;
  if (act) load_rows<GF>(kp, t, t.hash[i], sm.rs, sm.re);
  const int3 ci = PRECISE && act ? unpack_cell(kp.c3n[i]) : int3{0, 0, 0};
  bool staged = false;
  if (windows && GF == 1 && kp.stage_windows && !PRECISE) {
    const float4* const src[1] = {s.sh.rec};  // 32-byte records: two float4s per candidate
    staged = stage_window<Stencil<GF>::NR, 1>(*sm.wh, sm.win, kWinCapB, src, {2}, act, sm.rs, sm.re, sm.fb,
                                              s.flags, [](int r) { return Stencil<GF>::boundary_row(r); });
  }
  if (!act) return;
  const zsph_gpu_param_t& p = kp.p;
  const ShadowRec own = s.sh.load(i);
  const float4 pi = own.pr, vi = own.vp;
  const bool fi = fluid_of(pi.w);
  const float rho_self = reinterpret_cast<const float2*>(ptc.rhop)[i].x;  // old own density
  const float inv_h = kp.inv_h, c_fr = kp.c_fr, m = p.m;
  // The reference's second loop (delta_ns.cu:133-175) walks the same
  // neighbours with a constant matrix M: sum_j (M x_ij) f_j = M sum_j x_ij f_j,
  // so its sums (sx, sy, sz) ride along in the first walk and M is applied
  // once afterwards (same value, summed in a different rounding order).
  float Lxx = 0.f, Lxy = 0.f, Lxz = 0.f, Lyy = 0.f, Lyz = 0.f, Lzz = 0.f, divv = 0.f;
  float sx = 0.f, sy = 0.f, sz = 0.f;
  // reused lists: the boundary rows by the current cells (the lists' rows are the cells at build time)
  const int cy_i = REUSE ? kp.cur_cy[i] : 0;
  auto use1 = [&](const auto& nb) {
    const float dx = pi.x - nb.pr.x, dy = pi.y - nb.pr.y, dz = pi.z - nb.pr.z;
    if constexpr (REUSE) {
      if (!interacts(kp, dist2(dx, dy, dz))) return;
      const int row = nb.cy - cy_i;
      if (row < -GF || row >= GF) return;
    }
    const float q = sqrt_fast(dist2(dx, dy, dz)) * inv_h;
    const float a = 1.0f - 0.5f * q;
    const float fr = c_fr * (a * a * a);
    const float r1 = fabsf(nb.pr.w);
    const float frm = fr * m * rcp_fast(r1);
    const float tl = frm;
    Lxx -= dx * dx * tl; Lxy -= dx * dy * tl; Lxz -= dx * dz * tl;
    Lyy -= dy * dy * tl; Lyz -= dy * dz * tl; Lzz -= dz * dz * tl;
    const float f2 = frm * (r1 - rho_self);  // delta_ns.cu:163-164
    sx += dx * f2; sy += dy * f2; sz += dz * f2;
    if (fi && fluid_of(nb.pr.w)) {
      const float dvdx = (vi.x - nb.vp.x) * dx + (vi.y - nb.vp.y) * dy + (vi.z - nb.vp.z) * dz;
      divv -= tl * dvdx;
    }
  };
  const float4* win = sm.win;
  if constexpr (REUSE) {  // every list entry, classified by the current cells in use1
    walk<GF, false, NbB1C>(kp, s, i, pi, sm.rs, sm.re, sm.rs, i, kp.n - 1,
                           [&](int q) {
                             const ShadowRec r = s.sh.load(q);
                             return NbB1C{r.pr, r.vp, kp.cur_cy[q]};
                           }, use1);
  } else {
    if (staged)
      walk<GF, true, NbB1>(kp, s, i, pi, sm.rs, sm.re, sm.fb, 0, kWinCapB - 1,
                           [&](int q) { return NbB1{win[2 * q], win[2 * q + 1]}; }, use1);
    else
      walk<GF, true, NbB1, PRECISE>(kp, s, i, pi, sm.rs, sm.re, sm.rs, i, kp.n - 1,
                                    [&](int q) {
                                      const ShadowRec r = shadow_rec<PRECISE>(kp, s, q, ci);
                                      return NbB1{r.pr, r.vp};
                                    }, use1, ci);
  }
  // delta_ns.cu:99-114 (L is symmetric: L1 = (xx,xy,xz), L2 = (xy,yy,yz), L3 = (xz,yz,zz))
  const float det = Lxx * Lyy * Lzz + Lxy * Lyz * Lxz + Lxz * Lxy * Lyz - Lxz * Lyy * Lxz - Lxx * Lyz * Lyz -
                    Lxy * Lxy * Lzz;
  float M00, M01, M02, M10, M11, M12, M20, M21, M22;
  if (fabsf(det) > 1.8e-8f) {
    const float id = 1.0f / det;
    M00 = (Lyy * Lzz - Lyz * Lyz) * id;
    M01 = -(Lxy * Lzz - Lyz * Lxz) * id;
    M02 = (Lxy * Lyz - Lyy * Lxz) * id;
    M10 = -(Lxy * Lzz - Lxz * Lyz) * id;
    M11 = (Lxx * Lzz - Lxz * Lxz) * id;
    M12 = -(Lxx * Lyz - Lxy * Lxz) * id;
    M20 = (Lxy * Lyz - Lxz * Lyy) * id;
    M21 = -(Lxx * Lyz - Lxz * Lxy) * id;
    M22 = (Lxx * Lyy - Lxy * Lxy) * id;
  } else {
    M00 = 1.f; M01 = 0.f; M02 = 0.f;
    M10 = 0.f; M11 = 1.f; M12 = 0.f;
    M20 = 0.f; M21 = 0.f; M22 = 1.f;
  }
  const float gx = M00 * sx + M01 * sy + M02 * sz;
  const float gy = M10 * sx + M11 * sy + M12 * sz;
  const float gz = M20 * sx + M21 * sy + M22 * sz;
  reinterpret_cast<float4*>(t.dofv_grandrho)[i] = make_float4(gx, gy, gz, divv);
  if (!fi) reinterpret_cast<float2*>(ptc.rhop)[i] = make_float2(fabsf(pi.w), vi.w);
}

template <int GF, bool PRECISE = false, bool BATCH = false, bool REUSE = false>
__global__ void __launch_bounds__(kPairBlock) k_boundary(KParams kp_arg, Scratch s, zsph_ptc_t ptc, zsph_tmp_t t) {
  extern __shared__ __align__(16) unsigned char dsm[];
  boundary_one<GF, PRECISE, BATCH, REUSE>(kp_arg, s, ptc, t, blockIdx.x * kPairBlock + threadIdx.x,
                                          PairSmem<GF>(dsm), true);
}

struct NbG {  // governing
  float4 pr, vp, dg;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Learned-corrector aggregates of one fluid particle (FeatOut; the network's
// input order).  w = m / rho_j, grad W = F x_ij, e = r^2 / (r^2 + eta^2).
struct FeatAcc {
  float shep_f = 0.f, shep_w = 0.f;        // 0, 1: sum w W over fluid / wall j
  float gx = 0.f, gy = 0.f, gz = 0.f;      // 2-4: sum w F x_ij
  float dx = 0.f, dy = 0.f, dz = 0.f;      // 6-8: sum_fluid w F (divv_j - divv_i) x_ij
  float kx = 0.f, ky = 0.f, kz = 0.f;      // 9-11 (times divv_i): sum_fluid w F x_ij
  float lap_rho = 0.f;                     // 12: sum_fluid w F (rho_i - rho_j) 2e
  float lap_p = 0.f;                       // 13: sum w F (p_i - p_j) 2e
  float wx = 0.f, wy = 0.f, wz = 0.f;      // 28-30: pressure force of wall neighbours
};

// cuda_govering_ns (delta_ns.cu:179-267); MODE 1/2 fuses the prediction /
// correction of the same particle, written into `out` (a different buffer,
// so neighbours still read the unintegrated state).  FEAT (predictor stage
// of the learned form) also accumulates and writes the FeatOut aggregates.
// PRECISE: precision form (cell + offset positions).
// MINB: minimum resident CTAs per SM (register budget); the default six
// give 80 registers without spills for the plain variants.
// REUSE: as k_boundary's (entries re-tested at the current positions).
// governing_one: one thread's particle i, as boundary_one.
// List transfer, in the predictor's fused integration: particle i's
// predicted position (just written to `to`) goes to xfer_pos4, and the
// corrector is told to build its lists in full (*xfer_flag) if the half-step
// displacement exceeds the skin's allowance, a position is not finite, or
// the corrector's hash of the position (hash.cu:12-23, exactly as the search
// computes it) will kill the particle.
__device__ __forceinline__ void xfer_note_prediction(const KParams& kp, const zsph_ptc_t& from, const zsph_ptc_t& to,
                                                     int i) {
  const float x = to.pos[3 * i], y = to.pos[3 * i + 1], z = to.pos[3 * i + 2];
  const float d2 = dist2(x - from.pos[3 * i], y - from.pos[3 * i + 1], z - from.pos[3 * i + 2]);
  const zsph_gpu_param_t& p = kp.p;
  const int h = cell_hash(p, x, y, z, __frcp_rn(p.grid_size));
  const bool bad = !(d2 <= kp.disp2max) || h < 0 || h > p.grid_hash_max - p.grid_hash_min;
  kp.xfer_pos4[i] = make_float4(x, y, z, 0.0f);
  if (bad) atomicOr(kp.xfer_flag, 1);
}

template <int GF, int MODE, bool FEAT, bool PRECISE, bool BATCH, bool RIGID, bool REUSE>
__device__ __forceinline__ void governing_one(const KParams& kp_arg, const Scratch& s, const zsph_ptc_t& ptc,
                                              const zsph_tmp_t& t, const zsph_ptc_t& out, const FeatOut& fo, int i,
                                              const PairSmem<GF>& sm, bool windows) {
  KParams kp_scene;  // batched form: the parameters of the particle's scene
  if constexpr (BATCH) kp_scene = kp_of_particle(kp_arg, i);
  const KParams& kp = BATCH ? kp_scene : kp_arg;
  const bool act = i < kp.n;
  if (act) load_rows<GF>(kp, t, t.hash[i], sm.rs, sm.re);
  const int3 ci = PRECISE && act ? unpack_cell(kp.c3n[i]) : int3{0, 0, 0};
  const float4* dg = reinterpret_cast<const float4*>(t.dofv_grandrho);
  bool staged = false;
  if (windows && GF == 1 && kp.stage_windows && !PRECISE) {
    const float4* const src[2] = {s.sh.rec, dg};  // 32-byte records, then grad(rho)
    staged = stage_window<Stencil<GF>::NR, 2>(*sm.wh, sm.win, kWinCapG, src, {2, 1}, act, sm.rs, sm.re, sm.fb,
                                              s.flags, [](int) { return true; });
  }
  if (!act) return;
  const zsph_gpu_param_t& p = kp.p;
  const ShadowRec own = s.sh.load(i);
  const float4 pi = own.pr, vi = own.vp;
  const bool fi = fluid_of(pi.w);
  const float r0 = fabsf(pi.w), p0 = vi.w, ir0 = rcp_fast(r0);
  const float inv_h = kp.inv_h, c_fr = kp.c_fr, m = p.m;
  float4 g0 = dg[i];
  const float4 g0i = g0;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  FeatAcc fa;
  const bool rig = RIGID && ptc.type[i] == 2;
  float3 rf = make_float3(0.f, 0.f, 0.f);
  auto use = [&](const NbG& nb) {
    const float dx = pi.x - nb.pr.x, dy = pi.y - nb.pr.y, dz = pi.z - nb.pr.z;
    const float rr2 = dist2(dx, dy, dz);
    if constexpr (REUSE) {
      if (!interacts(kp, rr2)) return;
    }
    const float dvdx = (vi.x - nb.vp.x) * dx + (vi.y - nb.vp.y) * dy + (vi.z - nb.vp.z) * dz;
    const float q = sqrt_fast(rr2) * inv_h;
    const float a = 1.0f - 0.5f * q;
    const float fr = c_fr * (a * a * a);
    const float r1 = fabsf(nb.pr.w), p1 = nb.vp.w, ir1 = rcp_fast(r1);
    g0.x *= dx;  // order-dependent recurrence, delta_ns.cu:244-245
    g0.x += nb.dg.x * dx + (g0.y + nb.dg.y) * dy + (g0.z + nb.dg.z) * dz;
    const float frm = fr * m * ir1;
    acc.w += r0 * dvdx * frm;
    float vt = -(p0 + p1) * frm * ir0;
    if constexpr (FEAT) {
      if (fi) {
        const bool fj = fluid_of(nb.pr.w);
        const float e = rr2 * rcp_fast(rr2 + p.eta2);
        const float wW = -0.2f * p.h2 * frm * a * (2.0f * q + 1.0f);  // (m/rho_j) W, W = adh a^4 (2q+1)
        fa.gx += frm * dx; fa.gy += frm * dy; fa.gz += frm * dz;
        fa.lap_p += frm * (p0 - p1) * 2.0f * e;
        if (fj) {
          const float dd = frm * (nb.dg.w - g0i.w);
          fa.shep_f += wW;
          fa.dx += dd * dx; fa.dy += dd * dy; fa.dz += dd * dz;
          fa.kx += frm * dx; fa.ky += frm * dy; fa.kz += frm * dz;
          fa.lap_rho += frm * (r0 - r1) * 2.0f * e;
        } else {
          fa.shep_w += wW;
          fa.wx += vt * dx; fa.wy += vt * dy; fa.wz += vt * dz;
        }
      }
    }
    if (rig && fluid_of(nb.pr.w)) {  // the fluid's pressure force on a body particle
      rf.x += vt * dx;
      rf.y += vt * dy;
      rf.z += vt * dz;
    }
    if (fi && fluid_of(nb.pr.w)) {
      const float ire = rcp_fast(rr2 + p.eta2);
      acc.w += p.delta_h_cs * frm * ((r0 - r1) * 2.0f * rr2 * ire - g0.x);
      vt += p.h_cs_rho_m * fr * (g0.w + nb.dg.w + p.alpha * dvdx * ire) * ir0 * ir1;
    }
    acc.x += vt * dx;
    acc.y += vt * dy;
    acc.z += vt * dz;
  };
  const float4* win = sm.win;
  if (staged)
    walk<GF, false, NbG>(kp, s, i, pi, sm.rs, sm.re, sm.fb, 0, kWinCapG - 1,
                         [&](int q) { return NbG{win[2 * q], win[2 * q + 1], win[2 * kWinCapG + q]}; }, use);
  else
    walk<GF, false, NbG, PRECISE>(kp, s, i, pi, sm.rs, sm.re, sm.rs, i, kp.n - 1,
                                  [&](int q) {
                                    const ShadowRec r = shadow_rec<PRECISE>(kp, s, q, ci);
                                    return NbG{r.pr, r.vp, dg[q]};
                                  }, use, ci);
  if (rig) kp.rigid_f[i] = make_float4(rf.x, rf.y, rf.z, 0.f);
  acc.z += p.g;  // delta_ns.cu:264
  reinterpret_cast<float4*>(t.acc_drhodt)[i] = acc;
  if (!isfinite(acc.x + acc.y + acc.z + acc.w)) atomicOr(s.flags, ZSPH_FLAG_NAN);
  if constexpr (FEAT) {
    // D: this predictor-stage value minus the particle's previous corrector-stage value
    const float4 ap = fo.acc_prev ? fo.acc_prev[t.index[i]] : acc;
    const float4 dp = fi ? make_float4(acc.x - ap.x, acc.y - ap.y, acc.z - ap.z, acc.w - ap.w)
                         : make_float4(0.f, 0.f, 0.f, 0.f);
    if (fo.d_out) fo.d_out[i] = dp;
    float f[kFeat];
    if (fi) {
      const float fv[kFeat] = {fa.shep_f, fa.shep_w, fa.gx, fa.gy, fa.gz, g0i.w, fa.dx, fa.dy,
                               fa.dz, g0i.w * fa.kx, g0i.w * fa.ky, g0i.w * fa.kz, fa.lap_rho, fa.lap_p, acc.x, acc.y,
                               acc.z, acc.w, vi.x, vi.y, vi.z, r0 - p.rho0, g0i.x, g0i.y,
                               g0i.z, dp.x, dp.y, dp.z, fa.wx, fa.wy, fa.wz, dp.w};
#pragma unroll
      for (int k = 0; k < kFeat; ++k) f[k] = fv[k] * fo.scale[k];
    } else {
#pragma unroll
      for (int k = 0; k < kFeat; ++k) f[k] = 0.f;
    }
    if (fo.raw) {
      float4* dst = reinterpret_cast<float4*>(fo.raw) + (size_t)i * (kFeat / 4);
#pragma unroll
      for (int k = 0; k < kFeat / 4; ++k) dst[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
    }
    if (fo.tiles) {
      unsigned char* tile = fo.tiles + (size_t)(i >> 7) * 8192;
      const int r = i & 127;
#pragma unroll
      for (int cb = 0; cb < kFeat / 8; ++cb) {
        uint32_t u[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int c = cb * 8 + 2 * e;
          u[e] = fi ? pack_bf16x2((f[c] - fo.mean[c]) * fo.inv_std[c], (f[c + 1] - fo.mean[c + 1]) * fo.inv_std[c + 1])
                    : 0u;
        }
        // element (r, c) of a 128-row operand tile: ((c/8)*16 + r/8)*128 + (r%8)*16 + (c%8)*2
        *reinterpret_cast<uint4*>(tile + ((cb * 16 + (r >> 3)) << 7) + ((r & 7) << 4)) =
            make_uint4(u[0], u[1], u[2], u[3]);
      }
    }
    if (fo.acc_copy) fo.acc_copy[i] = acc;
  }
  if (MODE != 0) integrate_one<MODE, PRECISE>(kp, ptc, out, i, acc);
  if constexpr (MODE == 1 && !PRECISE && !BATCH && !REUSE)
    if (kp.xfer_pos4) xfer_note_prediction(kp, ptc, out, i);
}

template <int GF, int MODE, bool FEAT = false, bool PRECISE = false, bool BATCH = false, bool RIGID = false,
          int MINB = (FEAT || BATCH) ? 1 : 6, bool REUSE = false>
__global__ void __launch_bounds__(kPairBlock, MINB)
    k_governing(KParams kp_arg, Scratch s, zsph_ptc_t ptc, zsph_tmp_t t, zsph_ptc_t out, FeatOut fo) {
  extern __shared__ __align__(16) unsigned char dsm[];
  governing_one<GF, MODE, FEAT, PRECISE, BATCH, RIGID, REUSE>(kp_arg, s, ptc, t, out, fo,
                                                               blockIdx.x * kPairBlock + threadIdx.x,
                                                               PairSmem<GF>(dsm), true);
}

// ---- simple-SPH equations (the reference's simplesph target) --------------

struct NbS {  // simple boundary / governing
  float4 pr, vp;
  float dv;
};

// single_gpu_sph_src/equation/simple_ns.cu:3-97: scalar div(v) over fluid
// pairs of the boundary stencil into tmp.dofv; new wall (rho, p) (computed
// by k_walls) into ptc.rhop.  Walls read only fluid densities here, so the
// reference has no wall-density race in this kernel.
template <int GF>
__global__ void __launch_bounds__(kPairBlock) k_boundary_simple(KParams kp, Scratch s, zsph_ptc_t ptc,
                                                                zsph_tmp_t t) {
  extern __shared__ __align__(16) unsigned char dsm[];
  PairSmem<GF> sm(dsm);
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  load_rows<GF>(kp, t, t.hash[i], sm.rs, sm.re);
  const zsph_gpu_param_t& p = kp.p;
  const ShadowRec own = s.sh.load(i);
  const float4 pi = own.pr, vi = own.vp;
  const bool fi = fluid_of(pi.w);
  float divv = 0.f;
  if (fi)
    walk<GF, true, NbB1>(
        kp, s, i, pi, sm.rs, sm.re, sm.rs, i, kp.n - 1, [&](int q) {
          const ShadowRec r = s.sh.load(q);
          return NbB1{r.pr, r.vp};
        },
        [&](const NbB1& nb) {
          if (!fluid_of(nb.pr.w)) return;
          const float dx = pi.x - nb.pr.x, dy = pi.y - nb.pr.y, dz = pi.z - nb.pr.z;
          const float q = sqrt_fast(dist2(dx, dy, dz)) * kp.inv_h;
          const float a = 1.0f - 0.5f * q;
          const float fr = kp.c_fr * (a * a * a);
          const float dvdx = (vi.x - nb.vp.x) * dx + (vi.y - nb.vp.y) * dy + (vi.z - nb.vp.z) * dz;
          divv -= fr * dvdx * p.m * rcp_fast(nb.pr.w);
        });
  t.dofv[i] = divv;
  if (!fi) reinterpret_cast<float2*>(ptc.rhop)[i] = make_float2(fabsf(pi.w), vi.w);
}

// single_gpu_sph_src/equation/simple_ns.cu:99-180, with the same fused
// prediction / correction epilogue as k_governing.
template <int GF, int MODE>
__global__ void __launch_bounds__(kPairBlock) k_governing_simple(KParams kp, Scratch s, zsph_ptc_t ptc,
                                                                 zsph_tmp_t t, zsph_ptc_t out) {
  extern __shared__ __align__(16) unsigned char dsm[];
  PairSmem<GF> sm(dsm);
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  load_rows<GF>(kp, t, t.hash[i], sm.rs, sm.re);
  const zsph_gpu_param_t& p = kp.p;
  const ShadowRec own = s.sh.load(i);
  const float4 pi = own.pr, vi = own.vp;
  const bool fi = fluid_of(pi.w);
  const float r0 = fabsf(pi.w), p0 = vi.w, ir0 = rcp_fast(r0);
  const float d0 = t.dofv[i];
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  walk<GF, false, NbS>(
      kp, s, i, pi, sm.rs, sm.re, sm.rs, i, kp.n - 1, [&](int q) {
        const ShadowRec r = s.sh.load(q);
        return NbS{r.pr, r.vp, t.dofv[q]};
      },
      [&](const NbS& nb) {
        const float dx = pi.x - nb.pr.x, dy = pi.y - nb.pr.y, dz = pi.z - nb.pr.z;
        const float rr2 = dist2(dx, dy, dz);
        const float dvdx = (vi.x - nb.vp.x) * dx + (vi.y - nb.vp.y) * dy + (vi.z - nb.vp.z) * dz;
        const float q = sqrt_fast(rr2) * kp.inv_h;
        const float a = 1.0f - 0.5f * q;
        const float fr = kp.c_fr * (a * a * a);
        const float r1 = fabsf(nb.pr.w), p1 = nb.vp.w, ir1 = rcp_fast(r1);
        const float ire = rcp_fast(rr2 + p.eta2);
        acc.w += (r0 * dvdx * fr + (r0 - r1) * rr2 * fr * p.delta_h_cs * ire) * p.m * ir1;  // simple_ns.cu:162
        float vt = -(p0 + p1) * p.m * fr * ir0 * ir1;
        if (fi && fluid_of(nb.pr.w)) vt += p.h_cs_rho_m * fr * (d0 + nb.dv + p.alpha * dvdx * ire) * ir0 * ir1;
        acc.x += vt * dx;
        acc.y += vt * dy;
        acc.z += vt * dz;
      });
  acc.z += p.g;
  reinterpret_cast<float4*>(t.acc_drhodt)[i] = acc;
  if (!isfinite(acc.x + acc.y + acc.z + acc.w)) atomicOr(s.flags, ZSPH_FLAG_NAN);
  if (MODE != 0) integrate_one<MODE>(kp, ptc, out, i, acc);
}

// Drop-in cuda_prediction / cuda_correction: in place.
template <int MODE>
__global__ void __launch_bounds__(kSearchBlock) k_integrate(KParams kp, zsph_ptc_t ptc, zsph_tmp_t t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  if (ptc.type[i] != 1) return;
  integrate_one<MODE>(kp, ptc, ptc, i, reinterpret_cast<const float4*>(t.acc_drhodt)[i]);
}

inline int thread_blocks(int n) { return (n + kPairBlock - 1) / kPairBlock; }

// list build (grid factor 1) with the tuned number of cells per CTA
template <bool BATCH>
void launch_nblist_tuned(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                         cudaStream_t st) {
  // (eight cells per CTA would exceed the 48 KB of static shared memory)
  // default (0): two warps per CTA, what zsph_autotune picks on the dam-break cases
  // default segments per round (0): four
  const int segs = kp.tune_segs ? kp.tune_segs : kSegs;
  const int g4 = (kp.n + 127) / 128, g2 = (kp.n + 63) / 64;
  if (kp.tune_cw == 4) {
    if (segs == 2) k_nblist_seq<1, 4, BATCH, false, 2><<<g4, 128, 0, st>>>(kp, s, ptc, t);
    else if (segs == 3) k_nblist_seq<1, 4, BATCH, false, 3><<<g4, 128, 0, st>>>(kp, s, ptc, t);
    else k_nblist_seq<1, 4, BATCH, false, 4><<<g4, 128, 0, st>>>(kp, s, ptc, t);
  } else {
    if (segs == 2) k_nblist_seq<1, 2, BATCH, false, 2><<<g2, 64, 0, st>>>(kp, s, ptc, t);
    else if (segs == 3) k_nblist_seq<1, 2, BATCH, false, 3><<<g2, 64, 0, st>>>(kp, s, ptc, t);
    else k_nblist_seq<1, 2, BATCH, false, 4><<<g2, 64, 0, st>>>(kp, s, ptc, t);
  }
}

// governing (grid factor 1, fused prediction / correction, no shared-memory
// windows) with the tuned register budget
template <int MODE, bool BATCH>
void launch_governing_tuned(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                            const zsph_ptc_t& out, cudaStream_t st) {
  const FeatOut none{};
  const int nb = thread_blocks(kp.n), sm = pair_smem<1>(0, 0);
  // default (0): one resident CTA minimum (the largest register budget), what
  // zsph_autotune picks on the dam-break cases
  switch (kp.tune_minb) {
    case 6: k_governing<1, MODE, false, false, BATCH, false, 6><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none); break;
    case 8: k_governing<1, MODE, false, false, BATCH, false, 8><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none); break;
    default: k_governing<1, MODE, false, false, BATCH, false, 1><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none); break;
  }
}

// The wall pass: enough CTAs to fill the device, each looping over s.wl
// (its length is known on the device only).
template <int GF, bool PRECISE = false, bool BATCH = false>
void launch_walls(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, cudaStream_t st) {
  static int sms = 0;  // SMs of the device (the same for every B200)
  if (!sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
  }
  k_walls<GF, PRECISE, BATCH><<<min(thread_blocks(kp.n), sms * 16), kPairBlock, pair_smem<GF>(0, 0), st>>>(kp, s, t);
}

// zeroes the wall-list length before a list build appends to it
inline cudaError_t reset_walls(const Scratch& s, cudaStream_t st) {
  return cudaMemsetAsync(s.misc + kMiscWalls, 0, sizeof(int), st);
}

template <int GF>
cudaError_t boundary_gf(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                        cudaStream_t st, Prof* pf) {
  if (cudaError_t e = reset_walls(s, st)) return e;
  if (kp.scenes) {  // batched form (grid factor 1, delta equations)
    if (GF != 1 || kp.equations != ZSPH_EQ_DELTA || kp.c3o) return cudaErrorInvalidValue;
    launch_nblist_tuned<true>(kp, s, ptc, t, st);
    mark(pf, "nblist", st);
    launch_walls<1, false, true>(kp, s, t, st);
    mark(pf, "walls", st);
    k_boundary<1, false, true><<<thread_blocks(kp.n), kPairBlock, pair_smem<1>(0, 0), st>>>(kp, s, ptc, t);
    mark(pf, "boundary", st);
    return cudaGetLastError();
  }
  if (kp.c3o) {  // precision form (grid factor 1, delta equations)
    if (GF != 1 || kp.equations != ZSPH_EQ_DELTA) return cudaErrorInvalidValue;
    k_nblist_seq<1, kCellWarps, false, true><<<(kp.n + 32 * kCellWarps - 1) / (32 * kCellWarps), kCellWarps * 32, 0, st>>>(kp, s, ptc, t);
    mark(pf, "nblist", st);
    launch_walls<1, true>(kp, s, t, st);
    mark(pf, "walls", st);
    k_boundary<1, true><<<thread_blocks(kp.n), kPairBlock, pair_smem<1>(0, 0), st>>>(kp, s, ptc, t);
    mark(pf, "boundary", st);
    return cudaGetLastError();
  }
  if (GF == 1) launch_nblist_tuned<false>(kp, s, ptc, t, st);
  else k_nblist_seq<GF, kSeqWarps<GF>><<<(kp.n + 32 * kSeqWarps<GF> - 1) / (32 * kSeqWarps<GF>), kSeqWarps<GF> * 32, 0, st>>>(kp, s, ptc, t);
  mark(pf, "nblist", st);
  launch_walls<GF>(kp, s, t, st);
  mark(pf, "walls", st);
  if (kp.equations == ZSPH_EQ_SIMPLE)
    k_boundary_simple<GF><<<thread_blocks(kp.n), kPairBlock, pair_smem<GF>(0, 0), st>>>(kp, s, ptc, t);
  else
    k_boundary<GF><<<thread_blocks(kp.n), kPairBlock, pair_smem<GF>(kp.stage_windows ? 2 : 0, kWinCapB), st>>>(
        kp, s, ptc, t);
  mark(pf, "boundary", st);
  return cudaGetLastError();
}

template <int GF>
cudaError_t governing_gf(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t, int mode,
                         const zsph_ptc_t& out, cudaStream_t st, Prof* pf, const FeatOut* feat) {
  const int nb = thread_blocks(kp.n);
  if (kp.equations == ZSPH_EQ_SIMPLE) {
    const int ss = pair_smem<GF>(0, 0);
    if (mode == 0) k_governing_simple<GF, 0><<<nb, kPairBlock, ss, st>>>(kp, s, ptc, t, out);
    if (mode == 1) k_governing_simple<GF, 1><<<nb, kPairBlock, ss, st>>>(kp, s, ptc, t, out);
    if (mode == 2) k_governing_simple<GF, 2><<<nb, kPairBlock, ss, st>>>(kp, s, ptc, t, out);
    mark(pf, "governing", st);
    return cudaGetLastError();
  }
  if (kp.scenes) {  // batched form (grid factor 1, delta equations, no learned features)
    if (GF != 1 || feat || kp.c3o) return cudaErrorInvalidValue;
    const FeatOut none{};
    const int s1 = pair_smem<1>(0, 0);
    if (mode == 0) k_governing<1, 0, false, false, true><<<nb, kPairBlock, s1, st>>>(kp, s, ptc, t, out, none);
    if (mode == 1) launch_governing_tuned<1, true>(kp, s, ptc, t, out, st);
    if (mode == 2) launch_governing_tuned<2, true>(kp, s, ptc, t, out, st);
    mark(pf, "governing", st);
    return cudaGetLastError();
  }
  if (kp.c3o) {  // precision form (grid factor 1, delta equations, no learned features)
    if (GF != 1 || feat) return cudaErrorInvalidValue;
    const FeatOut none{};
    const int s1 = pair_smem<1>(0, 0);
    if (mode == 0) k_governing<1, 0, false, true><<<nb, kPairBlock, s1, st>>>(kp, s, ptc, t, out, none);
    if (kp.rigid_f) {  // floating body: also the fluid's force on its particles
      if (mode == 1) k_governing<1, 1, false, true, false, true><<<nb, kPairBlock, s1, st>>>(kp, s, ptc, t, out, none);
      if (mode == 2) k_governing<1, 2, false, true, false, true><<<nb, kPairBlock, s1, st>>>(kp, s, ptc, t, out, none);
    } else {
      if (mode == 1) k_governing<1, 1, false, true><<<nb, kPairBlock, s1, st>>>(kp, s, ptc, t, out, none);
      if (mode == 2) k_governing<1, 2, false, true><<<nb, kPairBlock, s1, st>>>(kp, s, ptc, t, out, none);
    }
    mark(pf, "governing", st);
    return cudaGetLastError();
  }
  const int sm = pair_smem<GF>(kp.stage_windows ? 3 : 0, kWinCapG);
  if (feat) {
    if (mode != 1) return cudaErrorInvalidValue;
    k_governing<GF, 1, true><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, *feat);
    mark(pf, "governing_feat", st);
    return cudaGetLastError();
  }
  const FeatOut none{};
  if (kp.rigid_f && mode != 0) {  // floating body, absolute positions
    if (GF != 1) return cudaErrorInvalidValue;
    if (mode == 1) k_governing<1, 1, false, false, false, true><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none);
    if (mode == 2) k_governing<1, 2, false, false, false, true><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none);
    mark(pf, "governing", st);
    return cudaGetLastError();
  }
  if (GF == 1 && !kp.stage_windows && mode != 0) {
    if (mode == 1) launch_governing_tuned<1, false>(kp, s, ptc, t, out, st);
    if (mode == 2) launch_governing_tuned<2, false>(kp, s, ptc, t, out, st);
    mark(pf, "governing", st);
    return cudaGetLastError();
  }
  if (mode == 0) k_governing<GF, 0><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none);
  if (mode == 1) k_governing<GF, 1><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none);
  if (mode == 2) k_governing<GF, 2><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, out, none);
  mark(pf, "governing", st);
  return cudaGetLastError();
}

template <int GF>
cudaError_t nblist_gf(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                      cudaStream_t st) {
  if (kp.scenes) {
    if (GF != 1) return cudaErrorInvalidValue;
    launch_nblist_tuned<true>(kp, s, ptc, t, st);
  } else if (kp.c3o) {
    if (GF != 1) return cudaErrorInvalidValue;
    k_nblist_seq<1, kCellWarps, false, true><<<(kp.n + 32 * kCellWarps - 1) / (32 * kCellWarps), kCellWarps * 32, 0, st>>>(kp, s, ptc, t);
  } else {
    k_nblist_seq<GF, kSeqWarps<GF>><<<(kp.n + 32 * kSeqWarps<GF> - 1) / (32 * kSeqWarps<GF>), kSeqWarps<GF> * 32, 0, st>>>(kp, s, ptc, t);
  }
  return cudaGetLastError();
}

// Learned form's corrector variants: wall (rho, p) of every non-fluid
// particle at the current (predicted) positions, from its fluid neighbours in
// the lists the predictor built that lie in the boundary rows by the current
// cells (delta_ns.cu:61-85, :116-131), each entry tested again against the
// exact threshold; summed in the lists' visit order and published in the
// packed shadows, and in ptc.rhop when no boundary pass follows (which would
// otherwise write it).
//
// k_cur_cells: each particle's y cell index at its current position, with
// the hash's arithmetic (hash.cu:13).
__global__ void __launch_bounds__(kSearchBlock) k_cur_cells(KParams kp, zsph_ptc_t ptc, int* cy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  cy[i] = (int)floorf(__fdiv_rn(__fsub_rn(ptc.pos[3 * i + 1], kp.p.grid_ymin), kp.p.grid_size));
}

template <int GF>
__global__ void __launch_bounds__(kPairBlock) k_walls_reuse(KParams kp, Scratch s, zsph_ptc_t ptc, zsph_tmp_t t,
                                                            int write_rhop) {
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  const float4 pi = s.sh.pr(i);
  if (fluid_of(pi.w)) return;
  const int c = t.hash[i];
  const int cnt = s.nb_cnt[i];
  const int cy_i = kp.cur_cy[i];
  float rsum = 0.0f, wsum = 0.0f;
  auto visit = [&](int j) {
    const float4 pj = s.sh.pr(j);
    if (!fluid_of(pj.w) || !interacts(kp, dist2(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z))) return;
    const int row = kp.cur_cy[j] - cy_i;  // the boundary rows by the current cells
    if (row < -GF || row >= GF) return;
    wall_term(kp, s, pi, j, rsum, wsum);
  };
  if (cnt != kOverflow) {
    for (int k = 0; k < cnt; ++k) {
      const unsigned e = s.nb[nb_vec(i, k >> 3) * 8 + (k & 7)];
      const int r = (int)(e >> kRowShift);
      int a, b;
      row_range<GF>(kp, t, c, r, a, b);
      const int j = a + (int)(e & kOffMask);
      if (j < b) visit(j);
    }
  } else {
    for (int r = 0; r < Stencil<GF>::NR; ++r) {
      int a, b;
      row_range<GF>(kp, t, c, r, a, b);
      for (int j = a; j < b; ++j)
        if (j != i) visit(j);
    }
  }
  const zsph_gpu_param_t& p = kp.p;
  if (fabsf(wsum) > 1e-8f) rsum = rsum / wsum; else rsum = 0.0f;
  if (rsum < 0.0f) rsum = 0.0f;
  const float rho = rsum / p.cs2 + p.rho0;
  s.sh.pr(i).w = -rho;  // still non-fluid
  s.sh.vp(i).w = rsum;
  if (write_rhop) reinterpret_cast<float2*>(ptc.rhop)[i] = make_float2(rho, rsum);
}

// Rigid-body contact (see launch_rigid_contact): one thread per particle,
// body particles only; the neighbours come from the particle's list (all
// stencil rows, visit order), the non-fluid ones of another body or of the
// walls within `dist` push back along the pair's normal.
__device__ __forceinline__ int body_range_of(const zsph_ptc_t& ptc, const BodyRange* br, int nb, int i) {
  if (ptc.type[i] != 2) return -1;
  const int id = ptc.table[i] + i;
  for (int b = 0; b < nb; ++b)
    if (id >= br[b].first && id < br[b].first + br[b].count) return b;
  return -1;
}

template <int GF, bool PRECISE>
__global__ void __launch_bounds__(kPairBlock) k_rigid_contact(KParams kp, Scratch s, zsph_ptc_t ptc, zsph_tmp_t t,
                                                              const BodyRange* br, int nb, float kn, float cn,
                                                              float dist) {
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  const int bi = body_range_of(ptc, br, nb, i);
  if (bi < 0) return;
  const int3 ci = PRECISE ? unpack_cell(kp.c3n[i]) : int3{0, 0, 0};
  const ShadowRec own = s.sh.load(i);
  const float inv_m = 1.0f / kp.p.m;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  auto visit = [&](int j) {
    if (ptc.type[j] == 1 || body_range_of(ptc, br, nb, j) == bi) return;
    const ShadowRec o = shadow_rec<PRECISE>(kp, s, j, ci);
    const float dx = own.pr.x - o.pr.x, dy = own.pr.y - o.pr.y, dz = own.pr.z - o.pr.z;
    const float r = __fsqrt_rn(dist2(dx, dy, dz));
    if (!(r < dist) || !(r > 0.f)) return;
    const float nx = dx / r, ny = dy / r, nz = dz / r;
    const float vn = (own.vp.x - o.vp.x) * nx + (own.vp.y - o.vp.y) * ny + (own.vp.z - o.vp.z) * nz;
    const float fc = fmaxf(kn * (dist - r) - cn * vn, 0.f) * inv_m;
    fx += fc * nx;
    fy += fc * ny;
    fz += fc * nz;
  };
  const int c = t.hash[i];
  const int cnt = s.nb_cnt[i];
  if (cnt != kOverflow) {
    for (int k = 0; k < cnt; ++k) {
      const unsigned e = s.nb[nb_vec(i, k >> 3) * 8 + (k & 7)];
      int a, b;
      row_range<GF>(kp, t, c, (int)(e >> kRowShift), a, b);
      const int j = a + (int)(e & kOffMask);
      if (j < b) visit(j);
    }
  } else {
    for (int r = 0; r < Stencil<GF>::NR; ++r) {
      int a, b;
      row_range<GF>(kp, t, c, r, a, b);
      for (int j = a; j < b; ++j)
        if (j != i) visit(j);
    }
  }
  float4 f = kp.rigid_f[i];
  f.x += fx;
  f.y += fy;
  f.z += fz;
  kp.rigid_f[i] = f;
}

// ---- batched form: the whole step in one persistent launch ----------------
//
// k_batch_persistent runs nsteps full steps of a batched handle (every scene)
// in one cooperative launch: the grid is at most what the GPU holds at once,
// every CTA stays resident, and the stages of a sub-step are separated by
// grid barriers instead of kernel boundaries.  Each stage loops over its
// work units with the same device code as the stage's own kernel
// (search_dev.cuh bodies, nblist_group, boundary_one, governing_one), so the
// arithmetic and the orders are those of the graph-of-launches step and each
// scene's result is still that of the scene run alone.  A CTA has 256
// threads: the search bodies' CTA, 8 list-build warps, or two 128-thread pair
// blocks.  The stages of a sub-step (from = old_, to = new_, as the fused
// step): hash and tickets | one-pass scan (tiles claimed in order) | scatter
// | crowded cells sorted, if the scan listed any | rank and gather | list
// build | wall pressure | boundary | governing with the prediction or
// correction into old_.
//
// Grid barrier: a CTA's thread 0 arrives on a counter and waits for the
// generation word to change; the last to arrive resets the counter and
// advances the generation.  The wait is bounded (spin_limit polls with a
// short sleep, about a second by default); a CTA that gives up raises
// ZSPH_FLAG_TIMEOUT and leaves the kernel, and so, within the same bound,
// does every other CTA.  `extra` adds arrivals that never come (self-test
// of the bound: with extra > 0 no barrier can complete).
constexpr int kPersistThreads = kSearchBlock;
static_assert(kPersistThreads == 2 * kPairBlock, "two pair blocks per persistent CTA");
constexpr int kPersistWarps = kPersistThreads / 32;

struct PersistArgs {
  KParams kp;
  Scratch s;
  zsph_ptc_t o, w;
  zsph_tmp_t t;
  unsigned* bar;  // [0] arrivals, [1] generation
  int nsteps;
  unsigned spin_limit;
  int extra;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier(const PersistArgs& a) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire_u32(a.bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(a.bar, 1u) + 1u;
    int ok = 1;
    if (arrived == gridDim.x + (unsigned)a.extra) {
      atomicExch(a.bar, 0u);
      __threadfence();
      atomicAdd(a.bar + 1, 1u);
    } else {
      unsigned spins = 0;
      while (ld_acquire_u32(a.bar + 1) == g) {
        if (++spins > a.spin_limit) {
          ok = 0;
          atomicOr(a.s.flags, ZSPH_FLAG_TIMEOUT);
          break;
        }
        __nanosleep(200);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int MODE>
__device__ __forceinline__ void persistent_pairs(const PersistArgs& a, unsigned char* dsm) {
  const KParams& kp = a.kp;
  const int half = threadIdx.x / kPairBlock, tid = threadIdx.x % kPairBlock;
  const PairSmem<1> sm(dsm + half * pair_smem<1>(0, 0), tid);
  const int nvb = (kp.n + kPairBlock - 1) / kPairBlock;
  const FeatOut none{};
  if (MODE == 0) {  // boundary
    for (int vb = 2 * blockIdx.x + half; vb < nvb; vb += 2 * gridDim.x)
      boundary_one<1, false, true, false>(kp, a.s, a.w, a.t, vb * kPairBlock + tid, sm, false);
  } else {          // governing, integrated into old_
    for (int vb = 2 * blockIdx.x + half; vb < nvb; vb += 2 * gridDim.x)
      governing_one<1, MODE, false, false, true, false, false>(kp, a.s, a.w, a.t, a.o, none, vb * kPairBlock + tid,
                                                               sm, false);
  }
}

__global__ void __launch_bounds__(kPersistThreads, 2) k_batch_persistent(PersistArgs a) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ int s_tile;
  const KParams& kp = a.kp;
  const Scratch& s = a.s;
  const int n = kp.n;
  const int hash_chunks = (n + kSearchBlock * kHashItems - 1) / (kSearchBlock * kHashItems);
  const int scan_tiles = (kp.G + kOneTile - 1) / kOneTile;
  const int scat_chunks = (n + kSearchBlock * kScatterItems - 1) / (kSearchBlock * kScatterItems);
  const int groups = (n + 31) / 32;
  const int wid = threadIdx.x >> 5;
  if (a.nsteps == 0 && !grid_barrier(a)) return;  // self-test: the barrier alone
  for (int step = 0; step < a.nsteps; ++step) {
    for (int sub = 1; sub <= 2; ++sub) {
      for (int c = blockIdx.x; c < hash_chunks; c += gridDim.x) {
        hash_count_body(kp, a.o, s, c);
        __syncthreads();  // its block-maximum scratch is reused by the next chunk
      }
      if (!grid_barrier(a)) return;
      for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&s.misc[5], 1);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= scan_tiles) break;
        scan_onepass_body(kp, s, a.t, tile);
      }
      if (!grid_barrier(a)) return;
      for (int c = blockIdx.x; c < scat_chunks; c += gridDim.x) scatter_body(kp, s, c);
      if (!grid_barrier(a)) return;
      const int listed = s.misc[3];
      if (listed > 0) {  // crowded cells: pre-sort their members (as the scatter's last CTA does)
        if (listed <= kBigListCap) {
          for (int e = blockIdx.x; e < listed; e += gridDim.x) {
            const int c = s.big_list[e];
            cta_sort_segment(s.perm + s.cell_lb[c], s.cell_lb[c + 1] - s.cell_lb[c]);
          }
        } else {
          for (int c = blockIdx.x; c < kp.G; c += gridDim.x) {
            const int lo = s.cell_lb[c], hi = s.cell_lb[c + 1];
            if (hi - lo > kBigSegment) cta_sort_segment(s.perm + lo, hi - lo);
          }
        }
      }
      if (!grid_barrier(a)) return;
      for (int t = blockIdx.x * kPersistThreads + threadIdx.x; t < n; t += gridDim.x * kPersistThreads)
        rank_gather_one<false>(kp, s, a.o, a.w, a.t, t);
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        s.misc[kMiscWalls] = 0;                // the wall list, appended by the list build
        s.misc[kMiscFluidEpoch] = s.misc[6];   // the cell stamps rank_gather_one wrote
      }
      if (!grid_barrier(a)) return;
      for (int g = blockIdx.x * kPersistWarps + wid; g < groups; g += gridDim.x * kPersistWarps)
        nblist_group<1, kPersistWarps, true, false>(kp, s, a.w, a.t, g, wid);
      if (!grid_barrier(a)) return;
      {
        const int nw = min(s.misc[kMiscWalls], n);
        const PairSmem<1> sm(dsm + (threadIdx.x / kPairBlock) * pair_smem<1>(0, 0), threadIdx.x % kPairBlock);
        for (int q = blockIdx.x * kPersistThreads + threadIdx.x; q < nw; q += gridDim.x * kPersistThreads)
          walls_one<1, false, true>(kp, s, a.t, s.wl[q], sm);
      }
      if (!grid_barrier(a)) return;
      persistent_pairs<0>(a, dsm);
      if (!grid_barrier(a)) return;
      if (sub == 1) persistent_pairs<1>(a, dsm);
      else persistent_pairs<2>(a, dsm);
      if (!grid_barrier(a)) return;
    }
  }
}

// Neighbour counts from the lists: governing stencil and boundary subset
// (-1 for a particle whose list overflowed).
template <int GF>
__global__ void __launch_bounds__(kSearchBlock) k_nb_counts(KParams kp, Scratch s, int* nb_boundary,
                                                            int* nb_governing) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  const int cnt = s.nb_cnt[i];
  if (cnt == kOverflow) {
    if (nb_boundary) nb_boundary[i] = -1;
    if (nb_governing) nb_governing[i] = -1;
    return;
  }
  int b = 0;
  for (int k = 0; k < cnt; ++k)
    b += Stencil<GF>::boundary_row((int)(s.nb[nb_vec(i, k >> 3) * 8 + (k & 7)] >> kRowShift));
  if (nb_boundary) nb_boundary[i] = b;
  if (nb_governing) nb_governing[i] = cnt;
}

// ---- list transfer: the corrector's lists made from the predictor's -------
//
// The corrector's neighbour set of a particle is every candidate of its
// stencil rows (cell bounds of the corrector's search) within 2h at the
// predicted positions.  For a particle that stays in its cell, those rows
// are the cells it had in the predictor's search, and a neighbour within 2h
// now was within 2h + skin then if no particle moved more than half the
// skin in the half step (the fused prediction checks that).  So its
// predictor list, its skin list (2h < r <= 2h + skin) and the particles
// handed over below hold the whole set: each is re-tested against the exact
// threshold at the predicted positions and kept only if its corrector slot
// lies in one of the particle's corrector row ranges (which reproduces the
// rows row_range drops and the excluded last particle).  Sorting the 16-bit
// entries (row << 11 | offset) restores the reference's visit order, so the
// lists equal those of a full build entry for entry.
//
// The particles that change cell (about 1 % per half step on the dam break),
// the predictor search's last particle (never anyone's candidate there),
// those whose predictor list or skin list overflowed and those whose rows
// meet stale cell bounds get a full search instead (k_xfer_classify lists
// them, k_xfer_search gives each a warp).  That search also hands
// such a particle to every neighbour whose predictor rows did not contain
// it, the only pairs the transferred lists can lack.

// Stale cell bounds: when a search's last particle is alone in its cell k,
// grid_end[c >= k] and grid_start[c > k] keep earlier values (sort.cu:30-60).
// A stencil row of cell c ends at cell c + XY + X + 1 at most, so only
// particles in cells from lo = k - (XY + X + 1) on have rows that can reach
// them.  k = lo = INT_MAX for a search without a lone last particle.
struct XStale {
  int kP, kC, loP, loC;  // predictor's and corrector's search
};
__device__ __forceinline__ XStale xfer_stale(const KParams& kp, const Scratch& s, const zsph_tmp_t& t) {
  const int n = kp.n, reach = kp.XY + kp.p.grid_xdim + 1;
  XStale x;
  x.kP = s.xf.hashP[n - 1] != s.xf.hashP[n - 2] ? s.xf.hashP[n - 1] : INT_MAX;
  x.kC = t.hash[n - 1] != t.hash[n - 2] ? t.hash[n - 1] : INT_MAX;
  x.loP = x.kP == INT_MAX ? INT_MAX : x.kP - reach;
  x.loC = x.kC == INT_MAX ? INT_MAX : x.kC - reach;
  return x;
}

// For a particle in cell c in both searches: whether one of its kept rows
// ends at a stale bound in one search only, or in both with a range that is
// not empty in both.  Rows that are stale and empty in both searches select
// nothing in either, and the transfer reproduces that through the corrector
// row ranges it checks every entry against.
__device__ bool xfer_stale_rows(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, const XStale& x, int c) {
  const zsph_gpu_param_t& p = kp.p;
  zsph_tmp_t tP = t;
  tP.grid_start = s.xf.gsP;
  tP.grid_end = s.xf.geP;
  for (int r = 0; r < 9; ++r) {
    const int cell = c + (r / 3 - 1) * kp.XY + (r % 3 - 1) * p.grid_xdim;
    if (cell - 1 < p.grid_hash_min || cell + 1 > p.grid_hash_max) continue;  // row_range drops it
    const bool sP = cell + 1 >= x.kP, sC = cell + 1 >= x.kC;
    if (!sP && !sC) continue;
    if (sP != sC) return true;
    int aP, bP, aC, bC;
    row_range<1>(kp, tP, c, r, aP, bP);
    row_range<1>(kp, t, c, r, aC, bC);
    if (aP < bP || aC < bC) return true;
  }
  return false;
}

// Whether corrector slot i gets a full search: the particle changed cell
// between the searches, was the predictor search's last particle (never a
// candidate there), its predictor list or skin list overflowed, or its rows
// meet stale bounds (above).  src = its predictor index.
__device__ __forceinline__ bool xfer_full(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, const XStale& x,
                                          int i, int& src) {
  src = t.index[i];
  const int cC = t.hash[i], cP = s.xf.hashP[src];
  if (cC != cP || src == kp.n - 1 || s.nb_cnt[src] == kOverflow || s.xf.sk_cnt[src] == kOverflow) return true;
  return (cC >= x.loP || cC >= x.loC) && xfer_stale_rows(kp, s, t, x, cC);
}

// Whether predictor cell cm lies in one of the stencil rows row_range keeps
// for cell cj (delta_ns.cu:39-46), i.e. a particle there (other than the
// search's last) was a candidate of a particle in cj.  Rows with stale
// bounds only matter where they are empty in both searches (xfer_full), and
// there the corrector row check drops the pair whatever this says.
__device__ __forceinline__ bool was_candidate(const KParams& kp, int cj, int cm) {
  const zsph_gpu_param_t& p = kp.p;
#pragma unroll
  for (int z = -1; z <= 1; ++z)
#pragma unroll
    for (int y = -1; y <= 1; ++y) {
      const int cell = cj + z * kp.XY + y * p.grid_xdim;
      if (cell - 1 >= p.grid_hash_min && cell + 1 <= p.grid_hash_max && cm >= cell - 1 && cm <= cell + 1)
        return true;
    }
  return false;
}

// Full-search particle (predictor index srcM, predictor cell cPM) found
// within 2h of corrector slot j: hand it to j unless j searches in full too
// or its predictor lists already hold the pair.  A slot without a full
// search kept its cell, so its corrector hash is its predictor cell.
__device__ __forceinline__ void xfer_hand_over(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, int j,
                                               int srcM, int cPM) {
  if (s.xf.fullb[j]) return;
  if (srcM != kp.n - 1 && was_candidate(kp, t.hash[j], cPM)) return;
  const int k = atomicAdd(s.xf.xcnt + j, 1);
  if (k < kXtra) s.xf.xl[(size_t)j * kXtra + k] = srcM;
  else atomicOr(s.xf.flag, 1);
}

// One warp's full search for corrector slot M: its list exactly as the
// full build makes it (each row's range as row_range gives it, stale
// bounds included; rows in order, candidates in order), plus the
// hand-overs.  The hand-over scans each row's cells' true particle range,
// the last particle included and rows at the ends of the hash range clamped
// instead of dropped, so it reaches every particle whose rows hold M; those
// ranges are disjoint, so no particle is handed M twice.
__device__ __forceinline__ void xfer_full_search(const KParams& kp, const Scratch& s, const zsph_ptc_t& cur,
                                                 const zsph_tmp_t& t, int M) {
  const zsph_gpu_param_t& p = kp.p;
  const int n = kp.n, lane = threadIdx.x & 31;
  const int srcM = t.index[M];
  const float px = cur.pos[3 * M], py = cur.pos[3 * M + 1], pz = cur.pos[3 * M + 2];
  const int cM = t.hash[M], cPM = s.xf.hashP[srcM], lastcell = t.hash[n - 1];
  int cnt = 0;
  bool ovf = false;
  for (int r = 0; r < 9; ++r) {
    int a, b;  // the row as the full build scans it
    row_range<1>(kp, t, cM, r, a, b);
    const int cell = cM + (r / 3 - 1) * kp.XY + (r % 3 - 1) * p.grid_xdim;
    const int cs = max(cell - 1, p.grid_hash_min), ce = min(cell + 1, p.grid_hash_max);
    int a2 = n, b2 = n;  // the true range of the row's cells (empty when they are off the grid)
    if (cs <= ce) {
      a2 = cs > lastcell ? n : max(t.grid_start[cs], 0);
      b2 = ce >= lastcell ? n : min(t.grid_end[ce], n);
    }
    // [lo, hi) in ascending order: the row's own range below the true one,
    // the true one, the own range above it (the first and last are empty
    // unless bounds are stale)
    auto scan = [&](int lo, int hi) {
      for (int j0 = lo; j0 < hi; j0 += 32) {
        const int j = j0 + lane;
        bool hit = false;
        if (j < hi && j != M)
          hit = interacts(kp, dist2(px - cur.pos[3 * j], py - cur.pos[3 * j + 1], pz - cur.pos[3 * j + 2]));
        const bool own = hit && j >= a && j < b;
        const unsigned om = __ballot_sync(0xffffffffu, own);
        bool bad = false;
        if (own) {
          const int k = cnt + __popc(om & lanemask_lt());
          const int off = j - a;
          if (k < kMaxNb && off <= kOffMask)
            s.xf.nb2[nb_vec(M, k >> 3) * 8 + (k & 7)] = (uint16_t)(((unsigned)r << kRowShift) | (unsigned)off);
          else
            bad = true;
        }
        cnt += __popc(om);
        ovf |= __any_sync(0xffffffffu, bad);
        if (hit && j >= a2 && j < b2) xfer_hand_over(kp, s, t, j, srcM, cPM);
      }
    };
    if (a2 < b2) {
      scan(a, min(b, a2));
      scan(a2, b2);
      scan(max(a, b2), b);
    } else {
      scan(a, b);
    }
  }
  if (cnt > 254) ovf = true;
  if (lane == 0) s.xf.nb_cnt2[M] = ovf ? kOverflow : (uint8_t)cnt;
  if (lane == 0 && ovf) atomicOr(s.flags, ZSPH_FLAG_NB_OVERFLOW);
}

// Corrector, after its search: each slot's class (fullb), its corrector
// slot in its predicted-position record (pos4[src].w), and the list of the
// slots that get a full search.  (The step needs n >= 64.)
__global__ void __launch_bounds__(kSearchBlock) k_xfer_classify(KParams kp, Scratch s, zsph_tmp_t t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool act = i < kp.n;
  int src = 0;
  bool full = false;
  if (act) {
    full = xfer_full(kp, s, t, xfer_stale(kp, s, t), i, src);
    reinterpret_cast<int*>(s.xf.pos4)[4 * (size_t)src + 3] = i;
    s.xf.fullb[i] = full ? 1 : 0;
  }
  const unsigned m = __ballot_sync(0xffffffffu, full);
  if (m) {
    int base = 0;
    if (lane == 0) {
      base = atomicAdd(s.xf.acount, __popc(m));
      atomicAdd(s.xf.stats + 2, (unsigned long long)__popc(m));
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    if (full) s.xf.alist[base + __popc(m & lanemask_lt())] = i;
  }
}

constexpr int kSearchWarps = 4;  // warps per CTA of k_xfer_search

// The full searches, one warp per listed slot (grid-stride over the list).
__global__ void __launch_bounds__(kSearchWarps * 32) k_xfer_search(KParams kp, Scratch s, zsph_ptc_t cur,
                                                                    zsph_tmp_t t) {
  const int na = *s.xf.acount;
  const int w0 = blockIdx.x * kSearchWarps + (threadIdx.x >> 5), nw = gridDim.x * kSearchWarps;
  for (int w = w0; w < na; w += nw) xfer_full_search(kp, s, cur, t, s.xf.alist[w]);
}

constexpr int kXferThreads = 64;            // threads (particles) per CTA of k_nblist_xfer
constexpr int kXBuf = kMaxNb + kSkinCap;    // a particle's merged predictor and skin entries

// Corrector: the transferred lists (see above), then each particle's packed
// shadow record, list count and wall-list entry exactly as the full build's
// end does (the walls' (rho, p) follow in k_walls).
// Returns at once when the full build runs instead (*s.xf.flag).
// Per particle: (1) its predictor list and skin list merged by their keys
// into shared memory (both are in the predictor's candidate order, so the
// merged entries, mapped to corrector slots, are out of order only where a
// neighbour changed cell); (2) eight entries at a time, their predicted
// positions loaded together, re-tested, and kept as corrector keys in place;
// (3) the hand-overs; (4) an insertion sort back into candidate order.
__global__ void __launch_bounds__(kXferThreads) k_nblist_xfer(KParams kp, Scratch s, zsph_ptc_t cur, zsph_tmp_t t) {
  constexpr int B = kXferThreads;
  // rows of kXBuf + 6 entries: 75 words, an odd stride, so the lanes' k-th
  // entries fall in different banks
  __shared__ __align__(16) uint16_t s_buf[B][kXBuf + 6];
  __shared__ int s_row[27 * B];  // predictor row starts, corrector row starts and ends
  if (*s.xf.flag) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(s.xf.stats, 1ull);
  const int tid = threadIdx.x;
  const int i = blockIdx.x * B + tid;
  if (i >= kp.n) return;
  const bool full = s.xf.fullb[i] != 0;
  const int c = t.hash[i];
  int cnt = 0;
  bool ovf = false;
  if (!full) {
    const int src = t.index[i];
    int* rsP = s_row + tid;
    int* rsC = s_row + 9 * B + tid;
    int* reC = s_row + 18 * B + tid;
    zsph_tmp_t tP = t;
    tP.grid_start = s.xf.gsP;
    tP.grid_end = s.xf.geP;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      int a, b;
      row_range<1>(kp, tP, c, r, a, b);
      rsP[r * B] = a;
      row_range<1>(kp, t, c, r, a, b);
      rsC[r * B] = a;
      reC[r * B] = b;
    }
    uint16_t* buf = s_buf[tid];
    // (1) merge
    const int cl = s.nb_cnt[src], ks = s.xf.sk_cnt[src];
    int m = 0, kk = 0;
    unsigned skn = ks > 0 ? s.xf.sk[sk_idx(src, 0)] : 0x10000u;
    const uint4* lst = reinterpret_cast<const uint4*>(s.nb);
    for (int k = 0; k < cl; k += 8) {
      const uint4 v = lst[nb_vec(src, k >> 3)];
      const unsigned wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        if (k + e < cl) {
          const unsigned ent = (wv[e >> 1] >> ((e & 1) * 16)) & 0xffffu;
          while (skn < ent) {
            buf[m++] = (uint16_t)skn;
            skn = ++kk < ks ? s.xf.sk[sk_idx(src, kk)] : 0x10000u;
          }
          buf[m++] = (uint16_t)ent;
        }
      }
    }
    for (; kk < ks; ++kk) buf[m++] = s.xf.sk[sk_idx(src, kk)];
    // (2) re-test at the predicted positions; keep as corrector keys
    const float4 pi = s.xf.pos4[src];
    auto keep = [&](float4 q, int hint) {
      if (!interacts(kp, dist2(pi.x - q.x, pi.y - q.y, pi.z - q.z))) return;
      const int jC = __float_as_int(q.w);
      int rr = hint;
      if (jC < rsC[rr * B] || jC >= reC[rr * B]) {  // the neighbour changed row (rare)
        rr = -1;
        for (int r = 0; r < 9; ++r)
          if (jC >= rsC[r * B] && jC < reC[r * B]) rr = r;
        if (rr < 0) return;  // in none of the particle's rows
      }
      const int off = jC - rsC[rr * B];
      if (cnt < kMaxNb && off <= kOffMask) buf[cnt] = (uint16_t)(((unsigned)rr << kRowShift) | (unsigned)off);
      else ovf = true;
      ++cnt;
    };
    const int nmax = kp.n - 1;
    for (int k0 = 0; k0 < m; k0 += 8) {
      float4 q[8];
      int rw[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        int jP = 0;
        rw[e] = -1;
        if (k0 + e < m) {
          const unsigned ent = buf[k0 + e];
          rw[e] = (int)(ent >> kRowShift);
          // inside the predictor row it came from, so below n; the clamp
          // only keeps the load in bounds should that ever not hold
          jP = min(max(rsP[rw[e] * B] + (int)(ent & kOffMask), 0), nmax);
        }
        q[e] = s.xf.pos4[jP];
      }
      // cnt <= k0 + e here: the keys written never overtake the entries not yet read
#pragma unroll
      for (int e = 0; e < 8; ++e)
        if (rw[e] >= 0) keep(q[e], rw[e]);
    }
    // (3) hand-overs (predictor indices of full-search particles)
    const int kx = min(s.xf.xcnt[i], kXtra);
    for (int k = 0; k < kx; ++k) keep(s.xf.pos4[min(max(s.xf.xl[(size_t)i * kXtra + k], 0), nmax)], 4);
    if (cnt > 254) ovf = true;
    if (!ovf) {
      // (4) the candidate order: ascending (row, offset)
      for (int k = 1; k < cnt; ++k) {
        const uint16_t v = buf[k];
        int j = k - 1;
        while (j >= 0 && buf[j] > v) {
          buf[j + 1] = buf[j];
          --j;
        }
        buf[j + 1] = v;
      }
      uint4* nbv = reinterpret_cast<uint4*>(s.xf.nb2);
      const uint32_t* bw = reinterpret_cast<const uint32_t*>(buf);  // rows are 4-byte aligned
      for (int k = 0; k < cnt; k += 8)
        nbv[nb_vec(i, k >> 3)] = make_uint4(bw[k / 2], bw[k / 2 + 1], bw[k / 2 + 2], bw[k / 2 + 3]);
    }
  } else {  // the list k_xfer_search wrote
    cnt = s.xf.nb_cnt2[i];
    ovf = cnt == kOverflow;
  }
  Scratch so = s;
  so.nb = s.xf.nb2;
  so.nb_cnt = s.xf.nb_cnt2;
  const float2 rp = reinterpret_cast<const float2*>(cur.rhop)[i];
  const float4 pc = make_float4(cur.pos[3 * i], cur.pos[3 * i + 1], cur.pos[3 * i + 2], packed_rho(rp.x, cur.type[i]));
  list_tail<1, false>(kp, so, cur, i, ovf ? 0 : cnt, ovf, pc, rp, true);  // every wall to the wall pass
}

}  // namespace

cudaError_t init_pair_kernels() {
  cudaError_t e = cudaSuccess;
  auto setb = [&](auto fn, int bytes) {
    if (!e) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  setb(k_boundary<1>, pair_smem<1>(2, kWinCapB));
  setb(k_boundary<2>, pair_smem<2>(2, kWinCapB));
  setb(k_governing<1, 0>, pair_smem<1>(3, kWinCapG));
  setb(k_governing<1, 1>, pair_smem<1>(3, kWinCapG));
  setb(k_governing<1, 2>, pair_smem<1>(3, kWinCapG));
  setb(k_governing<2, 0>, pair_smem<2>(3, kWinCapG));
  setb(k_governing<2, 1>, pair_smem<2>(3, kWinCapG));
  setb(k_governing<2, 2>, pair_smem<2>(3, kWinCapG));
  setb(k_governing<1, 1, true>, pair_smem<1>(3, kWinCapG));
  setb(k_governing<1, 1, false, false, false, true>, pair_smem<1>(3, kWinCapG));
  setb(k_governing<1, 2, false, false, false, true>, pair_smem<1>(3, kWinCapG));
  setb(k_governing<2, 1, true>, pair_smem<2>(3, kWinCapG));
  setb(k_boundary_simple<1>, pair_smem<1>(0, 0));
  setb(k_boundary_simple<2>, pair_smem<2>(0, 0));
  setb(k_governing_simple<1, 0>, pair_smem<1>(0, 0));
  setb(k_governing_simple<1, 1>, pair_smem<1>(0, 0));
  setb(k_governing_simple<1, 2>, pair_smem<1>(0, 0));
  setb(k_governing_simple<2, 0>, pair_smem<2>(0, 0));
  setb(k_governing_simple<2, 1>, pair_smem<2>(0, 0));
  setb(k_governing_simple<2, 2>, pair_smem<2>(0, 0));
  return e;
}

cudaError_t launch_boundary(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                            cudaStream_t st, Prof* pf) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor == 1) return boundary_gf<1>(kp, s, ptc, t, st, pf);
  if (kp.p.grid_factor == 2) return boundary_gf<2>(kp, s, ptc, t, st, pf);
  return cudaErrorInvalidValue;
}

cudaError_t launch_nblist(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                          cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor == 1) return nblist_gf<1>(kp, s, ptc, t, st);
  if (kp.p.grid_factor == 2) return nblist_gf<2>(kp, s, ptc, t, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_governing(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                             int mode, const zsph_ptc_t& out, cudaStream_t st, Prof* pf, const FeatOut* feat) {
  if (kp.n == 0) return cudaSuccess;
  if (feat && kp.equations != ZSPH_EQ_DELTA) return cudaErrorInvalidValue;
  if (kp.p.grid_factor == 1) return governing_gf<1>(kp, s, ptc, t, mode, out, st, pf, feat);
  if (kp.p.grid_factor == 2) return governing_gf<2>(kp, s, ptc, t, mode, out, st, pf, feat);
  return cudaErrorInvalidValue;
}

cudaError_t launch_integrate(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                             int correction, cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  const int nb = (kp.n + kSearchBlock - 1) / kSearchBlock;
  if (correction) k_integrate<2><<<nb, kSearchBlock, 0, st>>>(kp, ptc, t);
  else k_integrate<1><<<nb, kSearchBlock, 0, st>>>(kp, ptc, t);
  return cudaGetLastError();
}

cudaError_t launch_corrector_reuse(const KParams& kp_in, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                                  bool fresh_boundary, int mode, int* cy, cudaStream_t st) {
  if (kp_in.n == 0) return cudaSuccess;
  if (kp_in.p.grid_factor != 1 || kp_in.scenes || kp_in.c3o || kp_in.rigid_f || kp_in.stage_windows ||
      kp_in.equations != ZSPH_EQ_DELTA || (mode != 0 && mode != 2) || !cy)
    return cudaErrorInvalidValue;
  KParams kp = kp_in;
  kp.cur_cy = cy;
  cudaError_t e = launch_pack_shadows(kp, s, ptc, st);
  if (e) return e;
  k_cur_cells<<<(kp.n + kSearchBlock - 1) / kSearchBlock, kSearchBlock, 0, st>>>(kp, ptc, cy);
  const int nb = thread_blocks(kp.n), sm = pair_smem<1>(0, 0);
  k_walls_reuse<1><<<nb, kPairBlock, 0, st>>>(kp, s, ptc, t, fresh_boundary ? 0 : 1);
  if (fresh_boundary) k_boundary<1, false, false, true><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t);
  const FeatOut none{};
  if (mode == 2) k_governing<1, 2, false, false, false, false, 1, true><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, ptc, none);
  else k_governing<1, 0, false, false, false, false, 1, true><<<nb, kPairBlock, sm, st>>>(kp, s, ptc, t, ptc, none);
  return cudaGetLastError();
}

cudaError_t launch_rigid_contact(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                                 const BodyRange* ranges, int nb, float kn, float cn, float dist, cudaStream_t st) {
  if (kp.n == 0 || nb == 0) return cudaSuccess;
  if (kp.p.grid_factor != 1 || kp.scenes || !kp.rigid_f) return cudaErrorInvalidValue;
  const int blocks = thread_blocks(kp.n);
  if (kp.c3o) k_rigid_contact<1, true><<<blocks, kPairBlock, 0, st>>>(kp, s, ptc, t, ranges, nb, kn, cn, dist);
  else k_rigid_contact<1, false><<<blocks, kPairBlock, 0, st>>>(kp, s, ptc, t, ranges, nb, kn, cn, dist);
  return cudaGetLastError();
}

cudaError_t persistent_grid(int* grid) {
  int dev = 0, sms = 0, per_sm = 0;
  // 46 KB of static shared memory (the list build's staging) plus the two
  // pair blocks' row arrays: above the 48 KB a launch gets without opting in
  cudaError_t e = cudaFuncSetAttribute(k_batch_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * pair_smem<1>(0, 0));
  if (!e) e = cudaGetDevice(&dev);
  if (!e) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (!e) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persistent, kPersistThreads,
                                                            2 * pair_smem<1>(0, 0));
  if (!e && per_sm < 1) e = cudaErrorInvalidConfiguration;
  if (!e) *grid = per_sm * sms;
  return e;
}

cudaError_t launch_batch_persistent(const KParams& kp, const Scratch& s, const zsph_ptc_t& o, const zsph_ptc_t& w,
                                    const zsph_tmp_t& t, unsigned* bar, int nsteps, unsigned spin_limit, int extra,
                                    cudaStream_t st) {
  if (!kp.scenes || kp.p.grid_factor != 1 || kp.equations != ZSPH_EQ_DELTA || kp.c3o || kp.rigid_f ||
      kp.stage_windows)
    return cudaErrorInvalidValue;
  if (!ptc_aligned8(o) || !ptc_aligned8(w)) return cudaErrorMisalignedAddress;  // nothing launched
  int grid = 0;
  cudaError_t e = persistent_grid(&grid);
  if (e) return e;
  PersistArgs a{kp, s, o, w, t, bar, nsteps, spin_limit, extra};
  void* args[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)k_batch_persistent, dim3(grid), dim3(kPersistThreads), args,
                                     2 * pair_smem<1>(0, 0), st);
}

cudaError_t launch_xfer_pred_lists(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                                   cudaStream_t st, Prof* pf) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor != 1 || kp.scenes || kp.c3o || kp.stage_windows || kp.equations != ZSPH_EQ_DELTA || !s.xf.sk)
    return cudaErrorInvalidValue;
  if (cudaError_t e = reset_walls(s, st)) return e;
  const int segs = kp.tune_segs ? kp.tune_segs : kSegs;
  const int g4 = (kp.n + 127) / 128, g2 = (kp.n + 63) / 64;
  if (kp.tune_cw == 4) {
    if (segs == 2) k_nblist_seq<1, 4, false, false, 2, true><<<g4, 128, 0, st>>>(kp, s, ptc, t);
    else if (segs == 3) k_nblist_seq<1, 4, false, false, 3, true><<<g4, 128, 0, st>>>(kp, s, ptc, t);
    else k_nblist_seq<1, 4, false, false, 4, true><<<g4, 128, 0, st>>>(kp, s, ptc, t);
  } else {
    if (segs == 2) k_nblist_seq<1, 2, false, false, 2, true><<<g2, 64, 0, st>>>(kp, s, ptc, t);
    else if (segs == 3) k_nblist_seq<1, 2, false, false, 3, true><<<g2, 64, 0, st>>>(kp, s, ptc, t);
    else k_nblist_seq<1, 2, false, false, 4, true><<<g2, 64, 0, st>>>(kp, s, ptc, t);
  }
  mark(pf, "nblist", st);
  launch_walls<1>(kp, s, t, st);
  mark(pf, "walls", st);
  k_boundary<1><<<thread_blocks(kp.n), kPairBlock, pair_smem<1>(0, 0), st>>>(kp, s, ptc, t);
  mark(pf, "boundary", st);
  return cudaGetLastError();
}

cudaError_t launch_xfer_corr_lists(const KParams& kp, const Scratch& s, const zsph_ptc_t& cur, const zsph_tmp_t& t,
                                   cudaStream_t st, Prof* pf) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor != 1 || kp.scenes || kp.c3o || kp.stage_windows || kp.equations != ZSPH_EQ_DELTA || !s.xf.nb2)
    return cudaErrorInvalidValue;
  if (cudaError_t e = reset_walls(s, st)) return e;
  k_xfer_classify<<<(kp.n + kSearchBlock - 1) / kSearchBlock, kSearchBlock, 0, st>>>(kp, s, t);
  mark(pf, "xfer_classify", st);
  static int sms = 0;  // SMs of the device (the same for every B200)
  if (!sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
  }
  k_xfer_search<<<sms * 8, kSearchWarps * 32, 0, st>>>(kp, s, cur, t);
  mark(pf, "xfer_search", st);
  k_nblist_xfer<<<(kp.n + kXferThreads - 1) / kXferThreads, kXferThreads, 0, st>>>(kp, s, cur, t);
  mark(pf, "nblist_xfer", st);
  Scratch s2 = s;  // the walks read the corrector's lists
  s2.nb = s.xf.nb2;
  s2.nb_cnt = s.xf.nb_cnt2;
  const int segs = kp.tune_segs ? kp.tune_segs : kSegs;
  const int g4 = (kp.n + 127) / 128, g2 = (kp.n + 63) / 64;
  if (kp.tune_cw == 4) {
    if (segs == 2) k_nblist_fallback<4, 2><<<g4, 128, 0, st>>>(kp, s2, cur, t);
    else if (segs == 3) k_nblist_fallback<4, 3><<<g4, 128, 0, st>>>(kp, s2, cur, t);
    else k_nblist_fallback<4, 4><<<g4, 128, 0, st>>>(kp, s2, cur, t);
  } else {
    if (segs == 2) k_nblist_fallback<2, 2><<<g2, 64, 0, st>>>(kp, s2, cur, t);
    else if (segs == 3) k_nblist_fallback<2, 3><<<g2, 64, 0, st>>>(kp, s2, cur, t);
    else k_nblist_fallback<2, 4><<<g2, 64, 0, st>>>(kp, s2, cur, t);
  }
  mark(pf, "nblist_fallback", st);
  launch_walls<1>(kp, s2, t, st);
  mark(pf, "walls", st);
  k_boundary<1><<<thread_blocks(kp.n), kPairBlock, pair_smem<1>(0, 0), st>>>(kp, s2, cur, t);
  mark(pf, "boundary", st);
  return cudaGetLastError();
}

cudaError_t launch_nb_counts(const KParams& kp, const Scratch& s, int* nb_boundary, int* nb_governing,
                             cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  const int nb = (kp.n + kSearchBlock - 1) / kSearchBlock;
  if (kp.p.grid_factor == 1) k_nb_counts<1><<<nb, kSearchBlock, 0, st>>>(kp, s, nb_boundary, nb_governing);
  else if (kp.p.grid_factor == 2) k_nb_counts<2><<<nb, kSearchBlock, 0, st>>>(kp, s, nb_boundary, nb_governing);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace zsph
