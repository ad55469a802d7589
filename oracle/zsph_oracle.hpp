// ZSPH delta-SPH single-GPU step -- CPU ORACLE (test infrastructure only).
//
// This header restates, on the CPU, the algorithm of the reference solver's
// single-GPU delta-SPH step so that tests and the bench's CPU-baseline leg can
// check the CUDA path against it.  It is never linked into the product
// library.  Every function cites the reference file:line it follows
// (paths relative to the reference project root).
//
// The restatement is templated on the arithmetic type T:
//   T = float  : the FP32 instance.  Hash, sort and cell bounds use exactly the
//                reference's float operations, so they are bit-exact with the
//                reference CUDA path on the same input.  The pair distance
//                r^2 is formed as fma(dz,dz,fma(dy,dy,dx*dx)), the contraction
//                nvcc applies to the reference expression (checked against the
//                reference build's own outputs by tests/golden fixtures).
//   T = double : the FP64 oracle of the same equations with the same (float-
//                derived) constants; only the arithmetic precision differs.
//
// Deterministic wall-density semantics.  The reference's cuda_boundary_ns
// writes the extrapolated wall density in place (delta_ns.cu:130) while other
// threads read neighbour densities (delta_ns.cu:53,65,151,158): a race whose
// outcome depends on the schedule.  The oracle offers two deterministic
// orders that bracket it:
//   WALLS_FIRST (0): every neighbour read sees the new wall density; a wall
//                    particle's own loop-2 uses its old density (rhop_0 is
//                    loaded before the write, delta_ns.cu:25).  This is the
//                    semantics of the product kernels.
//   WALLS_OLD   (1): every neighbour read sees the old density.
//   WALLS_SPLIT (2): loop 1 (renormalisation matrix, div v) sees the old wall
//                    densities and loop 2 (grad rho) the new ones -- the
//                    outcome of the race when the reading and the writing
//                    threads run concurrently (each wall thread writes after
//                    its own loop 1, before the readers reach loop 2).
//
// The neighbour visit order is the reference's: stencil rows z = -gf..gf,
// y = -gf..gf-1 (boundary, delta_ns.cu:35-37) or y = -gf..gf (governing,
// delta_ns.cu:204-206); inside a row the contiguous sorted-particle range
// [grid_start[c-gf], grid_end[c+gf]) (delta_ns.cu:39-46).  The governing
// kernel's order-dependent recurrence on grad(rho).x (delta_ns.cu:244-245)
// therefore gives the same result as the reference's sequence.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace zsph_oracle {

enum { WALLS_FIRST = 0, WALLS_OLD = 1, WALLS_SPLIT = 2 };

// Derived constants; field meaning follows gpu_param_t
// (single_gpu_sph_src/header/data_structure.cuh:107-134) plus the host-side
// values the oracle needs (grid_num, dt, dt_max).
struct Params {
  float half_dt, h, g, m, rho0, adh, h2, eta2, cs2, alpha, delta_h_cs, h_cs_rho_m;
  float grid_size;
  int grid_factor;
  float grid_xmin, grid_ymin, grid_zmin;
  int grid_xdim, grid_ydim, grid_zdim, grid_hash_min, grid_hash_max, ptc_num;
  int grid_num;
  float dt, dt_max, cs, eta, r;
};

template <class T> struct State {
  T *pos, *vel, *rhop, *tmp_pos, *tmp_vel, *tmp_rhop;  // 3,3,2,3,3,2 per particle
  int *type, *table;
};

template <class T> struct Tmp {
  T *acc_drhodt, *dofv_grandrho;  // 4 per particle each
  int *index, *hash, *grid_start, *grid_end;
};

// float -> int conversion as the GPU's cvt.rzi.s32.f32 does it: truncation,
// saturation at the int range, NaN -> 0 (hash.cu:12-14 assigns floorf() to int).
template <class T> inline int cvt_rzi(T v) {
  if (std::isnan(v)) return 0;
  if (v >= (T)2147483647.0) return 2147483647;
  if (v <= (T)-2147483648.0) return (int)0x80000000;
  return (int)v;
}

// single_gpu_sph_src/lib/hash.cu:3-26
template <class T> void hash(const Params& p, State<T>& s, Tmp<T>& t) {
  const int n = p.ptc_num;
  const T gxmin = (T)p.grid_xmin, gymin = (T)p.grid_ymin, gzmin = (T)p.grid_zmin, gs = (T)p.grid_size;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const int hx = cvt_rzi<T>(std::floor((s.pos[3 * i + 0] - gxmin) / gs));
    const int hy = cvt_rzi<T>(std::floor((s.pos[3 * i + 1] - gymin) / gs));
    const int hz = cvt_rzi<T>(std::floor((s.pos[3 * i + 2] - gzmin) / gs));
    // two's complement wrap-around, as the GPU's 32-bit integer multiply-add
    const uint32_t X = (uint32_t)p.grid_xdim, Y = (uint32_t)p.grid_ydim;
    int h = (int)((uint32_t)hz * X * Y + (uint32_t)hy * X + (uint32_t)hx);
    if (h < p.grid_hash_min || h > p.grid_hash_max) {  // hash.cu:16-23
      s.type[i] = 100;
      s.pos[3 * i + 0] = gxmin; s.pos[3 * i + 1] = gymin; s.pos[3 * i + 2] = gzmin;
      s.vel[3 * i + 0] = 0; s.vel[3 * i + 1] = 0; s.vel[3 * i + 2] = 0;
      s.rhop[2 * i + 0] = (T)p.rho0; s.rhop[2 * i + 1] = 0;
      h = 0;
    }
    t.hash[i] = h;
    t.index[i] = i;  // hash.cu:24
  }
}

// single_gpu_sph_src/lib/sort.cu:3-6: thrust::sort_by_key(hash, index) is a
// stable ascending sort of the keys carrying the values.  Restated as a
// stable counting sort over the key range (keys are in [0, grid_num) after
// hash()); keys outside that range fall back to std::stable_sort.
template <class T> void sort_index(const Params& p, Tmp<T>& t) {
  const int n = p.ptc_num, G = p.grid_num;
  bool in_range = true;
  for (int i = 0; i < n; ++i) if (t.hash[i] < 0 || t.hash[i] >= G) { in_range = false; break; }
  std::vector<int> key(t.hash, t.hash + n), val(t.index, t.index + n);
  if (!in_range) {
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    for (int i = 0; i < n; ++i) { t.hash[i] = key[order[i]]; t.index[i] = val[order[i]]; }
    return;
  }
  std::vector<int> cnt((size_t)G + 1, 0);
  for (int i = 0; i < n; ++i) cnt[key[i] + 1]++;
  for (int c = 0; c < G; ++c) cnt[c + 1] += cnt[c];
  for (int i = 0; i < n; ++i) {
    const int d = cnt[key[i]]++;
    t.hash[d] = key[i];
    t.index[d] = val[i];
  }
}

// single_gpu_sph_src/lib/sort.cu:8-84: cell bounds from the sorted keys, with
// the reference's branch order (a change of key first, then tid==0, then
// tid==N-1), followed by the gather of all eight particle arrays and the
// table update table_new = table_old + old_index - tid (sort.cu:82).
template <class T> void sort_data(const Params& p, const State<T>& o, State<T>& w, Tmp<T>& t) {
  const int n = p.ptc_num;
  for (int tid = 0; tid < n; ++tid) {
    const int h = t.hash[tid];
    const int prev = tid > 0 ? t.hash[tid - 1] : h;
    if (h != prev) {  // sort.cu:30-40
      t.grid_start[h] = tid;
      t.grid_end[prev] = tid;
      for (int c = prev + 1; c < h; ++c) { t.grid_start[c] = tid; t.grid_end[c] = tid; }
    } else if (tid == 0) {  // sort.cu:41-50
      t.grid_start[h] = tid;
      for (int c = 0; c < h; ++c) { t.grid_end[c] = tid; t.grid_start[c] = tid; }
    } else if (tid == n - 1) {  // sort.cu:51-60
      t.grid_end[h] = tid;
      for (int c = h + 1; c <= p.grid_hash_max; ++c) { t.grid_end[c] = tid; t.grid_start[c] = tid; }
    }
  }
#pragma omp parallel for schedule(static)
  for (int tid = 0; tid < n; ++tid) {  // sort.cu:62-82
    const int oi = t.index[tid];
    for (int k = 0; k < 3; ++k) {
      w.pos[3 * tid + k] = o.pos[3 * oi + k];
      w.vel[3 * tid + k] = o.vel[3 * oi + k];
      w.tmp_pos[3 * tid + k] = o.tmp_pos[3 * oi + k];
      w.tmp_vel[3 * tid + k] = o.tmp_vel[3 * oi + k];
    }
    for (int k = 0; k < 2; ++k) {
      w.rhop[2 * tid + k] = o.rhop[2 * oi + k];
      w.tmp_rhop[2 * tid + k] = o.tmp_rhop[2 * oi + k];
    }
    w.type[tid] = o.type[oi];
    w.table[tid] = o.table[oi] + oi - tid;
  }
}

// Squared distance as the reference's dx.x*dx.x + dx.y*dx.y + dx.z*dx.z
// compiles on the GPU (left-to-right contraction into fused multiply-adds).
inline float rr2_of(float x, float y, float z) { return std::fmaf(z, z, std::fmaf(y, y, x * x)); }
inline double rr2_of(double x, double y, double z) { return x * x + y * y + z * z; }

// Visits the reference's stencil rows for particle i in order and calls
// f(j) for every j != i in each row's particle range.
// single_gpu_sph_src/equation/delta_ns.cu:35-48 (ylast = gf-1) and :204-217
// (ylast = gf).
template <class T, class F>
inline void for_each_candidate(const Params& p, const Tmp<T>& t, int i, int ylast, F&& f) {
  const int gf = p.grid_factor;
  for (int z = -gf; z <= gf; ++z)
    for (int y = -gf; y <= ylast; ++y) {
      int cs = t.hash[i] + z * p.grid_xdim * p.grid_ydim + y * p.grid_xdim;
      int ce = cs + gf;
      cs = cs - gf;
      if (cs >= p.grid_hash_min && ce <= p.grid_hash_max) {
        const int a = t.grid_start[cs], b = t.grid_end[ce];
        for (int j = a; j < b; ++j)
          if (j != i) f(j);
      }
    }
}

// Wall (type != 1) pressure extrapolation from fluid neighbours:
// single_gpu_sph_src/equation/delta_ns.cu:61-85 (sums) and :116-131 (result).
// Writes the new (rho, p) of every non-fluid particle into rho_new/p_new.
template <class T>
void wall_pressure(const Params& p, const State<T>& s, const Tmp<T>& t, std::vector<T>& rho_new,
                   std::vector<T>& p_new) {
  const int n = p.ptc_num;
  const T h = (T)p.h, adh = (T)p.adh, g = (T)p.g, cs2 = (T)p.cs2, rho0 = (T)p.rho0;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    rho_new[i] = s.rhop[2 * i];
    p_new[i] = s.rhop[2 * i + 1];
    if (s.type[i] == 1) continue;
    T rsum = 0, wsum = 0;
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    for_each_candidate(p, t, i, p.grid_factor - 1, [&](int j) {
      const T dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
      const T rr2 = rr2_of(dx, dy, dz);
      const T q = std::sqrt(rr2) / h;
      if (q <= (T)2) {
        const T a = (T)1 - q / (T)2;
        T w = a * a * a;
        w = w * a;
        w *= ((T)2 * q + (T)1) * adh;
        if (s.type[j] == 1) {
          const T rj = s.rhop[2 * j], pj = s.rhop[2 * j + 1];
          rsum += (pj - rj * ((T)0 * dx + (T)0 * dy + ((T)0 - g) * dz)) * w;
          wsum += w;
        }
      }
    });
    if (std::fabs(wsum) > (T)1e-8f) rsum = rsum / wsum; else rsum = 0;
    if (rsum < 0) rsum = 0;
    p_new[i] = rsum;
    rho_new[i] = rsum / cs2 + rho0;
  }
}

// single_gpu_sph_src/equation/delta_ns.cu:5-177 (cuda_boundary_ns) with the
// deterministic wall semantics described at the top of this file.
template <class T> void boundary(const Params& p, State<T>& s, Tmp<T>& t, int wall_mode) {
  const int n = p.ptc_num;
  std::vector<T> rho_new(n), p_new(n);
  wall_pressure(p, s, t, rho_new, p_new);
  std::vector<T> rho_old(n);
  for (int i = 0; i < n; ++i) rho_old[i] = s.rhop[2 * i];
  // Densities seen through neighbour reads in loop 1 and loop 2.
  const std::vector<T>& rho_nb = (wall_mode == WALLS_FIRST) ? rho_new : rho_old;
  const std::vector<T>& rho_nb2 = (wall_mode == WALLS_OLD) ? rho_old : rho_new;
  const T h = (T)p.h, adh = (T)p.adh, h2 = (T)p.h2, m = (T)p.m;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    T L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    T divv = 0;
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    const T vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
    const T rho0_i = rho_old[i];
    const int ti = s.type[i];
    // loop 1: delta_ns.cu:35-96
    for_each_candidate(p, t, i, p.grid_factor - 1, [&](int j) {
      const T d[3] = {px - s.pos[3 * j], py - s.pos[3 * j + 1], pz - s.pos[3 * j + 2]};
      const T dvx = vx - s.vel[3 * j], dvy = vy - s.vel[3 * j + 1], dvz = vz - s.vel[3 * j + 2];
      const T rr2 = rr2_of(d[0], d[1], d[2]);
      const T dvdx = dvx * d[0] + dvy * d[1] + dvz * d[2];
      const T q = std::sqrt(rr2) / h;
      if (q <= (T)2) {
        const T a = (T)1 - q / (T)2;
        T fr = a * a * a;
        fr *= (T)-5 * adh / h2;
        const T rj = rho_nb[j];
        const T tl = fr * m / rj;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) L[r][c] -= d[r] * d[c] * tl;
        if (ti == 1 && s.type[j] == 1) divv -= fr * dvdx * m / rj;
      }
    });
    // cofactor inverse: delta_ns.cu:99-114
    const T det = L[0][0] * L[1][1] * L[2][2] + L[0][1] * L[1][2] * L[2][0] + L[0][2] * L[1][0] * L[2][1] -
                  L[0][2] * L[1][1] * L[2][0] - L[0][0] * L[1][2] * L[2][1] - L[0][1] * L[1][0] * L[2][2];
    T M[3][3];
    if (std::fabs(det) > (T)1.8e-8f) {
      M[0][0] = (L[1][1] * L[2][2] - L[1][2] * L[2][1]) / det;
      M[0][1] = (T)-1 * (L[1][0] * L[2][2] - L[1][2] * L[2][0]) / det;
      M[0][2] = (L[1][0] * L[2][1] - L[1][1] * L[2][0]) / det;
      M[1][0] = (T)-1 * (L[0][1] * L[2][2] - L[0][2] * L[2][1]) / det;
      M[1][1] = (L[0][0] * L[2][2] - L[0][2] * L[2][0]) / det;
      M[1][2] = (T)-1 * (L[0][0] * L[2][1] - L[0][1] * L[2][0]) / det;
      M[2][0] = (L[0][1] * L[1][2] - L[0][2] * L[1][1]) / det;
      M[2][1] = (T)-1 * (L[0][0] * L[1][2] - L[0][2] * L[1][0]) / det;
      M[2][2] = (L[0][0] * L[1][1] - L[0][1] * L[1][0]) / det;
    } else {
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) M[r][c] = (r == c) ? (T)1 : (T)0;
    }
    // loop 2: delta_ns.cu:133-174
    T gr[3] = {0, 0, 0};
    for_each_candidate(p, t, i, p.grid_factor - 1, [&](int j) {
      const T d[3] = {px - s.pos[3 * j], py - s.pos[3 * j + 1], pz - s.pos[3 * j + 2]};
      const T rr2 = rr2_of(d[0], d[1], d[2]);
      const T q = std::sqrt(rr2) / h;
      if (q <= (T)2) {
        const T a = (T)1 - q / (T)2;
        T fr = (T)-5 * adh * a * a * a / h2;
        const T rj = rho_nb2[j];
        fr *= (rj - rho0_i) * m / rj;
        for (int r = 0; r < 3; ++r) gr[r] += (M[r][0] * d[0] + M[r][1] * d[1] + M[r][2] * d[2]) * fr;
      }
    });
    t.dofv_grandrho[4 * i + 0] = gr[0];
    t.dofv_grandrho[4 * i + 1] = gr[1];
    t.dofv_grandrho[4 * i + 2] = gr[2];
    t.dofv_grandrho[4 * i + 3] = divv;
  }
  // wall result written back: delta_ns.cu:117-131
  for (int i = 0; i < n; ++i)
    if (s.type[i] != 1) { s.rhop[2 * i] = rho_new[i]; s.rhop[2 * i + 1] = p_new[i]; }
}

// single_gpu_sph_src/equation/delta_ns.cu:179-267 (cuda_govering_ns)
template <class T> void governing(const Params& p, const State<T>& s, Tmp<T>& t) {
  const int n = p.ptc_num;
  const T h = (T)p.h, adh = (T)p.adh, h2 = (T)p.h2, m = (T)p.m, eta2 = (T)p.eta2;
  const T dhc = (T)p.delta_h_cs, hcrm = (T)p.h_cs_rho_m, alpha = (T)p.alpha, g = (T)p.g;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    T acc[4] = {0, 0, 0, 0};
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    const T vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
    const T r0 = s.rhop[2 * i], p0 = s.rhop[2 * i + 1];
    const int ti = s.type[i];
    T G0[4] = {t.dofv_grandrho[4 * i], t.dofv_grandrho[4 * i + 1], t.dofv_grandrho[4 * i + 2],
               t.dofv_grandrho[4 * i + 3]};
    for_each_candidate(p, t, i, p.grid_factor, [&](int j) {
      const T dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
      const T dvx = vx - s.vel[3 * j], dvy = vy - s.vel[3 * j + 1], dvz = vz - s.vel[3 * j + 2];
      const T rr2 = rr2_of(dx, dy, dz);
      const T dvdx = dvx * dx + dvy * dy + dvz * dz;
      const T q = std::sqrt(rr2) / h;
      if (q <= (T)2) {
        const T a = (T)1 - q / (T)2;
        const T fr = (T)-5 * adh * a * a * a / h2;
        const T r1 = s.rhop[2 * j], p1 = s.rhop[2 * j + 1];
        const T* G1 = &t.dofv_grandrho[4 * j];
        G0[0] *= dx;  // order-dependent recurrence, delta_ns.cu:244-245
        G0[0] += G1[0] * dx + (G0[1] + G1[1]) * dy + (G0[2] + G1[2]) * dz;
        acc[3] += r0 * dvdx * fr * m / r1;
        T vt = -(p0 + p1) * m * fr / (r0 * r1);
        if (ti == 1 && s.type[j] == 1) {
          acc[3] += dhc * fr * ((r0 - r1) * (T)2 * rr2 / (rr2 + eta2) - G0[0]) * m / r1;
          vt += hcrm * fr * (G0[3] + G1[3] + alpha * dvdx / (rr2 + eta2)) / (r0 * r1);
        }
        acc[0] += vt * dx;
        acc[1] += vt * dy;
        acc[2] += vt * dz;
      }
    });
    acc[2] += g;  // delta_ns.cu:264
    for (int k = 0; k < 4; ++k) t.acc_drhodt[4 * i + k] = acc[k];
  }
}

// Learned-corrector inputs (no reference counterpart): the 32 neighbour
// aggregates that the learned form's predictor-stage governing walk writes
// for each fluid particle (zeros for walls), restated as plain sums over the
// governing stencil's neighbours (q <= 2).  Reads dofv_grandrho from the
// boundary pass and acc_drhodt from governing(); out[32 i + k] = f_k * scale[k].
//  0 sum_fluid w W      1 sum_wall w W       2-4 sum w F x_ij      5 divv_i
//  6-8 sum_fluid w F (divv_j - divv_i) x_ij    9-11 divv_i sum_fluid w F x_ij
//  12 sum_fluid w F (rho_i - rho_j) 2e          13 sum w F (p_i - p_j) 2e
//  14-17 acc, drho/dt   18-20 v_i   21 rho_i - rho0   22-24 grad rho_i
//  25-27, 31 D = (acc, drho/dt) - the previous corrector-stage value of the
//  same particle (acc_prev, in the order before this search: index[i])
//  28-30 sum_wall -(p_i + p_j) m F x_ij / (rho_i rho_j)
//  w = m / rho_j, grad W = F x_ij, e = r^2/(r^2+eta^2)
template <class T>
void features(const Params& p, const State<T>& s, const Tmp<T>& t, const float* scale, const T* acc_prev, T* out) {
  const int n = p.ptc_num;
  const T h = (T)p.h, adh = (T)p.adh, h2 = (T)p.h2, m = (T)p.m, eta2 = (T)p.eta2, rho0 = (T)p.rho0;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    T f[32] = {};
    if (s.type[i] == 1) {
      const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
      const T vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
      const T r0 = s.rhop[2 * i], p0 = s.rhop[2 * i + 1];
      const T* G0 = &t.dofv_grandrho[4 * i];
      T k3[3] = {0, 0, 0};
      for_each_candidate(p, t, i, p.grid_factor, [&](int j) {
        const T d[3] = {px - s.pos[3 * j], py - s.pos[3 * j + 1], pz - s.pos[3 * j + 2]};
        const T rr2 = rr2_of(d[0], d[1], d[2]);
        const T q = std::sqrt(rr2) / h;
        if (!(q <= (T)2)) return;
        const T a = (T)1 - q / (T)2;
        const T fr = (T)-5 * adh * a * a * a / h2;
        const T r1 = s.rhop[2 * j], p1 = s.rhop[2 * j + 1];
        const T frm = fr * m / r1, e = rr2 / (rr2 + eta2);
        const T wW = adh * a * a * a * a * ((T)2 * q + (T)1) * m / r1;
        for (int c = 0; c < 3; ++c) f[2 + c] += frm * d[c];
        f[13] += frm * (p0 - p1) * (T)2 * e;
        if (s.type[j] == 1) {
          const T* G1 = &t.dofv_grandrho[4 * j];
          f[0] += wW;
          for (int c = 0; c < 3; ++c) {
            f[6 + c] += frm * (G1[3] - G0[3]) * d[c];
            k3[c] += frm * d[c];
          }
          f[12] += frm * (r0 - r1) * (T)2 * e;
        } else {
          f[1] += wW;
          const T vt = -(p0 + p1) * m * fr / (r0 * r1);
          for (int c = 0; c < 3; ++c) f[28 + c] += vt * d[c];
        }
      });
      f[5] = G0[3];
      for (int c = 0; c < 3; ++c) {
        f[9 + c] = G0[3] * k3[c];
        f[22 + c] = G0[c];
      }
      for (int c = 0; c < 4; ++c) f[14 + c] = t.acc_drhodt[4 * i + c];
      if (acc_prev) {
        const T* ap = &acc_prev[4 * (size_t)t.index[i]];
        for (int c = 0; c < 3; ++c) f[25 + c] = t.acc_drhodt[4 * i + c] - ap[c];
        f[31] = t.acc_drhodt[4 * i + 3] - ap[3];
      }
      f[18] = vx; f[19] = vy; f[20] = vz;
      f[21] = r0 - rho0;
    }
    for (int k = 0; k < 32; ++k) out[32 * (size_t)i + k] = f[k] * (T)scale[k];
  }
}

// single_gpu_sph_src/lib/time_int.cu:3-48
template <class T> void prediction(const Params& p, State<T>& s, const Tmp<T>& t) {
  const T hdt = (T)p.half_dt, rho0 = (T)p.rho0, cs2 = (T)p.cs2;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < p.ptc_num; ++i) {
    if (s.type[i] != 1) continue;
    for (int k = 0; k < 3; ++k) {
      s.tmp_pos[3 * i + k] = s.pos[3 * i + k];
      s.tmp_vel[3 * i + k] = s.vel[3 * i + k];
    }
    s.tmp_rhop[2 * i] = s.rhop[2 * i];
    s.tmp_rhop[2 * i + 1] = s.rhop[2 * i + 1];
    for (int k = 0; k < 3; ++k) s.pos[3 * i + k] += s.vel[3 * i + k] * hdt;
    for (int k = 0; k < 3; ++k) s.vel[3 * i + k] += t.acc_drhodt[4 * i + k] * hdt;
    T r = s.rhop[2 * i] + t.acc_drhodt[4 * i + 3] * hdt;
    if (r < rho0) r = rho0;
    s.rhop[2 * i] = r;
    s.rhop[2 * i + 1] = cs2 * (r - rho0);
  }
}

// single_gpu_sph_src/lib/time_int.cu:50-92
template <class T> void correction(const Params& p, State<T>& s, const Tmp<T>& t) {
  const T hdt = (T)p.half_dt, rho0 = (T)p.rho0, cs2 = (T)p.cs2;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < p.ptc_num; ++i) {
    if (s.type[i] != 1) continue;
    T v[3];
    for (int k = 0; k < 3; ++k) v[k] = s.vel[3 * i + k];
    for (int k = 0; k < 3; ++k) s.pos[3 * i + k] = s.tmp_pos[3 * i + k] + v[k] * hdt * (T)2;
    for (int k = 0; k < 3; ++k) s.vel[3 * i + k] = s.tmp_vel[3 * i + k] + t.acc_drhodt[4 * i + k] * hdt * (T)2;
    T r = s.tmp_rhop[2 * i] + t.acc_drhodt[4 * i + 3] * hdt * (T)2;
    if (r < rho0) r = rho0;
    s.rhop[2 * i] = r;
    s.rhop[2 * i + 1] = cs2 * (r - rho0);
  }
}

// One full step, single_gpu_sph_src/deltasph/main.cu:63-88: predictor
// sub-step sorts OLD into NEW, corrector sub-step sorts NEW back into OLD.
template <class T> void step(const Params& p, State<T>& o, State<T>& w, Tmp<T>& t, int wall_mode) {
  hash(p, o, t);
  sort_index(p, t);
  sort_data(p, o, w, t);
  boundary(p, w, t, wall_mode);
  governing(p, w, t);
  prediction(p, w, t);
  hash(p, w, t);
  sort_index(p, t);
  sort_data(p, w, o, t);
  boundary(p, o, t, wall_mode);
  governing(p, o, t);
  correction(p, o, t);
}

// Number of candidates j with q <= 2 in the given stencil (ylast = gf-1 for
// the boundary kernel's rows, gf for the governing kernel's), using the
// reference's distance test (delta_ns.cu:67-68, :238-240).
template <class T> void neighbor_count(const Params& p, const State<T>& s, const Tmp<T>& t, int ylast, int* out) {
  const T h = (T)p.h;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < p.ptc_num; ++i) {
    int c = 0;
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    for_each_candidate(p, t, i, ylast, [&](int j) {
      const T rr2 = rr2_of(px - s.pos[3 * j], py - s.pos[3 * j + 1], pz - s.pos[3 * j + 2]);
      if (std::sqrt(rr2) / h <= (T)2) ++c;
    });
    out[i] = c;
  }
}


// ---- simple-SPH equations (the reference's simplesph target) ---------------

// single_gpu_sph_src/equation/simple_ns.cu:3-97 (cuda_boundary_ns of the
// simple equations): wall pressure from fluid neighbours and the scalar
// div(v) = -sum F (v_ij . x_ij) m / rho_j over fluid pairs, one loop over the
// boundary stencil rows.  Walls read only fluid densities, so the in-place
// wall write (:94) has no reader in this kernel.
template <class T> void boundary_simple(const Params& p, State<T>& s, T* dofv, const Tmp<T>& t) {
  const int n = p.ptc_num;
  std::vector<T> rho_new(n), p_new(n);
  wall_pressure(p, s, t, rho_new, p_new);
  const T h = (T)p.h, adh = (T)p.adh, h2 = (T)p.h2, m = (T)p.m;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    T dv_sum = 0;
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    const T vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
    const int ti = s.type[i];
    for_each_candidate(p, t, i, p.grid_factor - 1, [&](int j) {
      const T dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
      const T dvdx = (vx - s.vel[3 * j]) * dx + (vy - s.vel[3 * j + 1]) * dy + (vz - s.vel[3 * j + 2]) * dz;
      const T q = std::sqrt(rr2_of(dx, dy, dz)) / h;
      if (q <= (T)2) {
        const T a = (T)1 - q / (T)2;
        T fr = a * a * a;
        fr *= (T)-5 * adh / h2;
        if (ti == 1 && s.type[j] == 1) dv_sum -= fr * dvdx * m / s.rhop[2 * j];  // simple_ns.cu:69-72
      }
    });
    dofv[i] = dv_sum;
  }
  for (int i = 0; i < n; ++i)  // simple_ns.cu:81-95
    if (s.type[i] != 1) { s.rhop[2 * i] = rho_new[i]; s.rhop[2 * i + 1] = p_new[i]; }
}

// single_gpu_sph_src/equation/simple_ns.cu:99-180 (cuda_govering_ns of the
// simple equations).
template <class T> void governing_simple(const Params& p, const State<T>& s, const T* dofv, Tmp<T>& t) {
  const int n = p.ptc_num;
  const T h = (T)p.h, adh = (T)p.adh, h2 = (T)p.h2, m = (T)p.m, eta2 = (T)p.eta2;
  const T dhc = (T)p.delta_h_cs, hcrm = (T)p.h_cs_rho_m, alpha = (T)p.alpha, g = (T)p.g;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    T acc[4] = {0, 0, 0, 0};
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    const T vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
    const T r0 = s.rhop[2 * i], p0 = s.rhop[2 * i + 1];
    const int ti = s.type[i];
    const T d0 = dofv[i];
    for_each_candidate(p, t, i, p.grid_factor, [&](int j) {
      const T dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
      const T dvdx = (vx - s.vel[3 * j]) * dx + (vy - s.vel[3 * j + 1]) * dy + (vz - s.vel[3 * j + 2]) * dz;
      const T rr2 = rr2_of(dx, dy, dz);
      const T q = std::sqrt(rr2) / h;
      if (q <= (T)2) {
        const T a = (T)1 - q / (T)2;
        const T fr = (T)-5 * adh * a * a * a / h2;
        const T r1 = s.rhop[2 * j], p1 = s.rhop[2 * j + 1];
        acc[3] += (r0 * dvdx * fr + (r0 - r1) * rr2 * fr * dhc / (rr2 + eta2)) * m / r1;  // simple_ns.cu:162
        T vt = -(p0 + p1) * m * fr / (r0 * r1);
        if (ti == 1 && s.type[j] == 1) vt += hcrm * fr * (d0 + dofv[j] + alpha * dvdx / (rr2 + eta2)) / (r0 * r1);
        acc[0] += vt * dx;
        acc[1] += vt * dy;
        acc[2] += vt * dz;
      }
    });
    acc[2] += g;
    for (int k = 0; k < 4; ++k) t.acc_drhodt[4 * i + k] = acc[k];
  }
}

// One step of the simplesph driver (same call order as main.cu:63-88).
template <class T> void step_simple(const Params& p, State<T>& o, State<T>& w, Tmp<T>& t, T* dofv) {
  hash(p, o, t);
  sort_index(p, t);
  sort_data(p, o, w, t);
  boundary_simple(p, w, dofv, t);
  governing_simple(p, w, dofv, t);
  prediction(p, w, t);
  hash(p, w, t);
  sort_index(p, t);
  sort_data(p, w, o, t);
  boundary_simple(p, o, dofv, t);
  governing_simple(p, o, dofv, t);
  correction(p, o, t);
}

// ---- 6DOF rigid body coupled to the fluid (no reference counterpart) ----
// Restates the product's FP64 body update (zsph_b200/csrc/precise.cu): the
// fluid's pressure force on each body particle (type 2, original index in
// [first, first + count)), summed into force and torque about the centre of
// mass; predictor / corrector of the pose with the angular acceleration of
// Test_6DOF/equation/acc_alpha.cpp:20-33 and the quaternion rate of
// Test_6DOF/equation/time_int.cpp:14-15; body particles placed from the pose.
struct Rigid {
  double x[3], v[3], w[3], q[4], xn[3], vn[3], wn[3], qn[4], F[3], T[3], I[9], Iinv[9], M, g;
  int first, count;
  const double* r0;  // [count][3] body-frame offsets
};

inline void rig_rot(const double* q, double* R) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z);     R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y);     R[7] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}
inline void rig_mv(const double* A, const double* v, double* r) {
  for (int a = 0; a < 3; ++a) r[a] = A[3 * a] * v[0] + A[3 * a + 1] * v[1] + A[3 * a + 2] * v[2];
}
inline void rig_mtv(const double* A, const double* v, double* r) {
  for (int a = 0; a < 3; ++a) r[a] = A[a] * v[0] + A[3 + a] * v[1] + A[6 + a] * v[2];
}
inline void rig_cross(const double* a, const double* b, double* r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
inline void rig_quat(const double* q0, const double* w, const double* qr, double dt, double* out) {
  const double a = -w[0] * qr[1] - w[1] * qr[2] - w[2] * qr[3];
  const double b = w[0] * qr[0] + w[1] * qr[3] - w[2] * qr[2];
  const double c = -w[0] * qr[3] + w[1] * qr[0] + w[2] * qr[1];
  const double d = w[0] * qr[2] - w[1] * qr[1] + w[2] * qr[0];
  double r[4] = {q0[0] + 0.5 * dt * a, q0[1] + 0.5 * dt * b, q0[2] + 0.5 * dt * c, q0[3] + 0.5 * dt * d};
  const double inv = 1.0 / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
  for (int k = 0; k < 4; ++k) out[k] = r[k] * inv;
}

// Contact between a body particle and a non-fluid particle that is not of
// its own body (a wall particle or another body's): within `dist`, a
// linear spring-dashpot along the pair's normal, kn (dist - r) - cn v_n,
// repulsive only (clamped at zero).  kn = 0 turns contact off.
struct Contact {
  double kn, cn, dist;
};

// the body owning particle i (type 2, original index table[i] + i inside a
// body's range), or -1
template <class T> int body_of(const State<T>& s, int i, const Rigid* bodies, int nb) {
  if (s.type[i] != 2) return -1;
  const int id = s.table[i] + i;
  for (int b = 0; b < nb; ++b)
    if (id >= bodies[b].first && id < bodies[b].first + bodies[b].count) return b;
  return -1;
}

// Force and torque of every body: the fluid's pressure force on each body
// particle (its acceleration per unit particle mass f, times m), plus the
// contact force of the particle's non-fluid neighbours of other bodies or
// walls; summed in FP64 over the body's particles in particle order.
template <class T>
void rigid_force_all(const Params& p, const State<T>& s, const Tmp<T>& t, Rigid* bodies, int nb, const Contact& ct) {
  const T h = (T)p.h, adh = (T)p.adh, h2 = (T)p.h2, m = (T)p.m;
  std::vector<double> F((size_t)3 * nb, 0.0), Tq((size_t)3 * nb, 0.0);
  for (int i = 0; i < p.ptc_num; ++i) {
    const int bi = body_of(s, i, bodies, nb);
    if (bi < 0) continue;
    const T px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
    const T r0 = s.rhop[2 * i], p0 = s.rhop[2 * i + 1];
    T f[3] = {0, 0, 0};
    for_each_candidate(p, t, i, p.grid_factor, [&](int j) {
      if (s.type[j] != 1) return;
      const T dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
      const T rr2 = rr2_of(dx, dy, dz);
      const T q = std::sqrt(rr2) / h;
      if (!(q <= (T)2)) return;
      const T a = (T)1 - q / (T)2;
      const T fr = (T)-5 * adh * a * a * a / h2;
      const T vt = -(p0 + s.rhop[2 * j + 1]) * m * fr / (r0 * s.rhop[2 * j]);
      f[0] += vt * dx;
      f[1] += vt * dy;
      f[2] += vt * dz;
    });
    if (ct.kn > 0) {
      const T vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
      const T d0 = (T)ct.dist, kn = (T)ct.kn, cn = (T)ct.cn;
      for_each_candidate(p, t, i, p.grid_factor, [&](int j) {
        if (s.type[j] == 1 || body_of(s, j, bodies, nb) == bi) return;
        const T dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
        const T r = std::sqrt(rr2_of(dx, dy, dz));
        if (!(r < d0) || !(r > (T)0)) return;
        const T nx = dx / r, ny = dy / r, nz = dz / r;
        const T vn = (vx - s.vel[3 * j]) * nx + (vy - s.vel[3 * j + 1]) * ny + (vz - s.vel[3 * j + 2]) * nz;
        T fc = kn * (d0 - r) - cn * vn;
        if (fc < (T)0) fc = (T)0;
        f[0] += fc * nx / m;
        f[1] += fc * ny / m;
        f[2] += fc * nz / m;
      });
    }
    const Rigid& b = bodies[bi];
    const double fv[3] = {(double)m * f[0], (double)m * f[1], (double)m * f[2]};
    const double r[3] = {(double)px - b.x[0], (double)py - b.x[1], (double)pz - b.x[2]};
    double tq[3];
    rig_cross(r, fv, tq);
    for (int a = 0; a < 3; ++a) {
      F[3 * bi + a] += fv[a];
      Tq[3 * bi + a] += tq[a];
    }
  }
  for (int b = 0; b < nb; ++b)
    for (int a = 0; a < 3; ++a) {
      bodies[b].F[a] = F[3 * b + a];
      bodies[b].T[a] = Tq[3 * b + a];
    }
}

template <class T> void rigid_force(const Params& p, const State<T>& s, const Tmp<T>& t, Rigid& b) {
  rigid_force_all(p, s, t, &b, 1, Contact{0, 0, 0});
}

inline void rigid_advance(Rigid& b, int mode, double half_dt) {
  double acc[3] = {b.F[0] / b.M, b.F[1] / b.M, b.F[2] / b.M + b.g};
  double R[9], tmp[3], tmp2[3], Iw[3], alpha[3];
  rig_rot(b.q, R);
  rig_mtv(R, b.w, tmp);
  rig_mv(b.I, tmp, tmp2);
  rig_mv(R, tmp2, Iw);
  rig_cross(b.w, Iw, tmp);
  for (int a = 0; a < 3; ++a) tmp[a] = b.T[a] - tmp[a];
  rig_mtv(R, tmp, tmp2);
  rig_mv(b.Iinv, tmp2, tmp);
  rig_mv(R, tmp, alpha);
  if (mode == 1) {
    for (int a = 0; a < 3; ++a) { b.xn[a] = b.x[a]; b.vn[a] = b.v[a]; b.wn[a] = b.w[a]; }
    for (int a = 0; a < 4; ++a) b.qn[a] = b.q[a];
    double qh[4];
    rig_quat(b.qn, b.wn, b.qn, half_dt, qh);
    for (int a = 0; a < 3; ++a) {
      b.x[a] = b.xn[a] + b.vn[a] * half_dt;
      b.v[a] = b.vn[a] + acc[a] * half_dt;
      b.w[a] = b.wn[a] + alpha[a] * half_dt;
    }
    for (int a = 0; a < 4; ++a) b.q[a] = qh[a];
  } else {
    const double dt = 2.0 * half_dt;
    double q1[4];
    rig_quat(b.qn, b.w, b.q, dt, q1);
    for (int a = 0; a < 3; ++a) {
      b.x[a] = b.xn[a] + b.v[a] * dt;
      b.v[a] = b.vn[a] + acc[a] * dt;
      b.w[a] = b.wn[a] + alpha[a] * dt;
    }
    for (int a = 0; a < 4; ++a) b.q[a] = q1[a];
  }
}

template <class T> void rigid_place(const Params& p, State<T>& s, const Rigid& b) {
  double R[9];
  rig_rot(b.q, R);
  for (int i = 0; i < p.ptc_num; ++i) {
    const int k = s.table[i] + i - b.first;
    if (s.type[i] != 2 || k < 0 || k >= b.count) continue;
    double r[3], w[3];
    rig_mv(R, b.r0 + 3 * (size_t)k, r);
    rig_cross(b.w, r, w);
    for (int a = 0; a < 3; ++a) {
      s.pos[3 * i + a] = (T)(b.x[a] + r[a]);
      s.vel[3 * i + a] = (T)(b.v[a] + w[a]);
    }
  }
}

// One step with the bodies: the plain step's call order, the bodies'
// forces, updates and placements after each sub-step's governing /
// integration.
template <class T>
void step_rigid_bodies(const Params& p, State<T>& o, State<T>& w, Tmp<T>& t, Rigid* bodies, int nb,
                       const Contact& ct, int wall_mode) {
  hash(p, o, t);
  sort_index(p, t);
  sort_data(p, o, w, t);
  boundary(p, w, t, wall_mode);
  governing(p, w, t);
  rigid_force_all(p, w, t, bodies, nb, ct);
  for (int b = 0; b < nb; ++b) rigid_advance(bodies[b], 1, (double)p.half_dt);
  prediction(p, w, t);
  for (int b = 0; b < nb; ++b) rigid_place(p, w, bodies[b]);
  hash(p, w, t);
  sort_index(p, t);
  sort_data(p, w, o, t);
  boundary(p, o, t, wall_mode);
  governing(p, o, t);
  rigid_force_all(p, o, t, bodies, nb, ct);
  for (int b = 0; b < nb; ++b) rigid_advance(bodies[b], 2, (double)p.half_dt);
  correction(p, o, t);
  for (int b = 0; b < nb; ++b) rigid_place(p, o, bodies[b]);
}

template <class T> void step_rigid(const Params& p, State<T>& o, State<T>& w, Tmp<T>& t, Rigid& b, int wall_mode) {
  step_rigid_bodies(p, o, w, t, &b, 1, Contact{0, 0, 0}, wall_mode);
}

}  // namespace zsph_oracle
