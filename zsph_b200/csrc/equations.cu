// delta-SPH pair-interaction kernels for sm_100a.
//
// Reference path replaced (single_gpu_sph_src/):
//   equation/delta_ns.cu:5-177   cuda_boundary_ns  -> k_nblist (list + wall pressure) + k_boundary
//   equation/delta_ns.cu:179-267 cuda_govering_ns  -> k_governing (optionally fused with time_int.cu)
//   lib/time_int.cu:3-92         cuda_prediction / cuda_correction -> k_integrate or k_governing epilogue
//
// Design.  The reference re-scans every candidate of the cell stencil in each
// of its three neighbour loops per sub-step, and every lane of a warp pays
// for the full pair arithmetic whenever any lane has a neighbour.  Here one
// kernel filters the candidates once per sub-step (the governing stencil is
// a superset of the boundary stencil) and writes, per particle, the list of
// interacting neighbours in the reference's visit order: stencil rows in
// (z, y) order, inside a row the sorted particle range.  Entries are 16-bit
// (row << 11 | offset inside the row's range), column-major so that a warp's
// accesses coalesce.  The pair kernels then walk their lists with all lanes
// converged.  The visit order is the reference's, so the order-dependent
// recurrence on grad(rho).x (delta_ns.cu:244-245) gets the same sequence.
//
// Neighbour test: the reference's q = sqrtf(r2)/h <= 2 (delta_ns.cu:67-68),
// with r2 formed as fma(dz,dz,fma(dy,dy,dx*dx)).  Far from the threshold the
// test is decided on r2 alone; within a relative 1e-5 of it the exact
// IEEE sqrt and division decide, so the neighbour set is the reference's.
//
// Wall densities: the reference writes them in place while neighbours read
// them (a race, delta_ns.cu:65,130,151).  Here k_nblist extrapolates every
// wall's (rho, p) first and publishes it in the packed shadows; k_boundary
// reads neighbours' densities from the shadows (new wall values) and a
// wall's own old density from ptc.rhop, and writes the new wall values to
// ptc.rhop at the end, when no reader is left.
#include "zsph_internal.cuh"

namespace zsph {
namespace {

// Plain coherent loads: some shadow fields are written while the kernel runs.
#define LDG(p) (*(p))

template <int GF> struct Stencil {
  static constexpr int W = 2 * GF + 1;  // rows per z-plane
  static constexpr int NR = W * W;      // governing rows (y = -GF..GF)
  __device__ static bool boundary_row(int r) { return (r % W) < 2 * GF; }  // y = -GF..GF-1
};

constexpr int kRowShift = 11;
constexpr int kOffMask = (1 << kRowShift) - 1;
constexpr uint8_t kOverflow = 255;

// Row ranges of particle i's stencil (delta_ns.cu:39-46), into shared memory
// columns rs/re (stride kPairBlock).
template <int GF>
__device__ __forceinline__ void load_rows(const KParams& kp, const zsph_tmp_t& t, int c, int* rs, int* re) {
  const zsph_gpu_param_t& p = kp.p;
#pragma unroll
  for (int r = 0; r < Stencil<GF>::NR; ++r) {
    const int z = r / Stencil<GF>::W - GF, y = r % Stencil<GF>::W - GF;
    const int cell = c + z * kp.XY + y * p.grid_xdim;
    const int cs = cell - GF, ce = cell + GF;
    int s = 0, e = 0;
    if (cs >= p.grid_hash_min && ce <= p.grid_hash_max) {
      // bounds a caller left stale are clamped to the particle range, so no
      // row can index outside the arrays (written bounds are always inside)
      s = max(LDG(&t.grid_start[cs]), 0);
      e = min(LDG(&t.grid_end[ce]), kp.n);
    }
    rs[r * kPairBlock] = s;
    re[r * kPairBlock] = e;
  }
}

__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

__device__ __forceinline__ bool interacts(const KParams& kp, float rr2) {
  if (rr2 > kp.r2hi) return false;
  if (rr2 < kp.r2lo) return true;
  return __fdiv_rn(__fsqrt_rn(rr2), kp.p.h) <= 2.0f;
}

// Calls f(j) for every interacting neighbour of i in visit order, from the
// list or, if the list overflowed, by re-filtering the stencil rows.
template <int GF, bool BOUNDARY_ONLY, class F>
__device__ __forceinline__ void visit(const KParams& kp, const Scratch& s, int i, float4 pi, const int* rs,
                                      const int* re, F&& f) {
  const int cnt = s.nb_cnt[i];
  if (cnt != kOverflow) {
    for (int k = 0; k < cnt; ++k) {
      const unsigned e = s.nb[(size_t)k * kp.n + i];
      const int r = (int)(e >> kRowShift);
      if (BOUNDARY_ONLY && !Stencil<GF>::boundary_row(r)) continue;
      f(rs[r * kPairBlock] + (int)(e & kOffMask));
    }
    return;
  }
  for (int r = 0; r < Stencil<GF>::NR; ++r) {
    if (BOUNDARY_ONLY && !Stencil<GF>::boundary_row(r)) continue;
    const int a = rs[r * kPairBlock], b = re[r * kPairBlock];
    for (int j = a; j < b; ++j) {
      if (j == i) continue;
      const float4 pj = LDG(&s.sh.pr[j]);
      if (interacts(kp, dist2(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z))) f(j);
    }
  }
}

// Filters the governing stencil of each particle into its neighbour list;
// with WALL, also extrapolates the (rho, p) of every non-fluid particle from
// its fluid neighbours in the boundary stencil (delta_ns.cu:61-85, :116-131)
// and publishes it in the shadows.
template <int GF, bool WALL>
__global__ void __launch_bounds__(kPairBlock) k_nblist(KParams kp, Scratch s, zsph_tmp_t t) {
  __shared__ int s_rs[Stencil<GF>::NR * kPairBlock];
  __shared__ int s_re[Stencil<GF>::NR * kPairBlock];
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  int* rs = s_rs + threadIdx.x;
  int* re = s_re + threadIdx.x;
  load_rows<GF>(kp, t, LDG(&t.hash[i]), rs, re);
  const float4 pi = s.sh.pr[i];
  int cnt = 0;
  bool ovf = false;
  int r = 0, j = rs[0], e = re[0], base = j;
  for (;;) {
    while (j >= e) {
      if (++r >= Stencil<GF>::NR) break;
      j = rs[r * kPairBlock];
      e = re[r * kPairBlock];
      base = j;
    }
    if (r >= Stencil<GF>::NR) break;
    if (j != i) {
      const float4 pj = LDG(&s.sh.pr[j]);
      if (interacts(kp, dist2(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z))) {
        const int off = j - base;
        if (cnt < kMaxNb && off <= kOffMask)
          s.nb[(size_t)cnt * kp.n + i] = (uint16_t)((r << kRowShift) | off);
        else
          ovf = true;
        ++cnt;
      }
    }
    ++j;
  }
  if (ovf) atomicOr(s.flags, ZSPH_FLAG_NB_OVERFLOW);
  s.nb_cnt[i] = ovf ? kOverflow : (uint8_t)cnt;
  if (!WALL) return;
  const int ti = s.sh.type[i];
  if (ti == 1) return;
  const zsph_gpu_param_t& p = kp.p;
  float rsum = 0.0f, wsum = 0.0f;
  visit<GF, true>(kp, s, i, pi, rs, re, [&](int jj) {
    if (LDG(&s.sh.type[jj]) != 1) return;
    const float4 pj = LDG(&s.sh.pr[jj]);
    const float dz = pi.z - pj.z;
    const float q = sqrtf(dist2(pi.x - pj.x, pi.y - pj.y, dz)) / p.h;
    const float a = 1.0f - q / 2.0f;
    float w = a * a * a;
    w = w * a;
    w *= (2.0f * q + 1.0f) * p.adh;
    const float p1 = LDG(&s.sh.vp[jj]).w;
    rsum += (p1 - pj.w * ((0.0f - p.g) * dz)) * w;
    wsum += w;
  });
  if (fabsf(wsum) > 1e-8f) rsum = rsum / wsum; else rsum = 0.0f;
  if (rsum < 0.0f) rsum = 0.0f;
  s.sh.pr[i].w = rsum / p.cs2 + p.rho0;
  s.sh.vp[i].w = rsum;
}

// cuda_boundary_ns main part (delta_ns.cu:35-174): renormalisation matrix and
// div(v) over the boundary stencil, cofactor inverse, renormalised grad(rho).
template <int GF>
__global__ void __launch_bounds__(kPairBlock) k_boundary(KParams kp, Scratch s, zsph_ptc_t ptc, zsph_tmp_t t) {
  __shared__ int s_rs[Stencil<GF>::NR * kPairBlock];
  __shared__ int s_re[Stencil<GF>::NR * kPairBlock];
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  int* rs = s_rs + threadIdx.x;
  int* re = s_re + threadIdx.x;
  load_rows<GF>(kp, t, LDG(&t.hash[i]), rs, re);
  const zsph_gpu_param_t& p = kp.p;
  const float4 pi = s.sh.pr[i];
  const float4 vi = s.sh.vp[i];
  const int ti = s.sh.type[i];
  const float rho_self = reinterpret_cast<const float2*>(ptc.rhop)[i].x;  // old own density
  float Lxx = 0.f, Lxy = 0.f, Lxz = 0.f, Lyy = 0.f, Lyz = 0.f, Lzz = 0.f, divv = 0.f;
  visit<GF, true>(kp, s, i, pi, rs, re, [&](int j) {
    const float4 pj = LDG(&s.sh.pr[j]);
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float q = sqrtf(dist2(dx, dy, dz)) / p.h;
    const float a = 1.0f - q / 2.0f;
    float fr = a * a * a;
    fr *= -5.0f * p.adh / p.h2;
    const float tl = fr * p.m / pj.w;
    Lxx -= dx * dx * tl; Lxy -= dx * dy * tl; Lxz -= dx * dz * tl;
    Lyy -= dy * dy * tl; Lyz -= dy * dz * tl; Lzz -= dz * dz * tl;
    if (ti == 1 && LDG(&s.sh.type[j]) == 1) {
      const float4 vj = LDG(&s.sh.vp[j]);
      const float dvdx = (vi.x - vj.x) * dx + (vi.y - vj.y) * dy + (vi.z - vj.z) * dz;
      divv -= fr * dvdx * p.m / pj.w;
    }
  });
  // delta_ns.cu:99-114 (L is symmetric: L1 = (xx,xy,xz), L2 = (xy,yy,yz), L3 = (xz,yz,zz))
  const float det = Lxx * Lyy * Lzz + Lxy * Lyz * Lxz + Lxz * Lxy * Lyz - Lxz * Lyy * Lxz - Lxx * Lyz * Lyz -
                    Lxy * Lxy * Lzz;
  float M00, M01, M02, M10, M11, M12, M20, M21, M22;
  if (fabsf(det) > 1.8e-8f) {
    M00 = (Lyy * Lzz - Lyz * Lyz) / det;
    M01 = -1.0f * (Lxy * Lzz - Lyz * Lxz) / det;
    M02 = (Lxy * Lyz - Lyy * Lxz) / det;
    M10 = -1.0f * (Lxy * Lzz - Lxz * Lyz) / det;
    M11 = (Lxx * Lzz - Lxz * Lxz) / det;
    M12 = -1.0f * (Lxx * Lyz - Lxy * Lxz) / det;
    M20 = (Lxy * Lyz - Lxz * Lyy) / det;
    M21 = -1.0f * (Lxx * Lyz - Lxz * Lxy) / det;
    M22 = (Lxx * Lyy - Lxy * Lxy) / det;
  } else {
    M00 = 1.f; M01 = 0.f; M02 = 0.f;
    M10 = 0.f; M11 = 1.f; M12 = 0.f;
    M20 = 0.f; M21 = 0.f; M22 = 1.f;
  }
  float gx = 0.f, gy = 0.f, gz = 0.f;
  visit<GF, true>(kp, s, i, pi, rs, re, [&](int j) {
    const float4 pj = LDG(&s.sh.pr[j]);
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float q = sqrtf(dist2(dx, dy, dz)) / p.h;
    const float a = 1.0f - q / 2.0f;
    float fr = -5.0f * p.adh * a * a * a / p.h2;
    fr *= (pj.w - rho_self) * p.m / pj.w;
    gx += (M00 * dx + M01 * dy + M02 * dz) * fr;
    gy += (M10 * dx + M11 * dy + M12 * dz) * fr;
    gz += (M20 * dx + M21 * dy + M22 * dz) * fr;
  });
  reinterpret_cast<float4*>(t.dofv_grandrho)[i] = make_float4(gx, gy, gz, divv);
  if (ti != 1) reinterpret_cast<float2*>(ptc.rhop)[i] = make_float2(pi.w, vi.w);
}

// time_int.cu:3-48 / :50-92 for one fluid particle, writing into `out`
// (which may alias `in`).  Non-fluid particles are copied unchanged.
template <int MODE>
__device__ __forceinline__ void integrate_one(const KParams& kp, const zsph_ptc_t& in, const zsph_ptc_t& out,
                                              int i, float4 acc) {
  const zsph_gpu_param_t& p = kp.p;
  const float3 pos = make_float3(in.pos[3 * i], in.pos[3 * i + 1], in.pos[3 * i + 2]);
  const float3 vel = make_float3(in.vel[3 * i], in.vel[3 * i + 1], in.vel[3 * i + 2]);
  const float2 rp = reinterpret_cast<const float2*>(in.rhop)[i];
  const int type = in.type[i];
  const bool alias = in.pos == out.pos;
  float3 tp = make_float3(in.tmp_pos[3 * i], in.tmp_pos[3 * i + 1], in.tmp_pos[3 * i + 2]);
  float3 tv = make_float3(in.tmp_vel[3 * i], in.tmp_vel[3 * i + 1], in.tmp_vel[3 * i + 2]);
  float2 trp = reinterpret_cast<const float2*>(in.tmp_rhop)[i];
  float3 np = pos, nv = vel;
  float2 nrp = rp;
  if (type == 1) {
    if (MODE == 1) {  // prediction
      tp = pos; tv = vel; trp = rp;
      np.x += vel.x * p.half_dt; np.y += vel.y * p.half_dt; np.z += vel.z * p.half_dt;
      nv.x += acc.x * p.half_dt; nv.y += acc.y * p.half_dt; nv.z += acc.z * p.half_dt;
      nrp.x += acc.w * p.half_dt;
    } else {  // correction
      np.x = tp.x + vel.x * p.half_dt * 2.0f;
      np.y = tp.y + vel.y * p.half_dt * 2.0f;
      np.z = tp.z + vel.z * p.half_dt * 2.0f;
      nv.x = tv.x + acc.x * p.half_dt * 2.0f;
      nv.y = tv.y + acc.y * p.half_dt * 2.0f;
      nv.z = tv.z + acc.z * p.half_dt * 2.0f;
      nrp.x = trp.x + acc.w * p.half_dt * 2.0f;
    }
    if (nrp.x < p.rho0) nrp.x = p.rho0;
    nrp.y = p.cs2 * (nrp.x - p.rho0);
  } else if (alias) {
    return;
  }
  out.pos[3 * i] = np.x; out.pos[3 * i + 1] = np.y; out.pos[3 * i + 2] = np.z;
  out.vel[3 * i] = nv.x; out.vel[3 * i + 1] = nv.y; out.vel[3 * i + 2] = nv.z;
  reinterpret_cast<float2*>(out.rhop)[i] = nrp;
  if (!alias || (MODE == 1 && type == 1)) {
    out.tmp_pos[3 * i] = tp.x; out.tmp_pos[3 * i + 1] = tp.y; out.tmp_pos[3 * i + 2] = tp.z;
    out.tmp_vel[3 * i] = tv.x; out.tmp_vel[3 * i + 1] = tv.y; out.tmp_vel[3 * i + 2] = tv.z;
    reinterpret_cast<float2*>(out.tmp_rhop)[i] = trp;
  }
  if (!alias) {
    out.type[i] = type;
    out.table[i] = in.table[i];
  }
}

// cuda_govering_ns (delta_ns.cu:179-267); MODE 1/2 fuses the prediction /
// correction of the same particle, written into `out` (a different buffer,
// so neighbours still read the unintegrated state).
template <int GF, int MODE>
__global__ void __launch_bounds__(kPairBlock) k_governing(KParams kp, Scratch s, zsph_ptc_t ptc, zsph_tmp_t t,
                                                          zsph_ptc_t out) {
  __shared__ int s_rs[Stencil<GF>::NR * kPairBlock];
  __shared__ int s_re[Stencil<GF>::NR * kPairBlock];
  const int i = blockIdx.x * kPairBlock + threadIdx.x;
  if (i >= kp.n) return;
  int* rs = s_rs + threadIdx.x;
  int* re = s_re + threadIdx.x;
  load_rows<GF>(kp, t, LDG(&t.hash[i]), rs, re);
  const zsph_gpu_param_t& p = kp.p;
  const float4 pi = s.sh.pr[i];
  const float4 vi = s.sh.vp[i];
  const int ti = s.sh.type[i];
  const float r0 = pi.w, p0 = vi.w;
  float4 g0 = reinterpret_cast<const float4*>(t.dofv_grandrho)[i];
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  visit<GF, false>(kp, s, i, pi, rs, re, [&](int j) {
    const float4 pj = LDG(&s.sh.pr[j]);
    const float4 vj = LDG(&s.sh.vp[j]);
    const float4 g1 = LDG(reinterpret_cast<const float4*>(t.dofv_grandrho) + j);
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float rr2 = dist2(dx, dy, dz);
    const float dvdx = (vi.x - vj.x) * dx + (vi.y - vj.y) * dy + (vi.z - vj.z) * dz;
    const float q = sqrtf(rr2) / p.h;
    const float a = 1.0f - q / 2.0f;
    const float fr = -5.0f * p.adh * a * a * a / p.h2;
    const float r1 = pj.w, p1 = vj.w;
    g0.x *= dx;  // order-dependent recurrence, delta_ns.cu:244-245
    g0.x += g1.x * dx + (g0.y + g1.y) * dy + (g0.z + g1.z) * dz;
    acc.w += r0 * dvdx * fr * p.m / r1;
    float vt = -(p0 + p1) * p.m * fr / (r0 * r1);
    if (ti == 1 && LDG(&s.sh.type[j]) == 1) {
      acc.w += p.delta_h_cs * fr * ((r0 - r1) * 2.0f * rr2 / (rr2 + p.eta2) - g0.x) * p.m / r1;
      vt += p.h_cs_rho_m * fr * (g0.w + g1.w + p.alpha * dvdx / (rr2 + p.eta2)) / (r0 * r1);
    }
    acc.x += vt * dx;
    acc.y += vt * dy;
    acc.z += vt * dz;
  });
  acc.z += p.g;  // delta_ns.cu:264
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

template <int GF>
cudaError_t boundary_gf(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                        cudaStream_t st, Prof* pf) {
  const int nb = (kp.n + kPairBlock - 1) / kPairBlock;
  k_nblist<GF, true><<<nb, kPairBlock, 0, st>>>(kp, s, t);
  mark(pf, "nblist_wall", st);
  k_boundary<GF><<<nb, kPairBlock, 0, st>>>(kp, s, ptc, t);
  mark(pf, "boundary", st);
  return cudaGetLastError();
}

template <int GF>
cudaError_t governing_gf(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t, int mode,
                         const zsph_ptc_t& out, cudaStream_t st, Prof* pf) {
  const int nb = (kp.n + kPairBlock - 1) / kPairBlock;
  if (mode == 0) k_governing<GF, 0><<<nb, kPairBlock, 0, st>>>(kp, s, ptc, t, out);
  if (mode == 1) k_governing<GF, 1><<<nb, kPairBlock, 0, st>>>(kp, s, ptc, t, out);
  if (mode == 2) k_governing<GF, 2><<<nb, kPairBlock, 0, st>>>(kp, s, ptc, t, out);
  mark(pf, "governing", st);
  return cudaGetLastError();
}

template <int GF>
cudaError_t nblist_gf(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, cudaStream_t st) {
  const int nb = (kp.n + kPairBlock - 1) / kPairBlock;
  k_nblist<GF, false><<<nb, kPairBlock, 0, st>>>(kp, s, t);
  return cudaGetLastError();
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
  for (int k = 0; k < cnt; ++k) b += Stencil<GF>::boundary_row((int)(s.nb[(size_t)k * kp.n + i] >> kRowShift));
  if (nb_boundary) nb_boundary[i] = b;
  if (nb_governing) nb_governing[i] = cnt;
}

}  // namespace

cudaError_t launch_boundary(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                            cudaStream_t st, Prof* pf) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor == 1) return boundary_gf<1>(kp, s, ptc, t, st, pf);
  if (kp.p.grid_factor == 2) return boundary_gf<2>(kp, s, ptc, t, st, pf);
  return cudaErrorInvalidValue;
}

cudaError_t launch_nblist(const KParams& kp, const Scratch& s, const zsph_tmp_t& t, cudaStream_t st) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor == 1) return nblist_gf<1>(kp, s, t, st);
  if (kp.p.grid_factor == 2) return nblist_gf<2>(kp, s, t, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_governing(const KParams& kp, const Scratch& s, const zsph_ptc_t& ptc, const zsph_tmp_t& t,
                             int mode, const zsph_ptc_t& out, cudaStream_t st, Prof* pf) {
  if (kp.n == 0) return cudaSuccess;
  if (kp.p.grid_factor == 1) return governing_gf<1>(kp, s, ptc, t, mode, out, st, pf);
  if (kp.p.grid_factor == 2) return governing_gf<2>(kp, s, ptc, t, mode, out, st, pf);
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
