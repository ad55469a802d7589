// ZSPH delta-SPH step -- FP64 GPU CHECKER (test infrastructure only).
//
// The T = double instance of the CPU oracle (zsph_oracle.hpp), run on the
// GPU so that full-size cases (millions of particles, thousands of steps)
// can be compared against an FP64 run of the same equations.  Each kernel is
// the oracle function of the same name with one thread per particle; the
// arithmetic and the neighbour visit order are the oracle's (the file is
// compiled with -fmad=false, as the oracle is with -ffp-contract=off), and
// the body's force and torque are summed over the body particles in sorted
// order, as the oracle's loop does, so the checker agrees with the CPU FP64
// oracle bit for bit (tests/test_gpu_precise.py pins that on a small case).
// Wall densities follow the oracle's WALLS_FIRST order.  Never linked into
// the product library.
#include <cuda_runtime.h>
#include <thrust/copy.h>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/sort.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "zsph_oracle.hpp"

using namespace zsph_oracle;

namespace {

struct DS {  // one particle buffer (reference layout, FP64)
  double *pos, *vel, *rhop, *tpos, *tvel, *trhop;
  int *type, *table;
};

struct DT {  // scratch of the step
  double *acc, *dg, *rho_new, *p_new, *fv, *fvc;
  int *index, *hash, *gs, *ge, *flag;
};

inline int blocks(int n) { return (n + 255) / 256; }

// single_gpu_sph_src/lib/hash.cu:3-26 (oracle hash<double>)
__global__ void g_hash(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num) return;
  const double gx = (double)p.grid_xmin, gy = (double)p.grid_ymin, gz = (double)p.grid_zmin;
  const double gsz = (double)p.grid_size;
  const int hx = (int)floor((s.pos[3 * i] - gx) / gsz);  // cvt.rzi: truncation, saturation, NaN -> 0
  const int hy = (int)floor((s.pos[3 * i + 1] - gy) / gsz);
  const int hz = (int)floor((s.pos[3 * i + 2] - gz) / gsz);
  const unsigned X = (unsigned)p.grid_xdim, Y = (unsigned)p.grid_ydim;
  int h = (int)((unsigned)hz * X * Y + (unsigned)hy * X + (unsigned)hx);
  if (h < p.grid_hash_min || h > p.grid_hash_max) {
    s.type[i] = 100;
    s.pos[3 * i] = gx; s.pos[3 * i + 1] = gy; s.pos[3 * i + 2] = gz;
    s.vel[3 * i] = 0; s.vel[3 * i + 1] = 0; s.vel[3 * i + 2] = 0;
    s.rhop[2 * i] = (double)p.rho0; s.rhop[2 * i + 1] = 0;
    h = 0;
  }
  t.hash[i] = h;
  t.index[i] = i;
}

// single_gpu_sph_src/lib/sort.cu:30-60: cell bounds with the reference's
// branch order; each thread writes only the cells of its own boundary.
__global__ void g_bounds(Params p, DT t) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = p.ptc_num;
  if (tid >= n) return;
  const int h = t.hash[tid];
  const int prev = tid > 0 ? t.hash[tid - 1] : h;
  if (h != prev) {
    t.gs[h] = tid;
    t.ge[prev] = tid;
    for (int c = prev + 1; c < h; ++c) { t.gs[c] = tid; t.ge[c] = tid; }
  } else if (tid == 0) {
    t.gs[h] = tid;
    for (int c = 0; c < h; ++c) { t.ge[c] = tid; t.gs[c] = tid; }
  } else if (tid == n - 1) {
    t.ge[h] = tid;
    for (int c = h + 1; c <= p.grid_hash_max; ++c) { t.ge[c] = tid; t.gs[c] = tid; }
  }
}

// single_gpu_sph_src/lib/sort.cu:62-82
__global__ void g_gather(Params p, DS o, DS w, DT t) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= p.ptc_num) return;
  const int oi = t.index[tid];
  for (int k = 0; k < 3; ++k) {
    w.pos[3 * tid + k] = o.pos[3 * oi + k];
    w.vel[3 * tid + k] = o.vel[3 * oi + k];
    w.tpos[3 * tid + k] = o.tpos[3 * oi + k];
    w.tvel[3 * tid + k] = o.tvel[3 * oi + k];
  }
  for (int k = 0; k < 2; ++k) {
    w.rhop[2 * tid + k] = o.rhop[2 * oi + k];
    w.trhop[2 * tid + k] = o.trhop[2 * oi + k];
  }
  w.type[tid] = o.type[oi];
  w.table[tid] = o.table[oi] + oi - tid;
}

// the oracle's for_each_candidate (delta_ns.cu:35-48, :204-217)
template <class F>
__device__ __forceinline__ void cand(const Params& p, const DT& t, int i, int ylast, F&& f) {
  const int gf = p.grid_factor;
  for (int z = -gf; z <= gf; ++z)
    for (int y = -gf; y <= ylast; ++y) {
      int cs = t.hash[i] + z * p.grid_xdim * p.grid_ydim + y * p.grid_xdim;
      int ce = cs + gf;
      cs = cs - gf;
      if (cs >= p.grid_hash_min && ce <= p.grid_hash_max) {
        const int a = t.gs[cs], b = t.ge[ce];
        for (int j = a; j < b; ++j)
          if (j != i) f(j);
      }
    }
}

__device__ __forceinline__ double rr2_of(double x, double y, double z) { return x * x + y * y + z * z; }

// delta_ns.cu:61-85, :116-131 (oracle wall_pressure<double>)
__global__ void g_wall_pressure(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num) return;
  t.rho_new[i] = s.rhop[2 * i];
  t.p_new[i] = s.rhop[2 * i + 1];
  if (s.type[i] == 1) return;
  const double h = p.h, adh = p.adh, g = p.g, cs2 = p.cs2, rho0 = p.rho0;
  double rsum = 0, wsum = 0;
  const double px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
  cand(p, t, i, p.grid_factor - 1, [&](int j) {
    const double dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
    const double q = sqrt(rr2_of(dx, dy, dz)) / h;
    if (q <= 2.0) {
      const double a = 1.0 - q / 2.0;
      double w = a * a * a;
      w = w * a;
      w *= (2.0 * q + 1.0) * adh;
      if (s.type[j] == 1) {
        const double rj = s.rhop[2 * j], pj = s.rhop[2 * j + 1];
        rsum += (pj - rj * (0.0 * dx + 0.0 * dy + (0.0 - g) * dz)) * w;
        wsum += w;
      }
    }
  });
  if (fabs(wsum) > (double)1e-8f) rsum = rsum / wsum; else rsum = 0;
  if (rsum < 0) rsum = 0;
  t.p_new[i] = rsum;
  t.rho_new[i] = rsum / cs2 + rho0;
}

// delta_ns.cu:5-177 (oracle boundary<double>, WALLS_FIRST)
__global__ void g_boundary(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num) return;
  const double h = p.h, adh = p.adh, h2 = p.h2, m = p.m;
  double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double divv = 0;
  const double px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
  const double vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
  const double rho0_i = s.rhop[2 * i];
  const int ti = s.type[i];
  cand(p, t, i, p.grid_factor - 1, [&](int j) {
    const double d[3] = {px - s.pos[3 * j], py - s.pos[3 * j + 1], pz - s.pos[3 * j + 2]};
    const double dvx = vx - s.vel[3 * j], dvy = vy - s.vel[3 * j + 1], dvz = vz - s.vel[3 * j + 2];
    const double rr2 = rr2_of(d[0], d[1], d[2]);
    const double dvdx = dvx * d[0] + dvy * d[1] + dvz * d[2];
    const double q = sqrt(rr2) / h;
    if (q <= 2.0) {
      const double a = 1.0 - q / 2.0;
      double fr = a * a * a;
      fr *= -5.0 * adh / h2;
      const double rj = t.rho_new[j];
      const double tl = fr * m / rj;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) L[r][c] -= d[r] * d[c] * tl;
      if (ti == 1 && s.type[j] == 1) divv -= fr * dvdx * m / rj;
    }
  });
  const double det = L[0][0] * L[1][1] * L[2][2] + L[0][1] * L[1][2] * L[2][0] + L[0][2] * L[1][0] * L[2][1] -
                     L[0][2] * L[1][1] * L[2][0] - L[0][0] * L[1][2] * L[2][1] - L[0][1] * L[1][0] * L[2][2];
  double M[3][3];
  if (fabs(det) > (double)1.8e-8f) {
    M[0][0] = (L[1][1] * L[2][2] - L[1][2] * L[2][1]) / det;
    M[0][1] = -1.0 * (L[1][0] * L[2][2] - L[1][2] * L[2][0]) / det;
    M[0][2] = (L[1][0] * L[2][1] - L[1][1] * L[2][0]) / det;
    M[1][0] = -1.0 * (L[0][1] * L[2][2] - L[0][2] * L[2][1]) / det;
    M[1][1] = (L[0][0] * L[2][2] - L[0][2] * L[2][0]) / det;
    M[1][2] = -1.0 * (L[0][0] * L[2][1] - L[0][1] * L[2][0]) / det;
    M[2][0] = (L[0][1] * L[1][2] - L[0][2] * L[1][1]) / det;
    M[2][1] = -1.0 * (L[0][0] * L[1][2] - L[0][2] * L[1][0]) / det;
    M[2][2] = (L[0][0] * L[1][1] - L[0][1] * L[1][0]) / det;
  } else {
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[r][c] = (r == c) ? 1.0 : 0.0;
  }
  double gr[3] = {0, 0, 0};
  cand(p, t, i, p.grid_factor - 1, [&](int j) {
    const double d[3] = {px - s.pos[3 * j], py - s.pos[3 * j + 1], pz - s.pos[3 * j + 2]};
    const double q = sqrt(rr2_of(d[0], d[1], d[2])) / h;
    if (q <= 2.0) {
      const double a = 1.0 - q / 2.0;
      double fr = -5.0 * adh * a * a * a / h2;
      const double rj = t.rho_new[j];
      fr *= (rj - rho0_i) * m / rj;
      for (int r = 0; r < 3; ++r) gr[r] += (M[r][0] * d[0] + M[r][1] * d[1] + M[r][2] * d[2]) * fr;
    }
  });
  t.dg[4 * i] = gr[0];
  t.dg[4 * i + 1] = gr[1];
  t.dg[4 * i + 2] = gr[2];
  t.dg[4 * i + 3] = divv;
}

// delta_ns.cu:117-131: the new wall values, written once no reader is left
__global__ void g_wall_write(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num || s.type[i] == 1) return;
  s.rhop[2 * i] = t.rho_new[i];
  s.rhop[2 * i + 1] = t.p_new[i];
}

// delta_ns.cu:179-267 (oracle governing<double>)
__global__ void g_governing(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num) return;
  const double h = p.h, adh = p.adh, h2 = p.h2, m = p.m, eta2 = p.eta2;
  const double dhc = p.delta_h_cs, hcrm = p.h_cs_rho_m, alpha = p.alpha, g = p.g;
  double acc[4] = {0, 0, 0, 0};
  const double px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
  const double vx = s.vel[3 * i], vy = s.vel[3 * i + 1], vz = s.vel[3 * i + 2];
  const double r0 = s.rhop[2 * i], p0 = s.rhop[2 * i + 1];
  const int ti = s.type[i];
  double G0[4] = {t.dg[4 * i], t.dg[4 * i + 1], t.dg[4 * i + 2], t.dg[4 * i + 3]};
  cand(p, t, i, p.grid_factor, [&](int j) {
    const double dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
    const double dvx = vx - s.vel[3 * j], dvy = vy - s.vel[3 * j + 1], dvz = vz - s.vel[3 * j + 2];
    const double rr2 = rr2_of(dx, dy, dz);
    const double dvdx = dvx * dx + dvy * dy + dvz * dz;
    const double q = sqrt(rr2) / h;
    if (q <= 2.0) {
      const double a = 1.0 - q / 2.0;
      const double fr = -5.0 * adh * a * a * a / h2;
      const double r1 = s.rhop[2 * j], p1 = s.rhop[2 * j + 1];
      const double* G1 = &t.dg[4 * j];
      G0[0] *= dx;  // delta_ns.cu:244-245
      G0[0] += G1[0] * dx + (G0[1] + G1[1]) * dy + (G0[2] + G1[2]) * dz;
      acc[3] += r0 * dvdx * fr * m / r1;
      double vt = -(p0 + p1) * m * fr / (r0 * r1);
      if (ti == 1 && s.type[j] == 1) {
        acc[3] += dhc * fr * ((r0 - r1) * 2.0 * rr2 / (rr2 + eta2) - G0[0]) * m / r1;
        vt += hcrm * fr * (G0[3] + G1[3] + alpha * dvdx / (rr2 + eta2)) / (r0 * r1);
      }
      acc[0] += vt * dx;
      acc[1] += vt * dy;
      acc[2] += vt * dz;
    }
  });
  acc[2] += g;
  for (int k = 0; k < 4; ++k) t.acc[4 * i + k] = acc[k];
}

// time_int.cu:3-48 (oracle prediction<double>)
__global__ void g_prediction(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num || s.type[i] != 1) return;
  const double hdt = p.half_dt, rho0 = p.rho0, cs2 = p.cs2;
  for (int k = 0; k < 3; ++k) {
    s.tpos[3 * i + k] = s.pos[3 * i + k];
    s.tvel[3 * i + k] = s.vel[3 * i + k];
  }
  s.trhop[2 * i] = s.rhop[2 * i];
  s.trhop[2 * i + 1] = s.rhop[2 * i + 1];
  for (int k = 0; k < 3; ++k) s.pos[3 * i + k] += s.vel[3 * i + k] * hdt;
  for (int k = 0; k < 3; ++k) s.vel[3 * i + k] += t.acc[4 * i + k] * hdt;
  double r = s.rhop[2 * i] + t.acc[4 * i + 3] * hdt;
  if (r < rho0) r = rho0;
  s.rhop[2 * i] = r;
  s.rhop[2 * i + 1] = cs2 * (r - rho0);
}

// time_int.cu:50-92 (oracle correction<double>)
__global__ void g_correction(Params p, DS s, DT t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num || s.type[i] != 1) return;
  const double hdt = p.half_dt, rho0 = p.rho0, cs2 = p.cs2;
  double v[3];
  for (int k = 0; k < 3; ++k) v[k] = s.vel[3 * i + k];
  for (int k = 0; k < 3; ++k) s.pos[3 * i + k] = s.tpos[3 * i + k] + v[k] * hdt * 2.0;
  for (int k = 0; k < 3; ++k) s.vel[3 * i + k] = s.tvel[3 * i + k] + t.acc[4 * i + k] * hdt * 2.0;
  double r = s.trhop[2 * i] + t.acc[4 * i + 3] * hdt * 2.0;
  if (r < rho0) r = rho0;
  s.rhop[2 * i] = r;
  s.rhop[2 * i + 1] = cs2 * (r - rho0);
}

// oracle rigid_force<double>, per body particle: its force m f and torque
// r x (m f) about the centre of mass; flag marks the body particles
__global__ void g_rigid_force(Params p, DS s, DT t, int first, int count, double cx, double cy, double cz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num) return;
  const int k = s.table[i] + i - first;
  t.flag[i] = 0;
  if (s.type[i] != 2 || k < 0 || k >= count) return;
  t.flag[i] = 1;
  const double h = p.h, adh = p.adh, h2 = p.h2, m = p.m;
  const double px = s.pos[3 * i], py = s.pos[3 * i + 1], pz = s.pos[3 * i + 2];
  const double r0 = s.rhop[2 * i], p0 = s.rhop[2 * i + 1];
  double f[3] = {0, 0, 0};
  cand(p, t, i, p.grid_factor, [&](int j) {
    if (s.type[j] != 1) return;
    const double dx = px - s.pos[3 * j], dy = py - s.pos[3 * j + 1], dz = pz - s.pos[3 * j + 2];
    const double q = sqrt(rr2_of(dx, dy, dz)) / h;
    if (!(q <= 2.0)) return;
    const double a = 1.0 - q / 2.0;
    const double fr = -5.0 * adh * a * a * a / h2;
    const double vt = -(p0 + s.rhop[2 * j + 1]) * m * fr / (r0 * s.rhop[2 * j]);
    f[0] += vt * dx;
    f[1] += vt * dy;
    f[2] += vt * dz;
  });
  const double fv[3] = {m * f[0], m * f[1], m * f[2]};
  const double r[3] = {px - cx, py - cy, pz - cz};
  double* o = t.fv + 6 * (size_t)i;
  o[0] = fv[0]; o[1] = fv[1]; o[2] = fv[2];
  o[3] = r[1] * fv[2] - r[2] * fv[1];
  o[4] = r[2] * fv[0] - r[0] * fv[2];
  o[5] = r[0] * fv[1] - r[1] * fv[0];
}

// the oracle's sum over body particles in sorted order (one thread)
__global__ void g_rigid_sum(const double* fvc, int count, double* out) {
  double F[6] = {0, 0, 0, 0, 0, 0};
  for (int e = 0; e < count; ++e)
    for (int a = 0; a < 6; ++a) F[a] += fvc[6 * e + a];
  for (int a = 0; a < 6; ++a) out[a] = F[a];
}

struct Six {  // force and torque of one body particle
  double a[6];
};
struct IsSet {
  __host__ __device__ bool operator()(int f) const { return f != 0; }
};

struct Pose {
  double R[9], x[3], v[3], w[3];
};

// oracle rigid_place<double>
__global__ void g_rigid_place(Params p, DS s, int first, int count, const double* r0, Pose b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.ptc_num) return;
  const int k = s.table[i] + i - first;
  if (s.type[i] != 2 || k < 0 || k >= count) return;
  const double* q = r0 + 3 * (size_t)k;
  double r[3];
  for (int a = 0; a < 3; ++a) r[a] = b.R[3 * a] * q[0] + b.R[3 * a + 1] * q[1] + b.R[3 * a + 2] * q[2];
  const double w[3] = {b.w[1] * r[2] - b.w[2] * r[1], b.w[2] * r[0] - b.w[0] * r[2], b.w[0] * r[1] - b.w[1] * r[0]};
  for (int a = 0; a < 3; ++a) {
    s.pos[3 * i + a] = b.x[a] + r[a];
    s.vel[3 * i + a] = b.v[a] + w[a];
  }
}

struct Checker {
  Params p{};
  int n = 0, G = 0;
  DS o{}, w{};
  DT t{};
  bool rigid = false;
  Rigid b{};
  double* r0 = nullptr;    // [count][3] on the device
  double* rsum = nullptr;  // [6]
  std::string err;
};

bool ck(Checker* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

template <class T> cudaError_t dmalloc(T*& ptr, size_t count) {
  return cudaMalloc(reinterpret_cast<void**>(&ptr), (count ? count : 1) * sizeof(T));
}

cudaError_t alloc_state(DS& s, int n) {
  cudaError_t e = cudaSuccess;
  double** f3[] = {&s.pos, &s.vel, &s.tpos, &s.tvel};
  for (double** q : f3) if (!e) e = dmalloc(*q, 3 * (size_t)n);
  if (!e) e = dmalloc(s.rhop, 2 * (size_t)n);
  if (!e) e = dmalloc(s.trhop, 2 * (size_t)n);
  if (!e) e = dmalloc(s.type, n);
  if (!e) e = dmalloc(s.table, n);
  return e;
}

void free_state(DS& s) {
  void* q[] = {s.pos, s.vel, s.tpos, s.tvel, s.rhop, s.trhop, s.type, s.table};
  for (void* x : q) if (x) cudaFree(x);
}

// oracle search + boundary + governing of one sub-step (sorts `from` into `to`)
cudaError_t substep_pairs(Checker* c, DS& from, DS& to) {
  const Params& p = c->p;
  const int nb = blocks(c->n);
  g_hash<<<nb, 256>>>(p, from, c->t);
  thrust::stable_sort_by_key(thrust::device, thrust::device_pointer_cast(c->t.hash),
                             thrust::device_pointer_cast(c->t.hash + c->n), thrust::device_pointer_cast(c->t.index));
  g_bounds<<<nb, 256>>>(p, c->t);
  g_gather<<<nb, 256>>>(p, from, to, c->t);
  g_wall_pressure<<<nb, 256>>>(p, to, c->t);
  g_boundary<<<nb, 256>>>(p, to, c->t);
  g_wall_write<<<nb, 256>>>(p, to, c->t);
  g_governing<<<nb, 256>>>(p, to, c->t);
  return cudaGetLastError();
}

// force and torque on the body (oracle rigid_force), its update on the host
// (oracle rigid_advance) and the placement of its particles (rigid_place)
cudaError_t rigid_substep(Checker* c, DS& s, int mode) {
  const Params& p = c->p;
  const int nb = blocks(c->n);
  g_rigid_force<<<nb, 256>>>(p, s, c->t, c->b.first, c->b.count, c->b.x[0], c->b.x[1], c->b.x[2]);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  // compact the body particles' six sums in sorted order, then sum them
  Six* src = reinterpret_cast<Six*>(c->t.fv);
  Six* dst = reinterpret_cast<Six*>(c->t.fvc);
  const int m = (int)(thrust::copy_if(thrust::device, thrust::device_pointer_cast(src),
                                      thrust::device_pointer_cast(src + c->n),
                                      thrust::device_pointer_cast(c->t.flag), thrust::device_pointer_cast(dst),
                                      IsSet()) -
                      thrust::device_pointer_cast(dst));
  g_rigid_sum<<<1, 1>>>(c->t.fvc, m, c->rsum);
  double F[6];
  e = cudaMemcpy(F, c->rsum, sizeof F, cudaMemcpyDeviceToHost);
  if (e) return e;
  for (int a = 0; a < 3; ++a) {
    c->b.F[a] = F[a];
    c->b.T[a] = F[3 + a];
  }
  rigid_advance(c->b, mode, (double)p.half_dt);
  return cudaSuccess;
}

cudaError_t place(Checker* c, DS& s) {
  Pose ps;
  rig_rot(c->b.q, ps.R);
  for (int a = 0; a < 3; ++a) {
    ps.x[a] = c->b.x[a];
    ps.v[a] = c->b.v[a];
    ps.w[a] = c->b.w[a];
  }
  g_rigid_place<<<blocks(c->n), 256>>>(c->p, s, c->b.first, c->b.count, c->r0, ps);
  return cudaGetLastError();
}

// oracle step<double> / step_rigid<double>
cudaError_t one_step(Checker* c) {
  const int nb = blocks(c->n);
  cudaError_t e = substep_pairs(c, c->o, c->w);
  if (!e && c->rigid) e = rigid_substep(c, c->w, 1);
  if (!e) g_prediction<<<nb, 256>>>(c->p, c->w, c->t);
  if (!e && c->rigid) e = place(c, c->w);
  if (!e) e = substep_pairs(c, c->w, c->o);
  if (!e && c->rigid) e = rigid_substep(c, c->o, 2);
  if (!e) g_correction<<<nb, 256>>>(c->p, c->o, c->t);
  if (!e && c->rigid) e = place(c, c->o);
  if (!e) e = cudaGetLastError();
  return e;
}

}  // namespace

extern "C" {

const char* gor_error(void* h) { return h ? static_cast<Checker*>(h)->err.c_str() : "null checker"; }

// Uploads an FP64 state in the reference layout (old buffer) with the
// oracle's derived constants.
void* gor_create(const Params* p, const double* pos, const double* vel, const double* rhop, const double* tpos,
                 const double* tvel, const double* trhop, const int* type, const int* table) {
  Checker* c = new Checker();
  c->p = *p;
  c->n = p->ptc_num;
  c->G = p->grid_num;
  const size_t n = (size_t)c->n;
  cudaError_t e = alloc_state(c->o, c->n);
  if (!e) e = alloc_state(c->w, c->n);
  DT& t = c->t;
  if (!e) e = dmalloc(t.acc, 4 * n);
  if (!e) e = dmalloc(t.dg, 4 * n);
  if (!e) e = dmalloc(t.rho_new, n);
  if (!e) e = dmalloc(t.p_new, n);
  if (!e) e = dmalloc(t.fv, 6 * n);
  if (!e) e = dmalloc(t.fvc, 6 * n);
  if (!e) e = dmalloc(t.index, n);
  if (!e) e = dmalloc(t.hash, n);
  if (!e) e = dmalloc(t.flag, n);
  if (!e) e = dmalloc(t.gs, (size_t)c->G);
  if (!e) e = dmalloc(t.ge, (size_t)c->G);
  if (!e) e = dmalloc(c->rsum, 6);
  if (!e) e = cudaMemset(t.gs, 0, sizeof(int) * (size_t)c->G);  // init.cu:110-111
  if (!e) e = cudaMemset(t.ge, 0, sizeof(int) * (size_t)c->G);
  if (!e) e = cudaMemset(t.dg, 0, sizeof(double) * 4 * n);
  if (!e) e = cudaMemset(t.acc, 0, sizeof(double) * 4 * n);
  struct Up { double* d; const double* h; size_t k; } up[] = {
      {c->o.pos, pos, 3}, {c->o.vel, vel, 3}, {c->o.rhop, rhop, 2},
      {c->o.tpos, tpos, 3}, {c->o.tvel, tvel, 3}, {c->o.trhop, trhop, 2}};
  for (auto& u : up)
    if (!e) e = u.h ? cudaMemcpy(u.d, u.h, sizeof(double) * u.k * n, cudaMemcpyHostToDevice)
                    : cudaMemset(u.d, 0, sizeof(double) * u.k * n);
  if (!e) e = cudaMemcpy(c->o.type, type, sizeof(int) * n, cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(c->o.table, table, sizeof(int) * n, cudaMemcpyHostToDevice);
  if (!ck(c, e, "gor_create")) {
    std::fprintf(stderr, "%s\n", c->err.c_str());
    return nullptr;
  }
  return c;
}

// Attaches the body (the oracle's Rigid, as attach_rigid computes it on the
// host, with its body-frame offsets r0[count][3]) and places its particles.
int gor_attach_rigid(void* h, const Rigid* b) {
  Checker* c = static_cast<Checker*>(h);
  c->b = *b;
  c->rigid = true;
  cudaError_t e = dmalloc(c->r0, 3 * (size_t)b->count);
  if (!e) e = cudaMemcpy(c->r0, b->r0, sizeof(double) * 3 * (size_t)b->count, cudaMemcpyHostToDevice);
  c->b.r0 = nullptr;
  if (!e) e = place(c, c->o);
  if (!e) e = cudaDeviceSynchronize();
  return ck(c, e, "gor_attach_rigid") ? 0 : 1;
}

int gor_step(void* h, int nsteps) {
  Checker* c = static_cast<Checker*>(h);
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < nsteps && !e; ++k) e = one_step(c);
  if (!e) e = cudaDeviceSynchronize();
  return ck(c, e, "gor_step") ? 0 : 1;
}

int gor_download(void* h, double* pos, double* vel, double* rhop, int* type, int* table) {
  Checker* c = static_cast<Checker*>(h);
  const size_t n = (size_t)c->n;
  cudaError_t e = cudaMemcpy(pos, c->o.pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(vel, c->o.vel, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(rhop, c->o.rhop, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(type, c->o.type, sizeof(int) * n, cudaMemcpyDeviceToHost);
  if (!e) e = cudaMemcpy(table, c->o.table, sizeof(int) * n, cudaMemcpyDeviceToHost);
  return ck(c, e, "gor_download") ? 0 : 1;
}

void gor_rigid(void* h, Rigid* out) {
  Checker* c = static_cast<Checker*>(h);
  *out = c->b;
}

void gor_destroy(void* h) {
  Checker* c = static_cast<Checker*>(h);
  if (!c) return;
  free_state(c->o);
  free_state(c->w);
  void* q[] = {c->t.acc, c->t.dg, c->t.rho_new, c->t.p_new, c->t.fv, c->t.fvc, c->t.index, c->t.hash,
               c->t.flag, c->t.gs, c->t.ge, c->r0, c->rsum};
  for (void* x : q) if (x) cudaFree(x);
  delete c;
}

}  // extern "C"
