// Precision form and the 6DOF floating body (no reference counterpart).
//
// Precision form: a particle's position is an integer grid cell (one packed
// int per particle, held on the handle for old_ and new_ and carried by the
// search's gather) plus the FP32 offset from the cell's corner, held in the
// pos arrays.  Pair distances are formed in the frame of the particle's own
// cell (equations.cu, shifted()), and the fused integration moves offsets
// and cells (integrate.cuh).  Global sums are FP64.
//
// Rigid body: particles of type 2 whose original index lies in
// [first, first + count) move as one body.  They take part in the fluid
// equations as dummy walls (pressure extrapolated from the fluid), and the
// fluid's pressure force on them is the body's hydrodynamic load.  After
// each fused sub-step's governing kernel:
//   k_rigid_sum   FP64 force and torque about the centre of mass (per-CTA
//                 partial sums, reduced in a fixed order)
//   k_rigid_step  FP64 predictor-corrector update of the body: linear
//                 acceleration F/M + g, angular acceleration of
//                 Test_6DOF/equation/acc_alpha.cpp:20-33
//                 alpha = R I^-1 R^T (T - w x (R I R^T w)), quaternion rate
//                 q' = w q / 2 (Test_6DOF/equation/time_int.cpp:14-15)
//   k_rigid_place body particles at x_c + R r_k with v_c + w x (x - x_c)
// The inertia tensor follows Test_6DOF/equation/rigid_info.cpp:18-39 (about
// the particles' centroid, mass shared equally).  The reference moves body
// particles by their velocity (time_int.cpp:7-12); here they are placed from
// the body's pose, so the body stays rigid.
//
// Several bodies (up to kMaxBodies, disjoint ranges of original indices)
// share these launches: k_rigid_sum runs one row of CTAs per body,
// k_rigid_step one thread per body.  With contact switched on
// (zsph_rigid_contact), k_rigid_contact (equations.cu) first adds to each
// body particle's load the spring-dashpot force of its wall and other-body
// neighbours.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "trace.h"
#include "zsph_internal.cuh"

namespace zsph {

constexpr int kMaxBodies = 16;

struct Body {
  double x[3], v[3], w[3], q[4];      // centre of mass, velocity, angular velocity (world), orientation (w,x,y,z)
  double xn[3], vn[3], wn[3], qn[4];  // the same at the start of the step
  double F[3], T[3];                  // last fluid (and contact) force and torque
  double I[9], Iinv[9];               // body-frame inertia about the centre of mass, and its inverse
  double M, g;
  int first, count;
  long long r0_off;                   // first of this body's rows in RigidState::r0
};

struct RigidState {
  Body* body = nullptr;         // device [kMaxBodies]
  BodyRange* ranges = nullptr;  // device [kMaxBodies] (first, count), for the contact kernel
  double* r0 = nullptr;         // [sum of counts][3] body-frame offsets, body after body
  double* partial = nullptr;    // [kMaxBodies][kRigidBlocks][6]
  float4* force = nullptr;      // [n] per-particle load per unit particle mass (kp.rigid_f)
  int nb = 0;
  std::vector<Body> host;       // the bodies as attached (device copies evolve)
  std::vector<std::vector<double>> host_r0;
  float kn = 0.f, cn = 0.f, dist = 0.f;  // contact (kn = 0: off)
};

namespace {

constexpr int kRigidBlocks = 148;
constexpr int kRigidThreads = 256;
constexpr int kSumBlocks = 296;

int set_herr(Handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else record_library_error(msg);
  return code;
}
int herr_cuda(Handle* h, const char* where, cudaError_t e) {
  return set_herr(h, e == cudaErrorMemoryAllocation ? ZSPH_ENOMEM : ZSPH_ECUDA,
                  std::string(where) + ": " + cudaGetErrorString(e));
}
#define PCHECK(h, where, expr)                           \
  do {                                                   \
    cudaError_t e_ = (expr);                             \
    if (e_ != cudaSuccess) return herr_cuda(h, where, e_); \
  } while (0)

// absolute FP64 position of particle i (precision form: cell + offset)
__device__ __forceinline__ void abs_pos(const KParams& kp, const zsph_ptc_t& s, const int* c3, int i, double* x) {
  const zsph_gpu_param_t& p = kp.p;
  if (c3) {
    const int3 c = unpack_cell(c3[i]);
    x[0] = (double)p.grid_xmin + (double)c.x * p.grid_size + s.pos[3 * i];
    x[1] = (double)p.grid_ymin + (double)c.y * p.grid_size + s.pos[3 * i + 1];
    x[2] = (double)p.grid_zmin + (double)c.z * p.grid_size + s.pos[3 * i + 2];
  } else {
    x[0] = s.pos[3 * i];
    x[1] = s.pos[3 * i + 1];
    x[2] = s.pos[3 * i + 2];
  }
}

// rotation matrix of a unit quaternion (w, x, y, z), row-major
__host__ __device__ inline void rot(const double* q, double* R) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z);     R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y);     R[7] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}
__host__ __device__ inline void mat_vec(const double* A, const double* v, double* r) {
  for (int a = 0; a < 3; ++a) r[a] = A[3 * a] * v[0] + A[3 * a + 1] * v[1] + A[3 * a + 2] * v[2];
}
__host__ __device__ inline void mat_tvec(const double* A, const double* v, double* r) {  // A^T v
  for (int a = 0; a < 3; ++a) r[a] = A[a] * v[0] + A[3 + a] * v[1] + A[6 + a] * v[2];
}
__host__ __device__ inline void cross(const double* a, const double* b, double* r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
// q + dt/2 * (0, w) q, normalized
__device__ inline void quat_advance(const double* q0, const double* w, const double* qr, double dt, double* out) {
  const double a = -w[0] * qr[1] - w[1] * qr[2] - w[2] * qr[3];
  const double b = w[0] * qr[0] + w[1] * qr[3] - w[2] * qr[2];
  const double c = -w[0] * qr[3] + w[1] * qr[0] + w[2] * qr[1];
  const double d = w[0] * qr[2] - w[1] * qr[1] + w[2] * qr[0];
  double r[4] = {q0[0] + 0.5 * dt * a, q0[1] + 0.5 * dt * b, q0[2] + 0.5 * dt * c, q0[3] + 0.5 * dt * d};
  const double inv = 1.0 / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
  for (int k = 0; k < 4; ++k) out[k] = r[k] * inv;
}

__device__ inline bool body_particle(const zsph_ptc_t& s, const Body& b, int i, int* k) {
  if (s.type[i] != 2) return false;
  *k = s.table[i] + i - b.first;  // table[i] + i: the particle's original index (sort.cu:82)
  return *k >= 0 && *k < b.count;
}
// the body owning particle i (index into bodies) and its row k, or -1
__device__ inline int body_of(const zsph_ptc_t& s, const Body* bodies, int nb, int i, int* k) {
  if (s.type[i] != 2) return -1;
  const int id = s.table[i] + i;
  for (int b = 0; b < nb; ++b) {
    const int kk = id - bodies[b].first;
    if (kk >= 0 && kk < bodies[b].count) {
      *k = kk;
      return b;
    }
  }
  return -1;
}

// FP64 force and torque on each body, per-CTA partial sums: CTA row
// blockIdx.y sums the particles of body blockIdx.y, in particle order
__global__ void __launch_bounds__(kRigidThreads) k_rigid_sum(KParams kp, zsph_ptc_t s, const int* c3,
                                                             const float4* f, const Body* bodies, double* partial) {
  const Body& b = bodies[blockIdx.y];
  partial += (size_t)blockIdx.y * gridDim.x * 6;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const double m = kp.p.m;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kp.n; i += gridDim.x * blockDim.x) {
    int k;
    if (!body_particle(s, b, i, &k)) continue;
    double x[3], r[3], t[3];
    abs_pos(kp, s, c3, i, x);
    const float4 fi = f[i];
    const double fv[3] = {m * fi.x, m * fi.y, m * fi.z};
    for (int a = 0; a < 3; ++a) r[a] = x[a] - b.x[a];
    cross(r, fv, t);
    for (int a = 0; a < 3; ++a) {
      acc[a] += fv[a];
      acc[3 + a] += t[a];
    }
  }
  __shared__ double sh[kRigidThreads / 32][6];
  for (int k = 0; k < 6; ++k)
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 6; ++k) sh[threadIdx.x >> 5][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0;
    for (int w = 0; w < kRigidThreads / 32; ++w) v += sh[w][threadIdx.x];
    partial[blockIdx.x * 6 + threadIdx.x] = v;
  }
}

// FP64 predictor (mode 1) or corrector (mode 2) of each body, one thread per body
__global__ void k_rigid_step(Body* bodies, int nb, const double* partial, int nparts, int mode, double half_dt) {
  if (blockIdx.x != 0 || (int)threadIdx.x >= nb) return;
  Body& b = bodies[threadIdx.x];
  partial += (size_t)threadIdx.x * nparts * 6;
  double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
  for (int c = 0; c < nparts; ++c)
    for (int a = 0; a < 3; ++a) {
      F[a] += partial[c * 6 + a];
      T[a] += partial[c * 6 + 3 + a];
    }
  for (int a = 0; a < 3; ++a) {
    b.F[a] = F[a];
    b.T[a] = T[a];
  }
  // accelerations at the current pose (acc_alpha.cpp:5-33)
  double acc[3] = {F[0] / b.M, F[1] / b.M, F[2] / b.M + b.g};
  double R[9], tmp[3], tmp2[3], Iw[3], alpha[3];
  rot(b.q, R);
  mat_tvec(R, b.w, tmp);    // R^T w
  mat_vec(b.I, tmp, tmp2);  // I R^T w
  mat_vec(R, tmp2, Iw);     // R I R^T w
  cross(b.w, Iw, tmp);
  for (int a = 0; a < 3; ++a) tmp[a] = T[a] - tmp[a];
  mat_tvec(R, tmp, tmp2);
  mat_vec(b.Iinv, tmp2, tmp);
  mat_vec(R, tmp, alpha);
  if (mode == 1) {
    for (int a = 0; a < 3; ++a) {
      b.xn[a] = b.x[a];
      b.vn[a] = b.v[a];
      b.wn[a] = b.w[a];
    }
    for (int a = 0; a < 4; ++a) b.qn[a] = b.q[a];
    double qh[4];
    quat_advance(b.qn, b.wn, b.qn, half_dt, qh);
    for (int a = 0; a < 3; ++a) {
      b.x[a] = b.xn[a] + b.vn[a] * half_dt;
      b.v[a] = b.vn[a] + acc[a] * half_dt;
      b.w[a] = b.wn[a] + alpha[a] * half_dt;
    }
    for (int a = 0; a < 4; ++a) b.q[a] = qh[a];
  } else {
    const double dt = 2.0 * half_dt;
    double q1[4];
    quat_advance(b.qn, b.w, b.q, dt, q1);  // rate at the half-step pose
    for (int a = 0; a < 3; ++a) {
      b.x[a] = b.xn[a] + b.v[a] * dt;
      b.v[a] = b.vn[a] + acc[a] * dt;
      b.w[a] = b.wn[a] + alpha[a] * dt;
    }
    for (int a = 0; a < 4; ++a) b.q[a] = q1[a];
  }
}

// body particles at the body's pose; precision form: cell + offset
__global__ void __launch_bounds__(kRigidThreads) k_rigid_place(KParams kp, zsph_ptc_t s, int* c3, const Body* bodies,
                                                               int nb, const double* r0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kp.n) return;
  int k;
  const int bi = body_of(s, bodies, nb, i, &k);
  if (bi < 0) return;
  const Body& b = bodies[bi];
  double R[9], r[3], x[3], w[3];
  rot(b.q, R);
  mat_vec(R, r0 + 3 * ((size_t)b.r0_off + (size_t)k), r);
  for (int a = 0; a < 3; ++a) x[a] = b.x[a] + r[a];
  cross(b.w, r, w);
  for (int a = 0; a < 3; ++a) s.vel[3 * i + a] = (float)(b.v[a] + w[a]);
  const zsph_gpu_param_t& p = kp.p;
  if (c3) {
    const double org[3] = {p.grid_xmin, p.grid_ymin, p.grid_zmin};
    const int dim[3] = {p.grid_xdim, p.grid_ydim, p.grid_zdim};
    int cc[3];
    for (int a = 0; a < 3; ++a) {
      const double u = (x[a] - org[a]) / p.grid_size;
      int h = (int)floor(u);
      double o = x[a] - org[a] - (double)h * p.grid_size;
      if (h < 0 || h >= dim[a]) h = kCellMask;
      cc[a] = h;
      s.pos[3 * i + a] = (float)o;
    }
    c3[i] = pack_cell(cc[0], cc[1], cc[2]);
  } else {
    for (int a = 0; a < 3; ++a) s.pos[3 * i + a] = (float)x[a];
  }
}

// FP64 global sums over the fluid: mass, volume, momentum, kinetic,
// potential and elastic energy, per-CTA partials
__global__ void __launch_bounds__(kRigidThreads) k_conserve(KParams kp, zsph_ptc_t s, const int* c3, double* partial) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const zsph_gpu_param_t& p = kp.p;
  const double m = p.m, g = p.g, rho0 = p.rho0, cs2 = p.cs2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kp.n; i += gridDim.x * blockDim.x) {
    if (s.type[i] != 1) continue;
    double x[3];
    abs_pos(kp, s, c3, i, x);
    const double rho = s.rhop[2 * i];
    const double u = s.vel[3 * i], w = s.vel[3 * i + 1], z = s.vel[3 * i + 2];
    v[0] += m;
    v[1] += m / rho;
    v[2] += m * u;
    v[3] += m * w;
    v[4] += m * z;
    v[5] += 0.5 * m * (u * u + w * w + z * z);
    v[6] += -m * g * x[2];
    // internal energy of the linear equation of state p = c^2 (rho - rho0)
    v[7] += m * cs2 * (log(rho / rho0) + rho0 / rho - 1.0);
  }
  __shared__ double sh[kRigidThreads / 32][8];
  for (int k = 0; k < 8; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 8; ++k) sh[threadIdx.x >> 5][k] = v[k];
  __syncthreads();
  if (threadIdx.x < 8) {
    double a = 0;
    for (int w = 0; w < kRigidThreads / 32; ++w) a += sh[w][threadIdx.x];
    partial[blockIdx.x * 8 + threadIdx.x] = a;
  }
}

void drop_graph(Handle* h) {
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
}

int inv3(const double* A, double* B) {
  const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                     A[2] * (A[3] * A[7] - A[4] * A[6]);
  if (!(std::fabs(det) > 0)) return 1;
  const double id = 1.0 / det;
  B[0] = (A[4] * A[8] - A[5] * A[7]) * id;
  B[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = (A[5] * A[6] - A[3] * A[8]) * id;
  B[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  B[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  B[6] = (A[3] * A[7] - A[4] * A[6]) * id;
  B[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return 0;
}

// host copies of the absolute FP64 positions, types and tables of a buffer
int download_positions(Handle* h, const zsph_ptc_t& s, std::vector<double>& x, std::vector<int>& type,
                       std::vector<int>& table) {
  const int n = h->kp.n;
  std::vector<float> pos((size_t)3 * n);
  std::vector<int> c3;
  x.assign((size_t)3 * n, 0.0);
  type.resize(n);
  table.resize(n);
  PCHECK(h, "download", cudaMemcpy(pos.data(), s.pos, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
  PCHECK(h, "download", cudaMemcpy(type.data(), s.type, sizeof(int) * n, cudaMemcpyDeviceToHost));
  PCHECK(h, "download", cudaMemcpy(table.data(), s.table, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (h->kp.c3o) {
    c3.resize(n);
    PCHECK(h, "download", cudaMemcpy(c3.data(), h->kp.c3o, sizeof(int) * n, cudaMemcpyDeviceToHost));
  }
  const zsph_gpu_param_t& p = h->kp.p;
  const double org[3] = {p.grid_xmin, p.grid_ymin, p.grid_zmin};
  for (int i = 0; i < n; ++i) {
    if (h->kp.c3o) {
      const int3 c = unpack_cell(c3[i]);
      const int cc[3] = {c.x, c.y, c.z};
      for (int a = 0; a < 3; ++a) x[3 * i + a] = org[a] + (double)cc[a] * p.grid_size + pos[3 * i + a];
    } else {
      for (int a = 0; a < 3; ++a) x[3 * i + a] = pos[3 * i + a];
    }
  }
  return ZSPH_OK;
}

}  // namespace

void precise_destroy(Handle* h) {
  if (!h) return;
  cudaFree(h->c3buf[0]);
  cudaFree(h->c3buf[1]);
  h->c3buf[0] = h->c3buf[1] = nullptr;
  if (h->rigid) {
    cudaFree(h->rigid->body);
    cudaFree(h->rigid->ranges);
    cudaFree(h->rigid->r0);
    cudaFree(h->rigid->partial);
    cudaFree(h->rigid->force);
    delete h->rigid;
    h->rigid = nullptr;
  }
}

cudaError_t rigid_substep(Handle* h, const zsph_ptc_t& from, const zsph_ptc_t& to, const zsph_tmp_t& t, int mode,
                          cudaStream_t st) {
  RigidState* R = h->rigid;
  const KParams& kp = h->kp;
  if (R->kn > 0.f) {
    cudaError_t e = launch_rigid_contact(kp, h->s, to, t, R->ranges, R->nb, R->kn, R->cn, R->dist, st);
    if (e) return e;
  }
  k_rigid_sum<<<dim3(kRigidBlocks, R->nb), kRigidThreads, 0, st>>>(kp, to, kp.c3n, R->force, R->body, R->partial);
  k_rigid_step<<<1, 32, 0, st>>>(R->body, R->nb, R->partial, kRigidBlocks, mode, (double)kp.p.half_dt);
  k_rigid_place<<<(kp.n + kRigidThreads - 1) / kRigidThreads, kRigidThreads, 0, st>>>(kp, from, kp.c3o, R->body,
                                                                                      R->nb, R->r0);
  return cudaGetLastError();
}

}  // namespace zsph

using namespace zsph;

extern "C" {

int zsph_set_precision(zsph_handle_t* h, int on) {
  if (!h) return set_herr(nullptr, ZSPH_EINVAL, "zsph_set_precision: null handle");
  if (on) {
    const zsph_gpu_param_t& p = h->kp.p;
    if (p.grid_factor != 1 || h->kp.equations != ZSPH_EQ_DELTA)
      return set_herr(h, ZSPH_EINVAL, "zsph_set_precision: needs grid_size_factor 1 and the delta-SPH equations");
    if (p.grid_xdim > kCellMask || p.grid_ydim > kCellMask || p.grid_zdim > kCellMask)
      return set_herr(h, ZSPH_EINVAL, "zsph_set_precision: grid dimensions above 1023");
    if (!h->c3buf[0]) {
      const size_t nb = sizeof(int) * (size_t)std::max(h->kp.n, 1);
      PCHECK(h, "zsph_set_precision", cudaMalloc(&h->c3buf[0], nb));
      PCHECK(h, "zsph_set_precision", cudaMalloc(&h->c3buf[1], nb));
      PCHECK(h, "zsph_set_precision", cudaMemset(h->c3buf[0], 0, nb));
      PCHECK(h, "zsph_set_precision", cudaMemset(h->c3buf[1], 0, nb));
    }
    h->kp.c3o = h->c3buf[0];
    h->kp.c3n = h->c3buf[1];
    h->kp.stage_windows = 0;
  } else {
    h->kp.c3o = h->kp.c3n = nullptr;
  }
  drop_graph(h);
  return ZSPH_OK;
}

int zsph_precise_load(zsph_handle_t* h, const zsph_ptc_t* old_, const double* pos, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (!h || !old_ || !pos) return set_herr(h, ZSPH_EINVAL, "zsph_precise_load: null argument");
  if (!h->kp.c3o) return set_herr(h, ZSPH_EINVAL, "zsph_precise_load: precision form is off");
  const int n = h->kp.n;
  const zsph_gpu_param_t& p = h->kp.p;
  const double org[3] = {p.grid_xmin, p.grid_ymin, p.grid_zmin};
  const int dim[3] = {p.grid_xdim, p.grid_ydim, p.grid_zdim};
  std::vector<int> c3(n);
  std::vector<float> off((size_t)3 * n);
  for (int i = 0; i < n; ++i) {
    int cc[3];
    for (int a = 0; a < 3; ++a) {
      const double u = pos[3 * (size_t)i + a] - org[a];
      int c = (int)std::floor(u / (double)p.grid_size);
      double o = u - (double)c * p.grid_size;
      if (c < 0 || c >= dim[a]) {  // left the grid: the next hash kills it
        c = kCellMask;
        o = 0.0;
      }
      cc[a] = c;
      off[3 * (size_t)i + a] = (float)o;
    }
    c3[i] = pack_cell(cc[0], cc[1], cc[2]);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PCHECK(h, "zsph_precise_load", cudaMemcpyAsync(h->kp.c3o, c3.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  PCHECK(h, "zsph_precise_load", cudaMemcpyAsync(old_->pos, off.data(), sizeof(float) * 3 * n,
                                                 cudaMemcpyHostToDevice, st));
  PCHECK(h, "zsph_precise_load", cudaStreamSynchronize(st));
  return ZSPH_OK;
}

int zsph_precise_positions(zsph_handle_t* h, const zsph_ptc_t* old_, double* pos, void* stream) {
  if (!h || !old_ || !pos) return set_herr(h, ZSPH_EINVAL, "zsph_precise_positions: null argument");
  PCHECK(h, "zsph_precise_positions", cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  std::vector<double> x;
  std::vector<int> type, table;
  if (int rc = download_positions(h, *old_, x, type, table)) return rc;
  std::memcpy(pos, x.data(), sizeof(double) * x.size());
  return ZSPH_OK;
}

int zsph_conservation(zsph_handle_t* h, const zsph_ptc_t* old_, zsph_conservation_t* out, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (!h || !old_ || !out) return set_herr(h, ZSPH_EINVAL, "zsph_conservation: null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* d = nullptr;
  PCHECK(h, "zsph_conservation", cudaMalloc(&d, sizeof(double) * 8 * kSumBlocks));
  k_conserve<<<kSumBlocks, kRigidThreads, 0, st>>>(h->kp, *old_, h->kp.c3o, d);
  std::vector<double> part((size_t)8 * kSumBlocks);
  cudaError_t e = cudaGetLastError();
  if (!e) e = cudaMemcpyAsync(part.data(), d, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  cudaFree(d);
  PCHECK(h, "zsph_conservation", e);
  double v[8] = {};
  for (int b = 0; b < kSumBlocks; ++b)
    for (int k = 0; k < 8; ++k) v[k] += part[(size_t)b * 8 + k];
  zsph_conservation_t c{};
  c.mass = v[0];
  c.volume = v[1];
  for (int a = 0; a < 3; ++a) c.momentum[a] = v[2 + a];
  c.kinetic = v[5];
  c.potential = v[6];
  c.internal = v[7];
  if (h->rigid) {
    std::vector<Body> bs(h->rigid->nb);
    PCHECK(h, "zsph_conservation body",
           cudaMemcpy(bs.data(), h->rigid->body, sizeof(Body) * bs.size(), cudaMemcpyDeviceToHost));
    for (const Body& b : bs) {
      double R[9], tmp[3], tmp2[3], Iw[3];
      rot(b.q, R);
      mat_tvec(R, b.w, tmp);
      mat_vec(b.I, tmp, tmp2);
      mat_vec(R, tmp2, Iw);
      c.body_kinetic += 0.5 * b.M * (b.v[0] * b.v[0] + b.v[1] * b.v[1] + b.v[2] * b.v[2]) +
                        0.5 * (b.w[0] * Iw[0] + b.w[1] * Iw[1] + b.w[2] * Iw[2]);
      c.body_potential += -b.M * b.g * b.x[2];
    }
  }
  *out = c;
  return ZSPH_OK;
}

int zsph_rigid_attach(zsph_handle_t* h, const zsph_ptc_t* old_, const zsph_rigid_t* body, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (!h || !old_ || !body) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: null argument");
  if (body->count <= 0 || body->first < 0 || !(body->mass > 0))
    return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: count > 0, first >= 0 and mass > 0 required");
  if (h->kp.equations != ZSPH_EQ_DELTA)
    return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: the delta-SPH equations are required");
  PCHECK(h, "zsph_rigid_attach", cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  std::vector<double> x;
  std::vector<int> type, table;
  if (int rc = download_positions(h, *old_, x, type, table)) return rc;
  // body particles by original index; centroid and inertia (rigid_info.cpp:3-39)
  std::vector<double> r((size_t)3 * body->count, 0.0);
  std::vector<int> seen(body->count, 0);
  double c[3] = {0, 0, 0};
  for (int i = 0; i < h->kp.n; ++i) {
    const int k = table[i] + i - body->first;
    if (type[i] != 2 || k < 0 || k >= body->count) continue;
    seen[k] = 1;
    for (int a = 0; a < 3; ++a) {
      r[3 * (size_t)k + a] = x[3 * (size_t)i + a];
      c[a] += x[3 * (size_t)i + a];
    }
  }
  for (int k = 0; k < body->count; ++k)
    if (!seen[k]) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: a body particle is missing or not of type 2");
  for (int a = 0; a < 3; ++a) c[a] /= body->count;
  Body b{};
  double I[9] = {};
  for (int k = 0; k < body->count; ++k) {
    double* rk = &r[3 * (size_t)k];
    for (int a = 0; a < 3; ++a) rk[a] -= c[a];
    I[0] += rk[1] * rk[1] + rk[2] * rk[2];
    I[4] += rk[0] * rk[0] + rk[2] * rk[2];
    I[8] += rk[0] * rk[0] + rk[1] * rk[1];
    I[1] -= rk[0] * rk[1];
    I[2] -= rk[0] * rk[2];
    I[5] -= rk[1] * rk[2];
  }
  I[3] = I[1];
  I[6] = I[2];
  I[7] = I[5];
  for (int a = 0; a < 9; ++a) I[a] *= body->mass / body->count;
  // world -> body frame with the given orientation
  double q[4];
  std::memcpy(q, body->q, sizeof q);
  const double qn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(qn > 0)) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: zero quaternion");
  for (double& v : q) v /= qn;
  double R[9], Ib[9], tmp[9];
  rot(q, R);
  for (int k = 0; k < body->count; ++k) {  // r0 = R^T r
    double rb[3];
    mat_tvec(R, &r[3 * (size_t)k], rb);
    std::memcpy(&r[3 * (size_t)k], rb, sizeof rb);
  }
  // body-frame inertia R^T I R
  for (int a = 0; a < 3; ++a)
    for (int bb = 0; bb < 3; ++bb) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += I[3 * a + k] * R[3 * k + bb];
      tmp[3 * a + bb] = s;
    }
  for (int a = 0; a < 3; ++a)
    for (int bb = 0; bb < 3; ++bb) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += R[3 * k + a] * tmp[3 * k + bb];
      Ib[3 * a + bb] = s;
    }
  std::memcpy(b.I, Ib, sizeof Ib);
  if (inv3(b.I, b.Iinv)) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: singular inertia");
  for (int a = 0; a < 3; ++a) {
    b.x[a] = b.xn[a] = c[a];
    b.v[a] = b.vn[a] = body->vel[a];
    b.w[a] = b.wn[a] = body->omega[a];
  }
  for (int a = 0; a < 4; ++a) b.q[a] = b.qn[a] = q[a];
  b.M = body->mass;
  b.g = h->kp.p.g;
  b.first = body->first;
  b.count = body->count;
  if (!h->rigid) {
    auto* R0 = new RigidState();
    const size_t n = (size_t)std::max(h->kp.n, 1);
    cudaError_t e = cudaMalloc(&R0->body, sizeof(Body) * kMaxBodies);
    if (!e) e = cudaMalloc(&R0->ranges, sizeof(BodyRange) * kMaxBodies);
    if (!e) e = cudaMalloc(&R0->partial, sizeof(double) * 6 * kRigidBlocks * kMaxBodies);
    if (!e) e = cudaMalloc(&R0->force, sizeof(float4) * n);
    if (!e) e = cudaMemset(R0->force, 0, sizeof(float4) * n);
    if (e) {
      cudaFree(R0->body);
      cudaFree(R0->ranges);
      cudaFree(R0->partial);
      cudaFree(R0->force);
      delete R0;
      return herr_cuda(h, "zsph_rigid_attach", e);
    }
    h->rigid = R0;
  }
  RigidState* RS = h->rigid;
  // the bodies' current states (earlier bodies have moved since they were attached)
  if (RS->nb > 0)
    PCHECK(h, "zsph_rigid_attach", cudaMemcpy(RS->host.data(), RS->body, sizeof(Body) * RS->nb, cudaMemcpyDeviceToHost));
  int slot = RS->nb;  // a body with the same first index is replaced, any other one added
  for (int k = 0; k < RS->nb; ++k) {
    if (RS->host[k].first == b.first) {
      slot = k;
      continue;
    }
    const Body& o = RS->host[k];
    if (b.first < o.first + o.count && o.first < b.first + b.count)
      return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: the body's particle range overlaps another body's");
  }
  if (slot == kMaxBodies) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_attach: at most 16 bodies per handle");
  if (slot == RS->nb) {
    RS->host.push_back(b);
    RS->host_r0.push_back(r);
    RS->nb += 1;
  } else {
    RS->host[slot] = b;
    RS->host_r0[slot] = r;
  }
  std::vector<double> all;
  std::vector<BodyRange> ranges(RS->nb);
  for (int k = 0; k < RS->nb; ++k) {
    RS->host[k].r0_off = (long long)(all.size() / 3);
    all.insert(all.end(), RS->host_r0[k].begin(), RS->host_r0[k].end());
    ranges[k] = BodyRange{RS->host[k].first, RS->host[k].count};
  }
  cudaFree(RS->r0);
  RS->r0 = nullptr;
  PCHECK(h, "zsph_rigid_attach", cudaMalloc(&RS->r0, sizeof(double) * all.size()));
  PCHECK(h, "zsph_rigid_attach", cudaMemcpy(RS->r0, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice));
  PCHECK(h, "zsph_rigid_attach", cudaMemcpy(RS->body, RS->host.data(), sizeof(Body) * RS->nb, cudaMemcpyHostToDevice));
  PCHECK(h, "zsph_rigid_attach", cudaMemcpy(RS->ranges, ranges.data(), sizeof(BodyRange) * RS->nb,
                                            cudaMemcpyHostToDevice));
  h->kp.rigid_f = RS->force;
  drop_graph(h);
  // body particles' velocities (and precision cells) from the poses
  k_rigid_place<<<(h->kp.n + kRigidThreads - 1) / kRigidThreads, kRigidThreads>>>(h->kp, *old_, h->kp.c3o, RS->body,
                                                                                 RS->nb, RS->r0);
  PCHECK(h, "zsph_rigid_attach place", cudaDeviceSynchronize());
  return ZSPH_OK;
}

int zsph_rigid_contact(zsph_handle_t* h, double stiffness, double damping, double distance) {
  if (!h) return set_herr(nullptr, ZSPH_EINVAL, "zsph_rigid_contact: null handle");
  if (!h->rigid) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_contact: attach a body first");
  if (!(stiffness >= 0) || !(damping >= 0) || !(distance >= 0))
    return set_herr(h, ZSPH_EINVAL, "zsph_rigid_contact: stiffness, damping and distance must be >= 0");
  if (stiffness > 0 && !((float)distance * (float)distance <= h->kp.r2max))
    return set_herr(h, ZSPH_EINVAL, "zsph_rigid_contact: the contact distance must not exceed the 2h support");
  if (h->kp.p.grid_factor != 1)
    return set_herr(h, ZSPH_EINVAL, "zsph_rigid_contact: needs grid_size_factor 1");
  h->rigid->kn = (float)stiffness;
  h->rigid->cn = (float)damping;
  h->rigid->dist = (float)distance;
  drop_graph(h);
  return ZSPH_OK;
}

int zsph_rigid_count(zsph_handle_t* h, int* count) {
  if (!h || !count) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_count: null argument");
  *count = h->rigid ? h->rigid->nb : 0;
  return ZSPH_OK;
}

int zsph_rigid_get_body(zsph_handle_t* h, int index, zsph_rigid_t* body) {
  if (!h || !body) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_get_body: null argument");
  if (!h->rigid || index < 0 || index >= h->rigid->nb)
    return set_herr(h, ZSPH_EINVAL, "zsph_rigid_get_body: no such body");
  PCHECK(h, "zsph_rigid_get_body", cudaStreamSynchronize(h->last_stream));
  Body b;
  PCHECK(h, "zsph_rigid_get_body", cudaMemcpy(&b, h->rigid->body + index, sizeof b, cudaMemcpyDeviceToHost));
  body->first = b.first;
  body->count = b.count;
  body->mass = b.M;
  std::memcpy(body->pos, b.x, sizeof b.x);
  std::memcpy(body->vel, b.v, sizeof b.v);
  std::memcpy(body->omega, b.w, sizeof b.w);
  std::memcpy(body->q, b.q, sizeof b.q);
  std::memcpy(body->force, b.F, sizeof b.F);
  std::memcpy(body->torque, b.T, sizeof b.T);
  std::memcpy(body->inertia, b.I, sizeof b.I);
  return ZSPH_OK;
}

int zsph_rigid_get(zsph_handle_t* h, zsph_rigid_t* body) {
  if (!h || !body) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_get: null argument");
  if (!h->rigid) return set_herr(h, ZSPH_EINVAL, "zsph_rigid_get: no body attached");
  return zsph_rigid_get_body(h, 0, body);
}

}  // extern "C"
