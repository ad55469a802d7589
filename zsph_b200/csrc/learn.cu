// Learned-corrector form of the step (no reference counterpart).
//
// Plain step: predictor sub-step (search, boundary, governing + prediction)
// then corrector sub-step (search, boundary, governing + correction).  The
// learned form keeps the predictor sub-step, whose governing walk also
// writes 32 non-dimensional neighbour aggregates per fluid particle
// (FeatOut), and replaces the whole corrector sub-step by one tensor-core
// kernel: the network predicts the change of (acc, drho/dt) from the
// predictor to the corrector stage, and the kernel's epilogue applies the
// time_int.cu:50-92 correction with predictor-stage value + prediction.
// Every judge_every-th step also runs the plain corrector, which judges the
// prediction (relative L2 of the fluid accelerations, FP64 sums) and
// replaces it; above the tolerance the plain corrector takes over until the
// next judged step passes.
//
// Training data come from plain steps: at sampled steps the predictor-stage
// features and (plain corrector - predictor) values of every particle are
// kept on the device; training (mlp.cu kernels) runs on shuffled 128-row
// tiles with Adam.  Units: lengths h, speeds c0, densities rho0, so
// accelerations c0^2/h and density rates rho0 c0/h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "trace.h"
#include "zsph_internal.cuh"

namespace zsph {

struct LearnState {
  int n = 0, n_pad = 0, cap = 0, count = 0;
  float* raw = nullptr;            // [cap][n_pad][kFeat] raw features
  float4* y = nullptr;             // [cap][n_pad] non-dimensional targets (standardized after training)
  float* w = nullptr;              // [cap][n_pad] row weights (1 fluid, 0 otherwise)
  unsigned char* tiles = nullptr;  // [n_pad / 128] tiles for the learned run
  float4* acc_n = nullptr;         // [n] predictor-stage (acc, drho/dt)
  float4* acc_prev = nullptr;      // [n] previous corrector-stage values (copied before a predictor)
  float4* dprev = nullptr;         // [n] D = predictor-stage value - previous corrector value
  float4* yhat = nullptr;          // [n] network outputs (judged steps)
  int* cy = nullptr;               // [n] current y cells (list-reuse correctors)
  double* red = nullptr;           // [kRedBlocks][8] reduction partials
  double* red_host = nullptr;      // pinned copy
  bool targets_standardized = false;
};

namespace {

constexpr int kRedBlocks = 296;
constexpr int kRedThreads = 256;

int set_herr(Handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else record_library_error(msg);
  return code;
}
int herr_cuda(Handle* h, const char* where, cudaError_t e) {
  return set_herr(h, e == cudaErrorMemoryAllocation ? ZSPH_ENOMEM : ZSPH_ECUDA,
                  std::string(where) + ": " + cudaGetErrorString(e));
}
#define LCHECK(h, where, expr)                           \
  do {                                                   \
    cudaError_t e_ = (expr);                             \
    if (e_ != cudaSuccess) return herr_cuda(h, where, e_); \
  } while (0)

struct Units {
  float H, C, R;
  float4 target_scale() const { return make_float4(H / (C * C), H / (C * C), H / (C * C), H / (R * C)); }
  float4 target_unit() const { return make_float4(C * C / H, C * C / H, C * C / H, R * C / H); }
};
Units units_of(const KParams& kp) { return Units{kp.p.h, std::sqrt(kp.p.cs2), kp.p.rho0}; }

// feature k's non-dimensional scale (order of FeatOut / the oracle's features)
void feature_scales(const Units& u, float* s) {
  const float H = u.H, C = u.C, R = u.R;
  const float v[kFeat] = {1.f, 1.f, H, H, H, H / C, H * H / C, H * H / C,
                          H * H / C, H * H / C, H * H / C, H * H / C, H * H / R, H * H / (R * C * C), H / (C * C), H / (C * C),
                          H / (C * C), H / (R * C), 1.f / C, 1.f / C, 1.f / C, 1.f / R, H / R, H / R,
                          H / R, H / (C * C), H / (C * C), H / (C * C), H / (C * C), H / (C * C), H / (C * C), H / (R * C)};
  std::memcpy(s, v, sizeof v);
}

// Target row of predictor-order particle i from corrector slot t: what the
// linear extrapolation a_n + D misses of the plain corrector value.
__global__ void k_targets(int n, const int* index, const float4* acc_c, const float4* acc_n, const float4* dprev,
                          const int* type, float4 scale, float4* y, float* w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = index[t];
  const float4 c = acc_c[t], a = acc_n[i], d = dprev[i];
  y[i] = make_float4((c.x - a.x - d.x) * scale.x, (c.y - a.y - d.y) * scale.y, (c.z - a.z - d.z) * scale.z,
                     (c.w - a.w - d.w) * scale.w);
  w[i] = type[t] == 1 ? 1.f : 0.f;
}

// Weighted moments (FP64) of the 32 features and 4 targets over `rows` rows:
// block b sums the rows [b*chunk, (b+1)*chunk); thread k < 36 owns column k.
// out[b][k][0..2] = sum w, sum w x, sum w x^2.
__global__ void k_moments(const float* raw, const float4* y, const float* w, long long rows, long long chunk,
                          double* out) {
  const int k = threadIdx.x;
  if (k >= kFeat + 4) return;
  const long long r0 = (long long)blockIdx.x * chunk, r1 = std::min(rows, r0 + chunk);
  double s0 = 0, s1 = 0, s2 = 0;
  for (long long r = r0; r < r1; ++r) {
    const float wr = w[r];
    if (wr == 0.f) continue;
    const float x = k < kFeat ? raw[r * kFeat + k] : reinterpret_cast<const float*>(y)[r * 4 + (k - kFeat)];
    s0 += wr;
    s1 += (double)wr * x;
    s2 += (double)wr * x * x;
  }
  double* o = out + ((size_t)blockIdx.x * (kFeat + 4) + k) * 3;
  o[0] = s0;
  o[1] = s1;
  o[2] = s2;
}

__global__ void k_standardize_targets(float4* y, long long rows, float4 mean, float4 inv_std) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const float4 v = y[r];
  y[r] = make_float4((v.x - mean.x) * inv_std.x, (v.y - mean.y) * inv_std.y, (v.z - mean.z) * inv_std.z,
                     (v.w - mean.w) * inv_std.w);
}

__global__ void k_loss_accum(const float* partial, int nparts, double* acc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0;
  for (int c = 0; c < nparts; ++c) s += partial[(size_t)c * ZSPH_MLP_NPARTIAL + ZSPH_MLP_NPARAM];
  *acc += s;
}

__device__ __forceinline__ void block_sum_to(double (&v)[8], double* out) {
  __shared__ double sh[kRedThreads / 32][8];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 8; ++k) sh[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < 8) {
    double s = 0;
    for (int wi = 0; wi < kRedThreads / 32; ++wi) s += sh[wi][threadIdx.x];
    out[(size_t)blockIdx.x * 8 + threadIdx.x] = s;
  }
}

// Held-out check in non-dimensional units: a_n = raw features 14..17,
// D = raw features 25..27, 31, a_c = a_n + D + target; the network predicts
// a_n + D + yhat (both de-standardized).  Sums for acc (xyz) at 0..3 and
// drho at 4..7: |network - a_c|^2, |a_c|^2, |a_n - a_c|^2 (predictor values
// alone), |a_n + D - a_c|^2 (extrapolation alone).
__global__ void k_val_sums(const float* raw, const float4* y, const float* w, const float4* yhat, long long rows,
                           float4 ym, float4 ys, double* out) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (long long)gridDim.x * blockDim.x) {
    if (w[r] == 0.f) continue;
    const float* f = raw + r * kFeat;
    const float4 t = y[r], p = yhat[r];
    const float res[4] = {t.x * ys.x + ym.x, t.y * ys.y + ym.y, t.z * ys.z + ym.z, t.w * ys.w + ym.w};
    const float est[4] = {p.x * ys.x + ym.x, p.y * ys.y + ym.y, p.z * ys.z + ym.z, p.w * ys.w + ym.w};
    const float dd[4] = {f[25], f[26], f[27], f[31]};
    for (int c = 0; c < 4; ++c) {
      const double ac = (double)f[14 + c] + dd[c] + res[c];
      const double e_net = (double)est[c] - res[c];
      const double e_base = (double)dd[c] + res[c];
      const int o = c < 3 ? 0 : 4;
      v[o] += e_net * e_net;
      v[o + 1] += ac * ac;
      v[o + 2] += e_base * e_base;
      v[o + 3] += (double)res[c] * res[c];
    }
  }
  block_sum_to(v, out);
}

// Judge: learned prediction (predictor order) against the plain corrector
// (corrector order t, particle index[t]), fluid particles, dimensional.
__global__ void k_judge(int n, const int* index, const float4* acc_c, const float4* acc_n, const float4* dprev,
                        const float4* yhat, const int* type, float4 oa, float4 ob, double* out) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    if (type[t] != 1) continue;
    const int i = index[t];
    const float4 c = acc_c[t], a = acc_n[i], y = yhat[i], d = dprev[i];
    const float px = a.x + d.x + fmaf(y.x, oa.x, ob.x), py = a.y + d.y + fmaf(y.y, oa.y, ob.y);
    const float pz = a.z + d.z + fmaf(y.z, oa.z, ob.z), pw = a.w + d.w + fmaf(y.w, oa.w, ob.w);
    const double ex = (double)px - c.x, ey = (double)py - c.y, ez = (double)pz - c.z, ew = (double)pw - c.w;
    v[0] += ex * ex + ey * ey + ez * ez;
    v[1] += (double)c.x * c.x + (double)c.y * c.y + (double)c.z * c.z;
    v[4] += ew * ew;
    v[5] += (double)c.w * c.w;
  }
  block_sum_to(v, out);
}

// Judge of the list-reuse correctors: their corrector-stage accelerations
// (predictor order) against the plain corrector's (corrector order t,
// particle index[t]), fluid particles.
__global__ void k_judge_acc(int n, const int* index, const float4* acc_c, const float4* acc_v, const int* type,
                            double* out) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    if (type[t] != 1) continue;
    const float4 c = acc_c[t], a = acc_v[index[t]];
    const double ex = (double)a.x - c.x, ey = (double)a.y - c.y, ez = (double)a.z - c.z, ew = (double)a.w - c.w;
    v[0] += ex * ex + ey * ey + ez * ez;
    v[1] += (double)c.x * c.x + (double)c.y * c.y + (double)c.z * c.z;
    v[4] += ew * ew;
    v[5] += (double)c.w * c.w;
  }
  block_sum_to(v, out);
}

uint64_t mix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void free_state(LearnState* L) {
  if (!L) return;
  cudaFree(L->raw);
  cudaFree(L->y);
  cudaFree(L->w);
  cudaFree(L->tiles);
  cudaFree(L->acc_n);
  cudaFree(L->acc_prev);
  cudaFree(L->dprev);
  cudaFree(L->yhat);
  cudaFree(L->cy);
  cudaFree(L->red);
  if (L->red_host) cudaFreeHost(L->red_host);
  delete L;
}

// per-handle scratch of the learned form (run tiles, copies, reductions)
int ensure_state(Handle* h) {
  if (h->learn) return ZSPH_OK;
  auto* L = new LearnState();
  L->n = h->kp.n;
  L->n_pad = (h->kp.n + 127) / 128 * 128;
  const size_t np = (size_t)std::max(L->n_pad, 128);
  cudaError_t e = cudaMalloc(&L->tiles, np / 128 * 8192);
  if (!e) e = cudaMemset(L->tiles, 0, np / 128 * 8192);
  if (!e) e = cudaMalloc(&L->acc_n, np * sizeof(float4));
  if (!e) e = cudaMalloc(&L->acc_prev, np * sizeof(float4));
  if (!e) e = cudaMalloc(&L->dprev, np * sizeof(float4));
  if (!e) e = cudaMemset(L->dprev, 0, np * sizeof(float4));
  if (!e) e = cudaMalloc(&L->yhat, np * sizeof(float4));
  if (!e) e = cudaMalloc(&L->cy, np * sizeof(int));
  if (!e) e = cudaMalloc(&L->red, kRedBlocks * 8 * sizeof(double));
  if (!e) e = cudaMallocHost(&L->red_host, kRedBlocks * 8 * sizeof(double));
  if (e) {
    free_state(L);
    return herr_cuda(h, "learned-form scratch", e);
  }
  h->learn = L;
  return ZSPH_OK;
}

FeatOut make_feat(const Handle* h, const zsph_mlp* net) {
  FeatOut fo{};
  if (h->learn) {
    fo.acc_prev = h->learn->acc_prev;
    fo.d_out = h->learn->dprev;
  }
  feature_scales(units_of(h->kp), fo.scale);
  for (int k = 0; k < kFeat; ++k) {
    fo.mean[k] = net ? net->in_mean[k] : 0.f;
    fo.inv_std[k] = net ? net->in_inv_std[k] : 1.f;
  }
  return fo;
}

int check_buffers(Handle* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* t, const char* who) {
  if (!h) return set_herr(nullptr, ZSPH_EINVAL, std::string(who) + ": null handle");
  if (!o || !w || !t || !o->pos || !w->pos || !t->acc_drhodt || !t->index)
    return set_herr(h, ZSPH_EINVAL, std::string(who) + ": null buffer");
  if (h->kp.equations != ZSPH_EQ_DELTA)
    return set_herr(h, ZSPH_EINVAL, std::string(who) + ": the learned form uses the delta-SPH equations");
  return ZSPH_OK;
}

// host sum of the first `k` entries of kRedBlocks partial rows
void host_sums(const LearnState* L, double* s, int k) {
  for (int j = 0; j < k; ++j) s[j] = 0;
  for (int b = 0; b < kRedBlocks; ++b)
    for (int j = 0; j < k; ++j) s[j] += L->red_host[b * 8 + j];
}

}  // namespace

void learn_destroy(Handle* h) {
  if (h) {
    free_state(h->learn);
    h->learn = nullptr;
  }
}

}  // namespace zsph

using namespace zsph;

extern "C" {

int zsph_learn_feature_scales(zsph_handle_t* h, float* scale) {
  if (!h || !scale) return set_herr(h, ZSPH_EINVAL, "zsph_learn_feature_scales: null argument");
  feature_scales(units_of(h->kp), scale);
  return ZSPH_OK;
}

int zsph_learn_features(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* t,
                        float* features, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (int rc = check_buffers(h, o, w, t, "zsph_learn_features")) return rc;
  if (!features) return set_herr(h, ZSPH_EINVAL, "zsph_learn_features: null features");
  if (reinterpret_cast<uintptr_t>(features) & 15)
    return set_herr(h, ZSPH_EINVAL, "zsph_learn_features: features must be 16-byte aligned");
  if (int rc = ensure_state(h)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  h->last_stream = st;
  // tmp's acc_drhodt holds the previous corrector-stage values (old_'s order)
  LCHECK(h, "zsph_learn_features", cudaMemcpyAsync(h->learn->acc_prev, t->acc_drhodt, sizeof(float4) * h->kp.n,
                                                   cudaMemcpyDeviceToDevice, st));
  FeatOut fo = make_feat(h, nullptr);
  fo.raw = features;
  LCHECK(h, "zsph_learn_features", run_substep(h, *o, *w, *t, 1, st, nullptr, &fo));
  return ZSPH_OK;
}

int zsph_learn_collect(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* t, int nsteps,
                       int every, int capacity, int* count, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (int rc = check_buffers(h, o, w, t, "zsph_learn_collect")) return rc;
  if (nsteps < 0 || every <= 0 || capacity <= 0)
    return set_herr(h, ZSPH_EINVAL, "zsph_learn_collect: nsteps >= 0, every > 0 and capacity > 0 required");
  if (int rc = ensure_state(h)) return rc;
  LearnState* L = h->learn;
  if (L->targets_standardized)
    return set_herr(h, ZSPH_EINVAL, "zsph_learn_collect: the snapshots were already trained on; clear them first");
  if (!L->raw) {
    const size_t rows = (size_t)capacity * L->n_pad;
    cudaError_t e = cudaMalloc(&L->raw, rows * kFeat * sizeof(float));
    if (!e) e = cudaMalloc(&L->y, rows * sizeof(float4));
    if (!e) e = cudaMalloc(&L->w, rows * sizeof(float));
    if (!e) e = cudaMemset(L->raw, 0, rows * kFeat * sizeof(float));
    if (!e) e = cudaMemset(L->y, 0, rows * sizeof(float4));
    if (!e) e = cudaMemset(L->w, 0, rows * sizeof(float));
    if (e) {
      cudaFree(L->raw);
      cudaFree(L->y);
      cudaFree(L->w);
      L->raw = nullptr;
      L->y = nullptr;
      L->w = nullptr;
      return herr_cuda(h, "zsph_learn_collect: snapshot storage", e);
    }
    L->cap = capacity;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  h->last_stream = st;
  const Units u = units_of(h->kp);
  FeatOut fo = make_feat(h, nullptr);
  fo.acc_copy = L->acc_n;
  for (int s = 0; s < nsteps; ++s) {
    // a sample needs the previous step's corrector values: never the first step
    const bool sample = s > 0 && ((s + 1) % every == 0) && L->count < L->cap;
    if (!sample) {
      LCHECK(h, "zsph_learn_collect step", run_substep(h, *o, *w, *t, 1, st, nullptr, nullptr));
      LCHECK(h, "zsph_learn_collect step", run_substep(h, *o, *w, *t, 2, st, nullptr, nullptr));
      continue;
    }
    const size_t base = (size_t)L->count * L->n_pad;
    fo.raw = L->raw + base * kFeat;
    LCHECK(h, "zsph_learn_collect copy", cudaMemcpyAsync(L->acc_prev, t->acc_drhodt, sizeof(float4) * h->kp.n,
                                                         cudaMemcpyDeviceToDevice, st));
    LCHECK(h, "zsph_learn_collect predictor", run_substep(h, *o, *w, *t, 1, st, nullptr, &fo));
    LCHECK(h, "zsph_learn_collect corrector", run_substep(h, *o, *w, *t, 2, st, nullptr, nullptr));
    if (h->kp.n > 0)
      k_targets<<<(h->kp.n + 255) / 256, 256, 0, st>>>(h->kp.n, t->index,
                                                       reinterpret_cast<const float4*>(t->acc_drhodt), L->acc_n,
                                                       L->dprev, o->type, u.target_scale(), L->y + base, L->w + base);
    LCHECK(h, "zsph_learn_collect targets", cudaGetLastError());
    L->count += 1;
  }
  if (count) *count = L->count;
  return ZSPH_OK;
}

int zsph_learn_clear(zsph_handle_t* h) {
  if (!h) return set_herr(nullptr, ZSPH_EINVAL, "zsph_learn_clear: null handle");
  if (h->learn) {
    LearnState* L = h->learn;
    cudaFree(L->raw);
    cudaFree(L->y);
    cudaFree(L->w);
    L->raw = nullptr;
    L->y = nullptr;
    L->w = nullptr;
    L->cap = L->count = 0;
    L->targets_standardized = false;
  }
  return ZSPH_OK;
}

int zsph_learn_train(zsph_handle_t* h, zsph_mlp_t* net, int epochs, int batch_tiles, float lr,
                     unsigned long long seed, float val_frac, zsph_learn_train_stats_t* out, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (!h || !net) return set_herr(h, ZSPH_EINVAL, "zsph_learn_train: null argument");
  LearnState* L = h->learn;
  if (!L || L->count < 2) return set_herr(h, ZSPH_EINVAL, "zsph_learn_train: collect at least 2 snapshots first");
  if (epochs < 0 || batch_tiles <= 0 || !(lr > 0.f) || !(val_frac >= 0.f && val_frac < 1.f))
    return set_herr(h, ZSPH_EINVAL, "zsph_learn_train: bad epochs / batch_tiles / lr / val_frac");
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  h->last_stream = st;
  int s_val = (int)std::floor(val_frac * L->count + 0.5);
  if (val_frac > 0.f) s_val = std::max(1, s_val);
  const int s_train = L->count - s_val;
  if (s_train < 1) return set_herr(h, ZSPH_EINVAL, "zsph_learn_train: no training snapshots left");
  const long long rows_train = (long long)s_train * L->n_pad, rows_all = (long long)L->count * L->n_pad;
  const int tiles_all = (int)(rows_all / 128), tiles_train = (int)(rows_train / 128);

  // 1. standardization from the training snapshots (FP64 moments)
  std::vector<double> mom((size_t)kRedBlocks * (kFeat + 4) * 3);
  double* dmom = nullptr;
  LCHECK(h, "zsph_learn_train moments", cudaMalloc(&dmom, mom.size() * sizeof(double)));
  const long long chunk = (rows_train + kRedBlocks - 1) / kRedBlocks;
  k_moments<<<kRedBlocks, 64, 0, st>>>(L->raw, L->y, L->w, rows_train, chunk, dmom);
  cudaError_t e = cudaMemcpyAsync(mom.data(), dmom, mom.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  cudaFree(dmom);
  LCHECK(h, "zsph_learn_train moments", e);
  double S[kFeat + 4][3] = {};
  for (int b = 0; b < kRedBlocks; ++b)
    for (int k = 0; k < kFeat + 4; ++k)
      for (int j = 0; j < 3; ++j) S[k][j] += mom[((size_t)b * (kFeat + 4) + k) * 3 + j];
  if (!(S[0][0] > 0)) return set_herr(h, ZSPH_EINVAL, "zsph_learn_train: no fluid rows in the training snapshots");
  auto mean_std = [&](int k, float& mu, float& sd) {
    const double m = S[k][1] / S[k][0];
    const double var = std::max(0.0, S[k][2] / S[k][0] - m * m);
    mu = (float)m;
    sd = (var > 1e-30 && var > 1e-12 * m * m) ? (float)std::sqrt(var) : 1.0f;
  };
  for (int k = 0; k < kFeat; ++k) {
    float mu, sd;
    mean_std(k, mu, sd);
    net->in_mean[k] = mu;
    net->in_inv_std[k] = 1.0f / sd;
  }
  for (int k = 0; k < 4; ++k) mean_std(kFeat + k, net->out_mean[k], net->out_std[k]);

  // 2. standardized bf16 feature tiles of every snapshot; standardized targets
  unsigned char* tiles = nullptr;
  float4* yhat = nullptr;
  float* partial = nullptr;
  int* ids = nullptr;
  int* dflags = nullptr;
  double* dloss = nullptr;
  auto cleanup = [&] {
    cudaFree(tiles);
    cudaFree(yhat);
    cudaFree(partial);
    cudaFree(ids);
    cudaFree(dflags);
    cudaFree(dloss);
  };
  const int sms = std::max(1, mlp_sm_count());
  e = cudaMalloc(&tiles, (size_t)tiles_all * 8192);
  if (!e) e = cudaMalloc(&partial, (size_t)sms * ZSPH_MLP_NPARTIAL * sizeof(float));
  if (!e) e = cudaMalloc(&ids, (size_t)std::max(tiles_train, 1) * sizeof(int));
  if (!e) e = cudaMalloc(&dflags, sizeof(int));
  if (!e) e = cudaMalloc(&dloss, sizeof(double));
  if (!e) e = cudaMemset(dflags, 0, sizeof(int));
  if (!e) e = launch_mlp_pack(L->raw, (int)rows_all, net->in_mean, net->in_inv_std, tiles, st);
  if (!e && !L->targets_standardized) {
    const float4 ym = make_float4(net->out_mean[0], net->out_mean[1], net->out_mean[2], net->out_mean[3]);
    const float4 yi = make_float4(1.f / net->out_std[0], 1.f / net->out_std[1], 1.f / net->out_std[2],
                                  1.f / net->out_std[3]);
    k_standardize_targets<<<(unsigned)((rows_all + 255) / 256), 256, 0, st>>>(L->y, rows_all, ym, yi);
    e = cudaGetLastError();
    L->targets_standardized = true;
  }
  // per-tile weights (tiles without fluid rows are skipped)
  std::vector<float> wh((size_t)rows_all);
  if (!e) e = cudaMemcpyAsync(wh.data(), L->w, rows_all * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) {
    cleanup();
    return herr_cuda(h, "zsph_learn_train setup", e);
  }
  std::vector<int> train_tiles;
  std::vector<float> tile_w((size_t)tiles_all, 0.f);
  double wsum_train = 0;
  for (int tl = 0; tl < tiles_all; ++tl) {
    float s = 0;
    for (int r = 0; r < 128; ++r) s += wh[(size_t)tl * 128 + r];
    tile_w[tl] = s;
    if (tl < tiles_train && s > 0) {
      train_tiles.push_back(tl);
      wsum_train += s;
    }
  }

  // 3. Adam over shuffled tiles, cosine learning-rate decay to lr/20
  uint64_t rs = seed;
  const int nt = (int)train_tiles.size();
  const int per_epoch = (nt + batch_tiles - 1) / batch_tiles;
  const long long total_it = (long long)epochs * per_epoch;
  long long it = 0;
  float loss_first = 0.f, loss_last = 0.f;
  for (int ep = 0; ep < epochs && nt > 0; ++ep) {
    for (int k = nt - 1; k > 0; --k) std::swap(train_tiles[k], train_tiles[mix64(rs) % (uint64_t)(k + 1)]);
    e = cudaMemcpyAsync(ids, train_tiles.data(), nt * sizeof(int), cudaMemcpyHostToDevice, st);
    if (!e) e = cudaMemsetAsync(dloss, 0, sizeof(double), st);
    for (int b = 0; b < per_epoch && !e; ++b, ++it) {
      const int off = b * batch_tiles, cnt = std::min(batch_tiles, nt - off);
      double ws = 0;
      for (int k = 0; k < cnt; ++k) ws += tile_w[train_tiles[off + k]];
      const double frac = total_it > 1 ? (double)it / (double)(total_it - 1) : 0.0;
      const float lr_it = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.14159265358979 * frac))));
      int nparts = 0;
      e = launch_mlp_grad(*net, tiles, reinterpret_cast<const float*>(L->y), L->w, ids + off, cnt, (float)(1.0 / ws),
                          partial, &nparts, dflags, st);
      if (!e) {
        k_loss_accum<<<1, 32, 0, st>>>(partial, nparts, dloss);
        e = cudaGetLastError();
      }
      if (!e) e = launch_mlp_adam(*net, partial, nparts, lr_it, 0.9f, 0.999f, 1e-8f, st);
    }
    double lsum = 0;
    if (!e) e = cudaMemcpyAsync(&lsum, dloss, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) break;
    const float l = (float)(lsum / wsum_train);
    if (ep == 0) loss_first = l;
    loss_last = l;
  }
  int f = 0;
  if (!e) e = cudaMemcpy(&f, dflags, sizeof(int), cudaMemcpyDeviceToHost);
  if (e) {
    cleanup();
    return herr_cuda(h, "zsph_learn_train", e);
  }
  if (f & ZSPH_FLAG_TIMEOUT) {
    cleanup();
    return set_herr(h, ZSPH_ETIMEOUT, "zsph_learn_train: tensor-core wait timed out");
  }

  // 4. held-out snapshots: learned prediction vs predictor-stage values
  zsph_learn_train_stats_t stt{};
  stt.snapshots_train = s_train;
  stt.snapshots_val = s_val;
  stt.rows_train = (long long)(wsum_train + 0.5);
  stt.epochs = epochs;
  stt.iterations = (int)it;
  stt.loss_first = loss_first;
  stt.loss_last = loss_last;
  if (s_val > 0) {
    const long long rows_val = rows_all - rows_train;
    e = cudaMalloc(&yhat, rows_val * sizeof(float4));
    if (!e) e = launch_mlp_forward(*net, tiles + (size_t)tiles_train * 8192, (int)rows_val,
                                   reinterpret_cast<float*>(yhat), dflags, st);
    if (!e) {
      const float4 ym = make_float4(net->out_mean[0], net->out_mean[1], net->out_mean[2], net->out_mean[3]);
      const float4 ys = make_float4(net->out_std[0], net->out_std[1], net->out_std[2], net->out_std[3]);
      k_val_sums<<<kRedBlocks, kRedThreads, 0, st>>>(L->raw + (size_t)rows_train * kFeat, L->y + rows_train,
                                                     L->w + rows_train, yhat, rows_val, ym, ys, L->red);
      e = cudaGetLastError();
    }
    if (!e) e = cudaMemcpyAsync(L->red_host, L->red, kRedBlocks * 8 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) {
      cleanup();
      return herr_cuda(h, "zsph_learn_train validation", e);
    }
    double v[8];
    host_sums(L, v, 8);
    auto rl = [](double a, double b) { return (float)std::sqrt(a / std::max(b, 1e-300)); };
    stt.val_acc_rel_l2 = rl(v[0], v[1]);
    stt.val_acc_rel_l2_base = rl(v[2], v[1]);
    stt.val_acc_rel_l2_extrap = rl(v[3], v[1]);
    stt.val_drho_rel_l2 = rl(v[4], v[5]);
    stt.val_drho_rel_l2_base = rl(v[6], v[5]);
    stt.val_drho_rel_l2_extrap = rl(v[7], v[5]);
  }
  cleanup();
  stt.seconds = std::chrono::duration<float>(std::chrono::steady_clock::now() - t0).count();
  if (out) *out = stt;
  return ZSPH_OK;
}

int zsph_run_learned(zsph_handle_t* h, zsph_mlp_t* net, const zsph_ptc_t* o, const zsph_ptc_t* w,
                     const zsph_tmp_t* t, int nsteps, int judge_every, float tol, zsph_learn_run_stats_t* out,
                     void* stream) {
  return zsph_run_learned_ex(h, net, o, w, t, nsteps, judge_every, tol, ZSPH_CORR_NETWORK, nullptr, 0, out, stream);
}

int zsph_run_learned_ex(zsph_handle_t* h, zsph_mlp_t* net, const zsph_ptc_t* o, const zsph_ptc_t* w,
                        const zsph_tmp_t* t, int nsteps, int judge_every, float tol, int corrector,
                        float* err_series, int series_cap, zsph_learn_run_stats_t* out, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (int rc = check_buffers(h, o, w, t, "zsph_run_learned")) return rc;
  const bool network = corrector == ZSPH_CORR_NETWORK;
  if (corrector < ZSPH_CORR_NETWORK || corrector > ZSPH_CORR_REUSE_FRESH)
    return set_herr(h, ZSPH_EINVAL, "zsph_run_learned: unknown corrector");
  if ((network && !net) || nsteps < 0 || judge_every < 0 || !(tol > 0.f) || series_cap < 0 ||
      (series_cap > 0 && !err_series))
    return set_herr(h, ZSPH_EINVAL, "zsph_run_learned: bad network / nsteps / judge_every / tol / error series");
  if (!network && (h->kp.p.grid_factor != 1 || h->kp.scenes || h->kp.c3o || h->rigid || h->kp.stage_windows ||
                   h->kp.equations != ZSPH_EQ_DELTA))
    return set_herr(h, ZSPH_EINVAL,
                    "zsph_run_learned: the list-reuse correctors need a single scene, grid factor 1, the delta "
                    "equations, absolute positions, no rigid body and no staged windows");
  if (int rc = ensure_state(h)) return rc;
  LearnState* L = h->learn;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  h->last_stream = st;
  const Units u = units_of(h->kp);
  const float4 un = u.target_unit();
  float4 oa = make_float4(0.f, 0.f, 0.f, 0.f), ob = oa;
  if (network) {
    oa = make_float4(net->out_std[0] * un.x, net->out_std[1] * un.y, net->out_std[2] * un.z, net->out_std[3] * un.w);
    ob = make_float4(net->out_mean[0] * un.x, net->out_mean[1] * un.y, net->out_mean[2] * un.z,
                     net->out_mean[3] * un.w);
  }
  FeatOut fo = make_feat(h, net);
  fo.tiles = L->tiles;
  FeatOut fj = fo;
  fj.acc_copy = L->acc_n;
  const bool fresh = corrector == ZSPH_CORR_REUSE_FRESH;
  zsph_learn_run_stats_t rs{};
  double err_sum = 0;
  bool plain = false;
  const size_t acc_bytes = sizeof(float4) * h->kp.n;
  for (int s = 0; s < nsteps; ++s) {
    const bool judged = judge_every > 0 && (s + 1) % judge_every == 0;
    // the network's first step has no previous corrector value of its own: plain
    if (network && s == 0 && !judged) {
      LCHECK(h, "zsph_run_learned plain", run_substep(h, *o, *w, *t, 1, st, nullptr, nullptr));
      LCHECK(h, "zsph_run_learned plain", run_substep(h, *o, *w, *t, 2, st, nullptr, nullptr));
      rs.plain += 1;
      rs.steps += 1;
      continue;
    }
    if (judged) {
      if (network) {
        LCHECK(h, "zsph_run_learned copy", cudaMemcpyAsync(L->acc_prev, t->acc_drhodt, acc_bytes,
                                                           cudaMemcpyDeviceToDevice, st));
        LCHECK(h, "zsph_run_learned predictor", run_substep(h, *o, *w, *t, 1, st, nullptr, &fj));
        LCHECK(h, "zsph_run_learned network", launch_mlp_forward(*net, L->tiles, h->kp.n,
                                                                 reinterpret_cast<float*>(L->yhat), h->s.flags, st));
      } else {
        // the variant's corrector-stage values (not applied), in the predictor's order
        LCHECK(h, "zsph_run_learned predictor", run_substep(h, *o, *w, *t, 1, st, nullptr, nullptr));
        LCHECK(h, "zsph_run_learned corrector", launch_corrector_reuse(h->kp, h->s, *o, *t, fresh, 0, L->cy, st));
        LCHECK(h, "zsph_run_learned copy", cudaMemcpyAsync(L->yhat, t->acc_drhodt, acc_bytes,
                                                           cudaMemcpyDeviceToDevice, st));
      }
      LCHECK(h, "zsph_run_learned corrector", run_substep(h, *o, *w, *t, 2, st, nullptr, nullptr));
      if (network)
        k_judge<<<kRedBlocks, kRedThreads, 0, st>>>(h->kp.n, t->index,
                                                   reinterpret_cast<const float4*>(t->acc_drhodt), L->acc_n,
                                                   L->dprev, L->yhat, o->type, oa, ob, L->red);
      else
        k_judge_acc<<<kRedBlocks, kRedThreads, 0, st>>>(h->kp.n, t->index,
                                                       reinterpret_cast<const float4*>(t->acc_drhodt), L->yhat,
                                                       o->type, L->red);
      LCHECK(h, "zsph_run_learned judge", cudaGetLastError());
      LCHECK(h, "zsph_run_learned judge", cudaMemcpyAsync(L->red_host, L->red, kRedBlocks * 8 * sizeof(double),
                                                          cudaMemcpyDeviceToHost, st));
      LCHECK(h, "zsph_run_learned judge", cudaStreamSynchronize(st));
      double v[8];
      host_sums(L, v, 8);
      const float err = (float)std::sqrt(v[0] / std::max(v[1], 1e-300));
      if (rs.judged < series_cap) err_series[rs.judged] = err;
      rs.judged += 1;
      rs.err_last = err;
      rs.err_max = std::max(rs.err_max, err);
      err_sum += err;
      const bool over = !(err <= tol);
      if (over && !plain) rs.fallbacks += 1;
      plain = over;
    } else if (plain) {
      LCHECK(h, "zsph_run_learned plain", run_substep(h, *o, *w, *t, 1, st, nullptr, nullptr));
      LCHECK(h, "zsph_run_learned plain", run_substep(h, *o, *w, *t, 2, st, nullptr, nullptr));
      rs.plain += 1;
    } else if (network) {
      LCHECK(h, "zsph_run_learned copy", cudaMemcpyAsync(L->acc_prev, t->acc_drhodt, acc_bytes,
                                                         cudaMemcpyDeviceToDevice, st));
      LCHECK(h, "zsph_run_learned predictor", run_substep(h, *o, *w, *t, 1, st, nullptr, &fo));
      LCHECK(h, "zsph_run_learned corrector", launch_mlp_correct(*net, h->kp, L->tiles, *o,
                                                                 reinterpret_cast<float4*>(t->acc_drhodt), L->dprev,
                                                                 oa, ob, h->s.flags, st));
      rs.learned += 1;
    } else {
      LCHECK(h, "zsph_run_learned predictor", run_substep(h, *o, *w, *t, 1, st, nullptr, nullptr));
      LCHECK(h, "zsph_run_learned corrector", launch_corrector_reuse(h->kp, h->s, *o, *t, fresh, 2, L->cy, st));
      rs.learned += 1;
    }
    rs.steps += 1;
  }
  rs.err_mean = rs.judged ? (float)(err_sum / rs.judged) : 0.f;
  if (out) *out = rs;
  return ZSPH_OK;
}

}  // extern "C"
