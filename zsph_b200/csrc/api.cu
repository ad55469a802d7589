// C ABI of the delta-SPH step (include/zsph.h): handle, buffers, entry
// points and the step driver.
//
// The step follows single_gpu_sph_src/deltasph/main.cu:63-88 (predictor
// sub-step OLD -> NEW, corrector sub-step back into OLD) with two changes
// that keep every result where the reference leaves it:
//  * the integration of each sub-step runs in the epilogue of the governing
//    kernel and writes the integrated particle into the other buffer, so the
//    neighbours still read the unintegrated state;
//  * hence sub-step 1 ends with the predicted state in OLD, and sub-step 2
//    sorts OLD into NEW again and writes the corrected state into OLD.
// After zsph_step, old_ holds exactly what the reference's OLD buffers hold
// (state sorted by the corrector's search), tmp holds the corrector's hash,
// index, cell bounds, acc_drhodt and dofv_grandrho; new_ is scratch.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "trace.h"
#include "zsph_internal.cuh"

using namespace zsph;

namespace {

std::mutex g_err_mu;
std::string g_err;

int set_err(zsph_handle* h, int code, const std::string& msg) {
  if (h) {
    h->err = msg;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
  }
  return code;
}

int cuda_fail(zsph_handle* h, const char* where, cudaError_t e) {
  return set_err(h, e == cudaErrorMemoryAllocation ? ZSPH_ENOMEM : ZSPH_ECUDA,
                 std::string(where) + ": " + cudaGetErrorString(e));
}

#define ZCHECK(h, where, expr)                       \
  do {                                               \
    cudaError_t e_ = (expr);                         \
    if (e_ != cudaSuccess) return cuda_fail(h, where, e_); \
  } while (0)

int validate_gparam(const zsph_gpu_param_t* p, int grid_num, std::string& why) {
  if (p->ptc_num < 0) { why = "ptc_num < 0"; return 1; }
  if (p->grid_xdim <= 0 || p->grid_ydim <= 0 || p->grid_zdim <= 0) { why = "grid dimensions must be positive"; return 1; }
  const long long g = (long long)p->grid_xdim * p->grid_ydim * p->grid_zdim;
  if (g != grid_num || g > 0x7fffffffLL - 2) { why = "grid_num != grid_xdim*grid_ydim*grid_zdim"; return 1; }
  if (p->grid_hash_min != 0 || p->grid_hash_max != grid_num - 1) { why = "grid_hash_min/max must be 0 and grid_num-1"; return 1; }
  if (p->grid_factor != 1 && p->grid_factor != 2) { why = "grid_factor (grid_size_factor) must be 1 or 2"; return 1; }
  if (!(p->h > 0.0f) || !(p->grid_size > 0.0f)) { why = "h and grid_size must be positive"; return 1; }
  return 0;
}

void fill_kparams(KParams& kp, const zsph_gpu_param_t& p, int grid_num) {
  kp.p = p;
  kp.n = p.ptc_num;
  kp.G = grid_num;
  kp.XY = p.grid_xdim * p.grid_ydim;
  const double R2 = 4.0 * (double)p.h * (double)p.h;
  kp.r2lo = (float)(R2 * (1.0 - 1e-5));
  kp.r2hi = (float)(R2 * (1.0 + 1e-5));
  // The reference's test q = sqrtf(r2)/h <= 2 (IEEE sqrt and division, both
  // monotone under round-to-nearest) holds exactly for r2 <= r2max, the
  // largest float that passes it; found here with the same float operations.
  volatile float hh = p.h;
  auto pass = [&](float r2) { volatile float q = std::sqrt(r2); q = q / hh; return q <= 2.0f; };
  float t = (float)R2;
  while (pass(t)) t = std::nextafter(t, INFINITY);
  while (!pass(t)) t = std::nextafter(t, -INFINITY);
  kp.r2max = t;
  kp.inv_h = 1.0f / p.h;
  kp.inv_gs = 1.0f / p.grid_size;
  kp.c_fr = -5.0f * p.adh / p.h2;
  // Shared-memory neighbour windows (TMA) are off by default: at 112 KB per
  // 128-particle CTA they limit the pair kernels to 8 warps per SM, which
  // measured slower than L1-cached global loads at 20 warps per SM.
  const char* sw = std::getenv("ZSPH_STAGE_WINDOWS");
  kp.stage_windows = (sw && sw[0] == '1') ? 1 : 0;
  kp.equations = ZSPH_EQ_DELTA;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int check_device(zsph_handle* h) {
  int d = -1;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) return cuda_fail(h, "cudaGetDevice", e);
  if (d != h->device) return set_err(h, ZSPH_EINVAL, "the handle's device is not the current CUDA device");
  return ZSPH_OK;
}

int check_ptc(zsph_handle* h, const zsph_ptc_t* p) {
  if (!p) return set_err(h, ZSPH_EINVAL, "null particle buffers");
  if (h->kp.n > 0 && (!p->pos || !p->vel || !p->rhop || !p->tmp_pos || !p->tmp_vel || !p->tmp_rhop || !p->type ||
                      !p->table))
    return set_err(h, ZSPH_EINVAL, "a particle array pointer is null");
  if (!ptc_aligned8(*p))
    return set_err(h, ZSPH_EINVAL, "particle float arrays must start on an 8-byte boundary (cudaMalloc alignment)");
  return ZSPH_OK;
}

int check_tmp(zsph_handle* h, const zsph_tmp_t* t) {
  if (!t) return set_err(h, ZSPH_EINVAL, "null scratch buffers");
  if (h->kp.n > 0 && (!t->acc_drhodt || !t->index || !t->hash || !t->grid_start || !t->grid_end))
    return set_err(h, ZSPH_EINVAL, "a tmp array pointer is null");
  if (h->kp.n > 0 && h->kp.equations == ZSPH_EQ_DELTA && !t->dofv_grandrho)
    return set_err(h, ZSPH_EINVAL, "tmp->dofv_grandrho is null (delta equations)");
  if (h->kp.n > 0 && h->kp.equations == ZSPH_EQ_SIMPLE && !t->dofv)
    return set_err(h, ZSPH_EINVAL, "tmp->dofv is null (simple equations)");
  return ZSPH_OK;
}

void free_xfer(Xfer& x) {
  void* ptrs[] = {x.nb2,   x.nb_cnt2, x.sk,  x.sk_cnt, x.pos4,  x.xl,     x.xcnt,
                  x.hashP, x.gsP,     x.geP, x.flag,   x.fullb, x.alist, x.acount, x.stats};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  std::memset(&x, 0, sizeof x);
}

void free_scratch(Scratch& s) {
  void* ptrs[] = {s.cnt, s.cell_lb, s.key, s.ticket, s.perm, s.val, s.tile_sum, s.tile_off, s.tile_last,
                  s.tile_state, s.misc, s.big_list, s.nb, s.nb_cnt, s.wl, s.cfe, s.flags, s.sh.rec};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  free_xfer(s.xf);
  std::memset(&s, 0, sizeof s);
}

template <class T> cudaError_t dalloc(T*& p, size_t count) {
  return cudaMalloc(reinterpret_cast<void**>(&p), (count ? count : 1) * sizeof(T));
}

// List transfer constants for a skin of xfer_skin * h: the skin lists'
// outer radius, and the largest half-step displacement for which every pair
// within 2h at the predicted positions lies within that radius at the old
// ones (with margins for the FP32 rounding of both distance tests).  A
// negative bound makes every step build in full.
void xfer_params(zsph_handle* h) {
  KParams& kp = h->kp;
  const double R = (2.0 + (double)h->xfer_skin) * (double)kp.p.h;
  kp.r2skin = (float)(R * R);
  const double d = 0.5 * (std::sqrt((double)kp.r2skin) * (1.0 - 1e-6) - std::sqrt((double)kp.r2max) * (1.0 + 1e-6));
  kp.disp2max = d > 0.0 ? (float)(d * d * (1.0 - 1e-6)) : -1.0f;
}

cudaError_t xfer_alloc(zsph_handle* h) {
  Xfer& x = h->s.xf;
  if (x.nb2) return cudaSuccess;
  const size_t n = (size_t)h->kp.n, G = (size_t)h->kp.G, n32 = (n + 31) & ~(size_t)31;
  cudaError_t e = dalloc(x.nb2, (size_t)kMaxNb * n32);
  if (!e) e = dalloc(x.nb_cnt2, n);
  if (!e) e = dalloc(x.sk, (size_t)kSkinCap * n32);
  if (!e) e = dalloc(x.sk_cnt, n);
  if (!e) e = dalloc(x.pos4, n);
  if (!e) e = dalloc(x.xl, (size_t)kXtra * n);
  if (!e) e = dalloc(x.xcnt, n);
  if (!e) e = dalloc(x.hashP, n);
  if (!e) e = dalloc(x.gsP, G);
  if (!e) e = dalloc(x.geP, G);
  if (!e) e = dalloc(x.flag, 1);
  if (!e) e = dalloc(x.fullb, n);
  if (!e) e = dalloc(x.alist, n);
  if (!e) e = dalloc(x.acount, 1);
  if (!e) e = dalloc(x.stats, 3);
  if (!e) e = cudaMemset(x.nb_cnt2, 0, n ? n : 1);
  if (!e) e = cudaMemset(x.sk_cnt, 0, n ? n : 1);
  if (!e) e = cudaMemset(x.xcnt, 0, (n ? n : 1) * sizeof(int));
  if (!e) e = cudaMemset(x.flag, 0, sizeof(int));
  if (!e) e = cudaMemset(x.stats, 0, 3 * sizeof(unsigned long long));
  if (!e) e = cudaDeviceSynchronize();
  if (e) free_xfer(x);
  return e;
}

// The plain step's corrector can take the list transfer: one scene, grid
// factor 1, delta equations, absolute positions, no rigid body, global loads.
bool xfer_eligible(const zsph_handle* h) {
  const KParams& kp = h->kp;
  return h->xfer_on && h->s.xf.nb2 && kp.n >= 64 && !kp.scenes && !kp.c3o && !kp.rigid_f && !h->rigid &&
         kp.equations == ZSPH_EQ_DELTA && kp.p.grid_factor == 1 && !kp.stage_windows;
}

// One step with the list transfer: the predictor sub-step also makes skin
// lists and records the predicted positions; the corrector's lists come from
// the predictor's (or a full build, when the device flag says so).  The
// user's tmp receives both searches' outputs as in the plain step, so cell
// bounds keep the reference's stale-value behaviour; the predictor's hash and
// bounds are copied aside for the transfer.
cudaError_t xfer_step(zsph_handle* h, const zsph_ptc_t& o, const zsph_ptc_t& w, const zsph_tmp_t& t, cudaStream_t st,
                      Prof* pf) {
  const Xfer& x = h->s.xf;
  const size_t n = (size_t)h->kp.n, G = (size_t)h->kp.G;
  cudaError_t e = launch_search(h->kp, h->s, h->tiles, o, w, t, st, pf);
  if (!e) e = cudaMemsetAsync(x.flag, 0, sizeof(int), st);
  if (!e) e = cudaMemsetAsync(x.xcnt, 0, n * sizeof(int), st);
  if (!e) e = cudaMemsetAsync(x.acount, 0, sizeof(int), st);
  if (!e) e = cudaMemcpyAsync(x.hashP, t.hash, n * sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (!e) e = cudaMemcpyAsync(x.gsP, t.grid_start, G * sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (!e) e = cudaMemcpyAsync(x.geP, t.grid_end, G * sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (!e) e = launch_xfer_pred_lists(h->kp, h->s, w, t, st, pf);
  KParams kp1 = h->kp;
  kp1.xfer_pos4 = x.pos4;
  kp1.xfer_flag = x.flag;
  if (!e) e = launch_governing(kp1, h->s, w, t, 1, o, st, pf);
  if (!e) e = launch_search(h->kp, h->s, h->tiles, o, w, t, st, pf);
  if (!e) e = launch_xfer_corr_lists(h->kp, h->s, w, t, st, pf);
  Scratch s2 = h->s;
  s2.nb = x.nb2;
  s2.nb_cnt = x.nb_cnt2;
  if (!e) e = launch_governing(h->kp, s2, w, t, 2, o, st, pf);
  return e;
}

// One sub-step of the fused path: search `from` into `to`, boundary on `to`,
// governing + integration of `to` written into `from`.
cudaError_t substep(zsph_handle* h, const zsph_ptc_t& from, const zsph_ptc_t& to, const zsph_tmp_t& t, int mode,
                    cudaStream_t st, Prof* pf, const FeatOut* feat = nullptr) {
  cudaError_t e;
  {
    const TraceRange r("search");
    e = launch_search(h->kp, h->s, h->tiles, from, to, t, st, pf);
  }
  if (!e) {
    const TraceRange r("boundary");
    e = launch_boundary(h->kp, h->s, to, t, st, pf);
  }
  if (!e) {
    const TraceRange r("governing");
    e = launch_governing(h->kp, h->s, to, t, mode, from, st, pf, feat);
  }
  if (!e && h->rigid && mode != 0) e = rigid_substep(h, from, to, t, mode, st);
  return e;
}

// the batched form's persistent kernel over nsteps steps (barrier words zeroed first)
cudaError_t persistent_steps(zsph_handle* h, const zsph_ptc_t& o, const zsph_ptc_t& w, const zsph_tmp_t& t,
                             int nsteps, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(h->pbar, 0, 2 * sizeof(unsigned), st);
  if (!e) e = launch_batch_persistent(h->kp, h->s, o, w, t, h->pbar, nsteps, h->spin_limit, 0, st);
  return e;
}

cudaError_t step_launches(zsph_handle* h, const zsph_ptc_t& o, const zsph_ptc_t& w, const zsph_tmp_t& t,
                          cudaStream_t st, Prof* pf = nullptr) {
  if (h->persistent && !pf) return persistent_steps(h, o, w, t, 1, st);
  if (xfer_eligible(h)) return xfer_step(h, o, w, t, st, pf);
  cudaError_t e = substep(h, o, w, t, 1, st, pf);
  if (!e) e = substep(h, o, w, t, 2, st, pf);
  return e;
}

}  // namespace

namespace zsph {
void record_library_error(const std::string& msg) { set_err(nullptr, ZSPH_OK, msg); }
cudaError_t run_substep(Handle* h, const zsph_ptc_t& from, const zsph_ptc_t& to, const zsph_tmp_t& t, int mode,
                        cudaStream_t st, Prof* pf, const FeatOut* feat) {
  return substep(static_cast<zsph_handle*>(h), from, to, t, mode, st, pf, feat);
}
}  // namespace zsph

extern "C" {

const char* zsph_version(void) { return "zsph-b200 0.1 (sm_100a)"; }

int zsph_last_error(zsph_handle_t* h, char* buf, int len) {
  std::string m;
  if (h) {
    m = h->err;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mu);
    m = g_err;
  }
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", m.c_str());
  return (int)m.size();
}

int zsph_alloc_ptc(zsph_ptc_t* p, int n) {
  if (!p || n < 0) return set_err(nullptr, ZSPH_EINVAL, "zsph_alloc_ptc: bad argument");
  std::memset(p, 0, sizeof *p);
  const size_t N = (size_t)(n ? n : 1);
  float** f3[] = {&p->pos, &p->vel, &p->tmp_pos, &p->tmp_vel};
  for (float** q : f3) {
    ZCHECK(nullptr, "zsph_alloc_ptc", cudaMalloc(reinterpret_cast<void**>(q), N * 3 * sizeof(float)));
    ZCHECK(nullptr, "zsph_alloc_ptc", cudaMemset(*q, 0, N * 3 * sizeof(float)));
  }
  float** f2[] = {&p->rhop, &p->tmp_rhop};
  for (float** q : f2) {
    ZCHECK(nullptr, "zsph_alloc_ptc", cudaMalloc(reinterpret_cast<void**>(q), N * 2 * sizeof(float)));
    ZCHECK(nullptr, "zsph_alloc_ptc", cudaMemset(*q, 0, N * 2 * sizeof(float)));
  }
  int** i1[] = {&p->type, &p->table};
  for (int** q : i1) {
    ZCHECK(nullptr, "zsph_alloc_ptc", cudaMalloc(reinterpret_cast<void**>(q), N * sizeof(int)));
    ZCHECK(nullptr, "zsph_alloc_ptc", cudaMemset(*q, 0, N * sizeof(int)));
  }
  return ZSPH_OK;
}

int zsph_free_ptc(zsph_ptc_t* p) {
  if (!p) return ZSPH_EINVAL;
  void* ptrs[] = {p->pos, p->vel, p->rhop, p->tmp_pos, p->tmp_vel, p->tmp_rhop, p->type, p->table};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  std::memset(p, 0, sizeof *p);
  return ZSPH_OK;
}

int zsph_alloc_tmp(zsph_tmp_t* t, int n, int grid_num) {
  if (!t || n < 0 || grid_num <= 0) return set_err(nullptr, ZSPH_EINVAL, "zsph_alloc_tmp: bad argument");
  std::memset(t, 0, sizeof *t);
  const size_t N = (size_t)(n ? n : 1), G = (size_t)grid_num;
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->acc_drhodt), N * 4 * sizeof(float)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->dofv_grandrho), N * 4 * sizeof(float)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->dofv), N * sizeof(float)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->index), N * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->hash), N * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->grid_start), G * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMalloc(reinterpret_cast<void**>(&t->grid_end), G * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->acc_drhodt, 0, N * 4 * sizeof(float)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->dofv_grandrho, 0, N * 4 * sizeof(float)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->dofv, 0, N * sizeof(float)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->index, 0, N * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->hash, 0, N * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->grid_start, 0, G * sizeof(int)));
  ZCHECK(nullptr, "zsph_alloc_tmp", cudaMemset(t->grid_end, 0, G * sizeof(int)));
  return ZSPH_OK;
}

int zsph_free_tmp(zsph_tmp_t* t) {
  if (!t) return ZSPH_EINVAL;
  void* ptrs[] = {t->acc_drhodt, t->dofv_grandrho, t->dofv, t->index, t->hash, t->grid_start, t->grid_end};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  std::memset(t, 0, sizeof *t);
  return ZSPH_OK;
}

int zsph_cpu_to_gpu(const zsph_ptc_t* p, const zsph_tmp_t* t, const float* pos, const float* vel, const float* rhop,
                    const int* type, const int* table, const float* acc, int n, void* stream) {
  if (!p || !t || n < 0) return set_err(nullptr, ZSPH_EINVAL, "zsph_cpu_to_gpu: bad argument");
  cudaStream_t st = as_stream(stream);
  const size_t N = (size_t)n;
  if (pos) ZCHECK(nullptr, "cpu_to_gpu pos", cudaMemcpyAsync(p->pos, pos, N * 12, cudaMemcpyHostToDevice, st));
  if (vel) ZCHECK(nullptr, "cpu_to_gpu vel", cudaMemcpyAsync(p->vel, vel, N * 12, cudaMemcpyHostToDevice, st));
  if (rhop) ZCHECK(nullptr, "cpu_to_gpu rhop", cudaMemcpyAsync(p->rhop, rhop, N * 8, cudaMemcpyHostToDevice, st));
  if (type) ZCHECK(nullptr, "cpu_to_gpu type", cudaMemcpyAsync(p->type, type, N * 4, cudaMemcpyHostToDevice, st));
  if (table) ZCHECK(nullptr, "cpu_to_gpu table", cudaMemcpyAsync(p->table, table, N * 4, cudaMemcpyHostToDevice, st));
  if (acc)
    ZCHECK(nullptr, "cpu_to_gpu acc", cudaMemcpyAsync(t->acc_drhodt, acc, N * 16, cudaMemcpyHostToDevice, st));
  else
    ZCHECK(nullptr, "cpu_to_gpu acc", cudaMemsetAsync(t->acc_drhodt, 0, N * 16, st));
  ZCHECK(nullptr, "cpu_to_gpu sync", cudaStreamSynchronize(st));
  return ZSPH_OK;
}

int zsph_gpu_to_cpu(const zsph_ptc_t* p, const zsph_tmp_t* t, float* pos, float* vel, float* rhop, int* type,
                    int* table, float* acc, int* hash, int n, void* stream) {
  if (!p || !t || n < 0) return set_err(nullptr, ZSPH_EINVAL, "zsph_gpu_to_cpu: bad argument");
  cudaStream_t st = as_stream(stream);
  const size_t N = (size_t)n;
  if (pos) ZCHECK(nullptr, "gpu_to_cpu pos", cudaMemcpyAsync(pos, p->pos, N * 12, cudaMemcpyDeviceToHost, st));
  if (vel) ZCHECK(nullptr, "gpu_to_cpu vel", cudaMemcpyAsync(vel, p->vel, N * 12, cudaMemcpyDeviceToHost, st));
  if (rhop) ZCHECK(nullptr, "gpu_to_cpu rhop", cudaMemcpyAsync(rhop, p->rhop, N * 8, cudaMemcpyDeviceToHost, st));
  if (type) ZCHECK(nullptr, "gpu_to_cpu type", cudaMemcpyAsync(type, p->type, N * 4, cudaMemcpyDeviceToHost, st));
  if (table) ZCHECK(nullptr, "gpu_to_cpu table", cudaMemcpyAsync(table, p->table, N * 4, cudaMemcpyDeviceToHost, st));
  if (acc) ZCHECK(nullptr, "gpu_to_cpu acc", cudaMemcpyAsync(acc, t->acc_drhodt, N * 16, cudaMemcpyDeviceToHost, st));
  if (hash) ZCHECK(nullptr, "gpu_to_cpu hash", cudaMemcpyAsync(hash, t->hash, N * 4, cudaMemcpyDeviceToHost, st));
  ZCHECK(nullptr, "gpu_to_cpu sync", cudaStreamSynchronize(st));
  return ZSPH_OK;
}

int zsph_create(const zsph_gpu_param_t* gp, int grid_num, zsph_handle_t** out) {
  if (!gp || !out) return set_err(nullptr, ZSPH_EINVAL, "zsph_create: null argument");
  *out = nullptr;
  std::string why;
  if (validate_gparam(gp, grid_num, why)) return set_err(nullptr, ZSPH_EINVAL, "zsph_create: " + why);
  zsph_handle* h = new zsph_handle();
  std::memset(&h->s, 0, sizeof h->s);
  fill_kparams(h->kp, *gp, grid_num);
  cudaError_t e = cudaGetDevice(&h->device);
  if (!e) e = init_pair_kernels();
  const size_t n = (size_t)gp->ptc_num, G = (size_t)grid_num;
  h->tiles = (grid_num + kScanTile - 1) / kScanTile;
  Scratch& s = h->s;
  if (!e) e = dalloc(s.cnt, G);
  if (!e) e = dalloc(s.cell_lb, G + 1);
  if (!e) e = dalloc(s.key, n);
  if (!e) e = dalloc(s.ticket, n);
  if (!e) e = dalloc(s.perm, n);
  if (!e) e = dalloc(s.val, n);
  if (!e) e = dalloc(s.tile_sum, (size_t)h->tiles);
  if (!e) e = dalloc(s.tile_off, (size_t)h->tiles);
  if (!e) e = dalloc(s.tile_last, (size_t)h->tiles);
  if (!e) e = dalloc(s.tile_state, (size_t)h->tiles);
  if (!e) e = dalloc(s.misc, kMiscWords);
  if (!e) e = dalloc(s.big_list, (size_t)kBigListCap);
  if (!e) e = dalloc(s.nb, (size_t)kMaxNb * ((n + 31) & ~(size_t)31));  // whole 32-particle list groups
  if (!e) e = dalloc(s.nb_cnt, n);
  if (!e) e = dalloc(s.wl, n);
  if (!e) e = dalloc(s.cfe, G);
  if (!e) e = dalloc(s.flags, 1);
  if (!e) e = dalloc(s.sh.rec, 2 * (size_t)n);
  if (!e) e = cudaMemset(s.cnt, 0, G * sizeof(int));
  if (!e) e = cudaMemset(s.cfe, 0, G * sizeof(int));
  if (!e) e = cudaMemset(s.misc, 0, kMiscWords * sizeof(int));
  if (!e) e = cudaMemset(s.tile_state, 0, (size_t)h->tiles * sizeof(unsigned long long));
  if (!e) e = cudaMemset(s.flags, 0, sizeof(int));
  if (!e) e = cudaMemset(s.nb_cnt, 0, n ? n : 1);
  if (!e) e = cudaDeviceSynchronize();
  if (!e) xfer_params(h);  // the list transfer stays off (and unallocated) until zsph_set_list_transfer
  if (e) {
    const int code = cuda_fail(nullptr, "zsph_create", e);
    free_scratch(h->s);
    delete h;
    return code;
  }
  *out = h;
  return ZSPH_OK;
}

int zsph_create_batch(const zsph_gpu_param_t* scenes, const int* grid_num, int nscenes, zsph_handle_t** out) {
  if (!scenes || !grid_num || !out || nscenes <= 0) return set_err(nullptr, ZSPH_EINVAL, "zsph_create_batch: bad argument");
  *out = nullptr;
  std::vector<SceneDev> tab((size_t)nscenes);
  std::vector<int> base(2 * (size_t)nscenes + 2, 0);
  long long N = 0, G = 0;
  for (int s = 0; s < nscenes; ++s) {
    std::string why;
    if (validate_gparam(&scenes[s], grid_num[s], why))
      return set_err(nullptr, ZSPH_EINVAL, "zsph_create_batch: scene " + std::to_string(s) + ": " + why);
    if (scenes[s].grid_factor != 1)
      return set_err(nullptr, ZSPH_EINVAL, "zsph_create_batch: every scene needs grid_size_factor 1");
    KParams k{};
    fill_kparams(k, scenes[s], grid_num[s]);
    SceneDev& d = tab[s];
    d.p = scenes[s];
    d.p.grid_hash_min = (int)G;  // the scene's cells in batch coordinates
    d.p.grid_hash_max = (int)(G + grid_num[s] - 1);
    d.XY = k.XY;
    d.r2lo = k.r2lo;
    d.r2hi = k.r2hi;
    d.r2max = k.r2max;
    d.inv_h = k.inv_h;
    d.inv_gs = k.inv_gs;
    d.c_fr = k.c_fr;
    base[s] = (int)N;
    base[nscenes + 1 + s] = (int)G;
    N += scenes[s].ptc_num;
    G += grid_num[s];
    if (N > 0x7fffffffLL / kMaxNb || G > 0x7fffffffLL - 2)
      return set_err(nullptr, ZSPH_EINVAL, "zsph_create_batch: batch too large");
  }
  base[nscenes] = (int)N;
  base[2 * nscenes + 1] = (int)G;
  // the handle sees one scene of N particles over a 1-D grid of G cells
  zsph_gpu_param_t all = scenes[0];
  all.ptc_num = (int)N;
  all.grid_xdim = (int)G;
  all.grid_ydim = 1;
  all.grid_zdim = 1;
  all.grid_hash_min = 0;
  all.grid_hash_max = (int)G - 1;
  zsph_handle_t* h = nullptr;
  if (int rc = zsph_create(&all, (int)G, &h)) return rc;
  cudaError_t e = cudaMalloc(&h->scene_tab, sizeof(SceneDev) * nscenes);
  if (!e) e = cudaMalloc(&h->scene_base, sizeof(int) * base.size());
  if (!e) e = cudaMemcpy(h->scene_tab, tab.data(), sizeof(SceneDev) * nscenes, cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(h->scene_base, base.data(), sizeof(int) * base.size(), cudaMemcpyHostToDevice);
  if (e) {
    const int code = cuda_fail(nullptr, "zsph_create_batch", e);
    zsph_destroy(h);
    return code;
  }
  h->kp.scenes = h->scene_tab;
  h->kp.scene_pbase = h->scene_base;
  h->kp.scene_cbase = h->scene_base + nscenes + 1;
  h->kp.nscenes = nscenes;
  h->kp.stage_windows = 0;
  *out = h;
  return ZSPH_OK;
}

void zsph_destroy(zsph_handle_t* h) {
  if (!h) return;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->graph_stream) cudaStreamDestroy(h->graph_stream);
  cudaFree(h->pbar);
  learn_destroy(h);
  precise_destroy(h);
  cudaFree(h->scene_tab);
  cudaFree(h->scene_base);
  free_scratch(h->s);
  delete h;
}

int zsph_set_params(zsph_handle_t* h, const zsph_gpu_param_t* gp) {
  if (!h || !gp) return set_err(h, ZSPH_EINVAL, "zsph_set_params: null argument");
  std::string why;
  if (validate_gparam(gp, h->kp.G, why)) return set_err(h, ZSPH_EINVAL, "zsph_set_params: " + why);
  if (gp->ptc_num != h->kp.n || gp->grid_xdim != h->kp.p.grid_xdim || gp->grid_ydim != h->kp.p.grid_ydim ||
      gp->grid_zdim != h->kp.p.grid_zdim)
    return set_err(h, ZSPH_EINVAL, "zsph_set_params: particle count and grid must not change");
  const int eq = h->kp.equations;
  fill_kparams(h->kp, *gp, h->kp.G);
  h->kp.equations = eq;
  xfer_params(h);
  if (h->graph) {  // kernel arguments changed: re-capture on the next zsph_run
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return ZSPH_OK;
}

int zsph_set_equations(zsph_handle_t* h, int equations) {
  if (!h) return set_err(nullptr, ZSPH_EINVAL, "null handle");
  if (equations != ZSPH_EQ_DELTA && equations != ZSPH_EQ_SIMPLE)
    return set_err(h, ZSPH_EINVAL, "zsph_set_equations: ZSPH_EQ_DELTA or ZSPH_EQ_SIMPLE");
  if (h->kp.equations != equations && h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->kp.equations = equations;
  return ZSPH_OK;
}

#define ENTRY_CHECKS(h)                                         \
  const zsph::TraceRange trace_range_(__func__);               \
  if (!h) return set_err(nullptr, ZSPH_EINVAL, "null handle"); \
  if (int rc_ = check_device(h)) return rc_;

int zsph_hash(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, ptc)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_hash", launch_hash(h->kp, h->s.flags, *ptc, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_sort_index(zsph_handle_t* h, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_sort_index", launch_sort_index(h->kp, h->s, h->tiles, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_sort_data(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, o)) return rc;
  if (int rc = check_ptc(h, w)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_sort_data", launch_sort_data(h->kp, h->s, h->tiles, *o, *w, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_neighbor_search(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp,
                         void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, o)) return rc;
  if (int rc = check_ptc(h, w)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_neighbor_search", launch_search(h->kp, h->s, h->tiles, *o, *w, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_boundary(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, ptc)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_boundary pack", launch_pack(h->kp, h->s, *ptc, *tmp, h->last_stream));
  ZCHECK(h, "zsph_boundary", launch_boundary(h->kp, h->s, *ptc, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_governing(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, ptc)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_governing pack", launch_pack(h->kp, h->s, *ptc, *tmp, h->last_stream));
  ZCHECK(h, "zsph_governing list", launch_nblist(h->kp, h->s, *ptc, *tmp, h->last_stream));
  ZCHECK(h, "zsph_governing", launch_governing(h->kp, h->s, *ptc, *tmp, 0, *ptc, h->last_stream));
  return ZSPH_OK;
}

int zsph_prediction(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, ptc)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_prediction", launch_integrate(h->kp, h->s, *ptc, *tmp, 0, h->last_stream));
  return ZSPH_OK;
}

int zsph_correction(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, ptc)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_correction", launch_integrate(h->kp, h->s, *ptc, *tmp, 1, h->last_stream));
  return ZSPH_OK;
}

int zsph_step(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, o)) return rc;
  if (int rc = check_ptc(h, w)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_step", step_launches(h, *o, *w, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_run(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp, int nsteps,
             void* stream) {
  ENTRY_CHECKS(h);
  if (nsteps < 0) return set_err(h, ZSPH_EINVAL, "zsph_run: nsteps < 0");
  if (int rc = check_ptc(h, o)) return rc;
  if (int rc = check_ptc(h, w)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  if (nsteps == 0 || h->kp.n == 0) return ZSPH_OK;
  if (h->persistent && h->persist_graph < 0) {  // graph capture refused: one launch for all steps
    ZCHECK(h, "zsph_run persistent", persistent_steps(h, *o, *w, *tmp, nsteps, h->last_stream));
    return ZSPH_OK;
  }
  const bool same = h->graph && !std::memcmp(&h->graph_old, o, sizeof *o) &&
                    !std::memcmp(&h->graph_new, w, sizeof *w) && !std::memcmp(&h->graph_tmp, tmp, sizeof *tmp);
  if (!same) {
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    if (!h->graph_stream) ZCHECK(h, "zsph_run stream", cudaStreamCreateWithFlags(&h->graph_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    ZCHECK(h, "zsph_run capture", cudaStreamBeginCapture(h->graph_stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    for (int k = 0; k < h->graph_steps && !le; ++k) le = step_launches(h, *o, *w, *tmp, h->graph_stream);
    cudaError_t ce = cudaStreamEndCapture(h->graph_stream, &g);
    if (h->persistent && (le || ce)) {  // a cooperative launch the capture does not take: run it directly
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      h->persist_graph = -1;
      ZCHECK(h, "zsph_run persistent", persistent_steps(h, *o, *w, *tmp, nsteps, h->last_stream));
      return ZSPH_OK;
    }
    if (le) { if (g) cudaGraphDestroy(g); return cuda_fail(h, "zsph_run launch", le); }
    if (ce) { if (g) cudaGraphDestroy(g); return cuda_fail(h, "zsph_run end capture", ce); }
    cudaError_t ie = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie && h->persistent) {
      cudaGetLastError();
      h->graph = nullptr;
      h->persist_graph = -1;
      ZCHECK(h, "zsph_run persistent", persistent_steps(h, *o, *w, *tmp, nsteps, h->last_stream));
      return ZSPH_OK;
    }
    if (ie) { h->graph = nullptr; return cuda_fail(h, "zsph_run instantiate", ie); }
    if (h->persistent) h->persist_graph = 1;
    h->graph_old = *o;
    h->graph_new = *w;
    h->graph_tmp = *tmp;
  }
  const int gs = std::max(h->graph_steps, 1);
  for (int k = 0; k < nsteps / gs; ++k) ZCHECK(h, "zsph_run launch", cudaGraphLaunch(h->graph, h->last_stream));
  for (int k = 0; k < nsteps % gs; ++k) ZCHECK(h, "zsph_run step", step_launches(h, *o, *w, *tmp, h->last_stream));
  return ZSPH_OK;
}

int zsph_autotune(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp, int trial_steps,
                  zsph_tune_t* out, void* stream) {
  ENTRY_CHECKS(h);
  if (trial_steps <= 0) return set_err(h, ZSPH_EINVAL, "zsph_autotune: trial_steps must be positive");
  if (int rc = check_ptc(h, o)) return rc;
  if (int rc = check_ptc(h, w)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  if (h->rigid) return set_err(h, ZSPH_EINVAL, "zsph_autotune: detach the rigid body first");
  cudaStream_t st = as_stream(stream);
  h->last_stream = st;
  const size_t n = (size_t)h->kp.n, G = (size_t)h->kp.G;
  // the state a step reads or carries over: old_, the cell bounds, the precision cells
  struct Piece { void* p; size_t bytes; };
  const Piece pieces[] = {{o->pos, 12 * n}, {o->vel, 12 * n}, {o->rhop, 8 * n}, {o->tmp_pos, 12 * n},
                          {o->tmp_vel, 12 * n}, {o->tmp_rhop, 8 * n}, {o->type, 4 * n}, {o->table, 4 * n},
                          {tmp->acc_drhodt, 16 * n}, {tmp->dofv_grandrho, 16 * n}, {tmp->grid_start, 4 * G},
                          {tmp->grid_end, 4 * G}, {h->kp.c3o, h->kp.c3o ? 4 * n : 0}};
  size_t total = 0;
  for (const Piece& pc : pieces) total += pc.p ? pc.bytes : 0;
  unsigned char* save = nullptr;
  ZCHECK(h, "zsph_autotune save", cudaMalloc(&save, total ? total : 1));
  auto copy = [&](bool to_save) -> cudaError_t {
    size_t off = 0;
    for (const Piece& pc : pieces) {
      if (!pc.p || !pc.bytes) continue;
      cudaError_t e = to_save ? cudaMemcpyAsync(save + off, pc.p, pc.bytes, cudaMemcpyDeviceToDevice, st)
                              : cudaMemcpyAsync(pc.p, save + off, pc.bytes, cudaMemcpyDeviceToDevice, st);
      if (e) return e;
      off += pc.bytes;
    }
    return cudaSuccess;
  };
  const int cws[] = {2, 4}, segss[] = {2, 3, 4}, minbs[] = {1, 6, 8}, spgs[] = {1, 4};
  zsph_tune_t best{};
  best.ms_per_step = 1e30f;
  float ms_default = 0.f;
  int count = 0;
  const KParams kp0 = h->kp;
  const int gs0 = h->graph_steps;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = copy(true);
  if (!e) e = cudaEventCreate(&e0);
  if (!e) e = cudaEventCreate(&e1);
  for (int cw : cws)
    for (int sg : segss)
    for (int mb : minbs)
      for (int spg : spgs) {
        if (e) break;
        h->kp.tune_cw = cw;
        h->kp.tune_segs = sg;
        h->kp.tune_minb = mb;
        h->graph_steps = spg;
        if (h->graph) {
          cudaGraphExecDestroy(h->graph);
          h->graph = nullptr;
        }
        e = copy(false);
        if (!e && zsph_run(h, o, w, tmp, spg, stream) != ZSPH_OK) e = cudaErrorUnknown;  // capture + warm-up
        const int launches = (trial_steps + spg - 1) / spg;
        if (!e) e = cudaEventRecord(e0, st);
        if (!e && zsph_run(h, o, w, tmp, launches * spg, stream) != ZSPH_OK) e = cudaErrorUnknown;
        if (!e) e = cudaEventRecord(e1, st);
        if (!e) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (!e) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e) break;
        ms /= (float)(launches * spg);
        ++count;
        if (cw == 2 && sg == 4 && mb == 1 && spg == 1) ms_default = ms;  // the untuned shapes
        if (ms < best.ms_per_step) {
          best.ms_per_step = ms;
          best.list_cells_per_cta = cw;
          best.list_segments = sg;
          best.governing_min_ctas = mb;
          best.steps_per_graph = spg;
        }
      }
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaError_t re = copy(false);
  if (!re) re = cudaStreamSynchronize(st);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(save);
  if (e || re || count == 0) {
    h->kp = kp0;
    h->graph_steps = gs0;
    if (e == cudaErrorUnknown) return ZSPH_ECUDA;  // the run's own error is in zsph_last_error
    return cuda_fail(h, "zsph_autotune", e ? e : re);
  }
  h->kp.tune_cw = best.list_cells_per_cta;
  h->kp.tune_segs = best.list_segments;
  h->kp.tune_minb = best.governing_min_ctas;
  h->graph_steps = best.steps_per_graph;
  best.candidates = count;
  best.ms_default = ms_default;
  if (out) *out = best;
  return ZSPH_OK;
}

int zsph_set_launch_shapes(zsph_handle_t* h, const zsph_tune_t* shapes) {
  if (!h) return set_err(nullptr, ZSPH_EINVAL, "null handle");
  if (!shapes) return set_err(h, ZSPH_EINVAL, "zsph_set_launch_shapes: null shapes");
  const int cw = shapes->list_cells_per_cta, mb = shapes->governing_min_ctas, spg = shapes->steps_per_graph;
  if (cw != 0 && cw != 2 && cw != 4)
    return set_err(h, ZSPH_EINVAL, "zsph_set_launch_shapes: list_cells_per_cta must be 0 (default), 2 or 4");
  if (mb != 0 && mb != 1 && mb != 6 && mb != 8)
    return set_err(h, ZSPH_EINVAL, "zsph_set_launch_shapes: governing_min_ctas must be 0 (default), 1, 6 or 8");
  if (spg != 0 && spg != 1 && spg != 4)
    return set_err(h, ZSPH_EINVAL, "zsph_set_launch_shapes: steps_per_graph must be 0 (default), 1 or 4");
  const int sg = shapes->list_segments;
  if (sg != 0 && sg != 2 && sg != 3 && sg != 4)
    return set_err(h, ZSPH_EINVAL, "zsph_set_launch_shapes: list_segments must be 0 (default), 2, 3 or 4");
  if (h->graph) {  // captured with the previous shapes
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->kp.tune_cw = cw;
  h->kp.tune_segs = sg;
  h->kp.tune_minb = mb;
  h->graph_steps = spg ? spg : 1;
  return ZSPH_OK;
}

int zsph_set_list_transfer(zsph_handle_t* h, int on, float skin) {
  ENTRY_CHECKS(h);
  if (!(skin >= 0.0f && skin <= 1.0f))
    return set_err(h, ZSPH_EINVAL, "zsph_set_list_transfer: skin must be in [0, 1] (a multiple of h)");
  if (on) ZCHECK(h, "zsph_set_list_transfer", xfer_alloc(h));
  if (h->graph) {  // captured with the other step form
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->xfer_on = on ? 1 : 0;
  h->xfer_skin = skin;
  xfer_params(h);
  return ZSPH_OK;
}

int zsph_list_transfer_info(zsph_handle_t* h, long long* transferred, long long* full_builds,
                            long long* full_searches) {
  ENTRY_CHECKS(h);
  unsigned long long v[3] = {0, 0, 0};
  if (h->s.xf.stats)
    ZCHECK(h, "zsph_list_transfer_info", cudaMemcpy(v, h->s.xf.stats, sizeof v, cudaMemcpyDeviceToHost));
  if (transferred) *transferred = (long long)v[0];
  if (full_builds) *full_builds = (long long)v[1];
  if (full_searches) *full_searches = (long long)v[2];
  return ZSPH_OK;
}

int zsph_set_batch_persistent(zsph_handle_t* h, int on) {
  ENTRY_CHECKS(h);
  if (on) {
    if (!h->kp.scenes) return set_err(h, ZSPH_EINVAL, "zsph_set_batch_persistent: a batched handle is required");
    int grid = 0;
    ZCHECK(h, "zsph_set_batch_persistent", persistent_grid(&grid));
    if (!h->pbar) ZCHECK(h, "zsph_set_batch_persistent", cudaMalloc(&h->pbar, 2 * sizeof(unsigned)));
    ZCHECK(h, "zsph_set_batch_persistent", cudaMemset(h->pbar, 0, 2 * sizeof(unsigned)));
  }
  h->persistent = on ? 1 : 0;
  h->persist_graph = 0;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return ZSPH_OK;
}

int zsph_persistent_info(zsph_handle_t* h, int* ctas, int* graph) {
  ENTRY_CHECKS(h);
  int g = 0;
  ZCHECK(h, "zsph_persistent_info", persistent_grid(&g));
  if (ctas) *ctas = g;
  if (graph) *graph = h->persist_graph;
  return ZSPH_OK;
}

int zsph_persistent_barrier_test(zsph_handle_t* h, int spin_limit, void* stream) {
  ENTRY_CHECKS(h);
  if (!h->persistent) return set_err(h, ZSPH_EINVAL, "zsph_persistent_barrier_test: persistent mode is off");
  if (spin_limit <= 0) return set_err(h, ZSPH_EINVAL, "zsph_persistent_barrier_test: spin_limit must be positive");
  cudaStream_t st = as_stream(stream);
  h->last_stream = st;
  ZCHECK(h, "zsph_persistent_barrier_test", cudaMemsetAsync(h->pbar, 0, 2 * sizeof(unsigned), st));
  ZCHECK(h, "zsph_persistent_barrier_test",
         launch_batch_persistent(h->kp, h->s, zsph_ptc_t{}, zsph_ptc_t{}, zsph_tmp_t{}, h->pbar, 0,
                                 (unsigned)spin_limit, 1, st));
  ZCHECK(h, "zsph_persistent_barrier_test", cudaStreamSynchronize(st));
  ZCHECK(h, "zsph_persistent_barrier_test", cudaMemsetAsync(h->pbar, 0, 2 * sizeof(unsigned), st));
  return zsph_status(h, nullptr, 1);
}

int zsph_status(zsph_handle_t* h, int* flags, int clear) {
  if (!h) return set_err(nullptr, ZSPH_EINVAL, "null handle");
  if (int rc = check_device(h)) return rc;
  ZCHECK(h, "zsph_status sync", cudaStreamSynchronize(h->last_stream));
  ZCHECK(h, "zsph_status last error", cudaGetLastError());
  int f = 0;
  ZCHECK(h, "zsph_status read", cudaMemcpy(&f, h->s.flags, sizeof f, cudaMemcpyDeviceToHost));
  if (clear) ZCHECK(h, "zsph_status clear", cudaMemset(h->s.flags, 0, sizeof(int)));
  if (flags) *flags = f;
  if (f & ZSPH_FLAG_NAN) return set_err(h, ZSPH_ENAN, "non-finite acceleration or density");
  if (f & ZSPH_FLAG_TIMEOUT) return set_err(h, ZSPH_ETIMEOUT, "a bounded wait in a kernel ran out");
  if (f & ZSPH_FLAG_BAD_KEY) return set_err(h, ZSPH_EINVAL, "zsph_sort_index: key outside [0, grid_num)");
  return ZSPH_OK;
}

int zsph_neighbor_counts(zsph_handle_t* h, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int* nb_boundary,
                         int* nb_governing, void* stream) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, ptc)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  h->last_stream = as_stream(stream);
  ZCHECK(h, "zsph_neighbor_counts pack", launch_pack(h->kp, h->s, *ptc, *tmp, h->last_stream));
  ZCHECK(h, "zsph_neighbor_counts list", launch_nblist(h->kp, h->s, *ptc, *tmp, h->last_stream));
  ZCHECK(h, "zsph_neighbor_counts", launch_nb_counts(h->kp, h->s, nb_boundary, nb_governing, h->last_stream));
  return ZSPH_OK;
}

int zsph_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
  if (kind < 1 || kind > 3) return set_err(nullptr, ZSPH_EINVAL, "zsph_memcpy: kind must be 1, 2 or 3");
  if (bytes == 0) return ZSPH_OK;
  cudaStream_t st = as_stream(stream);
  ZCHECK(nullptr, "zsph_memcpy", cudaMemcpyAsync(dst, src, bytes, (cudaMemcpyKind)kind, st));
  ZCHECK(nullptr, "zsph_memcpy sync", cudaStreamSynchronize(st));
  return ZSPH_OK;
}

int zsph_device_malloc(void** p, size_t bytes) {
  if (!p) return set_err(nullptr, ZSPH_EINVAL, "zsph_device_malloc: null argument");
  ZCHECK(nullptr, "zsph_device_malloc", cudaMalloc(p, bytes ? bytes : 1));
  return ZSPH_OK;
}

int zsph_device_free(void* p) {
  if (p) ZCHECK(nullptr, "zsph_device_free", cudaFree(p));
  return ZSPH_OK;
}

int zsph_device_synchronize(void) {
  ZCHECK(nullptr, "zsph_device_synchronize", cudaDeviceSynchronize());
  return ZSPH_OK;
}

}  // extern "C"

namespace {
int step_profiled(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp, void* stream,
                  float* ms, int cap, int* count, char* names, int names_len, bool groups) {
  ENTRY_CHECKS(h);
  if (int rc = check_ptc(h, o)) return rc;
  if (int rc = check_ptc(h, w)) return rc;
  if (int rc = check_tmp(h, tmp)) return rc;
  if (!ms || cap <= 0) return set_err(h, ZSPH_EINVAL, "zsph_step_profiled: no output slots");
  cudaStream_t st = as_stream(stream);
  h->last_stream = st;
  const int slots = cap + 1;
  std::vector<cudaEvent_t> ev(slots);
  std::vector<const char*> nm(slots, "");
  for (auto& e : ev) ZCHECK(h, "zsph_step_profiled event", cudaEventCreate(&e));
  // The step is captured into a graph whose event-record nodes bracket each
  // launch, then replayed once: the event intervals are then GPU time of each
  // kernel plus the graph's own gap to the next node, free of host launch cost.
  Prof pf;
  pf.ev = ev.data() + 1;
  pf.cap = cap;
  pf.names = nm.data() + 1;
  pf.external = true;
  pf.groups = groups;
  if (!h->graph_stream) {
    cudaError_t cs = cudaStreamCreateWithFlags(&h->graph_stream, cudaStreamNonBlocking);
    if (cs) {
      for (auto& e : ev) cudaEventDestroy(e);
      return cuda_fail(h, "zsph_step_profiled stream", cs);
    }
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t gx = nullptr;
  cudaError_t le = cudaStreamBeginCapture(h->graph_stream, cudaStreamCaptureModeThreadLocal);
  if (!le) {
    le = cudaEventRecordWithFlags(ev[0], h->graph_stream, cudaEventRecordExternal);
    if (!le) le = step_launches(h, *o, *w, *tmp, h->graph_stream, &pf);
    const cudaError_t ce = cudaStreamEndCapture(h->graph_stream, &g);
    if (!le) le = ce;
  }
  if (!le) le = cudaGraphInstantiate(&gx, g, 0);
  if (!le) le = cudaGraphLaunch(gx, st);
  cudaError_t se = cudaStreamSynchronize(st);
  if (gx) cudaGraphExecDestroy(gx);
  if (g) cudaGraphDestroy(g);
  const int n = pf.n;
  std::string all;
  for (int k = 0; k < n; ++k) {
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
    ms[k] = t;
    all += nm[k + 1];
    all += k + 1 < n ? "," : "";
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (le) return cuda_fail(h, "zsph_step_profiled launch", le);
  if (se) return cuda_fail(h, "zsph_step_profiled sync", se);
  if (names && names_len > 0) std::snprintf(names, (size_t)names_len, "%s", all.c_str());
  if (count) *count = n;
  return ZSPH_OK;
}

}  // namespace

extern "C" {

int zsph_step_profiled(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp,
                       void* stream, float* ms, int cap, int* count, char* names, int names_len) {
  return step_profiled(h, o, w, tmp, stream, ms, cap, count, names, names_len, false);
}

int zsph_step_profiled_groups(zsph_handle_t* h, const zsph_ptc_t* o, const zsph_ptc_t* w, const zsph_tmp_t* tmp,
                              void* stream, float* ms, int cap, int* count, char* names, int names_len) {
  return step_profiled(h, o, w, tmp, stream, ms, cap, count, names, names_len, true);
}

int zsph_launches_per_step(zsph_handle_t* h) {
  // per sub-step: hash_count, scan, scatter, rank_gather, nblist, walls,
  // boundary, governing; with the list transfer the corrector's nblist is
  // xfer_classify, xfer_search, nblist_xfer and nblist_fallback (one of the
  // last two returns at once)
  if (h && xfer_eligible(h)) return 8 + 11;
  return 2 * 8;
}

}  // extern "C"
