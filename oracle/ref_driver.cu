// Checker harness around the reference's OWN hot-path kernels, compiled
// unmodified from the reference sources for sm_100a (recipe:
// oracle/build_ref.sh).  It mirrors the reference's driver
// single_gpu_sph_src/deltasph/main.cu:10-90 without VTK input or output:
// case constants from set_cpu_param/set_gpu_param (lib/init.cu:153-251),
// device buffers from alloc_gpu_ptc_data/alloc_gpu_tmp_data (lib/init.cu:38-115),
// the __constant__ symbols par/tmp_data (main.cu:5-6), and the same launch
// sequence <<<ceil(N/256),256>>> per sub-step (main.cu:63-88).
//
// The only kernel written here is ref_count_neighbors, which counts, per
// particle, the candidates that pass the reference's own distance test
// (delta_ns.cu:61,67-68 / :236-240) over the reference's stencil rows, so that
// neighbour counts can be compared.  Test infrastructure only.
#include "equation.cuh"
#include "lib.cuh"

#include <cstring>
#include <sstream>

__constant__ gpu_param_t par;
__constant__ gpu_tmp_t tmp_data;

__global__ void ref_count_neighbors(gpu_ptc_t* tptc, int ylast, int* out) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  const gpu_ptc_t d = *tptc;
  if (index >= par.ptc_num) return;
  const float3 pos = d.pos[index];
  int count = 0;
  for (int z = -par.grid_factor; z <= par.grid_factor; z++) {
    for (int y = -par.grid_factor; y <= ylast; y++) {
      int cs = tmp_data.hash[index] + z * par.grid_xdim * par.grid_ydim + y * par.grid_xdim;
      int ce = cs + par.grid_factor;
      cs = cs - par.grid_factor;
      if (cs >= par.grid_hash_min && ce <= par.grid_hash_max) {
        cs = tmp_data.grid_start[cs];
        ce = tmp_data.grid_end[ce];
        for (int i = cs; i < ce; i++) {
          if (i != index) {
            float3 dx = d.pos[i];
            dx.x = pos.x - dx.x;
            dx.y = pos.y - dx.y;
            dx.z = pos.z - dx.z;
            float rr2 = dx.x * dx.x + dx.y * dx.y + dx.z * dx.z;
            float q = sqrtf(rr2) / par.h;
            if (q <= 2.0f) count++;
          }
        }
      }
    }
  }
  out[index] = count;
}

extern "C" {

typedef struct {
  float g, rho0, dx, h_factor, r_factor, eta_factor, cs_factor, delta, alpha;
  float xmin, xmax, ymin, ymax, zmin, zmax, grid_layer_factor, grid_size_factor;
  float dt;
  int ptc_num;
} rcase_t;

// Host particle arrays in the reference layout (3/3/2/3/3/2 floats, ints).
typedef struct {
  float *pos, *vel, *rhop, *tmp_pos, *tmp_vel, *tmp_rhop;
  int *type, *table;
} rstate_t;

typedef struct {
  float *acc_drhodt, *dofv_grandrho;  // 4 per particle
  int *index, *hash, *grid_start, *grid_end;
  int *nb_boundary, *nb_governing;  // neighbour counts (may be null)
  float* dofv;                      // scalar div(v) of the simple equations (may be null)
} rtmp_t;

static int g_err = 0;
static char g_msg[512];

static int fail(const char* where, cudaError_t e) {
  snprintf(g_msg, sizeof g_msg, "%s: %s", where, cudaGetErrorString(e));
  g_err = 1;
  return 1;
}

const char* ref_last_error(void) { return g_err ? g_msg : ""; }

static void to_param(const rcase_t* c, cpu_param_t* cp) {
  cpu_json_t j;
  j.g = c->g; j.rho0 = c->rho0; j.dx = c->dx; j.h_factor = c->h_factor; j.r_factor = c->r_factor;
  j.eta_factor = c->eta_factor; j.cs_factor = c->cs_factor; j.delta = c->delta; j.alpha = c->alpha;
  j.xmin = c->xmin; j.xmax = c->xmax; j.ymin = c->ymin; j.ymax = c->ymax; j.zmin = c->zmin; j.zmax = c->zmax;
  j.grid_layer_factor = c->grid_layer_factor; j.grid_size_factor = c->grid_size_factor;
  j.dt = c->dt; j.start_step = 0; j.current_step = 0; j.end_step = 0; j.output_step = 1;
  j.ptc_num = c->ptc_num; j.water_ptc_num = 0; j.air_ptc_num = 0; j.wall_ptc_num = 0; j.rigid_ptc_num = 0;
  j.thread_num = 1; j.gpu_id = 0;
  // the reference's host code prints banners to stdout; keep stdout for the caller
  std::ostringstream sink;
  std::streambuf* prev = std::cout.rdbuf(sink.rdbuf());
  set_cpu_param(cp, &j);  // reference host derivation (exits on dt > dt_max; callers pre-check)
  std::cout.rdbuf(prev);
}

// Derived constants as the reference computes them.
int ref_params(const rcase_t* c, gpu_param_t* gp, int* grid_num) {
  cpu_param_t cp;
  to_param(c, &cp);
  set_gpu_param(gp, &cp);
  *grid_num = cp.grid_num;
  return 0;
}

int ref_sizeof_gpu_param(void) { return (int)sizeof(gpu_param_t); }

struct Session {
  cpu_param_t cp;
  gpu_param_t gp;
  gpu_ptc_t old_, new_;
  gpu_tmp_t tmp;
  gpu_ptc_t *d_old = nullptr, *d_new = nullptr;
  int* d_count = nullptr;
  int grid, block;
};

static int open_session(const rcase_t* c, const rstate_t* in, Session& s) {
  memset(&s.tmp, 0, sizeof s.tmp);  // alloc_gpu_tmp_data sets dofv_grandrho or dofv, by build
  to_param(c, &s.cp);
  set_gpu_param(&s.gp, &s.cp);
  const int n = s.cp.ptc_num;
  alloc_gpu_ptc_data(&s.old_, &s.cp);
  alloc_gpu_ptc_data(&s.new_, &s.cp);
  alloc_gpu_tmp_data(&s.tmp, &s.cp);
  cpu_input_t ci;
  ci.pos = in->pos; ci.vel = in->vel; ci.rhop = in->rhop; ci.type = in->type; ci.table = in->table;
  std::vector<float> acc((size_t)4 * n, 0.0f);
  ci.acc_drhodt = acc.data();
  cpu_to_gpu(&s.old_, &s.tmp, &ci, &s.cp);
  cudaError_t e = cudaSuccess;
  if (in->tmp_pos) e = cudaMemcpy(s.old_.tmp_pos, in->tmp_pos, n * sizeof(float3), cudaMemcpyHostToDevice);
  if (!e && in->tmp_vel) e = cudaMemcpy(s.old_.tmp_vel, in->tmp_vel, n * sizeof(float3), cudaMemcpyHostToDevice);
  if (!e && in->tmp_rhop) e = cudaMemcpy(s.old_.tmp_rhop, in->tmp_rhop, n * sizeof(float2), cudaMemcpyHostToDevice);
  if (!e) e = cudaMalloc(&s.d_old, sizeof(gpu_ptc_t));
  if (!e) e = cudaMalloc(&s.d_new, sizeof(gpu_ptc_t));
  if (!e) e = cudaMalloc(&s.d_count, (size_t)n * sizeof(int));
  if (!e) e = cudaMemcpy(s.d_old, &s.old_, sizeof(gpu_ptc_t), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpy(s.d_new, &s.new_, sizeof(gpu_ptc_t), cudaMemcpyHostToDevice);
  if (!e) e = cudaMemcpyToSymbol(par, &s.gp, sizeof(gpu_param_t));
  if (!e) e = cudaMemcpyToSymbol(tmp_data, &s.tmp, sizeof(gpu_tmp_t));
  if (e) return fail("open_session", e);
  s.grid = (n + 255) / 256;
  s.block = 256;
  return 0;
}

static void close_session(Session& s) {
  cudaFree(s.d_old);
  cudaFree(s.d_new);
  cudaFree(s.d_count);
  delete_gpu_ptc_data(&s.old_);
  delete_gpu_ptc_data(&s.new_);
  cudaFree(s.tmp.acc_drhodt);
  if (s.tmp.dofv_grandrho) cudaFree(s.tmp.dofv_grandrho);
  if (s.tmp.dofv) cudaFree(s.tmp.dofv);
  cudaFree(s.tmp.hash);
  cudaFree(s.tmp.index);
  cudaFree(s.tmp.grid_start);
  cudaFree(s.tmp.grid_end);
}

static int copy_out(Session& s, const gpu_ptc_t& src, rstate_t* out, rtmp_t* t) {
  const int n = s.cp.ptc_num, G = s.cp.grid_num;
  cudaError_t e = cudaDeviceSynchronize();
  if (out) {
    if (!e && out->pos) e = cudaMemcpy(out->pos, src.pos, n * sizeof(float3), cudaMemcpyDeviceToHost);
    if (!e && out->vel) e = cudaMemcpy(out->vel, src.vel, n * sizeof(float3), cudaMemcpyDeviceToHost);
    if (!e && out->rhop) e = cudaMemcpy(out->rhop, src.rhop, n * sizeof(float2), cudaMemcpyDeviceToHost);
    if (!e && out->tmp_pos) e = cudaMemcpy(out->tmp_pos, src.tmp_pos, n * sizeof(float3), cudaMemcpyDeviceToHost);
    if (!e && out->tmp_vel) e = cudaMemcpy(out->tmp_vel, src.tmp_vel, n * sizeof(float3), cudaMemcpyDeviceToHost);
    if (!e && out->tmp_rhop) e = cudaMemcpy(out->tmp_rhop, src.tmp_rhop, n * sizeof(float2), cudaMemcpyDeviceToHost);
    if (!e && out->type) e = cudaMemcpy(out->type, src.type, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (!e && out->table) e = cudaMemcpy(out->table, src.table, n * sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (t) {
    if (!e && t->acc_drhodt) e = cudaMemcpy(t->acc_drhodt, s.tmp.acc_drhodt, n * sizeof(float4), cudaMemcpyDeviceToHost);
    if (!e && t->dofv_grandrho && s.tmp.dofv_grandrho)
      e = cudaMemcpy(t->dofv_grandrho, s.tmp.dofv_grandrho, n * sizeof(float4), cudaMemcpyDeviceToHost);
    if (!e && t->dofv && s.tmp.dofv) e = cudaMemcpy(t->dofv, s.tmp.dofv, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (!e && t->index) e = cudaMemcpy(t->index, s.tmp.index, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (!e && t->hash) e = cudaMemcpy(t->hash, s.tmp.hash, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (!e && t->grid_start) e = cudaMemcpy(t->grid_start, s.tmp.grid_start, G * sizeof(int), cudaMemcpyDeviceToHost);
    if (!e && t->grid_end) e = cudaMemcpy(t->grid_end, s.tmp.grid_end, G * sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (e) return fail("copy_out", e);
  return 0;
}

static int count_out(Session& s, gpu_ptc_t* d, rtmp_t* t) {
  const int n = s.cp.ptc_num;
  cudaError_t e = cudaSuccess;
  if (t && t->nb_boundary) {
    ref_count_neighbors<<<s.grid, s.block>>>(d, s.gp.grid_factor - 1, s.d_count);
    e = cudaMemcpy(t->nb_boundary, s.d_count, n * sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (!e && t && t->nb_governing) {
    ref_count_neighbors<<<s.grid, s.block>>>(d, s.gp.grid_factor, s.d_count);
    e = cudaMemcpy(t->nb_governing, s.d_count, n * sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (e) return fail("count_out", e);
  return 0;
}

// One predictor sub-step of main.cu:63-73 on the input state, stopping after
// `stage` kernels: 1 = hash, 2 = +sort_index, 3 = +sort_data, 4 = +boundary,
// 5 = +governing, 6 = +prediction.  Returns the sorted (NEW) buffers.
int ref_substep(const rcase_t* c, const rstate_t* in, int stage, rstate_t* out, rtmp_t* t) {
  g_err = 0;
  Session s;
  if (open_session(c, in, s)) return 1;
  if (stage >= 1) cuda_ptc_hash<<<s.grid, s.block>>>(s.d_old);
  if (stage >= 2) cuda_sort_index(s.tmp, s.cp);
  if (stage >= 3) cuda_sort_data<<<s.grid, s.block>>>(s.d_old, s.d_new);
  if (stage >= 4) cuda_boundary_ns<<<s.grid, s.block>>>(s.d_new);
  if (stage >= 5) cuda_govering_ns<<<s.grid, s.block>>>(s.d_new);
  if (stage >= 6) cuda_prediction<<<s.grid, s.block>>>(s.d_new);
  cudaError_t e = cudaDeviceSynchronize();
  int rc = e ? fail("ref_substep", e) : 0;
  if (!rc) rc = copy_out(s, stage >= 3 ? s.new_ : s.old_, out, t);
  if (!rc && stage >= 3) rc = count_out(s, s.d_new, t);
  close_session(s);
  return rc;
}

// `nsteps` full steps of main.cu:58-90 (two sub-steps each); returns the
// OLD buffers and the scratch arrays after the last sub-step.  If ms_per_step
// is given, the steps after `warmup` ones are timed with CUDA events.
int ref_run(const rcase_t* c, const rstate_t* in, int warmup, int nsteps, rstate_t* out, rtmp_t* t,
            float* ms_per_step) {
  g_err = 0;
  Session s;
  if (open_session(c, in, s)) return 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int i = 0; i < warmup + nsteps; ++i) {
    if (i == warmup) cudaEventRecord(e0);
    cuda_ptc_hash<<<s.grid, s.block>>>(s.d_old);
    cuda_sort_index(s.tmp, s.cp);
    cuda_sort_data<<<s.grid, s.block>>>(s.d_old, s.d_new);
    cuda_boundary_ns<<<s.grid, s.block>>>(s.d_new);
    cuda_govering_ns<<<s.grid, s.block>>>(s.d_new);
    cuda_prediction<<<s.grid, s.block>>>(s.d_new);
    cuda_ptc_hash<<<s.grid, s.block>>>(s.d_new);
    cuda_sort_index(s.tmp, s.cp);
    cuda_sort_data<<<s.grid, s.block>>>(s.d_new, s.d_old);
    cuda_boundary_ns<<<s.grid, s.block>>>(s.d_old);
    cuda_govering_ns<<<s.grid, s.block>>>(s.d_old);
    cuda_correction<<<s.grid, s.block>>>(s.d_old);
  }
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  if (!e) e = cudaGetLastError();
  int rc = e ? fail("ref_run", e) : 0;
  if (!rc && ms_per_step && nsteps > 0) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    *ms_per_step = ms / nsteps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = copy_out(s, s.old_, out, t);
  if (!rc) rc = count_out(s, s.d_old, t);
  close_session(s);
  return rc;
}

// The loop of ref_run with a CUDA event after each of a step's twelve launch
// slots (main.cu:63-88: hash, sort_index, sort_data, boundary, governing,
// prediction, then the same five and correction), so that where the step's
// time goes can be read per slot.  A slot's time is the interval between the
// events around it; for the two cuda_sort_index slots it includes every gap
// the host leaves on the device while Thrust allocates and frees its
// temporary storage (lib/sort.cu:5 uses Thrust's default allocator, i.e. a
// cudaMalloc and a cudaFree per call).  The host time of each
// cuda_sort_index call is measured with a steady clock.
//   slot_ms[12]      per-step mean of each slot (ms)
//   host_sort_ms[2]  per-step mean host duration of the two sort calls (ms)
//   ms_per_step      first event to last, per step
// Events add a few microseconds per launch; ref_run gives the step time
// without them.
int ref_run_profiled(const rcase_t* c, const rstate_t* in, int warmup, int nsteps, float* ms_per_step,
                     float* slot_ms, float* host_sort_ms) {
  g_err = 0;
  if (nsteps <= 0) return 0;
  Session s;
  if (open_session(c, in, s)) return 1;
  const int kSlots = 12;
  std::vector<cudaEvent_t> ev((size_t)nsteps * (kSlots + 1));
  for (auto& e : ev) cudaEventCreate(&e);
  double host_ms[2] = {0.0, 0.0};
  for (int i = 0; i < warmup + nsteps; ++i) {
    const bool timed = i >= warmup;
    cudaEvent_t* e = timed ? &ev[(size_t)(i - warmup) * (kSlots + 1)] : nullptr;
    auto mark = [&](int k) {
      if (timed) cudaEventRecord(e[k]);
    };
    auto sort = [&](int which) {
      auto t0 = std::chrono::steady_clock::now();
      cuda_sort_index(s.tmp, s.cp);
      auto t1 = std::chrono::steady_clock::now();
      if (timed) host_ms[which] += std::chrono::duration<double, std::milli>(t1 - t0).count();
    };
    mark(0);
    cuda_ptc_hash<<<s.grid, s.block>>>(s.d_old);
    mark(1);
    sort(0);
    mark(2);
    cuda_sort_data<<<s.grid, s.block>>>(s.d_old, s.d_new);
    mark(3);
    cuda_boundary_ns<<<s.grid, s.block>>>(s.d_new);
    mark(4);
    cuda_govering_ns<<<s.grid, s.block>>>(s.d_new);
    mark(5);
    cuda_prediction<<<s.grid, s.block>>>(s.d_new);
    mark(6);
    cuda_ptc_hash<<<s.grid, s.block>>>(s.d_new);
    mark(7);
    sort(1);
    mark(8);
    cuda_sort_data<<<s.grid, s.block>>>(s.d_new, s.d_old);
    mark(9);
    cuda_boundary_ns<<<s.grid, s.block>>>(s.d_old);
    mark(10);
    cuda_govering_ns<<<s.grid, s.block>>>(s.d_old);
    mark(11);
    cuda_correction<<<s.grid, s.block>>>(s.d_old);
    mark(12);
  }
  cudaError_t err = cudaDeviceSynchronize();
  if (!err) err = cudaGetLastError();
  int rc = err ? fail("ref_run_profiled", err) : 0;
  if (!rc) {
    double slot[kSlots] = {0.0};
    double total = 0.0;
    for (int st = 0; st < nsteps; ++st) {
      cudaEvent_t* e = &ev[(size_t)st * (kSlots + 1)];
      for (int k = 0; k < kSlots; ++k) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e[k], e[k + 1]);
        slot[k] += ms;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e[0], e[kSlots]);
      total += ms;
    }
    for (int k = 0; k < kSlots; ++k)
      if (slot_ms) slot_ms[k] = (float)(slot[k] / nsteps);
    if (host_sort_ms) {
      host_sort_ms[0] = (float)(host_ms[0] / nsteps);
      host_sort_ms[1] = (float)(host_ms[1] / nsteps);
    }
    if (ms_per_step) *ms_per_step = (float)(total / nsteps);
  }
  for (auto& e : ev) cudaEventDestroy(e);
  close_session(s);
  return rc;
}

}  // extern "C"
