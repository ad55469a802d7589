// zsph_compat_run: the reference's driver program on this library's C ABI.
//
// Restates single_gpu_sph_src/deltasph/main.cu:8-147 step for step with the
// public entry points, so a reference case directory runs unchanged:
//   read_json            -> zsph_read_json(json_path)
//   set_cpu_param        -> zsph_set_cpu_param (includes check_dt, init.cu:218)
//   read_vtk             -> zsph_read_vtk(input_path + "/input.vtk")  (read_vkt.cu:5)
//   cudaSetDevice(gpu_id)
//   set_gpu_param, alloc_gpu_*, cpu_to_gpu
//   mul_thread_creat     -> zsph_writer_create(output_path, thread_num writers)
//   step loop            -> the twelve launches of main.cu:63-88 through the
//                           drop-in entry points (ZSPH_COMPAT_SEPARATE), or one
//                           zsph_step per step (ZSPH_COMPAT_FUSED)
//   output every output_step -> zsph_writer_submit (output_path/zsph<i>.vtk)
// The reference's simplesph program is the same driver linked with
// equation/simple_ns.cu; ZSPH_COMPAT_SIMPLE selects those equations.
// Differences: no per-step console output and no exit(): every failure is a
// ZSPH_* status with its message in zsph_last_error(NULL, ...).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "trace.h"
#include "zsph_internal.cuh"

namespace {

int fail(int code, const std::string& m) {
  zsph::record_library_error("zsph_compat_run: " + m);
  return code;
}

std::string last_error(zsph_handle_t* h) {
  char b[512];
  zsph_last_error(h, b, (int)sizeof b);
  return b;
}

// The run log the reference prints to stdout as per-step timings
// (deltasph/main.cu:60-95), as JSON lines in the file that the environment
// variable ZSPH_METRICS names (no log without it): at every output step, the
// steps and wall time since the previous line (the stream synchronised first,
// so the time covers the device work), particle-steps/s, the device status
// bits and the FP64 conservation sums of the state (zsph_conservation).
struct MetricsLog {
  std::FILE* f = nullptr;
  std::chrono::steady_clock::time_point t0;
  int steps = 0;
  ~MetricsLog() {
    if (f) std::fclose(f);
  }
  void start() { t0 = std::chrono::steady_clock::now(); }
  int line(zsph_handle_t* h, const zsph_ptc_t& o, int step, int n, cudaStream_t st, std::string& what) {
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce) {
      what = std::string("metrics: ") + cudaGetErrorString(ce);
      return ZSPH_ECUDA;
    }
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    zsph_conservation_t c{};
    int rc = zsph_conservation(h, &o, &c, st);
    if (rc) {
      what = "metrics: " + last_error(h);
      return rc;
    }
    int flags = 0;
    rc = zsph_status(h, &flags, 0);
    if (rc == ZSPH_ECUDA) {
      what = "metrics: " + last_error(h);
      return rc;
    }
    // a non-finite sum (a state that blew up) is written as null, so every line stays JSON
    auto num = [](double x) {
      char b[32];
      if (!std::isfinite(x)) return std::string("null");
      std::snprintf(b, sizeof b, "%.17g", x);
      return std::string(b);
    };
    std::fprintf(f,
                 "{\"step\": %d, \"steps\": %d, \"seconds\": %.6f, \"particle_steps_per_s\": %.6e, "
                 "\"flags\": %d, \"mass\": %s, \"volume\": %s, \"momentum\": [%s, %s, %s], "
                 "\"kinetic\": %s, \"potential\": %s, \"internal\": %s}\n",
                 step, steps, dt, dt > 0 ? (double)n * steps / dt : 0.0, flags, num(c.mass).c_str(),
                 num(c.volume).c_str(), num(c.momentum[0]).c_str(), num(c.momentum[1]).c_str(),
                 num(c.momentum[2]).c_str(), num(c.kinetic).c_str(), num(c.potential).c_str(),
                 num(c.internal).c_str());
    if (std::fflush(f) != 0) {
      what = "metrics: write failed";
      return ZSPH_EIO;
    }
    steps = 0;
    start();
    return ZSPH_OK;
  }
};

int compat_run(const char* json_path, int mode, int* steps_done) {
  bool simple = (mode & ZSPH_COMPAT_SIMPLE) != 0;
  mode &= ~ZSPH_COMPAT_SIMPLE;
  if (mode != ZSPH_COMPAT_SEPARATE && mode != ZSPH_COMPAT_FUSED) return fail(ZSPH_EINVAL, "unknown mode");
  zsph_json_t j;
  char err[256] = {0};
  int rc = zsph_read_json(json_path, &j, err, (int)sizeof err);
  if (rc) return fail(rc, std::string("read_json: ") + err);
  zsph_case_options_t opt;
  rc = zsph_read_case_options(json_path, &opt, err, (int)sizeof err);
  if (rc) return fail(rc, std::string("case options: ") + err);
  if (opt.equations == ZSPH_EQ_SIMPLE) simple = true;
  zsph_cpu_param_t cp;
  rc = zsph_set_cpu_param(&cp, &j);
  if (rc) return fail(rc, "set_cpu_param: " + last_error(nullptr));
  const int n = cp.ptc_num;
  if (n < 0) return fail(ZSPH_EINVAL, "negative ptc_num in the case file");
  MetricsLog metrics;
  const char* mpath = std::getenv("ZSPH_METRICS");
  if (mpath && *mpath) {
    metrics.f = std::fopen(mpath, "w");
    if (!metrics.f) return fail(ZSPH_EIO, std::string("cannot open the metrics log ") + mpath);
  }
  std::vector<float> pos(3 * (size_t)n), vel(3 * (size_t)n), rhop(2 * (size_t)n), acc(4 * (size_t)n);
  std::vector<int> type((size_t)n), table((size_t)n);
  const std::string input = std::string(cp.input_path) + "/input.vtk";
  rc = zsph_read_vtk(input.c_str(), n, cp.rho0, 0, pos.data(), vel.data(), rhop.data(), acc.data(), type.data(),
                     table.data());
  if (rc) return fail(rc, "read_vtk: " + last_error(nullptr));
  cudaError_t ce = cudaSetDevice(cp.gpu_id);
  if (ce) return fail(ZSPH_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));
  zsph_gpu_param_t gp;
  rc = zsph_set_gpu_param(&gp, &cp);
  if (rc) return fail(rc, "set_gpu_param: " + last_error(nullptr));

  zsph_ptc_t o{}, w{};
  zsph_tmp_t t{};
  zsph_handle_t* h = nullptr;
  zsph_writer_t* wr = nullptr;
  cudaStream_t st = nullptr;
  int done = 0;
  std::string what;
  rc = zsph_alloc_ptc(&o, n);
  if (!rc) rc = zsph_alloc_ptc(&w, n);
  if (!rc) rc = zsph_alloc_tmp(&t, n, cp.grid_num);
  if (!rc) rc = zsph_cpu_to_gpu(&o, &t, pos.data(), vel.data(), rhop.data(), type.data(), table.data(), acc.data(),
                                n, nullptr);
  if (rc) what = "device buffers: " + last_error(nullptr);
  if (!rc && (ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) {
    rc = ZSPH_ECUDA;
    what = std::string("stream: ") + cudaGetErrorString(ce);
  }
  int first = cp.start_step;
  if (!rc && opt.resume[0]) {  // the state, cell bounds and step of a snapshot replace the input's
    // the input's upload ran on the legacy stream: let it land before the snapshot overwrites it
    if ((ce = cudaDeviceSynchronize()) != cudaSuccess) {
      rc = ZSPH_ECUDA;
      what = std::string("resume: ") + cudaGetErrorString(ce);
    }
    int step = 0;
    if (!rc) {
      rc = zsph_snapshot_load(opt.resume, &o, &t, n, cp.grid_num, &step, st);
      if (rc) what = "resume: " + last_error(nullptr);
      else first = step;
    }
  }
  if (!rc) {
    rc = zsph_create(&gp, cp.grid_num, &h);
    if (rc) what = "create: " + last_error(nullptr);
  }
  if (!rc && simple) {
    rc = zsph_set_equations(h, ZSPH_EQ_SIMPLE);
    if (rc) what = "set_equations: " + last_error(h);
  }
  if (!rc) {
    rc = zsph_writer_create(cp.output_path, n, ZSPH_OUT_REFERENCE, cp.thread_num > 0 ? cp.thread_num : 1, &wr);
    if (rc) what = "writer: " + last_error(nullptr);
  }
  void* s = st;
  metrics.start();
  for (int i = first; !rc && i < cp.end_step; ++i) {
    if (mode == ZSPH_COMPAT_FUSED) {
      rc = zsph_step(h, &o, &w, &t, s);
    } else {  // main.cu:63-88
      rc = zsph_hash(h, &o, &t, s);
      if (!rc) rc = zsph_sort_index(h, &t, s);
      if (!rc) rc = zsph_sort_data(h, &o, &w, &t, s);
      if (!rc) rc = zsph_boundary(h, &w, &t, s);
      if (!rc) rc = zsph_governing(h, &w, &t, s);
      if (!rc) rc = zsph_prediction(h, &w, &t, s);
      if (!rc) rc = zsph_hash(h, &w, &t, s);
      if (!rc) rc = zsph_sort_index(h, &t, s);
      if (!rc) rc = zsph_sort_data(h, &w, &o, &t, s);
      if (!rc) rc = zsph_boundary(h, &o, &t, s);
      if (!rc) rc = zsph_governing(h, &o, &t, s);
      if (!rc) rc = zsph_correction(h, &o, &t, s);
    }
    if (rc) {
      what = "step " + std::to_string(i) + ": " + last_error(h);
      break;
    }
    ++metrics.steps;
    if (cp.output_step > 0 && i % cp.output_step == 0) {  // main.cu:95-124
      rc = zsph_writer_submit(wr, &o, &t, i, s);
      if (rc) what = "output: " + last_error(nullptr);
      if (!rc && metrics.f) rc = metrics.line(h, o, i, n, st, what);
    }
    if (!rc && opt.snapshot_every > 0 && (i + 1) % opt.snapshot_every == 0) {  // the state before step i + 1
      const std::string snap = std::string(cp.output_path) + "/snapshot" + std::to_string(i + 1) + ".zsnap";
      rc = zsph_snapshot_save(snap.c_str(), &o, &t, n, cp.grid_num, i + 1, st);
      if (rc) what = "snapshot: " + last_error(nullptr);
    }
    ++done;
  }
  if (!rc && h) {
    int flags = 0;
    rc = zsph_status(h, &flags, 0);
    if (rc) what = "status: " + last_error(h);
  }
  if (wr) {
    const int wrc = zsph_writer_destroy(wr);  // writes the pending files
    if (!rc && wrc) {
      rc = wrc;
      what = "writer: " + last_error(nullptr);
    }
  }
  if (h) zsph_destroy(h);
  if (st) cudaStreamDestroy(st);
  zsph_free_ptc(&o);
  zsph_free_ptc(&w);
  zsph_free_tmp(&t);
  if (steps_done) *steps_done = done;
  return rc ? fail(rc, what) : ZSPH_OK;
}

}  // namespace

extern "C" {

int zsph_compat_run(const char* json_path, int mode, int* steps_done) {
  const zsph::TraceRange trace_range_(__func__);
  if (steps_done) *steps_done = 0;
  if (!json_path) return fail(ZSPH_EINVAL, "null json path");
  // No C++ exception leaves through the C ABI (a std::bad_alloc for the host
  // copies of a very large case, for example): it becomes an error code.
  try {
    return compat_run(json_path, mode, steps_done);
  } catch (const std::exception& e) {
    return fail(ZSPH_EIO, e.what());
  } catch (...) {
    return fail(ZSPH_EIO, "unknown error");
  }
}

}  // extern "C"
