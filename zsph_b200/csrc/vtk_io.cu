// Particle file IO without libVTK.
//
// zsph_write_vtk     <- single_gpu_sph_src/io/write_vtk.cu:29-130 (legacy VTK,
//                       BINARY, big-endian, "DATASET UNSTRUCTURED_GRID" with
//                       POINTS and POINT_DATA arrays selected by flags, the
//                       run-time form of the reference's ZSPH_OUTPUT_* macros)
// zsph_read_vtk      <- single_gpu_sph_src/io/read_vkt.cu:3-92 (points, point
//                       arrays "p", "rho", "vel", "acc", "type", "table" with the
//                       reference's defaults)
// zsph_writer_*      <- single_gpu_sph_src/io/mul_thread.cu:3-81 and the output
//                       hand-off of deltasph/main.cu:101-142: a pool of writer
//                       threads, each with pinned host buffers.  The device-to-host
//                       copy is issued on the caller's stream and the thread
//                       writes output_path/zsph<step>.vtk once the copy's event has
//                       completed; threads sleep on a condition variable instead
//                       of spinning on an atomic flag.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "trace.h"
#include "zsph_internal.cuh"

namespace {

uint32_t bswap32(uint32_t v) { return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24); }
uint64_t bswap64(uint64_t v) {
  return ((uint64_t)bswap32((uint32_t)v) << 32) | bswap32((uint32_t)(v >> 32));
}

template <class T> void put_be(std::string& out, const T* v, size_t count) {
  static_assert(sizeof(T) == 4, "32-bit values");
  const size_t at = out.size();
  out.resize(at + count * 4);
  for (size_t k = 0; k < count; ++k) {
    uint32_t u;
    std::memcpy(&u, &v[k], 4);
    u = bswap32(u);
    std::memcpy(&out[at + 4 * k], &u, 4);
  }
}

int fail(int code, const std::string& m) {
  zsph::record_library_error(m);
  return code;
}

// Legacy VTK tokenizer over an in-memory file: text tokens separated by
// whitespace, with raw big-endian binary blocks read at the current offset.
struct Cursor {
  const std::string& s;
  size_t p = 0;
  explicit Cursor(const std::string& d) : s(d) {}
  std::string line() {
    size_t e = s.find('\n', p);
    if (e == std::string::npos) e = s.size();
    std::string l = s.substr(p, e - p);
    p = e < s.size() ? e + 1 : e;
    if (!l.empty() && l.back() == '\r') l.pop_back();
    return l;
  }
  std::string token() {
    while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
    size_t b = p;
    while (p < s.size() && !std::isspace((unsigned char)s[p])) ++p;
    return s.substr(b, p - b);
  }
  void skip_line_end() {  // after the last header token of a binary block
    while (p < s.size() && s[p] != '\n') ++p;
    if (p < s.size()) ++p;
  }
};

// Bytes per value of a binary block's data type; 0 for a type this reader
// does not take.  The reference's writer uses float, double and int.
size_t binary_width(const std::string& type) {
  if (type == "double" || type == "vtktypeint64") return 8;
  if (type == "float" || type == "int" || type == "vtktypeint32") return 4;
  return 0;
}

// Reads `count` values of `type` (float, double, int) as doubles.  The count
// comes from the file, so it is checked against the bytes left before anything
// is allocated: a binary block needs count * width bytes, an ASCII one at least
// one character per value.  Returns an empty string or the reason it failed.
std::string read_values(Cursor& c, bool binary, const std::string& type, long long count, std::vector<double>& out) {
  if (count < 0) return "negative value count";
  const size_t left = c.s.size() - std::min(c.p, c.s.size());
  if (!binary) {
    if ((unsigned long long)count > left) return "fewer values than declared";
    out.resize((size_t)count);
    for (size_t k = 0; k < (size_t)count; ++k) {
      const std::string t = c.token();
      if (t.empty()) return "fewer values than declared";
      out[k] = std::strtod(t.c_str(), nullptr);
    }
    return "";
  }
  const size_t w = binary_width(type);
  if (w == 0) return "unsupported binary data type \"" + type + "\"";
  c.skip_line_end();
  const size_t avail = c.s.size() - c.p;
  if ((unsigned long long)count > avail / w) return "fewer bytes than declared";
  out.resize((size_t)count);
  for (size_t k = 0; k < (size_t)count; ++k) {
    const char* q = c.s.data() + c.p + k * w;
    if (w == 8) {
      uint64_t u;
      std::memcpy(&u, q, 8);
      u = bswap64(u);
      if (type == "double") {
        double d;
        std::memcpy(&d, &u, 8);
        out[k] = d;
      } else {
        int64_t i;
        std::memcpy(&i, &u, 8);
        out[k] = (double)i;
      }
    } else {
      uint32_t u;
      std::memcpy(&u, q, 4);
      u = bswap32(u);
      if (type == "float") {
        float f;
        std::memcpy(&f, &u, 4);
        out[k] = f;
      } else {
        int32_t i;
        std::memcpy(&i, &u, 4);
        out[k] = i;
      }
    }
  }
  c.p += (size_t)count * w;
  return "";
}

// A count or component number from the file's text; -1 when it is not a
// plain non-negative decimal number.
long long parse_count(const std::string& t) {
  if (t.empty() || t.size() > 18) return -1;
  for (char ch : t)
    if (ch < '0' || ch > '9') return -1;
  return std::strtoll(t.c_str(), nullptr, 10);
}

struct Array {
  std::string type;  // float, double, int, ...
  int comps = 1;
  std::vector<double> v;
};

int read_vtk_file(const char* path, int n, float rho0, int accept_float, float* pos, float* vel, float* rhop,
                  float* acc, int* type, int* table) {
  if (!path || n < 0) return fail(ZSPH_EINVAL, "zsph_read_vtk: bad argument");
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(ZSPH_EIO, std::string("zsph_read_vtk: cannot open ") + path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string data = ss.str();
  Cursor c(data);
  if (c.line().rfind("# vtk DataFile", 0) != 0) return fail(ZSPH_EIO, "zsph_read_vtk: not a legacy VTK file");
  c.line();  // title
  std::string fmt = c.token();
  const bool binary = (fmt == "BINARY");
  if (!binary && fmt != "ASCII") return fail(ZSPH_EIO, "zsph_read_vtk: format must be ASCII or BINARY");
  std::vector<double> pts;
  std::vector<std::pair<std::string, Array>> arrays;
  long long npts = -1;
  auto values = [&](const std::string& what, const std::string& ty, long long count, std::vector<double>& out) {
    const std::string why = read_values(c, binary, ty, count, out);
    return why.empty() ? ZSPH_OK : fail(ZSPH_EIO, "zsph_read_vtk: " + what + ": " + why);
  };
  // VTK's own legacy writer follows an array with a METADATA block
  // (COMPONENT_NAMES, INFORMATION n and its entries) that ends at an empty
  // line, between the arrays of a FIELD too: skipped whole.
  auto skip_metadata = [&] {
    c.line();
    while (c.p < c.s.size()) {
      const std::string l = c.line();
      if (l.find_first_not_of(" \t") == std::string::npos) break;
    }
  };
  for (;;) {
    const std::string kw = c.token();
    if (kw.empty()) break;
    int rc = ZSPH_OK;
    if (kw == "DATASET") {
      if (c.token() != "UNSTRUCTURED_GRID") return fail(ZSPH_EIO, "zsph_read_vtk: dataset must be UNSTRUCTURED_GRID");
    } else if (kw == "POINTS") {
      const std::string cnt = c.token();
      npts = parse_count(cnt);
      const std::string ty = c.token();
      if (npts != n)  // read_vkt.cu:14 asserts this
        return fail(ZSPH_EINVAL, "zsph_read_vtk: file has " + cnt + " points, ptc_num is " + std::to_string(n));
      rc = values("POINTS", ty, npts * 3, pts);
    } else if (kw == "CELLS" || kw == "CELL_TYPES") {
      // The cells are read past, not kept.  Version 5.1 files give CELLS as
      // an OFFSETS and a CONNECTIVITY block, each with its own data type;
      // older ones as one int block.
      const long long a = parse_count(c.token());
      const long long b = kw == "CELLS" ? parse_count(c.token()) : a;
      if (a < 0 || b < 0) return fail(ZSPH_EIO, "zsph_read_vtk: bad " + kw + " size");
      std::vector<double> skip;
      const size_t at = c.p;
      if (kw == "CELLS" && c.token() == "OFFSETS") {
        rc = values("CELLS offsets", c.token(), a, skip);
        if (rc == ZSPH_OK && c.token() != "CONNECTIVITY")
          return fail(ZSPH_EIO, "zsph_read_vtk: CELLS: CONNECTIVITY expected after OFFSETS");
        if (rc == ZSPH_OK) rc = values("CELLS connectivity", c.token(), b, skip);
      } else {
        c.p = at;
        rc = values(kw, "int", b, skip);
      }
    } else if (kw == "POINT_DATA" || kw == "CELL_DATA") {
      c.token();
    } else if (kw == "SCALARS") {
      Array a;
      const std::string name = c.token();
      a.type = c.token();
      // optional component count (1 to 4), then LOOKUP_TABLE
      std::string t = c.token();
      if (t != "LOOKUP_TABLE") {
        const long long comps = parse_count(t);
        if (comps < 1 || comps > 4) return fail(ZSPH_EIO, "zsph_read_vtk: SCALARS " + name + ": bad component count " + t);
        a.comps = (int)comps;
        t = c.token();
      }
      c.token();  // table name
      rc = values("SCALARS " + name, a.type, (long long)n * a.comps, a.v);
      arrays.emplace_back(name, std::move(a));
    } else if (kw == "VECTORS") {
      Array a;
      const std::string name = c.token();
      a.type = c.token();
      a.comps = 3;
      rc = values("VECTORS " + name, a.type, (long long)n * 3, a.v);
      arrays.emplace_back(name, std::move(a));
    } else if (kw == "FIELD") {
      c.token();
      const long long narr = parse_count(c.token());
      if (narr < 0) return fail(ZSPH_EIO, "zsph_read_vtk: bad FIELD array count");
      for (long long k = 0; k < narr && rc == ZSPH_OK; ++k) {
        Array a;
        std::string name = c.token();
        while (name == "METADATA") {
          skip_metadata();
          name = c.token();
        }
        const long long comps = parse_count(c.token());
        const long long tuples = parse_count(c.token());
        a.type = c.token();
        if (comps < 1 || comps > 16 || tuples < 0)
          return fail(ZSPH_EIO, "zsph_read_vtk: field " + name + ": bad component or tuple count");
        if (tuples > (1LL << 40)) return fail(ZSPH_EIO, "zsph_read_vtk: field " + name + ": fewer values than declared");
        a.comps = (int)comps;
        rc = values("field " + name, a.type, tuples * comps, a.v);
        arrays.emplace_back(name, std::move(a));
      }
    } else if (kw == "LOOKUP_TABLE") {
      c.line();
    } else if (kw == "METADATA") {
      skip_metadata();
    } else {
      return fail(ZSPH_EIO, "zsph_read_vtk: unexpected keyword " + kw);
    }
    if (rc != ZSPH_OK) return rc;
  }
  if (npts < 0) return fail(ZSPH_EIO, "zsph_read_vtk: no POINTS");
  // read_vkt.cu:61-83: p, vel, acc, rho must be double arrays (a float array is
  // ignored and the default used) unless accept_float; type and table int
  // arrays.  An array that is taken must hold one tuple of the expected width
  // per point (1 for p, rho, type, table; 3 for vel, acc): a shorter or wider
  // one is an error rather than a read past its end.
  std::string bad;
  auto find = [&](const char* name, bool want_int, int comps) -> const Array* {
    for (auto& kv : arrays)
      if (kv.first == name) {
        const Array& arr = kv.second;
        const std::string& t = arr.type;
        const bool taken = want_int ? (t == "int") : (t == "double" || (accept_float && t == "float"));
        if (!taken) return nullptr;
        if (arr.comps != comps || arr.v.size() != (size_t)n * (size_t)comps) {
          if (bad.empty())
            bad = std::string("zsph_read_vtk: array \"") + name + "\" holds " + std::to_string(arr.v.size()) +
                  " values in tuples of " + std::to_string(arr.comps) + "; expected " + std::to_string(n) +
                  " tuples of " + std::to_string(comps);
          return nullptr;
        }
        return &arr;
      }
    return nullptr;
  };
  const Array* ap = find("p", false, 1);
  const Array* ar = find("rho", false, 1);
  const Array* av = find("vel", false, 3);
  const Array* aa = find("acc", false, 3);
  const Array* at = find("type", true, 1);
  const Array* ab = find("table", true, 1);
  if (!bad.empty()) return fail(ZSPH_EIO, bad);
  if (!at) return fail(ZSPH_EIO, "zsph_read_vtk: the int array \"type\" is required");  // read_vkt.cu:101
  for (int i = 0; i < n; ++i) {  // read_vkt.cu:85-126
    for (int k = 0; k < 3; ++k) {
      if (pos) pos[3 * i + k] = (float)pts[3 * (size_t)i + k];
      if (vel) vel[3 * i + k] = av ? (float)av->v[3 * (size_t)i + k] : 0.0f;
      if (acc) acc[4 * i + k] = aa ? (float)aa->v[3 * (size_t)i + k] : 0.0f;
    }
    if (acc) acc[4 * i + 3] = 0.0f;
    if (rhop) {
      rhop[2 * i] = ar ? (float)ar->v[i] : rho0;
      rhop[2 * i + 1] = ap ? (float)ap->v[i] : 0.0f;
    }
    if (type) type[i] = (int)at->v[i];
    if (table) table[i] = ab ? (int)ab->v[i] : 0;
  }
  return ZSPH_OK;
}

}  // namespace

extern "C" {

int zsph_write_vtk(const char* path, int n, const float* pos, const float* vel, const float* rhop, const int* type,
                   const float* acc, const int* hash, const int* table, int flags) {
  const zsph::TraceRange trace_range_(__func__);
  if (!path || n < 0 || (n > 0 && !pos)) return fail(ZSPH_EINVAL, "zsph_write_vtk: bad argument");
  // No C++ exception leaves through the C ABI (a std::bad_alloc for a very
  // large n, for example): it becomes an error code.
  try {
    std::string out;
    out.reserve((size_t)n * 48 + 512);
    std::ostringstream hdr;
    hdr << "# vtk DataFile Version 3.0\nzsph data\nBINARY\nDATASET UNSTRUCTURED_GRID\n";  // write_vtk.cu:36-39
    hdr << "POINTS " << n << " float\n";
    out += hdr.str();
    put_be(out, pos, (size_t)n * 3);
    out += "\nPOINT_DATA " + std::to_string(n) + "\n";
    auto scalar_f = [&](const char* name, const float* base, int stride) {
      out += std::string("SCALARS ") + name + " float 1\nLOOKUP_TABLE default\n";
      const size_t at = out.size();
      out.resize(at + (size_t)n * 4);
      for (int i = 0; i < n; ++i) {
        uint32_t u;
        std::memcpy(&u, &base[(size_t)i * stride], 4);
        u = bswap32(u);
        std::memcpy(&out[at + 4 * (size_t)i], &u, 4);
      }
      out += "\n";
    };
    auto scalar_i = [&](const char* name, const int* v) {
      out += std::string("SCALARS ") + name + " int 1\nLOOKUP_TABLE default\n";
      put_be(out, v, (size_t)n);
      out += "\n";
    };
    auto vector_f = [&](const char* name, const float* base, int stride) {
      out += std::string("VECTORS ") + name + " float\n";
      const size_t at = out.size();
      out.resize(at + (size_t)n * 12);
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
          uint32_t u;
          std::memcpy(&u, &base[(size_t)i * stride + k], 4);
          u = bswap32(u);
          std::memcpy(&out[at + 12 * (size_t)i + 4 * k], &u, 4);
        }
      out += "\n";
    };
    if ((flags & ZSPH_OUT_RHO) && rhop) scalar_f("rho", rhop, 2);
    if ((flags & ZSPH_OUT_P) && rhop) scalar_f("p", rhop + 1, 2);           // write_vtk.cu:66-74
    if ((flags & ZSPH_OUT_TYPE) && type) scalar_i("type", type);            // :76-84
    if ((flags & ZSPH_OUT_HASH) && hash) scalar_i("hash", hash);            // :86-94
    if ((flags & ZSPH_OUT_TABLE) && table) scalar_i("table", table);
    if ((flags & ZSPH_OUT_VEL) && vel) vector_f("vel", vel, 3);             // :106-116
    if ((flags & ZSPH_OUT_ACC) && acc) vector_f("acc", acc, 4);             // :118-128
    std::ofstream f(path, std::ios::binary);
    if (!f) return fail(ZSPH_EIO, std::string("zsph_write_vtk: cannot open ") + path);
    f.write(out.data(), (std::streamsize)out.size());
    return f ? ZSPH_OK : fail(ZSPH_EIO, std::string("zsph_write_vtk: write failed: ") + path);
  } catch (const std::exception& e) {
    return fail(ZSPH_EIO, std::string("zsph_write_vtk: ") + e.what());
  } catch (...) {
    return fail(ZSPH_EIO, "zsph_write_vtk: unknown error");
  }
}

int zsph_read_vtk(const char* path, int n, float rho0, int accept_float, float* pos, float* vel, float* rhop,
                  float* acc, int* type, int* table) {
  const zsph::TraceRange trace_range_(__func__);
  // A malformed file must come back as an error code, never as a C++
  // exception through the C ABI (a std::bad_alloc, for example).
  try {
    return read_vtk_file(path, n, rho0, accept_float, pos, vel, rhop, acc, type, table);
  } catch (const std::exception& e) {
    return fail(ZSPH_EIO, std::string("zsph_read_vtk: ") + e.what());
  } catch (...) {
    return fail(ZSPH_EIO, "zsph_read_vtk: unknown error");
  }
}

}  // extern "C"

// ---- writer pool ------------------------------------------------------------

struct zsph_writer {
  struct Slot {
    float *pos = nullptr, *vel = nullptr, *rhop = nullptr, *acc = nullptr;
    int *type = nullptr, *hash = nullptr, *table = nullptr;
    cudaEvent_t done = nullptr;
    int step = 0;
    bool busy = false;
  };
  std::string out_dir;
  int n = 0, flags = 0;
  std::vector<Slot> slots;
  std::deque<int> queue;  // slots with a pending copy, in submission order
  std::mutex mu;
  std::condition_variable cv_work, cv_free;
  std::vector<std::thread> threads;
  bool stop = false;
  int errors = 0;
  std::string first_error;

  void run() {
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return;
        k = queue.front();
        queue.pop_front();
      }
      Slot& s = slots[k];
      cudaError_t e = cudaEventSynchronize(s.done);
      int rc = ZSPH_OK;
      std::string fname = out_dir + "/zsph" + std::to_string(s.step) + ".vtk";  // mul_thread.cu:63
      if (e == cudaSuccess)
        rc = zsph_write_vtk(fname.c_str(), n, s.pos, s.vel, s.rhop, s.type, s.acc, s.hash, s.table, flags);
      {
        std::lock_guard<std::mutex> lk(mu);
        if (e != cudaSuccess || rc != ZSPH_OK) {
          if (!errors++) first_error = e != cudaSuccess ? cudaGetErrorString(e) : "cannot write " + fname;
        }
        s.busy = false;
      }
      cv_free.notify_all();
    }
  }
};

extern "C" {

int zsph_writer_create(const char* output_path, int ptc_num, int flags, int nthreads, zsph_writer_t** out) {
  if (!output_path || ptc_num < 0 || nthreads < 1 || !out) return fail(ZSPH_EINVAL, "zsph_writer_create: bad argument");
  *out = nullptr;
  zsph_writer* w = nullptr;
  try {  // host allocation failures become a status code, not an exception through the C ABI
    w = new zsph_writer();
    w->out_dir = output_path;
    w->n = ptc_num;
    w->flags = flags;
    w->slots.resize((size_t)nthreads);
  } catch (const std::exception& ex) {
    delete w;
    return fail(ZSPH_EIO, std::string("zsph_writer_create: ") + ex.what());
  }
  const size_t N = (size_t)(ptc_num ? ptc_num : 1);
  cudaError_t e = cudaSuccess;
  for (auto& s : w->slots) {
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.pos), N * 12);
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.vel), N * 12);
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.rhop), N * 8);
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.acc), N * 16);
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.type), N * 4);
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.hash), N * 4);
    if (!e) e = cudaMallocHost(reinterpret_cast<void**>(&s.table), N * 4);
    if (!e) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
  }
  if (e) {
    zsph_writer_destroy(w);
    return fail(ZSPH_ECUDA, std::string("zsph_writer_create: ") + cudaGetErrorString(e));
  }
  try {
    for (int t = 0; t < nthreads; ++t) w->threads.emplace_back([w] { w->run(); });
  } catch (const std::exception& ex) {  // a thread that could not start: stop and join the others
    zsph_writer_destroy(w);
    return fail(ZSPH_EIO, std::string("zsph_writer_create: cannot start a writer thread: ") + ex.what());
  }
  *out = w;
  return ZSPH_OK;
}

int zsph_writer_submit(zsph_writer_t* w, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int step, void* stream) {
  const zsph::TraceRange trace_range_(__func__);
  if (!w || !ptc || !tmp) return fail(ZSPH_EINVAL, "zsph_writer_submit: bad argument");
  int k = -1;
  {
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv_free.wait(lk, [&] {
      for (size_t i = 0; i < w->slots.size(); ++i)
        if (!w->slots[i].busy) return true;
      return false;
    });
    for (size_t i = 0; i < w->slots.size(); ++i)
      if (!w->slots[i].busy) { k = (int)i; break; }
    w->slots[(size_t)k].busy = true;
  }
  auto& s = w->slots[(size_t)k];
  s.step = step;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t N = (size_t)w->n;
  const int fl = w->flags;
  cudaError_t e = cudaMemcpyAsync(s.pos, ptc->pos, N * 12, cudaMemcpyDeviceToHost, st);  // gmemcpy.cu:5
  if (!e && (fl & ZSPH_OUT_VEL)) e = cudaMemcpyAsync(s.vel, ptc->vel, N * 12, cudaMemcpyDeviceToHost, st);
  if (!e && (fl & (ZSPH_OUT_RHO | ZSPH_OUT_P))) e = cudaMemcpyAsync(s.rhop, ptc->rhop, N * 8, cudaMemcpyDeviceToHost, st);
  if (!e && (fl & ZSPH_OUT_TYPE)) e = cudaMemcpyAsync(s.type, ptc->type, N * 4, cudaMemcpyDeviceToHost, st);
  if (!e && (fl & ZSPH_OUT_TABLE)) e = cudaMemcpyAsync(s.table, ptc->table, N * 4, cudaMemcpyDeviceToHost, st);
  if (!e && (fl & ZSPH_OUT_HASH)) e = cudaMemcpyAsync(s.hash, tmp->hash, N * 4, cudaMemcpyDeviceToHost, st);
  if (!e && (fl & ZSPH_OUT_ACC)) e = cudaMemcpyAsync(s.acc, tmp->acc_drhodt, N * 16, cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaEventRecord(s.done, st);
  if (e) {
    std::lock_guard<std::mutex> lk(w->mu);
    s.busy = false;
    return fail(ZSPH_ECUDA, std::string("zsph_writer_submit: ") + cudaGetErrorString(e));
  }
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->queue.push_back(k);
  }
  w->cv_work.notify_one();
  return ZSPH_OK;
}

int zsph_writer_destroy(zsph_writer_t* w) {
  if (!w) return ZSPH_OK;
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->stop = true;
  }
  w->cv_work.notify_all();
  for (auto& t : w->threads) t.join();
  int rc = w->errors ? ZSPH_EIO : ZSPH_OK;
  if (w->errors) fail(ZSPH_EIO, "zsph_writer: " + w->first_error);
  for (auto& s : w->slots) {
    void* bufs[] = {s.pos, s.vel, s.rhop, s.acc, s.type, s.hash, s.table};
    for (void* b : bufs)
      if (b) cudaFreeHost(b);
    if (s.done) cudaEventDestroy(s.done);
  }
  delete w;
  return rc;
}

}  // extern "C"
