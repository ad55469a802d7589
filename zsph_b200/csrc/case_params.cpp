// Host-side case set-up: JSON case reader and derived constants.
//
// zsph_read_json       <- single_gpu_sph_src/io/read_json.cu:5-51
// zsph_set_cpu_param   <- single_gpu_sph_src/lib/init.cu:153-219
// zsph_set_gpu_param   <- single_gpu_sph_src/lib/init.cu:221-251
// zsph_check_dt        <- single_gpu_sph_src/lib/check.cu:3-18
//
// The derivation keeps the reference's float arithmetic (left-to-right
// products, sqrt/abs of a float through their float overloads, the literal
// 3.1415926f, truncating grid dimensions) so that the constants, and with them
// the cell hashes, are bit-identical to the reference's.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "../../include/zsph.h"
#include "trace.h"

namespace {

// Minimal JSON reader for the reference's flat case file: one object whose
// values are numbers, strings, booleans or null; nested values are parsed
// and skipped.  Numbers keep their text so that ints and floats convert the
// way nlohmann::json's get<> does (any number converts to float or int).
struct JValue {
  enum Kind { NUM, STR, OTHER } kind = OTHER;
  double num = 0.0;
  std::string str;
};

class JParser {
 public:
  explicit JParser(const std::string& s) : s_(s) {}
  bool parse(std::map<std::string, JValue>& out, std::string& err) {
    ws();
    if (!eat('{')) return fail(err, "expected '{' at top level");
    ws();
    if (eat('}')) return true;
    for (;;) {
      ws();
      std::string key;
      if (!str(key)) return fail(err, "expected a string key");
      ws();
      if (!eat(':')) return fail(err, "expected ':' after key \"" + key + "\"");
      ws();
      JValue v;
      if (!value(v)) return fail(err, "bad value for key \"" + key + "\"");
      out[key] = v;
      ws();
      if (eat(',')) continue;
      if (eat('}')) break;
      return fail(err, "expected ',' or '}'");
    }
    ws();
    if (p_ != s_.size()) return fail(err, "trailing characters after the object");
    return true;
  }

 private:
  const std::string& s_;
  size_t p_ = 0;
  bool fail(std::string& err, const std::string& m) {
    char b[64];
    snprintf(b, sizeof b, " (at byte %zu)", p_);
    err = m + b;
    return false;
  }
  void ws() {
    while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
  }
  bool eat(char c) {
    if (p_ < s_.size() && s_[p_] == c) { ++p_; return true; }
    return false;
  }
  bool str(std::string& o) {
    if (!eat('"')) return false;
    while (p_ < s_.size() && s_[p_] != '"') {
      char c = s_[p_++];
      if (c == '\\' && p_ < s_.size()) {
        char e = s_[p_++];
        switch (e) {
          case 'n': o += '\n'; break;
          case 't': o += '\t'; break;
          case 'r': o += '\r'; break;
          case 'b': o += '\b'; break;
          case 'f': o += '\f'; break;
          case 'u': p_ += 4; o += '?'; break;
          default: o += e;
        }
      } else {
        o += c;
      }
    }
    return eat('"');
  }
  bool value(JValue& v) {
    if (p_ >= s_.size()) return false;
    char c = s_[p_];
    if (c == '"') { v.kind = JValue::STR; return str(v.str); }
    if (c == '{' || c == '[') return skip_nested();
    if (s_.compare(p_, 4, "true") == 0) { p_ += 4; return true; }
    if (s_.compare(p_, 5, "false") == 0) { p_ += 5; return true; }
    if (s_.compare(p_, 4, "null") == 0) { p_ += 4; return true; }
    const char* b = s_.c_str() + p_;
    char* e = nullptr;
    double d = std::strtod(b, &e);
    if (e == b) return false;
    p_ += (size_t)(e - b);
    v.kind = JValue::NUM;
    v.num = d;
    return true;
  }
  bool skip_nested() {
    int depth = 0;
    while (p_ < s_.size()) {
      char c = s_[p_];
      if (c == '"') { std::string t; if (!str(t)) return false; continue; }
      if (c == '{' || c == '[') ++depth;
      if (c == '}' || c == ']') { --depth; if (depth == 0) { ++p_; return true; } }
      ++p_;
    }
    return false;
  }
};

void set_err(char* err, int len, const std::string& m) {
  if (err && len > 0) {
    std::snprintf(err, (size_t)len, "%s", m.c_str());
  }
}

void copy_str(char* dst, size_t cap, const std::string& s) {
  std::snprintf(dst, cap, "%s", s.c_str());
}

}  // namespace

namespace {

int read_json_file(const char* path, zsph_json_t* out, char* err, int errlen) {
  std::ifstream f(path);
  if (!f) { set_err(err, errlen, std::string("cannot open ") + path); return ZSPH_EIO; }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  std::map<std::string, JValue> kv;
  std::string perr;
  if (!JParser(text).parse(kv, perr)) { set_err(err, errlen, "JSON parse error: " + perr); return ZSPH_EIO; }
  std::memset(out, 0, sizeof *out);
  std::string missing;
  auto num = [&](const char* k, double& v) -> bool {
    auto it = kv.find(k);
    if (it == kv.end() || it->second.kind != JValue::NUM) {
      if (missing.empty()) missing = std::string(it == kv.end() ? "missing key: " : "key is not a number: ") + k;
      return false;
    }
    v = it->second.num;
    return true;
  };
  auto fnum = [&](const char* k, float& dst) { double v; if (num(k, v)) dst = (float)v; };
  // An int key takes any number and truncates it, as nlohmann's get<int> does;
  // one outside the int range (where the conversion is undefined) is an error.
  auto inum = [&](const char* k, int& dst) {
    double v;
    if (!num(k, v)) return;
    if (!(v > -2147483649.0 && v < 2147483648.0)) {
      if (missing.empty()) missing = std::string("key is out of the int range: ") + k;
      return;
    }
    dst = (int)v;
  };
  auto sval = [&](const char* k, char* dst, size_t cap) {
    auto it = kv.find(k);
    if (it == kv.end() || it->second.kind != JValue::STR) {
      if (missing.empty()) missing = std::string(it == kv.end() ? "missing key: " : "key is not a string: ") + k;
      return;
    }
    copy_str(dst, cap, it->second.str);
  };
  // read_json.cu:12-49, same keys in the same order
  fnum("g", out->g);
  fnum("rho0", out->rho0);
  fnum("dx", out->dx);
  fnum("h_factor", out->h_factor);
  fnum("r_factor", out->r_factor);
  fnum("eta_factor", out->eta_factor);
  fnum("cs_factor", out->cs_factor);
  fnum("delta", out->delta);
  fnum("alpha", out->alpha);
  fnum("xmin", out->xmin);
  fnum("xmax", out->xmax);
  fnum("ymin", out->ymin);
  fnum("ymax", out->ymax);
  fnum("zmin", out->zmin);
  fnum("zmax", out->zmax);
  fnum("grid_layer_factor", out->grid_layer_factor);
  fnum("grid_size_factor", out->grid_size_factor);
  fnum("dt", out->dt);
  inum("start_step", out->start_step);
  inum("current_step", out->current_step);
  inum("end_step", out->end_step);
  inum("output_step", out->output_step);
  inum("ptc_num", out->ptc_num);
  inum("water_ptc_num", out->water_ptc_num);
  inum("air_ptc_num", out->air_ptc_num);
  inum("wall_ptc_num", out->wall_ptc_num);
  inum("rigid_ptc_num", out->rigid_ptc_num);
  inum("thread_num", out->thread_num);
  inum("gpu_id", out->gpu_id);
  sval("input_path", out->input_path, sizeof out->input_path);
  sval("output_path", out->output_path, sizeof out->output_path);
  sval("git_hash", out->git_hash, sizeof out->git_hash);
  if (!missing.empty()) { set_err(err, errlen, missing); return ZSPH_EIO; }
  set_err(err, errlen, "");
  return ZSPH_OK;
}

}  // namespace

extern "C" int zsph_read_json(const char* path, zsph_json_t* out, char* err, int errlen) {
  const zsph::TraceRange trace_range_(__func__);
  if (!path || !out) { set_err(err, errlen, "null argument"); return ZSPH_EINVAL; }
  // No C++ exception leaves through the C ABI: it becomes an error code.
  try {
    return read_json_file(path, out, err, errlen);
  } catch (const std::exception& e) {
    set_err(err, errlen, std::string("zsph_read_json: ") + e.what());
    return ZSPH_EIO;
  } catch (...) {
    set_err(err, errlen, "zsph_read_json: unknown error");
    return ZSPH_EIO;
  }
}

namespace {

int read_options_file(const char* path, zsph_case_options_t* out, char* err, int errlen) {
  std::ifstream f(path);
  if (!f) { set_err(err, errlen, std::string("cannot open ") + path); return ZSPH_EIO; }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  std::map<std::string, JValue> kv;
  std::string perr;
  if (!JParser(text).parse(kv, perr)) { set_err(err, errlen, "JSON parse error: " + perr); return ZSPH_EIO; }
  std::memset(out, 0, sizeof *out);
  out->equations = ZSPH_EQ_DELTA;
  auto bad = [&](const std::string& m) { set_err(err, errlen, m); return ZSPH_EINVAL; };
  auto it = kv.find("equations");
  if (it != kv.end()) {
    if (it->second.kind != JValue::STR) return bad("key is not a string: equations");
    if (it->second.str == "delta") out->equations = ZSPH_EQ_DELTA;
    else if (it->second.str == "simple") out->equations = ZSPH_EQ_SIMPLE;
    else return bad("equations must be \"delta\" or \"simple\", not \"" + it->second.str + "\"");
  }
  it = kv.find("eos");
  if (it != kv.end()) {
    if (it->second.kind != JValue::STR) return bad("key is not a string: eos");
    if (it->second.str != "linear")
      return bad("eos \"" + it->second.str + "\" is not implemented; the reference's code uses \"linear\"");
  }
  it = kv.find("snapshot_every");
  if (it != kv.end()) {
    const double v = it->second.num;
    if (it->second.kind != JValue::NUM || !(v >= 0.0 && v < 2147483648.0) || v != (double)(long long)v)
      return bad("snapshot_every must be a whole number >= 0");
    out->snapshot_every = (int)v;
  }
  it = kv.find("resume");
  if (it != kv.end()) {
    if (it->second.kind != JValue::STR) return bad("key is not a string: resume");
    if (it->second.str.size() >= sizeof out->resume) return bad("resume: path too long");
    copy_str(out->resume, sizeof out->resume, it->second.str);
  }
  set_err(err, errlen, "");
  return ZSPH_OK;
}

}  // namespace

extern "C" int zsph_read_case_options(const char* path, zsph_case_options_t* out, char* err, int errlen) {
  const zsph::TraceRange trace_range_(__func__);
  if (!path || !out) { set_err(err, errlen, "null argument"); return ZSPH_EINVAL; }
  try {
    return read_options_file(path, out, err, errlen);
  } catch (const std::exception& e) {
    set_err(err, errlen, std::string("zsph_read_case_options: ") + e.what());
    return ZSPH_EIO;
  } catch (...) {
    set_err(err, errlen, "zsph_read_case_options: unknown error");
    return ZSPH_EIO;
  }
}

extern "C" int zsph_check_dt(const zsph_cpu_param_t* param, float* dt_max_out) {
  if (!param) return ZSPH_EINVAL;
  // check.cu:6: 0.25 is a double literal; sqrt of a float argument.
  const float arg = -param->g * (param->zmax - param->zmin);
  const float dt_max = (float)(0.25 * (double)param->h / (double)std::sqrt(arg));
  if (dt_max_out) *dt_max_out = dt_max;
  return (param->dt <= dt_max) ? ZSPH_OK : ZSPH_EINVAL;  // check.cu:9-17
}

extern "C" int zsph_set_cpu_param(zsph_cpu_param_t* p, const zsph_json_t* j) {
  if (!p || !j) return ZSPH_EINVAL;
  std::memset(p, 0, sizeof *p);
  p->g = j->g;
  p->m = j->rho0 * j->dx * j->dx * j->dx;  // init.cu:157
  p->rho0 = j->rho0;
  p->dx = j->dx;
  p->h = j->h_factor * j->dx;
  p->r = j->r_factor * j->h_factor * j->dx;
  p->eta = j->eta_factor * j->h_factor * j->dx;
  p->cs = j->cs_factor * std::sqrt(std::fabs(j->g) * (j->zmax - j->zmin));  // init.cu:163
  p->delta = j->delta;
  p->alpha = j->alpha;
  p->adh = 21.0f / (16.0f * 3.1415926f * p->h * p->h * p->h);  // init.cu:166
  p->xmin = j->xmin; p->xmax = j->xmax;
  p->ymin = j->ymin; p->ymax = j->ymax;
  p->zmin = j->zmin; p->zmax = j->zmax;
  p->grid_size = j->r_factor * j->h_factor * j->dx / j->grid_size_factor;  // init.cu:177
  p->grid_factor = (int)j->grid_size_factor;
  p->grid_xmin = j->xmin - p->grid_size * j->grid_layer_factor;
  p->grid_xmax = j->xmax + p->grid_size * j->grid_layer_factor;
  p->grid_ymin = j->ymin - p->grid_size * j->grid_layer_factor;
  p->grid_ymax = j->ymax + p->grid_size * j->grid_layer_factor;
  p->grid_zmin = j->zmin - p->grid_size * j->grid_layer_factor;
  p->grid_zmax = j->zmax + p->grid_size * j->grid_layer_factor;
  p->grid_xdim = (int)((p->grid_xmax - p->grid_xmin) / p->grid_size);  // init.cu:185-187
  p->grid_ydim = (int)((p->grid_ymax - p->grid_ymin) / p->grid_size);
  p->grid_zdim = (int)((p->grid_zmax - p->grid_zmin) / p->grid_size);
  p->grid_num = p->grid_xdim * p->grid_ydim * p->grid_zdim;
  p->grid_hash_min = 0;
  p->grid_hash_max = p->grid_num - 1;
  p->ptc_num = j->ptc_num;
  p->water_ptc_num = j->water_ptc_num;
  p->air_ptc_num = j->air_ptc_num;
  p->wall_ptc_num = j->wall_ptc_num;
  p->rigid_ptc_num = j->rigid_ptc_num;
  p->thread_num = j->thread_num;
  p->gpu_id = j->gpu_id;
  std::memcpy(p->input_path, j->input_path, sizeof p->input_path);
  std::memcpy(p->output_path, j->output_path, sizeof p->output_path);
  std::memcpy(p->git_hash, j->git_hash, sizeof p->git_hash);
  p->dt = j->dt;
  p->start_step = j->start_step;
  p->current_step = j->current_step;
  p->end_step = j->end_step;
  p->output_step = j->output_step;
  return zsph_check_dt(p, nullptr);  // init.cu:218
}

extern "C" int zsph_set_gpu_param(zsph_gpu_param_t* g, const zsph_cpu_param_t* c) {
  if (!g || !c) return ZSPH_EINVAL;
  g->half_dt = c->dt / 2.0f;  // init.cu:223
  g->h = c->h;
  g->g = c->g;
  g->m = c->m;
  g->rho0 = c->rho0;
  g->adh = c->adh;
  g->h2 = c->h * c->h;
  g->eta2 = c->eta * c->eta;
  g->cs2 = c->cs * c->cs;
  g->alpha = c->alpha;
  g->delta_h_cs = c->delta * c->h * c->cs;        // init.cu:233
  g->h_cs_rho_m = c->h * c->cs * c->rho0 * c->m;  // init.cu:234
  g->grid_factor = c->grid_factor;
  g->grid_size = c->grid_size;
  g->grid_xmin = c->grid_xmin;
  g->grid_ymin = c->grid_ymin;
  g->grid_zmin = c->grid_zmin;
  g->grid_xdim = c->grid_xdim;
  g->grid_ydim = c->grid_ydim;
  g->grid_zdim = c->grid_zdim;
  g->grid_hash_min = c->grid_hash_min;
  g->grid_hash_max = c->grid_hash_max;
  g->ptc_num = c->ptc_num;
  return ZSPH_OK;
}
