// Checkpoint and resume: a binary snapshot of one particle buffer set and of
// the tmp arrays.
//
// The reference has no snapshot.  Its only resume state is the start_step /
// current_step pair of the case file (single_gpu_sph_src/io/read_json.cu:32-35)
// plus an input.vtk, and its VTK output does not read back as that input: the
// writer emits float arrays and never rho (io/write_vtk.cu:56-128), while the
// reader takes only double arrays (io/read_vkt.cu:27-39).  A snapshot here
// holds every array the next step reads, bit for bit, so a run resumed from it
// continues exactly as the saved run does.
//
// File layout (host byte order, checked on load through a marker word):
//   header   "ZSPHSNAP", u32 version, u32 byte-order marker 0x01020304,
//            i32 ptc_num, i32 grid_num, i32 step, u32 array count   (32 bytes)
//   per array: char name[16], u64 bytes, u64 checksum                (32 bytes)
//              then the array's bytes
// Arrays are the non-null members of zsph_ptc_t and zsph_tmp_t, in struct
// order; each has a fixed size from ptc_num and grid_num.  The checksum is a
// 64-bit multiply-rotate hash of the array's 32-bit words: it catches
// truncated or damaged files, it is not a cryptographic digest.
//
// A load reads the file twice: the first pass checks the header, every array's
// size and checksum and that each destination array is present, so a damaged
// file is refused before anything is written; the second pass copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "trace.h"
#include "zsph_internal.cuh"

namespace {

constexpr char kMagic[8] = {'Z', 'S', 'P', 'H', 'S', 'N', 'A', 'P'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kByteOrder = 0x01020304u;
constexpr size_t kChunk = size_t(16) << 20;  // bytes per staged copy and per read

struct FileHeader {
  char magic[8];
  uint32_t version, byte_order;
  int32_t ptc_num, grid_num, step;
  uint32_t narrays;
};
struct ArrayHeader {
  char name[16];
  uint64_t bytes, checksum;
};
static_assert(sizeof(FileHeader) == 32 && sizeof(ArrayHeader) == 32, "snapshot header layout");

struct Slot {
  const char* name;
  void* ptr;
  uint64_t bytes;
  bool required;  // needed to resume bit for bit
};

// The arrays of a snapshot, in file order.  Required: the state the next step
// reads (positions, velocities, densities and pressures, types, the original
// index table) and the cell bounds, whose entries from earlier searches can
// survive a search (the reference never clears them, sort.cu:30-60).
std::vector<Slot> slots(const zsph_ptc_t& p, const zsph_tmp_t& t, int n, int G) {
  const uint64_t N = (uint64_t)n * 4, C = (uint64_t)G * 4;
  return {{"pos", p.pos, 3 * N, true},         {"vel", p.vel, 3 * N, true},
          {"rhop", p.rhop, 2 * N, true},       {"tmp_pos", p.tmp_pos, 3 * N, false},
          {"tmp_vel", p.tmp_vel, 3 * N, false}, {"tmp_rhop", p.tmp_rhop, 2 * N, false},
          {"type", p.type, N, true},           {"table", p.table, N, true},
          {"acc_drhodt", t.acc_drhodt, 4 * N, false}, {"dofv_grandrho", t.dofv_grandrho, 4 * N, false},
          {"dofv", t.dofv, N, false},          {"index", t.index, N, false},
          {"hash", t.hash, N, false},          {"grid_start", t.grid_start, C, true},
          {"grid_end", t.grid_end, C, true}};
}

// 64-bit hash of a run of 32-bit words, fed in pieces whose sizes are
// multiples of 4 bytes.
struct Checksum {
  uint64_t h = 0x243F6A8885A308D3ull, words = 0;
  void add(const unsigned char* p, size_t nbytes) {
    for (size_t k = 0; k + 4 <= nbytes; k += 4) {
      uint32_t w;
      std::memcpy(&w, p + k, 4);
      h ^= (uint64_t)w * 0x9E3779B97F4A7C15ull;
      h = (h << 29) | (h >> 35);
      h *= 0xBF58476D1CE4E5B9ull;
    }
    words += nbytes / 4;
  }
  uint64_t value() const {
    uint64_t x = h ^ words;
    x ^= x >> 31;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 29;
    return x;
  }
};

int fail(int code, const std::string& m) {
  zsph::record_library_error(m);
  return code;
}

struct File {
  std::FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

bool same_name(const char* a, const char* b) { return std::strncmp(a, b, 16) == 0; }

int save(const char* who, const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int n, int G, int step,
         bool device, cudaStream_t st) {
  if (!path || !ptc || !tmp || n < 0 || G < 1) return fail(ZSPH_EINVAL, std::string(who) + ": bad argument");
  std::vector<Slot> all = slots(*ptc, *tmp, n, G), used;
  for (const Slot& s : all) {
    if (s.ptr) used.push_back(s);
    else if (s.required) return fail(ZSPH_EINVAL, std::string(who) + ": array " + s.name + " is null");
  }
  // written under a temporary name and renamed at the end, so that a failed
  // save never replaces an earlier good snapshot at `path`
  const std::string part = std::string(path) + ".part";
  File out;
  out.f = std::fopen(part.c_str(), "wb");
  if (!out.f) return fail(ZSPH_EIO, std::string(who) + ": cannot open " + part);
  struct Cleanup {
    File& f;
    const std::string& name;
    bool keep = false;
    ~Cleanup() {
      if (!keep) {
        if (f.f) std::fclose(f.f);
        f.f = nullptr;
        std::remove(name.c_str());
      }
    }
  } cleanup{out, part};
  FileHeader fh{};
  std::memcpy(fh.magic, kMagic, 8);
  fh.version = kVersion;
  fh.byte_order = kByteOrder;
  fh.ptc_num = n;
  fh.grid_num = G;
  fh.step = step;
  fh.narrays = (uint32_t)used.size();
  if (std::fwrite(&fh, sizeof fh, 1, out.f) != 1) return fail(ZSPH_EIO, std::string(who) + ": write failed");
  std::vector<unsigned char> stage(device ? kChunk : 0);
  for (const Slot& s : used) {
    ArrayHeader ah{};
    std::snprintf(ah.name, sizeof ah.name, "%s", s.name);
    ah.bytes = s.bytes;
    const long at = std::ftell(out.f);
    if (at < 0 || std::fwrite(&ah, sizeof ah, 1, out.f) != 1) return fail(ZSPH_EIO, std::string(who) + ": write failed");
    Checksum cs;
    for (uint64_t o = 0; o < s.bytes; o += kChunk) {
      const size_t len = (size_t)std::min<uint64_t>(kChunk, s.bytes - o);
      const unsigned char* src = static_cast<const unsigned char*>(s.ptr) + o;
      if (device) {
        cudaError_t e = cudaMemcpyAsync(stage.data(), src, len, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) return fail(ZSPH_ECUDA, std::string(who) + ": copy of " + s.name + ": " + cudaGetErrorString(e));
        src = stage.data();
      }
      cs.add(src, len);
      if (std::fwrite(src, 1, len, out.f) != len) return fail(ZSPH_EIO, std::string(who) + ": write failed");
    }
    ah.checksum = cs.value();
    if (std::fseek(out.f, at, SEEK_SET) != 0 || std::fwrite(&ah, sizeof ah, 1, out.f) != 1 ||
        std::fseek(out.f, 0, SEEK_END) != 0)
      return fail(ZSPH_EIO, std::string(who) + ": write failed");
  }
  const int closed = std::fclose(out.f);
  out.f = nullptr;
  if (closed != 0) return fail(ZSPH_EIO, std::string(who) + ": write failed");
  if (std::rename(part.c_str(), path) != 0) return fail(ZSPH_EIO, std::string(who) + ": cannot rename to " + path);
  cleanup.keep = true;
  return ZSPH_OK;
}

int load(const char* who, const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int n, int G, int* step,
         bool device, cudaStream_t st) {
  if (!path || !ptc || !tmp || n < 0 || G < 1) return fail(ZSPH_EINVAL, std::string(who) + ": bad argument");
  const std::string w = std::string(who) + ": " + path;
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return fail(ZSPH_EIO, std::string(who) + ": cannot open " + path);
  FileHeader fh{};
  if (std::fread(&fh, sizeof fh, 1, in.f) != 1 || std::memcmp(fh.magic, kMagic, 8) != 0)
    return fail(ZSPH_EIO, w + ": not a snapshot file");
  if (fh.byte_order != kByteOrder) return fail(ZSPH_EIO, w + ": written on a host of the other byte order");
  if (fh.version != kVersion) return fail(ZSPH_EIO, w + ": snapshot version " + std::to_string(fh.version));
  if (fh.ptc_num != n || fh.grid_num != G)
    return fail(ZSPH_EINVAL, w + ": holds " + std::to_string(fh.ptc_num) + " particles and " +
                                 std::to_string(fh.grid_num) + " cells; the buffers have " + std::to_string(n) +
                                 " and " + std::to_string(G));
  const std::vector<Slot> all = slots(*ptc, *tmp, n, G);
  if (fh.narrays > all.size()) return fail(ZSPH_EIO, w + ": too many arrays");
  // pass 1: sizes, names and checksums of every array in the file
  std::vector<long> data_at(all.size(), -1);
  std::vector<unsigned char> buf(kChunk);
  for (uint32_t a = 0; a < fh.narrays; ++a) {
    ArrayHeader ah{};
    if (std::fread(&ah, sizeof ah, 1, in.f) != 1) return fail(ZSPH_EIO, w + ": truncated");
    size_t k = 0;
    while (k < all.size() && !same_name(ah.name, all[k].name)) ++k;
    if (k == all.size()) return fail(ZSPH_EIO, w + ": unknown array");
    if (data_at[k] >= 0) return fail(ZSPH_EIO, w + ": array " + all[k].name + " appears twice");
    if (ah.bytes != all[k].bytes)
      return fail(ZSPH_EIO, w + ": array " + all[k].name + " has " + std::to_string(ah.bytes) + " bytes, expected " +
                                std::to_string(all[k].bytes));
    data_at[k] = std::ftell(in.f);
    Checksum cs;
    for (uint64_t o = 0; o < ah.bytes; o += kChunk) {
      const size_t len = (size_t)std::min<uint64_t>(kChunk, ah.bytes - o);
      if (std::fread(buf.data(), 1, len, in.f) != len) return fail(ZSPH_EIO, w + ": truncated in " + all[k].name);
      cs.add(buf.data(), len);
    }
    if (cs.value() != ah.checksum) return fail(ZSPH_EIO, w + ": checksum mismatch in " + all[k].name);
  }
  if (std::fgetc(in.f) != EOF) return fail(ZSPH_EIO, w + ": trailing bytes after the last array");
  for (size_t k = 0; k < all.size(); ++k)
    if (all[k].ptr && data_at[k] < 0) return fail(ZSPH_EIO, w + ": lacks array " + all[k].name);
  // pass 2: copy into every non-null destination
  for (size_t k = 0; k < all.size(); ++k) {
    if (!all[k].ptr) continue;
    if (std::fseek(in.f, data_at[k], SEEK_SET) != 0) return fail(ZSPH_EIO, w + ": seek failed");
    for (uint64_t o = 0; o < all[k].bytes; o += kChunk) {
      const size_t len = (size_t)std::min<uint64_t>(kChunk, all[k].bytes - o);
      unsigned char* dst = static_cast<unsigned char*>(all[k].ptr) + o;
      if (std::fread(device ? buf.data() : dst, 1, len, in.f) != len) return fail(ZSPH_EIO, w + ": read failed");
      if (device) {
        cudaError_t e = cudaMemcpyAsync(dst, buf.data(), len, cudaMemcpyHostToDevice, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) return fail(ZSPH_ECUDA, std::string(who) + ": copy of " + all[k].name + ": " + cudaGetErrorString(e));
      }
    }
  }
  if (step) *step = fh.step;
  return ZSPH_OK;
}

// No C++ exception (a failed host allocation, for example) leaves through the C ABI.
template <class F>
int guarded(const char* who, F&& f) {
  const zsph::TraceRange trace_range(who);
  try {
    return f();
  } catch (const std::exception& e) {
    return fail(ZSPH_EIO, std::string(who) + ": " + e.what());
  } catch (...) {
    return fail(ZSPH_EIO, std::string(who) + ": unknown error");
  }
}

}  // namespace

extern "C" {

int zsph_snapshot_save(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num, int grid_num,
                       int step, void* stream) {
  return guarded("zsph_snapshot_save", [&] {
    return save("zsph_snapshot_save", path, ptc, tmp, ptc_num, grid_num, step, true, static_cast<cudaStream_t>(stream));
  });
}

int zsph_snapshot_load(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num, int grid_num,
                       int* step, void* stream) {
  return guarded("zsph_snapshot_load", [&] {
    return load("zsph_snapshot_load", path, ptc, tmp, ptc_num, grid_num, step, true, static_cast<cudaStream_t>(stream));
  });
}

int zsph_snapshot_save_host(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num,
                            int grid_num, int step) {
  return guarded("zsph_snapshot_save_host", [&] {
    return save("zsph_snapshot_save_host", path, ptc, tmp, ptc_num, grid_num, step, false, nullptr);
  });
}

int zsph_snapshot_load_host(const char* path, const zsph_ptc_t* ptc, const zsph_tmp_t* tmp, int ptc_num,
                            int grid_num, int* step) {
  return guarded("zsph_snapshot_load_host", [&] {
    return load("zsph_snapshot_load_host", path, ptc, tmp, ptc_num, grid_num, step, false, nullptr);
  });
}

}  // extern "C"
