// zsph_sort_index_noalloc: the stable cell-key sort of zsph_sort_index for
// callers that cannot allocate device memory.
//
// Who needs it: zsph_sort_index works through a handle, and zsph_create
// allocates the handle's scratch with cudaMalloc.  Some callers must not
// allocate device memory once they are running: an application whose device
// memory is entirely reserved by another allocator (a framework's caching
// allocator, a fixed memory budget), or a time-critical loop in which
// cudaMalloc/cudaFree, which may synchronise the device, are not acceptable.
// This entry point needs no handle and allocates nothing: its scratch is the
// file-scope device array below, of a fixed maximum size that every GPU which
// loads the library holds until the process exits.
//
// Limits: at most kNoAllocMaxParticles particles and kNoAllocMaxCells cells;
// larger problems are rejected with ZSPH_EINVAL (use zsph_sort_index).
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture on the device.  The address belongs to the
// device's context: the lookup is kept together with the context's id
// (cuCtxGetId, reached through the runtime's driver entry points, so the
// library does not link libcuda), and a call made in a different context, for
// example after cudaDeviceReset, looks the address up again.  The first call
// after such a reset is then a set-up call too and must also come before any
// stream capture.
//
// Keys: hash values must lie in [0, grid_num).  A key outside that range is
// sorted as if it were 0 (negative keys) or grid_num - 1 (keys too large) and
// is written back clamped; this entry point does not report it, since the
// only place it could report it is the shared array, which the next call
// clears.  zsph_sort_index on a handle reports the same condition as
// ZSPH_EINVAL through zsph_status.
//
// Sharing: every call on a device uses the same array, which keeps the last
// call's contents.  Each call clears the parts that must start at zero.  Calls
// whose work overlaps on the GPU (different streams, or different host
// threads) race on the array and must be serialised by the caller.
#include <cstdio>
#include <mutex>
#include <string>

#include "zsph_internal.cuh"

namespace {

using namespace zsph;

constexpr int kNoAllocMaxParticles = 131072;
constexpr int kNoAllocMaxCells = 131072;
constexpr int kNoAllocMaxTiles = (kNoAllocMaxCells + kScanTile - 1) / kScanTile;
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Byte offsets of the scratch regions inside the array (all 256-byte aligned).
constexpr size_t kOffCnt = 0;
constexpr size_t kOffCellLb = kOffCnt + align256(sizeof(int) * kNoAllocMaxCells);
constexpr size_t kOffKey = kOffCellLb + align256(sizeof(int) * (kNoAllocMaxCells + 1));
constexpr size_t kOffTicket = kOffKey + align256(sizeof(int) * kNoAllocMaxParticles);
constexpr size_t kOffPerm = kOffTicket + align256(sizeof(int) * kNoAllocMaxParticles);
constexpr size_t kOffVal = kOffPerm + align256(sizeof(int) * kNoAllocMaxParticles);
constexpr size_t kOffTileSum = kOffVal + align256(sizeof(int) * kNoAllocMaxParticles);
constexpr size_t kOffTileOff = kOffTileSum + align256(sizeof(int) * kNoAllocMaxTiles);
constexpr size_t kOffTileLast = kOffTileOff + align256(sizeof(int) * kNoAllocMaxTiles);
constexpr size_t kOffMisc = kOffTileLast + align256(sizeof(int) * kNoAllocMaxTiles);
constexpr size_t kOffBigList = kOffMisc + align256(sizeof(int) * 8);
constexpr size_t kOffFlags = kOffBigList + align256(sizeof(int) * kBigListCap);
constexpr size_t kNoAllocBytes = kOffFlags + align256(sizeof(int));  // about 3.2 MB

// The scratch.  In host code this name is only a host-side stand-in for the
// device array: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocBytes];

std::mutex g_mu;
unsigned char* g_base[kMaxDevices] = {};
unsigned long long g_ctx[kMaxDevices] = {};  // id of the context g_base[dev] was looked up in

// errors are reported through zsph_last_error(NULL, ...)
int fail(int code, const std::string& m) {
  record_library_error(m);
  return code;
}

}  // namespace

extern "C" {

int zsph_sort_index_noalloc(const zsph_gpu_param_t* gparam, int grid_num, const zsph_tmp_t* tmp, void* stream) {
  if (!gparam || !tmp) return fail(ZSPH_EINVAL, "zsph_sort_index_noalloc: null argument");
  const int n = gparam->ptc_num;
  if (n < 0 || grid_num < 1) return fail(ZSPH_EINVAL, "zsph_sort_index_noalloc: need ptc_num >= 0 and grid_num >= 1");
  if (n > kNoAllocMaxParticles || grid_num > kNoAllocMaxCells) {
    char b[200];
    std::snprintf(b, sizeof b,
                  "zsph_sort_index_noalloc: %d particles / %d cells exceed its fixed scratch (at most %d particles "
                  "and %d cells); use zsph_sort_index",
                  n, grid_num, kNoAllocMaxParticles, kNoAllocMaxCells);
    return fail(ZSPH_EINVAL, b);
  }
  if (n > 0 && (!tmp->hash || !tmp->index)) return fail(ZSPH_EINVAL, "zsph_sort_index_noalloc: null hash or index");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ZSPH_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(ZSPH_EINVAL, "zsph_sort_index_noalloc: device index too large");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_base[dev] || ctx == 0 || ctx != g_ctx[dev]) {  // once per device and context, with that device current
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_sort_scratch);
      if (e != cudaSuccess) {
        g_base[dev] = nullptr;
        record_library_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return ZSPH_ECUDA;
      }
      g_base[dev] = static_cast<unsigned char*>(p);
      g_ctx[dev] = current_context_id();  // the lookup made the device's context current if it was not
    }
    base = g_base[dev];
  }
  Scratch s{};
  s.cnt = reinterpret_cast<int*>(base + kOffCnt);
  s.cell_lb = reinterpret_cast<int*>(base + kOffCellLb);
  s.key = reinterpret_cast<int*>(base + kOffKey);
  s.ticket = reinterpret_cast<int*>(base + kOffTicket);
  s.perm = reinterpret_cast<int*>(base + kOffPerm);
  s.val = reinterpret_cast<int*>(base + kOffVal);
  s.tile_sum = reinterpret_cast<int*>(base + kOffTileSum);
  s.tile_off = reinterpret_cast<int*>(base + kOffTileOff);
  s.tile_last = reinterpret_cast<int*>(base + kOffTileLast);
  s.misc = reinterpret_cast<int*>(base + kOffMisc);
  s.big_list = reinterpret_cast<int*>(base + kOffBigList);
  s.flags = reinterpret_cast<int*>(base + kOffFlags);
  KParams kp{};
  kp.p = *gparam;
  kp.n = n;
  kp.G = grid_num;
  const int tiles = (grid_num + kScanTile - 1) / kScanTile;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: clear what must start at zero
  e = cudaMemsetAsync(s.cnt, 0, sizeof(int) * (size_t)grid_num, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.misc, 0, sizeof(int) * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.flags, 0, sizeof(int), st);
  if (e == cudaSuccess) e = launch_sort_index(kp, s, tiles, *tmp, st);
  if (e != cudaSuccess) return fail(ZSPH_ECUDA, std::string("zsph_sort_index_noalloc: ") + cudaGetErrorString(e));
  return ZSPH_OK;
}

}  // extern "C"
