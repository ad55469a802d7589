// The id of the calling thread's current CUDA context, for host-side state
// that belongs to one device context: the allocation-free sort's scratch
// address (noalloc.cu) and the network kernels' shared-memory attributes
// (mlp.cu).  Such state is lost when the context goes (cudaDeviceReset, for
// example), and another device of the same process has its own, so it is
// kept per device together with this id and set up again when the id
// differs.  cuCtxGetId is reached through the runtime's driver entry points,
// so the library does not link libcuda.
#include <cuda.h>  // CUcontext / CUresult types only; the entry points come from the runtime
#include <cuda_runtime.h>

#include <mutex>

#include "zsph_internal.cuh"

namespace zsph {
namespace {

using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;
std::once_flag g_entry_once;

}  // namespace

unsigned long long current_context_id() {
  std::call_once(g_entry_once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(p);
    p = nullptr;
    q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(p);
  });
  if (!g_ctx_get_current || !g_ctx_get_id) return 0;
  CUcontext c = nullptr;
  if (g_ctx_get_current(&c) != CUDA_SUCCESS || !c) return 0;
  unsigned long long id = 0;
  if (g_ctx_get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

}  // namespace zsph
