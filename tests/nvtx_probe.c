/* NVTX injection library for the CPU test of the library's trace ranges
 * (tests/test_nvtx_cpu.py).  The NVTX 3 header code inside libzsph_b200.so
 * loads it when NVTX_INJECTION64_PATH names it, through the documented tool
 * entry point InitializeInjectionNvtx2; it then appends "push <name>" for each
 * nvtxRangePushA and "pop" for each nvtxRangePop to the file ZSPH_NVTX_LOG. */
#include <stdio.h>
#include <stdlib.h>

#include <nvtx3/nvToolsExt.h> /* also declares the tool-side types (nvtxDetail/nvtxTypes.h) */

static FILE* g_log;

static int NVTX_API push_a(const char* message) {
  if (g_log) {
    fprintf(g_log, "push %s\n", message ? message : "");
    fflush(g_log);
  }
  return 0;
}

static int NVTX_API pop(void) {
  if (g_log) {
    fprintf(g_log, "pop\n");
    fflush(g_log);
  }
  return 0;
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_table) {
  const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get_table(NVTX_ETID_CALLBACKS);
  NvtxFunctionTable table = 0;
  unsigned int size = 0;
  if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size) || size <= NVTX_CBID_CORE_RangePop)
    return 0;
  *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)push_a;
  *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)pop;
  const char* path = getenv("ZSPH_NVTX_LOG");
  g_log = path ? fopen(path, "w") : NULL;
  return 1;
}
