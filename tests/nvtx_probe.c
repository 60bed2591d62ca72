/* A minimal NVTX tool for tests/test_nvtx.py: loaded by the NVTX runtime through
 * NVTX_INJECTION64_PATH, it replaces the range push / pop callbacks and writes one line
 * per call to the file named by CPT_NVTX_LOG. Uses the tool-side interface of the
 * public NVTX v3 headers (nvtxDetail/nvtxTypes.h). */
#include <stdio.h>
#include <stdlib.h>
#include <nvtx3/nvToolsExt.h>

static FILE* g_log;

static int NVTX_API probe_push(const char* message)
{
    if (g_log) {
        fprintf(g_log, "push %s\n", message ? message : "");
        fflush(g_log);
    }
    return 0;
}

static int NVTX_API probe_pop(void)
{
    if (g_log) {
        fprintf(g_log, "pop\n");
        fflush(g_log);
    }
    return 0;
}

int NVTX_API InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_table)
{
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get_table(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable core = 0;
    unsigned int size = 0;
    const char* path = getenv("CPT_NVTX_LOG");
    if (!cb || !path || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &core, &size)) return 0;
    if (size <= NVTX_CBID_CORE_RangePop) return 0;
    *core[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)probe_push;
    *core[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)probe_pop;
    g_log = fopen(path, "w");
    return g_log != 0;
}
