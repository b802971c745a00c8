/* A minimal NVTX injection library for the tests (TEST INFRASTRUCTURE ONLY): loaded by the NVTX
 * code compiled into libmqb200 when NVTX_INJECTION64_PATH names it, it records the names of the
 * ranges pushed (nvtxRangePushA) and counts the pops, so a test can check the library's ranges
 * without a profiler or a GPU. */
#include <nvtx3/nvToolsExt.h>
#include <string.h>

#define MAX_NAMES 256
static char g_names[MAX_NAMES][64];
static int g_pushes = 0, g_pops = 0;

static int record_push(const char *message) {
    if (g_pushes < MAX_NAMES) {
        strncpy(g_names[g_pushes], message ? message : "", sizeof(g_names[0]) - 1);
        g_names[g_pushes][sizeof(g_names[0]) - 1] = '\0';
    }
    return g_pushes++;
}

static int record_pop(void) { return g_pops++; }

/* The NVTX loader calls this once; the core module's function table gets our push and pop. */
int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_export_table) {
    const NvtxExportTableCallbacks *cb = (const NvtxExportTableCallbacks *)get_export_table(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable table = 0;
    unsigned int size = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size)) return 0;
    if (size <= NVTX_CBID_CORE_RangePop) return 0;
    *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)record_push;
    *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)record_pop;
    return 1;
}

int recorder_pushes(void) { return g_pushes; }
int recorder_pops(void) { return g_pops; }
const char *recorder_name(int i) { return i >= 0 && i < g_pushes && i < MAX_NAMES ? g_names[i] : ""; }
