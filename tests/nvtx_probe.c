/* nvtx_probe.c -- a minimal NVTX tool for the tracing test: loaded through
 * NVTX_INJECTION64_PATH, it takes over the push and pop callbacks of the
 * NVTX core module and records the name of every range pushed, and the
 * deepest nesting seen.  Built by tests/test_trace.py with the host compiler.
 * Test infrastructure only. */
#define NVTX_NO_IMPL
#include <nvtx3/nvToolsExt.h>
#include <string.h>

#define PROBE_MAX 256
static char g_names[PROBE_MAX][64];
static int g_count = 0;
static int g_depth = 0;
static int g_max_depth = 0;

static int NVTX_API probe_push(const char* message) {
    if (g_count < PROBE_MAX) {
        strncpy(g_names[g_count], message ? message : "", 63);
        g_names[g_count][63] = '\0';
        ++g_count;
    }
    ++g_depth;
    if (g_depth > g_max_depth) g_max_depth = g_depth;
    return g_depth - 1;
}

static int NVTX_API probe_pop(void) {
    --g_depth;
    return g_depth;
}

int probe_count(void) { return g_count; }
const char* probe_name(int i) { return (i >= 0 && i < g_count) ? g_names[i] : ""; }
int probe_depth(void) { return g_depth; }
int probe_max_depth(void) { return g_max_depth; }

int NVTX_API InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_export_table) {
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get_export_table(NVTX_ETID_CALLBACKS);
    if (!cb || !cb->GetModuleFunctionTable) return 0;
    NvtxFunctionTable table = 0;
    unsigned int size = 0;
    if (!cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size) || !table) return 0;
    if (size <= NVTX_CBID_CORE_RangePop) return 0;
    *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)probe_push;
    *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)probe_pop;
    return 1;
}
