/* nvtx_probe.c — an NVTX 3 injection library for the tests: loaded through
 * NVTX_INJECTION64_PATH, it takes over the domain create / push / pop callbacks and writes one
 * line per event to the file named by VOSS_NVTX_LOG ("domain <name>", "push <name>", "pop"). */
#include <nvtx3/nvToolsExt.h>
#include <stdio.h>
#include <stdlib.h>

static FILE* g_log;
static struct nvtxDomainRegistration_st* g_domain = (struct nvtxDomainRegistration_st*)&g_log;

static nvtxDomainHandle_t NVTX_API probe_domain_create(const char* name) {
  fprintf(g_log, "domain %s\n", name);
  fflush(g_log);
  return g_domain;
}

static int NVTX_API probe_push(nvtxDomainHandle_t d, const nvtxEventAttributes_t* a) {
  (void)d;
  fprintf(g_log, "push %s\n", a->messageType == NVTX_MESSAGE_TYPE_ASCII ? a->message.ascii : "?");
  fflush(g_log);
  return 0;
}

static int NVTX_API probe_pop(nvtxDomainHandle_t d) {
  (void)d;
  fprintf(g_log, "pop\n");
  fflush(g_log);
  return 0;
}

int NVTX_API InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get) {
  const char* path = getenv("VOSS_NVTX_LOG");
  if (!path || !(g_log = fopen(path, "w"))) return 0;
  const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get(NVTX_ETID_CALLBACKS);
  NvtxFunctionTable t = 0;
  unsigned int n = 0;
  if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE2, &t, &n) || n < NVTX_CBID_CORE2_DomainCreateA)
    return 0;
  *t[NVTX_CBID_CORE2_DomainCreateA] = (NvtxFunctionPointer)probe_domain_create;
  *t[NVTX_CBID_CORE2_DomainRangePushEx] = (NvtxFunctionPointer)probe_push;
  *t[NVTX_CBID_CORE2_DomainRangePop] = (NvtxFunctionPointer)probe_pop;
  return 1;
}
