/* nvtx_probe.c - a minimal NVTX injection library for the tracing test.
 *
 * Named by NVTX_INJECTION64_PATH, it is loaded by the first NVTX call of the
 * process (the loader and the callback tables are the public NVTX3 injection
 * interface, nvtx3/nvtxDetail/nvtxInit.h and nvtxTypes.h). It records every
 * domain creation and every domain range push and pop, in order, and hands
 * the record to the test through nvtx_probe_dump(). Test infrastructure: the
 * library under test never loads it by itself.
 */
#include <nvtx3/nvToolsExt.h>

#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#define PROBE_DOMAINS 16
#define PROBE_LOG 65536

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static char g_domains[PROBE_DOMAINS][64];
static int g_ndomains = 0;
static char g_log[PROBE_LOG];
static size_t g_used = 0;
static int g_dropped = 0;

/* Domain handles are 1-based indexes into g_domains. */
static const char* domain_name(nvtxDomainHandle_t d) {
  const intptr_t i = (intptr_t)d;
  return (i >= 1 && i <= g_ndomains) ? g_domains[i - 1] : "";
}

static void append(const char* kind, nvtxDomainHandle_t d, const char* message) {
  char line[256];
  const int n = snprintf(line, sizeof line, "%s\t%s\t%lu\t%s\n", kind, domain_name(d), (unsigned long)pthread_self(),
                         message != NULL ? message : "");
  if (n <= 0) return;
  pthread_mutex_lock(&g_lock);
  if (g_used + (size_t)n < PROBE_LOG) {
    memcpy(g_log + g_used, line, (size_t)n);
    g_used += (size_t)n;
  } else {
    g_dropped = 1;
  }
  pthread_mutex_unlock(&g_lock);
}

static nvtxDomainHandle_t NVTX_API probe_domain_create(const char* name) {
  pthread_mutex_lock(&g_lock);
  intptr_t handle = 0;
  if (g_ndomains < PROBE_DOMAINS) {
    snprintf(g_domains[g_ndomains], sizeof g_domains[0], "%s", name != NULL ? name : "");
    handle = ++g_ndomains;
  }
  pthread_mutex_unlock(&g_lock);
  return (nvtxDomainHandle_t)handle;
}

static int NVTX_API probe_push(nvtxDomainHandle_t d, const nvtxEventAttributes_t* a) {
  const char* message = (a != NULL && a->messageType == NVTX_MESSAGE_TYPE_ASCII) ? a->message.ascii : "";
  append("push", d, message);
  return 0;
}

static int NVTX_API probe_pop(nvtxDomainHandle_t d) {
  append("pop", d, "");
  return 0;
}

int NVTX_API InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get_export_table) {
  const NvtxExportTableCallbacks* callbacks = (const NvtxExportTableCallbacks*)get_export_table(NVTX_ETID_CALLBACKS);
  if (callbacks == NULL) return 0;
  NvtxFunctionTable table = 0;
  unsigned int size = 0;
  if (!callbacks->GetModuleFunctionTable(NVTX_CB_MODULE_CORE2, &table, &size) || table == 0) return 0;
  if (size < NVTX_CBID_CORE2_DomainCreateA) return 0;
  *table[NVTX_CBID_CORE2_DomainCreateA] = (NvtxFunctionPointer)probe_domain_create;
  *table[NVTX_CBID_CORE2_DomainRangePushEx] = (NvtxFunctionPointer)probe_push;
  *table[NVTX_CBID_CORE2_DomainRangePop] = (NvtxFunctionPointer)probe_pop;
  return 1;
}

/* Copies the record (tab-separated lines: push|pop, domain, thread, message)
 * into out; returns its length, or -1 when it did not fit or lines were lost. */
long nvtx_probe_dump(char* out, size_t capacity) {
  pthread_mutex_lock(&g_lock);
  long n = (long)g_used;
  if (g_dropped || g_used + 1 > capacity) {
    n = -1;
  } else {
    memcpy(out, g_log, g_used);
    out[g_used] = '\0';
  }
  pthread_mutex_unlock(&g_lock);
  return n;
}
