/* A minimal NVTX tool for the tests: NVTX loads it through
 * NVTX_INJECTION64_PATH and calls InitializeInjectionNvtx2, which installs
 * handlers for nvtxRangePushA and nvtxRangePop.  Every push and pop is
 * written to the file named by PGMG_NVTX_LOG as one line,
 *
 *     <thread id> push <path>
 *     <thread id> pop <path>
 *
 * where <path> is the thread's stack of open range names joined by '/', so a
 * test can check both the ranges and their nesting.  Injection interface:
 * nvtx3/nvtxDetail/nvtxTypes.h (export table NVTX_ETID_CALLBACKS = 1, module
 * NVTX_CB_MODULE_CORE = 1, slots NVTX_CBID_CORE_RangePushA = 9 and
 * NVTX_CBID_CORE_RangePop = 11). */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/syscall.h>
#include <unistd.h>

typedef void (*fn_ptr)(void);
typedef fn_ptr** fn_table;
typedef struct {
    size_t struct_size;
    int (*get_module_table)(int module, fn_table* out_table, unsigned int* out_size);
} callbacks_table;
typedef const void* (*get_export_table_fn)(uint32_t id);

enum { kMaxDepth = 64, kMaxPath = 4096 };

static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
static FILE* g_out = NULL;
static __thread char t_path[kMaxPath];
static __thread int t_len[kMaxDepth];
static __thread int t_depth = 0;

static void emit(const char* what) {
    pthread_mutex_lock(&g_mu);
    if (g_out) fprintf(g_out, "%ld %s %s\n", (long)syscall(SYS_gettid), what, t_path);
    pthread_mutex_unlock(&g_mu);
}

static int on_push(const char* name) {
    if (t_depth < kMaxDepth) {
        int len = (int)strlen(t_path);
        t_len[t_depth] = len;
        snprintf(t_path + len, (size_t)(kMaxPath - len), "%s%s", len ? "/" : "", name ? name : "");
    }
    t_depth++;
    emit("push");
    return t_depth - 1;
}

static int on_pop(void) {
    if (t_depth == 0) {
        emit("pop-unmatched");
        return -1;
    }
    emit("pop");
    t_depth--;
    if (t_depth < kMaxDepth) t_path[t_len[t_depth]] = '\0';
    return t_depth;
}

int InitializeInjectionNvtx2(get_export_table_fn get_export_table) {
    const callbacks_table* cb = (const callbacks_table*)get_export_table(1);
    fn_table table = NULL;
    unsigned int n = 0;
    if (!cb || !cb->get_module_table(1, &table, &n) || !table) return 0;
    pthread_mutex_lock(&g_mu);
    if (!g_out) {
        const char* path = getenv("PGMG_NVTX_LOG");
        if (path) g_out = fopen(path, "w");
        if (g_out) setvbuf(g_out, NULL, _IOLBF, 0);
    }
    pthread_mutex_unlock(&g_mu);
    if (!g_out) return 0;
    if (n > 9 && table[9]) *table[9] = (fn_ptr)on_push;
    if (n > 11 && table[11]) *table[11] = (fn_ptr)on_pop;
    return 1;
}
