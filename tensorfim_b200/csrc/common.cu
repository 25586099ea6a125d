// Error state, buffers and small helpers shared by the engine.
#include <cstdarg>
#include <cstring>

#include "tfim_internal.h"

namespace tfim {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
const char* get_error() { return g_err; }

int DevBuf::reserve(size_t need) {
    if (need <= bytes && p) return TFIM_OK;
    release();
    size_t cap = need < 4096 ? 4096 : need + need / 4;
    cudaError_t e = cudaMalloc(&p, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        bytes = 0;
        set_error("device allocation of %zu bytes failed: %s", cap, cudaGetErrorString(e));
        return TFIM_E_NOMEM;
    }
    bytes = cap;
    return TFIM_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

int HostBuf::reserve(size_t need) {
    if (need <= bytes && p) return TFIM_OK;
    release();
    size_t cap = need < 4096 ? 4096 : need + need / 4;
    cudaError_t e = cudaMallocHost(&p, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        bytes = 0;
        set_error("pinned host allocation of %zu bytes failed: %s", cap, cudaGetErrorString(e));
        return TFIM_E_NOMEM;
    }
    bytes = cap;
    return TFIM_OK;
}
void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

}  // namespace tfim

extern "C" {

const char* tfim_version(void) { return "tensorfim-b200 0.1 (sm_100a)"; }
const char* tfim_last_error(void) { return tfim::get_error(); }

void tfim_mine_opts_default(tfim_mine_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->engine = TFIM_ENGINE_BATCHED;
    o->counter = TFIM_COUNTER_AUTO;
    o->wave_cap = 0;
    o->lookahead = 1;
    o->use_graphs = 0;
}

}  // extern "C"
