// Error state, buffers and small helpers shared by the engine.
#include <cstdarg>
#include <cstring>
#include <map>
#include <mutex>

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

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};

cudaMemPool_t device_pool(int dev) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (cudaMemPoolCreate(&g_pools[dev], &props) != cudaSuccess) {
            cudaGetLastError();
            g_pools[dev] = nullptr;
            return nullptr;
        }
        uint64_t keep = 16ull << 30;   // cached bytes kept across frees
        cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return g_pools[dev];
}

std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pinned_free;   // size class -> block
}  // namespace

int dev_alloc(void** p, size_t bytes, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool = device_pool(dev);
    cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, s) : cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        return TFIM_E_NOMEM;
    }
    return TFIM_OK;
}

void dev_free(void* p, cudaStream_t s) {
    if (!p) return;
    int dev = 0;
    cudaGetDevice(&dev);
    if (device_pool(dev)) cudaFreeAsync(p, s);
    else cudaFree(p);
}

void* pinned_alloc(size_t bytes, size_t* got) {
    size_t cls = 4096;
    while (cls < bytes) cls <<= 1;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pinned_free.find(cls);
        if (it != g_pinned_free.end()) {
            void* p = it->second;
            g_pinned_free.erase(it);
            *got = cls;
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, cls) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *got = cls;
    return p;
}

void pinned_free(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pinned_free.emplace(bytes, p);
}

int DevBuf::reserve(size_t need) {
    if (need <= bytes && p) return TFIM_OK;
    release();
    size_t cap = need < 4096 ? 4096 : need + need / 4;
    TFIM_TRY(dev_alloc(&p, cap, stream));
    bytes = cap;
    return TFIM_OK;
}
void DevBuf::release() {
    dev_free(p, stream);
    p = nullptr;
    bytes = 0;
}

int HostBuf::reserve(size_t need) {
    if (need <= bytes && p) return TFIM_OK;
    release();
    size_t got = 0;
    p = pinned_alloc(need, &got);
    if (!p) {
        bytes = 0;
        set_error("pinned host allocation of %zu bytes failed", need);
        return TFIM_E_NOMEM;
    }
    bytes = got;
    return TFIM_OK;
}
void HostBuf::release() {
    pinned_free(p, bytes);
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
    o->proj_auto = -1;
}

}  // extern "C"
