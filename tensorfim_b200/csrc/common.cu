// Error state, buffers and small helpers shared by the engine.
#include <dlfcn.h>

#include <cstdarg>
#include <cstdlib>
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
        // freed blocks stay cached in the pool up to half the device's memory, so that closing
        // a database and opening the next one does not unmap and remap its buffers
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            total_b = 32ull << 30;
        }
        uint64_t keep = (uint64_t)total_b / 2;
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

// ------------------------------------------------------------------ tuning table
namespace {
std::mutex g_tune_mu;
bool g_tune_init = false;
tfim_tuning g_tune;
std::string g_tune_src = "built-in";

void tuning_builtin(tfim_tuning* t) {
    memset(t, 0, sizeof *t);
    t->wave_rows = 4096;
    t->l3_slices_per_sm = 8.f;
    t->b1_tiles_per_sm = 4.f;
    t->b1_min_rows = 16;
    t->b1_min_cols = 16;
    t->proj_auto = kTuneProjAuto;
    t->rate_b1_bitops = kTuneB1BitOps;
    t->rate_lop3_bitops = kTuneLop3BitOps;
    t->rate_pair_incr = kTunePairIncrements;
    t->i8_min_rows = 128;
    t->i8_min_cols = 128;
    t->rate_i8_bitops = 3.0e14;
    t->tc_min_work = 1536;
    t->tc_min_density = 0.5f;
    t->tc_tiles_per_sm = 8.f;
    t->gram_min_rows = 32;
    t->l3_dense_slices_per_sm = 128.f;
}

bool tuning_valid(const tfim_tuning& t) {
    return t.wave_rows >= 16 && t.wave_rows <= (1 << 20) && t.l3_slices_per_sm > 0.f && t.l3_slices_per_sm <= 1024.f &&
           t.b1_tiles_per_sm > 0.f && t.b1_tiles_per_sm <= 1024.f && t.b1_min_rows >= 1 && t.b1_min_cols >= 1 &&
           (t.proj_auto == 0 || t.proj_auto == 1) && t.rate_b1_bitops > 0 && t.rate_lop3_bitops > 0 && t.rate_pair_incr > 0 &&
           t.i8_min_rows >= 1 && t.i8_min_cols >= 1 && t.rate_i8_bitops > 0 && t.tc_min_work >= 1 &&
           t.tc_min_density >= 0.f && t.tc_min_density <= 2.f && t.tc_tiles_per_sm > 0.f && t.tc_tiles_per_sm <= 1024.f &&
           t.gram_min_rows >= 1 && t.l3_dense_slices_per_sm > 0.f && t.l3_dense_slices_per_sm <= 1024.f;
}

// Flat JSON object of numbers: {"key": value, ...}.  Unknown keys are ignored.
int tuning_parse(const std::string& text, tfim_tuning* t) {
    struct Key { const char* name; int kind; void* dst; };   // kind 0 int, 1 float, 2 double
    const Key keys[] = {{"wave_rows", 0, &t->wave_rows},       {"l3_slices_per_sm", 1, &t->l3_slices_per_sm},
                        {"b1_tiles_per_sm", 1, &t->b1_tiles_per_sm}, {"b1_min_rows", 0, &t->b1_min_rows},
                        {"b1_min_cols", 0, &t->b1_min_cols},   {"proj_auto", 0, &t->proj_auto},
                        {"rate_b1_bitops", 2, &t->rate_b1_bitops}, {"rate_lop3_bitops", 2, &t->rate_lop3_bitops},
                        {"rate_pair_incr", 2, &t->rate_pair_incr}, {"i8_min_rows", 0, &t->i8_min_rows},
                        {"i8_min_cols", 0, &t->i8_min_cols}, {"rate_i8_bitops", 2, &t->rate_i8_bitops},
                        {"tc_min_work", 0, &t->tc_min_work}, {"tc_min_density", 1, &t->tc_min_density},
                        {"tc_tiles_per_sm", 1, &t->tc_tiles_per_sm}, {"gram_min_rows", 0, &t->gram_min_rows},
                        {"l3_dense_slices_per_sm", 1, &t->l3_dense_slices_per_sm}};
    for (const Key& k : keys) {
        const std::string pat = std::string("\"") + k.name + "\"";
        const size_t at = text.find(pat);
        if (at == std::string::npos) continue;
        size_t colon = text.find(':', at + pat.size());
        if (colon == std::string::npos) return TFIM_E_INVALID;
        const char* b = text.c_str() + colon + 1;
        char* e = nullptr;
        const double v = strtod(b, &e);
        if (e == b) return TFIM_E_INVALID;
        if (k.kind == 0) *(int32_t*)k.dst = (int32_t)v;
        else if (k.kind == 1) *(float*)k.dst = (float)v;
        else *(double*)k.dst = v;
    }
    return TFIM_OK;
}

int tuning_load_locked(const char* path) {
    FILE* f = fopen(path, "rb");
    TFIM_CHECK(f, TFIM_E_IO, "cannot open tuning table %s", path);
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    fclose(f);
    tfim_tuning t = g_tune;
    TFIM_CHECK(tuning_parse(text, &t) == TFIM_OK, TFIM_E_INVALID, "malformed tuning table %s", path);
    TFIM_CHECK(tuning_valid(t), TFIM_E_INVALID, "tuning table %s holds a value out of range", path);
    g_tune = t;
    g_tune_src = path;
    return TFIM_OK;
}

// First use: built-in values, then the table shipped beside the library if present.
void tuning_init_locked() {
    if (g_tune_init) return;
    g_tune_init = true;
    tuning_builtin(&g_tune);
    Dl_info info;
    if (dladdr((const void*)&tuning_builtin, &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        const size_t slash = so.rfind('/');
        const std::string dir = slash == std::string::npos ? std::string(".") : so.substr(0, slash);
        const std::string path = dir + "/../tuning.json";
        FILE* f = fopen(path.c_str(), "rb");
        if (f) {
            fclose(f);
            tuning_load_locked(path.c_str());   // a bad table leaves the built-in values
        }
    }
}
}  // namespace

tfim_tuning tuning() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tuning_init_locked();
    return g_tune;
}

}  // namespace tfim

extern "C" {

void tfim_tuning_get(tfim_tuning* out) {
    if (out) *out = tfim::tuning();
}

int tfim_tuning_set(const tfim_tuning* t) {
    TFIM_CHECK(t, TFIM_E_INVALID, "null tuning table");
    TFIM_CHECK(tfim::tuning_valid(*t), TFIM_E_INVALID, "tuning value out of range");
    std::lock_guard<std::mutex> lk(tfim::g_tune_mu);
    tfim::tuning_init_locked();
    tfim::g_tune = *t;
    tfim::g_tune_src = "set by the caller";
    return TFIM_OK;
}

int tfim_tuning_load(const char* path) {
    TFIM_CHECK(path, TFIM_E_INVALID, "null path");
    std::lock_guard<std::mutex> lk(tfim::g_tune_mu);
    tfim::tuning_init_locked();
    return tfim::tuning_load_locked(path);
}

const char* tfim_tuning_source(void) {
    std::lock_guard<std::mutex> lk(tfim::g_tune_mu);
    tfim::tuning_init_locked();
    return tfim::g_tune_src.c_str();
}

const char* tfim_version(void) { return "tensorfim-b200 0.1 (sm_100a)"; }
const char* tfim_last_error(void) { return tfim::get_error(); }

void tfim_mine_opts_default(tfim_mine_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->engine = TFIM_ENGINE_RESIDENT;
    o->counter = TFIM_COUNTER_AUTO;
    o->wave_cap = 0;
    o->lookahead = 1;
    o->use_graphs = 0;
    o->proj_auto = -1;
    o->superset = 0;
}

}  // extern "C"
