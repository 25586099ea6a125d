// extern "C" entry points of libtfim (declared in include/tfim.h).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <numeric>
#include <string>

#include "tfim_internal.h"

namespace tfim {
int ingest_csr(tfim_ctx* c, const int64_t* off, const int32_t* items, int64_t n_rows, double thr);
int ingest_bitmap(tfim_ctx* c, const uint32_t* rows, int32_t n_rows, int64_t n_bits, int32_t n_counted);

namespace {

int make_ctx(int32_t device, tfim_ctx** out) {
    TFIM_CHECK(out != nullptr, TFIM_E_INVALID, "null output handle");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) {
        cudaGetLastError();
        set_error("no CUDA device available (%s)", e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
        return TFIM_E_CUDA;
    }
    TFIM_CHECK(device >= 0 && device < n, TFIM_E_INVALID, "device %d out of range (%d devices)", device, n);
    TFIM_CUDA(cudaSetDevice(device));
    tfim_ctx* c = new (std::nothrow) tfim_ctx();
    TFIM_CHECK(c != nullptr, TFIM_E_NOMEM, "context allocation failed");
    c->device = device;
    static std::atomic<uint64_t> next_uid{1};
    c->uid = next_uid.fetch_add(1);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->ev_span0) != cudaSuccess || cudaEventCreate(&c->ev_span1) != cudaSuccess) {
        set_error("stream/event creation failed: %s", cudaGetErrorString(cudaGetLastError()));
        tfim_close(c);
        return TFIM_E_CUDA;
    }
    for (auto& b : c->d_scratch) b.stream = c->stream;
    c->d_masks.stream = c->stream;
    c->d_group.stream = c->stream;
    *out = c;
    return TFIM_OK;
}

// A context of a sharded database.  Before the ingest's first collective every rank learns
// whether any rank rejected its arguments, and that the values in `agree` are equal on all
// ranks, so a bad call fails everywhere instead of leaving the others waiting.
int make_sharded_ctx(int32_t device, const tfim_group* g, bool args_ok, const std::vector<int64_t>& agree,
                     const char* what, tfim_ctx** out) {
    TFIM_CHECK(out != nullptr, TFIM_E_INVALID, "null output handle");
    *out = nullptr;
    TFIM_CHECK(g && g->world >= 1 && g->rank >= 0 && g->rank < g->world && (g->world == 1 || g->allreduce),
               TFIM_E_INVALID, "%s: invalid tfim_group", what);
    tfim_ctx* c = nullptr;
    TFIM_TRY(make_ctx(device, &c));
    c->group = *g;
    c->sharded = true;
    std::vector<int64_t> v(1 + 2 * agree.size());
    v[0] = args_ok ? 0 : 1;
    for (size_t i = 0; i < agree.size(); i++) { v[1 + 2 * i] = agree[i]; v[2 + 2 * i] = -agree[i]; }
    int rc = group_reduce_host(c, v.data(), (int32_t)v.size(), TFIM_RED_MAX);
    if (rc == TFIM_OK && v[0]) {
        set_error(args_ok ? "%s: another rank's arguments were rejected" : "%s: invalid arguments", what);
        rc = TFIM_E_INVALID;
    }
    for (size_t i = 0; rc == TFIM_OK && i < agree.size(); i++)
        if (v[1 + 2 * i] != -v[2 + 2 * i]) {
            set_error("%s: argument %zu differs across the group", what, i);
            rc = TFIM_E_INVALID;
        }
    if (rc != TFIM_OK) { tfim_close(c); return rc; }
    *out = c;
    return TFIM_OK;
}

}  // namespace

// Per-node masks + one count job over every counted row (the reference counting contract).
int count_wave_impl(tfim_ctx* c, int32_t b, int32_t min_count, const int32_t* d_items, const MatDesc* d_mats,
                    int32_t* d_counts, int32_t* d_nfreq, cudaStream_t s) {
    const int32_t d = c->n_counted;
    // masks: one pool row per node
    TFIM_TRY(c->d_masks.reserve((size_t)b * (size_t)c->W * 4));
    TFIM_TRY(launch_materialize(c->d_bitmap, c->W, c->d_masks.as<uint32_t>(), d_mats, d_items, b, s));
    if (d == 0) return launch_nfreq(d_counts, b, 0, min_count, d_nfreq, s);
    // host-built job/tile tables (independent of the list contents)
    const int32_t counter = c->counter_pref;
    const tfim_tuning tn = tuning();
    const bool i8 = counter == TFIM_COUNTER_I8 ||
                    (counter == TFIM_COUNTER_AUTO && b >= tn.i8_min_rows && d >= tn.i8_min_cols);
    const bool b1 = !i8 && (counter == TFIM_COUNTER_TENSOR ||
                            (counter == TFIM_COUNTER_AUTO && b >= tn.b1_min_rows && d >= tn.b1_min_cols));
    std::vector<JobDesc> jobs(1);
    jobs[0].base_slot = -1; jobs[0].base_item = -1;
    jobs[0].n_rows = b; jobs[0].n_cols = d; jobs[0].row_off = 0; jobs[0].col_off = 0; jobs[0].out_off = 0;
    jobs[0].self_col = -1; jobs[0].pad = 0;
    std::vector<RowDesc> rows(b);
    for (int32_t i = 0; i < b; i++) rows[i] = RowDesc{i, -1};
    std::vector<int32_t> cols(d);
    std::iota(cols.begin(), cols.end(), 0);
    std::vector<TileDesc> tiles;
    const int64_t W = c->W;
    if (i8) {
        // 128 x 128 tiles, word slices of 64-word multiples
        const int64_t base = (int64_t)((b + 127) / 128) * ((d + 127) / 128);
        const int64_t want = (int64_t)(tn.b1_tiles_per_sm * 148);
        int64_t ks = std::max<int64_t>(1, (want + base - 1) / base);
        ks = std::min<int64_t>(ks, W / 64);
        const int64_t kslice = ((W / 64 + ks - 1) / ks) * 64;
        for (int64_t w0 = 0; w0 < W; w0 += kslice)
            for (int32_t r0 = 0; r0 < b; r0 += 128)
                for (int32_t c0 = 0; c0 < d; c0 += 128)
                    tiles.push_back(TileDesc{0, r0, std::min(128, b - r0), c0, std::min(d, c0 + 128), (int32_t)w0,
                                             (int32_t)std::min<int64_t>(W, w0 + kslice), 0});
    } else if (b1) {
        const int64_t base = (int64_t)((b + kB1Rows - 1) / kB1Rows) * ((d + kB1Cols - 1) / kB1Cols);
        const int64_t want = (int64_t)(tn.b1_tiles_per_sm * 148);
        int64_t ks = std::max<int64_t>(1, (want + base - 1) / base);
        ks = std::min<int64_t>(ks, W / 64);
        const int64_t kslice = ((W / 64 + ks - 1) / ks) * 64;
        for (int64_t w0 = 0; w0 < W; w0 += kslice)
            for (int32_t r0 = 0; r0 < b; r0 += kB1Rows)
                for (int32_t c0 = 0; c0 < d; c0 += kB1Cols)
                    tiles.push_back(TileDesc{0, r0, std::min(kB1Rows, b - r0), c0, std::min(d, c0 + kB1Cols), (int32_t)w0,
                                             (int32_t)std::min<int64_t>(W, w0 + kslice), 0});
    } else {
        const int64_t chunk = std::min<int64_t>(W, kLop3Chunk);
        for (int32_t r0 = 0; r0 < b; r0 += kLop3Rows)
            for (int32_t c0 = 0; c0 < d; c0 += 64)
                for (int64_t w0 = 0; w0 < W; w0 += chunk)
                    tiles.push_back(TileDesc{0, r0, std::min(kLop3Rows, b - r0), c0, std::min(d, c0 + 64), (int32_t)w0,
                                             (int32_t)std::min<int64_t>(W, w0 + chunk), 0});
    }
    const size_t o_rows = 64, o_cols = o_rows + ((rows.size() * sizeof(RowDesc) + 15) & ~size_t(15));
    const size_t o_tiles = o_cols + ((cols.size() * 4 + 15) & ~size_t(15));
    const size_t total = o_tiles + tiles.size() * sizeof(TileDesc);
    TFIM_TRY(c->h_scratch[0].reserve(total));
    TFIM_TRY(c->d_scratch[0].reserve(total));
    unsigned char* hp = c->h_scratch[0].as<unsigned char>();
    memcpy(hp, jobs.data(), sizeof(JobDesc));
    memcpy(hp + o_rows, rows.data(), rows.size() * sizeof(RowDesc));
    memcpy(hp + o_cols, cols.data(), cols.size() * 4);
    memcpy(hp + o_tiles, tiles.data(), tiles.size() * sizeof(TileDesc));
    unsigned char* dp = c->d_scratch[0].as<unsigned char>();
    if (s != c->stream) {
        // buffers are allocated in the context stream's order: the caller's stream waits
        TFIM_CUDA(cudaEventRecord(c->ev0, c->stream));
        TFIM_CUDA(cudaStreamWaitEvent(s, c->ev0, 0));
    }
    TFIM_CUDA(cudaMemcpyAsync(dp, hp, total, cudaMemcpyHostToDevice, s));
    TFIM_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)b * d * 4, s));
    CountArgs a;
    a.bitmap = c->d_bitmap; a.W = W; a.masks = c->d_masks.as<uint32_t>();
    a.jobs = (const JobDesc*)dp; a.rows = (const RowDesc*)(dp + o_rows); a.cols = (const int32_t*)(dp + o_cols);
    a.tiles = (const TileDesc*)(dp + o_tiles); a.n_tiles = (int32_t)tiles.size(); a.out = d_counts;
    c->used_i8 = i8;
    TFIM_TRY(i8 ? launch_count_i8(a, s) : b1 ? launch_count_b1(a, s) : launch_count_lop3(a, s));
    TFIM_TRY(group_reduce(c, d_counts, (int64_t)b * d, TFIM_DT_I32, TFIM_RED_SUM, s));
    TFIM_TRY(launch_nfreq(d_counts, b, d, min_count, d_nfreq, s));
    // the host staging buffer may be reused by the next call only after this copy ran
    TFIM_CUDA(cudaStreamSynchronize(s));
    return TFIM_OK;
}

namespace {

__global__ void k_mats_from_offsets(const int64_t* __restrict__ off, int32_t b, MatDesc* __restrict__ mats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b) return;
    MatDesc m;
    m.dst = i; m.src = -1; m.off = (int32_t)off[i]; m.n = (int32_t)(off[i + 1] - off[i]);
    mats[i] = m;
}

std::string cpu_name() {
    std::ifstream f("/proc/cpuinfo");
    std::string line;
    while (std::getline(f, line))
        if (line.rfind("model name", 0) == 0) {
            size_t p = line.find(':');
            if (p != std::string::npos) {
                std::string s = line.substr(p + 1);
                size_t b = s.find_first_not_of(" \t");
                return b == std::string::npos ? s : s.substr(b);
            }
        }
    return "Unknown CPU";
}

}  // namespace
}  // namespace tfim

using namespace tfim;

extern "C" {

int tfim_open_db(const int64_t* row_offsets, const int32_t* items, int64_t n_rows, double support_threshold,
                 int32_t device, tfim_ctx** out) {
    TFIM_CHECK(out != nullptr, TFIM_E_INVALID, "null output handle");
    *out = nullptr;
    TFIM_CHECK(row_offsets != nullptr && n_rows >= 0, TFIM_E_INVALID, "invalid transaction set");
    TFIM_CHECK(n_rows == 0 || row_offsets[n_rows] == 0 || items != nullptr, TFIM_E_INVALID, "null items");
    TFIM_CHECK(support_threshold > 0.0 && support_threshold <= 1.0 && std::isfinite(support_threshold), TFIM_E_INVALID,
               "support threshold %g outside (0, 1]", support_threshold);
    tfim_ctx* c = nullptr;
    TFIM_TRY(make_ctx(device, &c));
    int rc = ingest_csr(c, row_offsets, items, n_rows, support_threshold);
    if (rc != TFIM_OK) { tfim_close(c); return rc; }
    *out = c;
    return TFIM_OK;
}

}  // extern "C"

namespace {
int open_from_text(const TextSource& src, double thr, int32_t device, tfim_ctx** out) {
    TFIM_CHECK(out != nullptr, TFIM_E_INVALID, "null output handle");
    *out = nullptr;
    TFIM_CHECK(thr > 0.0 && thr <= 1.0 && std::isfinite(thr), TFIM_E_INVALID, "support threshold %g outside (0, 1]", thr);
    tfim_ctx* c = nullptr;
    TFIM_TRY(make_ctx(device, &c));
    int64_t* d_off = nullptr;
    int32_t* d_items = nullptr;
    int64_t n_rows = 0, nnz = 0;
    int rc = parse_text_device(src, c->stream, &d_off, &d_items, &n_rows, &nnz);
    if (rc == TFIM_OK) rc = ingest_device_csr(c, d_off, d_items, n_rows, nnz, thr);
    dev_free(d_off, c->stream);
    dev_free(d_items, c->stream);
    if (rc != TFIM_OK) { tfim_close(c); return rc; }
    *out = c;
    return TFIM_OK;
}
}  // namespace

extern "C" {

int tfim_open_text(const char* bytes, int64_t n_bytes, double support_threshold, int32_t device, tfim_ctx** out) {
    TFIM_CHECK(n_bytes >= 0 && (bytes != nullptr || n_bytes == 0), TFIM_E_INVALID, "invalid transaction file bytes");
    TextSource src;
    src.host = bytes ? bytes : "";
    src.n_bytes = n_bytes;
    return open_from_text(src, support_threshold, device, out);
}

int tfim_open_file(const char* path, double support_threshold, int32_t device, tfim_ctx** out) {
    TFIM_CHECK(out != nullptr, TFIM_E_INVALID, "null output handle");
    *out = nullptr;
    TFIM_CHECK(path != nullptr, TFIM_E_INVALID, "null path");
    const int fd = open(path, O_RDONLY | O_CLOEXEC);
    TFIM_CHECK(fd >= 0, TFIM_E_IO, "%s open failed", path);
    struct stat st{};
    if (fstat(fd, &st) != 0 || !S_ISREG(st.st_mode)) {
        close(fd);
        set_error("%s is not a readable regular file", path);
        return TFIM_E_IO;
    }
    TextSource src;
    src.fd = fd;
    src.n_bytes = (int64_t)st.st_size;
    const int rc = open_from_text(src, support_threshold, device, out);
    close(fd);
    return rc;
}

int tfim_parse_text(const char* bytes, int64_t n_bytes, int32_t device, int64_t* row_offsets, int64_t rows_cap,
                    int32_t* items, int64_t items_cap, int64_t* n_rows, int64_t* n_items) {
    TFIM_CHECK(n_bytes >= 0 && (bytes != nullptr || n_bytes == 0) && n_rows && n_items, TFIM_E_INVALID,
               "tfim_parse_text: invalid arguments");
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev <= 0) {
        cudaGetLastError();
        set_error("no CUDA device available");
        return TFIM_E_CUDA;
    }
    TFIM_CHECK(device >= 0 && device < n_dev, TFIM_E_INVALID, "device %d out of range (%d devices)", device, n_dev);
    TFIM_CUDA(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    TFIM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    TextSource src;
    src.host = bytes ? bytes : "";
    src.n_bytes = n_bytes;
    int64_t* d_off = nullptr;
    int32_t* d_items = nullptr;
    int64_t rows = 0, nnz = 0;
    int rc = parse_text_device(src, s, &d_off, &d_items, &rows, &nnz);
    if (rc == TFIM_OK) {
        *n_rows = rows;
        *n_items = nnz;
        if (row_offsets && items && rows_cap >= rows + 1 && items_cap >= nnz) {
            if (cudaMemcpyAsync(row_offsets, d_off, (size_t)(rows + 1) * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                (nnz > 0 && cudaMemcpyAsync(items, d_items, (size_t)nnz * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                set_error("device-to-host copy of the parsed transactions failed");
                rc = TFIM_E_CUDA;
            }
        } else if (row_offsets || items) {
            set_error("tfim_parse_text: output capacity too small (%lld rows + 1, %lld items needed)", (long long)rows,
                      (long long)nnz);
            rc = TFIM_E_NOMEM;
        }
    }
    dev_free(d_off, s);
    dev_free(d_items, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

int tfim_open_bitmap(const uint32_t* rows, int32_t n_rows, int64_t n_bits, int32_t n_counted, int32_t device,
                     tfim_ctx** out) {
    TFIM_CHECK(out != nullptr, TFIM_E_INVALID, "null output handle");
    *out = nullptr;
    tfim_ctx* c = nullptr;
    TFIM_TRY(make_ctx(device, &c));
    int rc = ingest_bitmap(c, rows, n_rows, n_bits, n_counted);
    if (rc != TFIM_OK) { tfim_close(c); return rc; }
    *out = c;
    return TFIM_OK;
}

int tfim_open_db_sharded(const int64_t* row_offsets, const int32_t* items, int64_t n_rows, double support_threshold,
                         int32_t device, const tfim_group* group, tfim_ctx** out) {
    const bool ok = row_offsets != nullptr && n_rows >= 0 && (n_rows == 0 || row_offsets[0] == 0) &&
                    (n_rows == 0 || row_offsets[n_rows] >= 0) && (n_rows == 0 || row_offsets[n_rows] == 0 || items != nullptr) &&
                    support_threshold > 0.0 && support_threshold <= 1.0 && std::isfinite(support_threshold);
    int64_t thr_bits = 0;
    memcpy(&thr_bits, &support_threshold, 8);
    tfim_ctx* c = nullptr;
    TFIM_TRY(make_sharded_ctx(device, group, ok, {thr_bits}, "tfim_open_db_sharded", &c));
    int rc = ingest_csr(c, row_offsets, items, n_rows, support_threshold);
    if (rc != TFIM_OK) { tfim_close(c); return rc; }
    *out = c;
    return TFIM_OK;
}

int tfim_open_bitmap_sharded(const uint32_t* rows, int32_t n_rows, int64_t n_bits, int32_t n_counted, int32_t device,
                             const tfim_group* group, tfim_ctx** out) {
    const bool ok = rows != nullptr && n_rows > 0 && n_bits > 0 && n_counted >= 0 && n_counted <= n_rows;
    tfim_ctx* c = nullptr;
    TFIM_TRY(make_sharded_ctx(device, group, ok, {n_rows, n_counted}, "tfim_open_bitmap_sharded", &c));
    int rc = ingest_bitmap(c, rows, n_rows, n_bits, n_counted);
    if (rc != TFIM_OK) { tfim_close(c); return rc; }
    *out = c;
    return TFIM_OK;
}

int tfim_db_info_get(const tfim_ctx* c, tfim_db_info* out) {
    TFIM_CHECK(c && out, TFIM_E_INVALID, "null argument");
    *out = c->info;
    return TFIM_OK;
}

int tfim_dense_to_orig(const tfim_ctx* c, int32_t* out) {
    TFIM_CHECK(c && (out || c->dense_to_orig.empty()), TFIM_E_INVALID, "null argument");
    std::copy(c->dense_to_orig.begin(), c->dense_to_orig.end(), out);
    return TFIM_OK;
}

int tfim_dense_freq(const tfim_ctx* c, int32_t* out) {
    TFIM_CHECK(c && (out || (c->from_db ? c->dense_freq.empty() : c->bit_support.empty())), TFIM_E_INVALID,
               "null argument");
    if (c->from_db) std::copy(c->dense_freq.begin(), c->dense_freq.end(), out);
    else std::copy(c->bit_support.begin(), c->bit_support.end(), out);
    return TFIM_OK;
}

int tfim_set_counter(tfim_ctx* c, int32_t counter) {
    TFIM_CHECK(c, TFIM_E_INVALID, "null context");
    TFIM_CHECK((counter >= TFIM_COUNTER_AUTO && counter <= TFIM_COUNTER_TENSOR) || counter == TFIM_COUNTER_I8,
               TFIM_E_INVALID, "unknown counter %d", counter);
    // (TFIM_COUNTER_PROJ applies to the search's family counts only)
    c->counter_pref = counter;
    return TFIM_OK;
}

int tfim_count_wave(tfim_ctx* c, const int32_t* item_lists, const int64_t* list_offsets, int32_t b, int32_t min_count,
                    int32_t* counts_out, int32_t* nfreq_out) {
    TFIM_CHECK(c && list_offsets && counts_out && nfreq_out && b >= 0, TFIM_E_INVALID, "tfim_count_wave: invalid arguments");
    if (b == 0) return TFIM_OK;
    TFIM_CUDA(cudaSetDevice(c->device));
    const int32_t n_rows_total = c->info.n_dense;
    TFIM_CHECK(list_offsets[0] == 0, TFIM_E_INVALID, "list_offsets[0] must be 0");
    for (int32_t i = 0; i < b; i++) {
        const int64_t len = list_offsets[i + 1] - list_offsets[i];
        TFIM_CHECK(len >= 0, TFIM_E_INVALID, "list_offsets must be non-decreasing");
        TFIM_CHECK(len <= kMaxListLen, TFIM_E_DEPTH, "node %d lists %lld items; at most %d", i, (long long)len, kMaxListLen);
        for (int64_t q = list_offsets[i]; q < list_offsets[i + 1]; q++)
            TFIM_CHECK(item_lists[q] >= 0 && item_lists[q] < n_rows_total, TFIM_E_INVALID, "item %d out of range", item_lists[q]);
    }
    const int64_t n_items = list_offsets[b];
    const int32_t d = c->n_counted;
    cudaStream_t s = c->stream;
    // device staging: items, mats, counts, nfreq
    const size_t o_items = 0;
    const size_t o_mats = (((size_t)std::max<int64_t>(n_items, 1) * 4) + 15) & ~size_t(15);
    const size_t o_counts = o_mats + (((size_t)b * sizeof(MatDesc) + 15) & ~size_t(15));
    const size_t o_nfreq = o_counts + (((size_t)b * d * 4 + 15) & ~size_t(15));
    const size_t total = o_nfreq + (size_t)b * 4;
    TFIM_TRY(c->d_scratch[1].reserve(total));
    TFIM_TRY(c->h_scratch[1].reserve(o_counts));
    unsigned char* hp = c->h_scratch[1].as<unsigned char>();
    if (n_items) memcpy(hp + o_items, item_lists, (size_t)n_items * 4);
    MatDesc* hm = (MatDesc*)(hp + o_mats);
    for (int32_t i = 0; i < b; i++) hm[i] = MatDesc{i, -1, (int32_t)list_offsets[i], (int32_t)(list_offsets[i + 1] - list_offsets[i])};
    unsigned char* dp = c->d_scratch[1].as<unsigned char>();
    TFIM_CUDA(cudaMemcpyAsync(dp, hp, o_counts, cudaMemcpyHostToDevice, s));
    TFIM_TRY(count_wave_impl(c, b, min_count, (const int32_t*)(dp + o_items), (const MatDesc*)(dp + o_mats),
                             (int32_t*)(dp + o_counts), (int32_t*)(dp + o_nfreq), s));
    TFIM_CUDA(cudaMemcpyAsync(counts_out, dp + o_counts, (size_t)b * d * 4, cudaMemcpyDeviceToHost, s));
    TFIM_CUDA(cudaMemcpyAsync(nfreq_out, dp + o_nfreq, (size_t)b * 4, cudaMemcpyDeviceToHost, s));
    TFIM_CUDA(cudaStreamSynchronize(s));
    if (c->used_i8) TFIM_TRY(count_i8_status(true));
    return TFIM_OK;
}

int tfim_count_wave_device(tfim_ctx* c, const int32_t* d_item_lists, const int64_t* d_list_offsets, int32_t b,
                           int32_t max_len, int32_t min_count, int32_t* d_counts_out, int32_t* d_nfreq_out, void* stream) {
    TFIM_CHECK(c && d_list_offsets && d_counts_out && d_nfreq_out && b >= 0, TFIM_E_INVALID,
               "tfim_count_wave_device: invalid arguments");
    TFIM_CHECK(max_len >= 0 && max_len <= kMaxListLen, TFIM_E_DEPTH, "max_len %d exceeds %d", max_len, kMaxListLen);
    if (b == 0) return TFIM_OK;
    TFIM_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    TFIM_TRY(c->d_scratch[2].reserve((size_t)b * sizeof(MatDesc)));
    TFIM_TRY(c->d_masks.reserve((size_t)b * (size_t)c->W * 4));
    if (s != c->stream) {
        TFIM_CUDA(cudaEventRecord(c->ev0, c->stream));
        TFIM_CUDA(cudaStreamWaitEvent(s, c->ev0, 0));
    }
    k_mats_from_offsets<<<(b + 255) / 256, 256, 0, s>>>(d_list_offsets, b, c->d_scratch[2].as<MatDesc>());
    TFIM_CUDA(cudaGetLastError());
    return count_wave_impl(c, b, min_count, d_item_lists, c->d_scratch[2].as<MatDesc>(), d_counts_out, d_nfreq_out, s);
}

int tfim_mine(tfim_ctx* c, const tfim_mine_opts* opts, tfim_mine_stats* stats) {
    TFIM_CHECK(c, TFIM_E_INVALID, "null context");
    TFIM_CHECK(c->from_db, TFIM_E_STATE, "tfim_mine needs a context opened with tfim_open_db");
    TFIM_CUDA(cudaSetDevice(c->device));
    tfim_mine_opts o;
    if (opts) o = *opts;
    else {
        tfim_mine_opts_default(&o);
        if (c->sharded) o.engine = TFIM_ENGINE_BATCHED;
    }
    TFIM_CHECK(o.engine == TFIM_ENGINE_PLAIN || o.engine == TFIM_ENGINE_BATCHED || o.engine == TFIM_ENGINE_RESIDENT,
               TFIM_E_INVALID, "unknown engine %d", o.engine);
    TFIM_CHECK(!(c->sharded && o.engine == TFIM_ENGINE_RESIDENT), TFIM_E_STATE,
               "the resident engine keeps its counts on the device between waves and does not run on a "
               "transaction-sharded context: use the batched or plain engine");
    tfim_mine_stats st;
    memset(&st, 0, sizeof st);
    c->mfis.clear();
    c->mined = false;
    cudaEvent_t e_begin = c->ev_span0, e_end = c->ev_span1;
    TFIM_CUDA(cudaEventRecord(e_begin, c->stream));
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    if (o.engine == TFIM_ENGINE_PLAIN) rc = mine_plain(c, &o, &st);
    else if (o.engine == TFIM_ENGINE_BATCHED) rc = mine_batched(c, &o, &st);
    else rc = mine_resident(c, &o, &st);
    cudaEventRecord(e_end, c->stream);
    cudaEventSynchronize(e_end);
    const auto t1 = std::chrono::steady_clock::now();
    float span_ms = 0;
    cudaEventElapsedTime(&span_ms, e_begin, e_end);
    if (rc != TFIM_OK) return rc;
    st.device_ms = span_ms;
    st.host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count() - st.sync_ms;
    if (!c->mfis.ordered) {
        // descending support; ties by descending item lists (deterministic order)
        const MfiSet& M = c->mfis;
        auto before = [&](int32_t a, int32_t b) {
            if (M.sup[a] != M.sup[b]) return M.sup[a] > M.sup[b];
            return std::lexicographical_compare(M.items.begin() + M.off[b], M.items.begin() + M.off[b + 1],
                                                M.items.begin() + M.off[a], M.items.begin() + M.off[a + 1]);
        };
        // sort on a packed key (support, first item), then order equal keys fully
        std::vector<std::pair<uint64_t, int32_t>> keyed(M.size());
        for (size_t k = 0; k < M.size(); k++) {
            const uint32_t first = M.off[k + 1] > M.off[k] ? (uint32_t)M.items[M.off[k]] : 0u;
            keyed[k] = {((uint64_t)(0xFFFFFFFFu - (uint32_t)M.sup[k]) << 32) | (uint64_t)(0xFFFFFFFFu - first), (int32_t)k};
        }
        std::sort(keyed.begin(), keyed.end());
        std::vector<int32_t> idx(M.size());
        for (size_t k = 0; k < M.size(); k++) idx[k] = keyed[k].second;
        for (size_t a = 0; a < keyed.size();) {
            size_t b = a + 1;
            while (b < keyed.size() && keyed[b].first == keyed[a].first) b++;
            if (b - a > 1) std::sort(idx.begin() + a, idx.begin() + b, before);
            a = b;
        }
        MfiSet S;
        S.items.reserve(M.items.size());
        S.off.reserve(M.size() + 1);
        S.sup.reserve(M.size());
        for (int32_t k : idx) S.add(M.items.data() + M.off[k], (size_t)(M.off[k + 1] - M.off[k]), M.sup[k]);
        c->mfis.items.swap(S.items);
        c->mfis.off.swap(S.off);
        c->mfis.sup.swap(S.sup);
        c->mfis.ordered = true;
    }
    st.n_mfi = (int64_t)c->mfis.size();
    // computation time as the reference reports it: search and counting, bitmap resident,
    // results in host memory in their output order
    const auto t2 = std::chrono::steady_clock::now();
    st.mine_seconds = std::chrono::duration<double>(t2 - t0).count();
    st.readback_ms += std::chrono::duration<double, std::milli>(t2 - t1).count();
    c->mined = true;
    c->last_stats = st;
    if (stats) *stats = st;
    return TFIM_OK;
}

int tfim_set_proposal(tfim_ctx* c, tfim_mlp* mlp, float threshold) {
    TFIM_CHECK(c, TFIM_E_INVALID, "null context");
    c->proposal = mlp;
    c->proposal_threshold = threshold;
    return TFIM_OK;
}

int64_t tfim_lookahead_log(const tfim_ctx* c, float* feats, float* labels, int64_t cap) {
    if (!c) { set_error("null context"); return -TFIM_E_INVALID; }
    const int64_t n = (int64_t)c->la_labels.size();
    const int64_t k = std::min<int64_t>(n, std::max<int64_t>(cap, 0));
    if (k > 0) {
        if (!feats || !labels) { set_error("null buffers"); return -TFIM_E_INVALID; }
        memcpy(feats, c->la_feats.data(), (size_t)k * 32 * sizeof(float));
        memcpy(labels, c->la_labels.data(), (size_t)k * sizeof(float));
    }
    return n;
}

int64_t tfim_num_mfis(const tfim_ctx* c) { return c && c->mined ? (int64_t)c->mfis.size() : -1; }

int64_t tfim_mfi_item_total(const tfim_ctx* c) { return c && c->mined ? (int64_t)c->mfis.items.size() : -1; }

int tfim_get_mfis(const tfim_ctx* c, int32_t* items, int64_t* offsets, int32_t* supports) {
    TFIM_CHECK(c && items && offsets && supports, TFIM_E_INVALID, "null argument");
    TFIM_CHECK(c->mined, TFIM_E_STATE, "tfim_get_mfis before tfim_mine");
    const MfiSet& M = c->mfis;
    const int32_t* map = c->dense_to_orig.data();
    for (size_t q = 0; q < M.items.size(); q++) items[q] = map[M.items[q]];
    std::copy(M.off.begin(), M.off.end(), offsets);
    std::copy(M.sup.begin(), M.sup.end(), supports);
    return TFIM_OK;
}

int tfim_write_results(const tfim_ctx* c, const char* trans_set_file, const char* result_path, double prep_s,
                       double comp_s) {
    TFIM_CHECK(c && trans_set_file && result_path, TFIM_E_INVALID, "null argument");
    TFIM_CHECK(c->mined, TFIM_E_STATE, "tfim_write_results before tfim_mine");
    FILE* f = fopen(result_path, "w");
    TFIM_CHECK(f != nullptr, TFIM_E_IO, "cannot open %s for writing", result_path);
    const tfim_db_info& I = c->info;
    fprintf(f, "==================================================================\n");
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, c->device) == cudaSuccess) {
        fprintf(f, "GPU %d: %s\n", c->device, p.name);
        fprintf(f, "     Multi-Processor Count: %d\n", p.multiProcessorCount);
        fprintf(f, "     Max Threads Per Multi-Processor: %d\n", p.maxThreadsPerMultiProcessor);
        fprintf(f, "     Warp Size: %d\n", p.warpSize);
        fprintf(f, "     Max Threads Per Block: %d\n", p.maxThreadsPerBlock);
        fprintf(f, "     Compute Capability: %d.%d\n", p.major, p.minor);
        fprintf(f, "     Number of Multi-Processors: %d\n\n", p.multiProcessorCount);
    }
    const long lc = sysconf(_SC_NPROCESSORS_ONLN);
    fprintf(f, "CPU: %s\n", cpu_name().c_str());
    fprintf(f, "     Number of Logical Cores: %ld\n\n", lc);
    int rt = 0;
    cudaRuntimeGetVersion(&rt);
    fprintf(f, "CUDA Version: %d.%d\n", rt / 1000, (rt % 1000) / 10);
    fprintf(f, "Engine: %s\n", tfim_version());
    fprintf(f, "==================================================================\n");
    fprintf(f, "transSetFile: %s\n", trans_set_file);
    fprintf(f, "dimension: %lld\n", (long long)I.dimension);
    fprintf(f, "transNum: %lld\n", (long long)I.trans_num);
    fprintf(f, "itemIDmin: %lld\n", (long long)I.item_id_min);
    fprintf(f, "itemIDmax: %lld\n", (long long)I.item_id_max_dense);
    fprintf(f, "transLengthMin: %lld\n", (long long)I.trans_len_min);
    fprintf(f, "transLengthMax: %lld\n", (long long)I.trans_len_max);
    fprintf(f, "transLengthMean: %g\n", I.trans_len_mean);
    fprintf(f, "\nsupportThreshold: %g\n\n", I.support_threshold);
    fprintf(f, "dimensionReduced: %lld\n", (long long)I.dimension_reduced);
    fprintf(f, "transNumReduced: %lld\n", (long long)I.trans_num_reduced);
    fprintf(f, "transLengthReducedMin: %lld\n", (long long)I.trans_len_red_min);
    fprintf(f, "transLengthReducedMax: %lld\n", (long long)I.trans_len_red_max);
    fprintf(f, "transLengthReducedMean: %g\n", I.trans_len_red_mean);
    fprintf(f, "\nGPUtaskPercentage: 100%%\n");
    fprintf(f, "==================================================================\n");
    fprintf(f, "preprocessing_time(s): %g\n", prep_s);
    fprintf(f, "computation_time(s): %g\n", comp_s);
    fprintf(f, "total_time(s): %g\n", prep_s + comp_s);
    fprintf(f, "\nMFIsNumber: %lld\n", (long long)c->mfis.size());
    fprintf(f, "============================List of MFIs:=============================\n");
    const MfiSet& M = c->mfis;
    for (size_t k = 0; k < M.size(); k++) {
        fprintf(f, "%zuth: %lld { ", k + 1, (long long)(M.off[k + 1] - M.off[k]));
        for (int64_t q = M.off[k]; q < M.off[k + 1]; q++) fprintf(f, "%d ", c->dense_to_orig[M.items[q]]);
        fprintf(f, "}   support: %g  frequency: %d\n", (double)M.sup[k] / (double)I.trans_num, M.sup[k]);
    }
    fprintf(f, "==================================================================\n");
    const bool ok = ferror(f) == 0;
    fclose(f);
    TFIM_CHECK(ok, TFIM_E_IO, "write to %s failed", result_path);
    return TFIM_OK;
}

int tfim_release_cached(int32_t device) { return tfim::release_cached(device); }

void tfim_close(tfim_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->engine) tfim::free_engine(c->engine);
    c->engine = nullptr;
    tfim::stash_resident(c);   // pools for the next database opened on this device
    if (c->resident) tfim::free_resident(c->resident, c->stream);
    c->resident = nullptr;
    tfim::dev_free(c->d_bitmap, c->stream);
    tfim::dev_free(c->d_red_off, c->stream);
    tfim::dev_free(c->d_red_items, c->stream);
    for (auto& b : c->d_scratch) b.release();
    for (auto& b : c->h_scratch) b.release();
    c->d_masks.release();
    c->d_group.release();
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev_span0) cudaEventDestroy(c->ev_span0);
    if (c->ev_span1) cudaEventDestroy(c->ev_span1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"
