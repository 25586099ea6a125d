// Device parse of a transaction file: the bytes go to HBM once, and two passes over them
// build the CSR transaction set that ingest starts from.
//
// Semantics are the reference's byte scanner, readTransSetFile
// (code/engine/src/kernel_bitmap.cu:205-233), restated per byte so that every byte can be
// classified independently:
//   * every '\n' ends a row (empty rows included);
//   * a maximal run of digits is an item id, unless the byte before the run is '-' (the
//     scanner consumes "-<digits>" and drops it);
//   * every other byte separates;
//   * a last row without a closing '\n' is kept only when it holds an id (:232).
// The scanner's digit loop accumulates in a `long` and stores `(int)v`; ids here accumulate
// modulo 2^32 and are stored as int32, which is the same value for every run of up to 18
// digits (longer runs overflow the reference's `long`, which C leaves undefined).
//
// Pass 1 (k_parse_count): one block per 4 KiB tile, 16 bytes per thread from one 16-byte
// load; per tile the number of '\n' bytes and of id starts.  An exclusive scan over tiles
// gives every tile its first row and first item.  Pass 2 (k_parse_write): the tile and a
// 64-byte halo staged in shared memory, a block scan of the per-thread counts, then each
// thread writes its ids (value parsed from shared memory, from global memory past the halo)
// and, per '\n', the row end offset (ids before it).  Both passes read the text once from
// HBM; the bytes beyond the file are spaces, so no pass needs a bounds test per byte.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kParseThreads = 256;
constexpr int kParseBpt = 16;                              // bytes per thread
constexpr int kParseTile = kParseThreads * kParseBpt;      // 4096 bytes per block
constexpr int kParseHalo = 64;                             // staged bytes past the tile

struct Cnt {
    long long nl, st;   // newlines, id starts
};
struct CntSum {
    __host__ __device__ Cnt operator()(const Cnt& a, const Cnt& b) const { return Cnt{a.nl + b.nl, a.st + b.st}; }
};

__device__ __forceinline__ bool is_digit(uint32_t c) { return c - '0' < 10u; }

// Flags of the 16 bytes in `w` (little-endian: byte j = bits 8j..8j+7); `prev` is the byte
// before them.  Bit j of *nl: byte j is '\n'; bit j of *st: an id starts at byte j.
__device__ __forceinline__ void byte_flags(const uint4 w, uint32_t prev, uint32_t* nl, uint32_t* st) {
    const uint32_t wd[4] = {w.x, w.y, w.z, w.w};
    uint32_t n = 0, s = 0;
    bool pd = is_digit(prev), pm = prev == '-';
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const uint32_t c = (wd[j >> 2] >> ((j & 3) * 8)) & 0xffu;
        const bool d = is_digit(c);
        n |= (uint32_t)(c == '\n') << j;
        s |= (uint32_t)(d && !pd && !pm) << j;
        pd = d;
        pm = c == '-';
    }
    *nl = n;
    *st = s;
}

__global__ void __launch_bounds__(kParseThreads) k_parse_count(const uint8_t* __restrict__ text, Cnt* __restrict__ tile_cnt) {
    const int64_t i0 = (int64_t)blockIdx.x * kParseTile + threadIdx.x * kParseBpt;
    const uint4 w = __ldg(reinterpret_cast<const uint4*>(text + i0));
    const uint32_t prev = i0 > 0 ? __ldg(text + i0 - 1) : ' ';
    uint32_t nl, st;
    byte_flags(w, prev, &nl, &st);
    typedef cub::BlockReduce<int, kParseThreads> BR;
    __shared__ typename BR::TempStorage t1, t2;
    const int bn = BR(t1).Sum(__popc(nl));
    const int bs = BR(t2).Sum(__popc(st));
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = Cnt{bn, bs};
}

__global__ void __launch_bounds__(kParseThreads) k_parse_write(const uint8_t* __restrict__ text, const Cnt* __restrict__ tile_base,
                                                              int64_t* __restrict__ off, int32_t* __restrict__ items) {
    __shared__ __align__(16) uint8_t tile[kParseTile + kParseHalo];
    typedef cub::BlockScan<unsigned long long, kParseThreads> BS;
    __shared__ typename BS::TempStorage ts;
    const int64_t t0 = (int64_t)blockIdx.x * kParseTile;
    const int64_t i0 = t0 + threadIdx.x * kParseBpt;
    const uint4 w = __ldg(reinterpret_cast<const uint4*>(text + i0));
    reinterpret_cast<uint4*>(tile)[threadIdx.x] = w;
    if (threadIdx.x < kParseHalo / 16)
        reinterpret_cast<uint4*>(tile + kParseTile)[threadIdx.x] =
            __ldg(reinterpret_cast<const uint4*>(text + t0 + kParseTile) + threadIdx.x);
    const uint32_t prev = i0 > 0 ? __ldg(text + i0 - 1) : ' ';
    uint32_t nl, st;
    byte_flags(w, prev, &nl, &st);
    // per-thread (newlines, id starts) packed into one 64-bit word; a tile holds at most 4096 of each
    unsigned long long mine = ((unsigned long long)__popc(nl) << 32) | (unsigned long long)__popc(st), pre;
    BS(ts).ExclusiveSum(mine, pre);
    __syncthreads();   // the staged tile is complete before any thread reads past its own bytes
    const Cnt base = tile_base[blockIdx.x];
    int64_t r = base.nl + (int64_t)(pre >> 32);
    int64_t o = base.st + (int64_t)(pre & 0xffffffffull);
    const uint32_t any = nl | st;
    if (!any) return;
    for (int j = 0; j < kParseBpt; j++) {
        if (st >> j & 1u) {
            uint32_t v = 0;
            int k = threadIdx.x * kParseBpt + j;
            for (; k < kParseTile + kParseHalo; k++) {
                const uint32_t c = tile[k];
                if (!is_digit(c)) break;
                v = v * 10u + (c - '0');
            }
            if (k == kParseTile + kParseHalo) {   // a run longer than the halo: continue in global memory
                for (const uint8_t* p = text + t0 + k;; p++) {
                    const uint32_t c = *p;
                    if (!is_digit(c)) break;
                    v = v * 10u + (c - '0');
                }
            }
            items[o++] = (int32_t)v;
        }
        if (nl >> j & 1u) off[++r] = o;
    }
}

// A last row without a closing newline counts only when it holds an id.
__global__ void k_parse_tail(int64_t* off, int64_t n_nl, int64_t n_ids, int64_t* n_rows) {
    off[0] = 0;
    const int64_t before = n_nl > 0 ? off[n_nl] : 0;
    if (n_ids > before) {
        off[n_nl + 1] = n_ids;
        *n_rows = n_nl + 1;
    } else {
        *n_rows = n_nl;
    }
}

// ------------------------------------------------------------------ upload
// Copy the file bytes into d_text.  A pinned host buffer goes in one copy; otherwise worker
// threads fill pinned chunks (memcpy from the host buffer, or pread from the file) and each
// enqueues its chunk's copy on its own stream, so reading chunk k+1 overlaps copying chunk k.
constexpr size_t kUploadChunk = 8u << 20;

int upload_text(const TextSource& src, uint8_t* d_text, cudaStream_t s) {
    const int64_t n = src.n_bytes;
    if (n == 0) return TFIM_OK;
    if (src.host) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, src.host) == cudaSuccess && at.type == cudaMemoryTypeHost) {
            TFIM_CUDA(cudaMemcpyAsync(d_text, src.host, (size_t)n, cudaMemcpyHostToDevice, s));
            return TFIM_OK;
        }
        cudaGetLastError();
    }
    const int64_t n_chunks = (n + (int64_t)kUploadChunk - 1) / (int64_t)kUploadChunk;
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int n_workers = (int)std::min<int64_t>(n_chunks, std::min(hw, 8));
    std::atomic<int> failed{0};
    std::vector<std::string> errs(n_workers);
    std::vector<cudaStream_t> streams(n_workers, nullptr);
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    auto work = [&](int wk) {
        cudaSetDevice(dev);
        cudaStream_t ws = nullptr;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        void* buf[2] = {nullptr, nullptr};
        size_t got[2] = {0, 0};
        bool used[2] = {false, false};
        auto fail = [&](const char* what) {
            errs[wk] = what;
            failed.store(1);
        };
        if (cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
            fail("stream or event creation failed");
        } else {
            buf[0] = pinned_alloc(kUploadChunk, &got[0]);
            buf[1] = pinned_alloc(kUploadChunk, &got[1]);
            if (!buf[0] || !buf[1]) fail("pinned staging allocation failed");
        }
        int slot = 0;
        for (int64_t k = wk; !failed.load() && k < n_chunks; k += n_workers, slot ^= 1) {
            if (used[slot] && cudaEventSynchronize(ev[slot]) != cudaSuccess) { fail("host-to-device copy failed"); break; }
            const int64_t at = k * (int64_t)kUploadChunk;
            const size_t len = (size_t)std::min<int64_t>((int64_t)kUploadChunk, n - at);
            if (src.host) {
                memcpy(buf[slot], src.host + at, len);
            } else {
                size_t done = 0;
                while (done < len) {
                    const ssize_t r = pread(src.fd, (char*)buf[slot] + done, len - done, (off_t)(at + (int64_t)done));
                    if (r <= 0) break;
                    done += (size_t)r;
                }
                if (done != len) { fail("reading the transaction file failed (short read)"); break; }
            }
            if (cudaMemcpyAsync(d_text + at, buf[slot], len, cudaMemcpyHostToDevice, ws) != cudaSuccess ||
                cudaEventRecord(ev[slot], ws) != cudaSuccess) {
                fail("host-to-device copy failed");
                break;
            }
            used[slot] = true;
        }
        if (ws) cudaStreamSynchronize(ws);   // the staging buffers go back to the cache only when idle
        for (int b = 0; b < 2; b++) {
            if (buf[b]) pinned_free(buf[b], got[b]);
            if (ev[b]) cudaEventDestroy(ev[b]);
        }
        streams[wk] = ws;
    };
    std::vector<std::thread> th;
    for (int wk = 1; wk < n_workers; wk++) th.emplace_back(work, wk);
    work(0);
    for (auto& t : th) t.join();
    for (auto ws : streams)
        if (ws) cudaStreamDestroy(ws);
    if (failed.load()) {
        for (auto& e : errs)
            if (!e.empty()) { set_error("%s", e.c_str()); break; }
        return TFIM_E_CUDA;
    }
    return TFIM_OK;
}

}  // namespace

int parse_text_device(const TextSource& src, cudaStream_t s, int64_t** d_off_out, int32_t** d_items_out,
                      int64_t* n_rows_out, int64_t* nnz_out) {
    *d_off_out = nullptr;
    *d_items_out = nullptr;
    const int64_t n = src.n_bytes;
    TFIM_CHECK(n >= 0 && (n == 0 || src.host || src.fd >= 0), TFIM_E_INVALID, "invalid transaction file bytes");
    const int64_t n_tiles = std::max<int64_t>(1, (n + kParseTile - 1) / kParseTile);
    // one spare tile past the last: the write pass stages its halo from there
    const size_t text_bytes = (size_t)(n_tiles + 1) * kParseTile;
    uint8_t* d_text = nullptr;
    Cnt* d_cnt = nullptr;   // tile counts, then tile bases, then the totals
    int64_t* d_off = nullptr;
    int32_t* d_items = nullptr;
    void* d_tmp = nullptr;
    int rc = TFIM_OK;
    auto cleanup = [&](int r) {
        dev_free(d_text, s);
        dev_free(d_cnt, s);
        dev_free(d_tmp, s);
        if (r != TFIM_OK) {
            dev_free(d_off, s);
            dev_free(d_items, s);
        }
        return r;
    };
    if ((rc = dev_alloc((void**)&d_text, text_bytes, s)) || (rc = dev_alloc((void**)&d_cnt, (size_t)(2 * n_tiles + 1) * sizeof(Cnt), s)))
        return cleanup(rc);
    if (cudaMemsetAsync(d_text + n, ' ', text_bytes - (size_t)n, s) != cudaSuccess) {
        set_error("padding the transaction text failed");
        return cleanup(TFIM_E_CUDA);
    }
    // the upload's worker streams write into memory allocated in stream order on `s`
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("transaction text buffer set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
        return cleanup(TFIM_E_CUDA);
    }
    if ((rc = upload_text(src, d_text, s))) return cleanup(rc);
    Cnt* cnt = d_cnt;
    Cnt* base = d_cnt + n_tiles;
    k_parse_count<<<(unsigned)n_tiles, kParseThreads, 0, s>>>(d_text, cnt);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveScan(nullptr, tb, cnt, base, CntSum(), Cnt{0, 0}, (int64_t)n_tiles, s);
    if ((rc = dev_alloc(&d_tmp, tb, s))) return cleanup(rc);
    cub::DeviceScan::ExclusiveScan(d_tmp, tb, cnt, base, CntSum(), Cnt{0, 0}, (int64_t)n_tiles, s);
    Cnt tot[2];
    cudaMemcpyAsync(&tot[0], base + n_tiles - 1, sizeof(Cnt), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&tot[1], cnt + n_tiles - 1, sizeof(Cnt), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        set_error("transaction file parse (count pass) failed: %s", cudaGetErrorString(cudaGetLastError()));
        return cleanup(TFIM_E_CUDA);
    }
    const int64_t n_nl = tot[0].nl + tot[1].nl, n_ids = tot[0].st + tot[1].st;
    if ((rc = dev_alloc((void**)&d_off, (size_t)(n_nl + 2) * 8, s)) ||
        (rc = dev_alloc((void**)&d_items, (size_t)std::max<int64_t>(n_ids, 1) * 4, s)))
        return cleanup(rc);
    k_parse_write<<<(unsigned)n_tiles, kParseThreads, 0, s>>>(d_text, base, d_off, d_items);
    int64_t* d_rows = reinterpret_cast<int64_t*>(d_cnt + 2 * n_tiles);
    k_parse_tail<<<1, 1, 0, s>>>(d_off, n_nl, n_ids, d_rows);
    int64_t rows = 0;
    cudaMemcpyAsync(&rows, d_rows, 8, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        set_error("transaction file parse (write pass) failed: %s", cudaGetErrorString(cudaGetLastError()));
        return cleanup(TFIM_E_CUDA);
    }
    *d_off_out = d_off;
    *d_items_out = d_items;
    *n_rows_out = rows;
    *nnz_out = n_ids;
    return cleanup(TFIM_OK);
}

}  // namespace tfim
