// Device ingest: F1 occurrence histogram, frequency compaction and the vertical bitmap.
//
// Semantics follow the reference's host pipeline (code/engine/src/kernel_bitmap.cu):
//   getItemsFrequenc :269-298   occurrence counts (a repeated id in one row counts twice)
//   main :806                   frequencyThreshold = transNum * supportThreshold (double)
//   reduceTransSet :692-703     drop ids with count < threshold, then empty rows
//   main :815-816               dimensionReduced: ids (0 included) with freq/transNum > thr
//   buildBitmap :342-380        survivors = ids 1..max with count >= threshold, dense ids in
//                               ascending original order; a frequent id 0 is parked after
//                               them; bit t of row x set iff reduced row t holds x
// The work is done on the GPU: one histogram pass, one pass that measures reduced rows,
// a scan that numbers the surviving rows, and one scatter pass that sets the bits.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <numeric>

#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

struct ScanStats {
    int32_t id_min, id_max;
    int32_t neg;        // any negative id seen
    int32_t bad_off;    // any decreasing offset seen
    long long len_min, len_max;
    unsigned long long len_sum;
    long long red_min, red_max;
    unsigned long long red_sum;
    unsigned long long red_sq_sum;   // sum of squared reduced lengths: pair-counting work
};

__global__ void k_item_minmax(const int32_t* __restrict__ items, int64_t nnz, ScanStats* st) {
    int32_t mn = INT_MAX, mx = INT_MIN, neg = 0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = items[j];
        mn = min(mn, v);
        mx = max(mx, v);
        neg |= (v < 0);
    }
    typedef cub::BlockReduce<int32_t, 256> BR;
    __shared__ typename BR::TempStorage t1;
    int32_t bmn = BR(t1).Reduce(mn, cub::Min());
    __syncthreads();
    int32_t bmx = BR(t1).Reduce(mx, cub::Max());
    __syncthreads();
    int32_t bneg = BR(t1).Reduce(neg, cub::Max());
    if (threadIdx.x == 0) {
        atomicMin(&st->id_min, bmn);
        atomicMax(&st->id_max, bmx);
        if (bneg) atomicExch(&st->neg, 1);
    }
}

__global__ void k_row_lengths(const int64_t* __restrict__ off, int64_t n_rows, ScanStats* st) {
    long long mn = LLONG_MAX, mx = 0;
    unsigned long long sum = 0;
    int bad = 0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
        long long len = (long long)(off[r + 1] - off[r]);
        bad |= (len < 0);
        mn = min(mn, len);
        mx = max(mx, len);
        sum += (unsigned long long)(len > 0 ? len : 0);
    }
    typedef cub::BlockReduce<long long, 256> BR;
    typedef cub::BlockReduce<unsigned long long, 256> BRU;
    typedef cub::BlockReduce<int, 256> BRI;
    __shared__ typename BR::TempStorage t1;
    __shared__ typename BRU::TempStorage t2;
    __shared__ typename BRI::TempStorage t3;
    long long bmn = BR(t1).Reduce(mn, cub::Min());
    __syncthreads();
    long long bmx = BR(t1).Reduce(mx, cub::Max());
    unsigned long long bs = BRU(t2).Sum(sum);
    int bb = BRI(t3).Reduce(bad, cub::Max());
    if (threadIdx.x == 0) {
        atomicMin(&st->len_min, bmn);
        atomicMax(&st->len_max, bmx);
        atomicAdd(&st->len_sum, bs);
        if (bb) atomicExch(&st->bad_off, 1);
    }
}

__global__ void k_hist(const int32_t* __restrict__ items, int64_t nnz, int32_t* __restrict__ freq) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&freq[items[j]], 1);
}

// The same histogram when the id space fits in shared memory: every block counts a strided
// share of the items in a private shared histogram (no global atomics; the skewed ids of a
// long-tailed database collide only within a block) and writes it to partial[block]; the
// column sums are taken by k_hist_sum.
constexpr int kHistSmemBins = 48 * 1024;
__global__ void __launch_bounds__(1024) k_hist_smem(const int32_t* __restrict__ items, int64_t nnz, int32_t bins,
                                                    int32_t* __restrict__ partial) {
    extern __shared__ int32_t h[];
    for (int i = threadIdx.x; i < bins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[__ldg(items + j)], 1);
    __syncthreads();
    int32_t* out = partial + (int64_t)blockIdx.x * bins;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) out[i] = h[i];
}
__global__ void k_hist_sum(const int32_t* __restrict__ partial, int32_t parts, int32_t bins, int32_t* __restrict__ freq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bins) return;
    int32_t v = 0;
    for (int b = 0; b < parts; b++) v += partial[(int64_t)b * bins + i];
    freq[i] = v;
}

// Per row: the reduced length (occurrences of ids that survive the threshold, id 0
// included when frequent); 0 marks a row that reduction removes.
__global__ void k_reduced_rows(const int64_t* __restrict__ off, const int32_t* __restrict__ items, int64_t n_rows,
                               const int32_t* __restrict__ map, int32_t* __restrict__ red_len, ScanStats* st) {
    long long mn = LLONG_MAX, mx = 0;
    unsigned long long sum = 0, sq = 0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
        int32_t len = 0;
        for (int64_t j = off[r]; j < off[r + 1]; j++) len += (map[items[j]] >= 0);
        red_len[r] = len;
        if (len > 0) {
            mn = min(mn, (long long)len);
            mx = max(mx, (long long)len);
            sum += (unsigned long long)len;
            sq += (unsigned long long)len * (unsigned long long)len;
        }
    }
    typedef cub::BlockReduce<long long, 256> BR;
    typedef cub::BlockReduce<unsigned long long, 256> BRU;
    __shared__ typename BR::TempStorage t1;
    __shared__ typename BRU::TempStorage t2;
    long long bmn = BR(t1).Reduce(mn, cub::Min());
    __syncthreads();
    long long bmx = BR(t1).Reduce(mx, cub::Max());
    unsigned long long bs = BRU(t2).Sum(sum);
    __syncthreads();
    unsigned long long bq = BRU(t2).Sum(sq);
    if (threadIdx.x == 0) {
        atomicMin(&st->red_min, bmn);
        atomicMax(&st->red_max, bmx);
        atomicAdd(&st->red_sum, bs);
        atomicAdd(&st->red_sq_sum, bq);
    }
}

struct IsPositive {
    __host__ __device__ int32_t operator()(int32_t v) const { return v > 0; }
};

// The reduced transaction list in dense ids (reduced row rr = surviving row r).
__global__ void k_write_reduced(const int64_t* __restrict__ off, const int32_t* __restrict__ items, int64_t n_rows,
                                const int32_t* __restrict__ map, const int32_t* __restrict__ red_len,
                                const int64_t* __restrict__ red_idx, const int64_t* __restrict__ item_off,
                                int64_t* __restrict__ red_off, int32_t* __restrict__ red_items) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
        if (red_len[r] == 0) continue;
        const int64_t rr = red_idx[r];
        int64_t o = item_off[r];
        red_off[rr] = o;
        for (int64_t j = off[r]; j < off[r + 1]; j++) {
            const int32_t d = map[items[j]];
            if (d >= 0) red_items[o++] = d;
        }
    }
}

// One thread per reduced row: set the row's bit in the row of each of its items.  Rows
// of one warp are consecutive, so their bits for one item share a 32-bit word; the warp
// merges equal (item, word) targets before the atomic.
__global__ void k_scatter_bits(const int64_t* __restrict__ red_off, const int32_t* __restrict__ red_items, int64_t n_red,
                               uint32_t* __restrict__ bm, int64_t W) {
    for (int64_t r0 = blockIdx.x * (int64_t)blockDim.x; r0 < n_red; r0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t rr = r0 + threadIdx.x;
        const bool live = rr < n_red;
        int64_t j = live ? red_off[rr] : 0, je = live ? red_off[rr + 1] : 0;
        while (__any_sync(0xffffffffu, j < je)) {
            int32_t d = -1;
            if (j < je) { d = red_items[j]; j++; }
            const unsigned long long key = d >= 0 ? ((unsigned long long)(uint32_t)d << 32) | (unsigned long long)(rr >> 5) : ~0ull;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const uint32_t bit = d >= 0 ? (1u << (rr & 31)) : 0u;
            uint32_t acc = bit;
            for (int k = 0; k < 32; k++) {
                const uint32_t v = __shfl_sync(0xffffffffu, bit, k);
                if ((peers >> k) & 1u) acc |= v;
            }
            const int leader = __ffs(peers) - 1;
            if (d >= 0 && (int)(threadIdx.x & 31) == leader) atomicOr(&bm[(int64_t)d * W + (rr >> 5)], acc);
        }
    }
}

__global__ void k_row_popc(const uint32_t* __restrict__ bm, int64_t W, int32_t n, int32_t* __restrict__ out) {
    const int row = blockIdx.x;
    if (row >= n) return;
    const uint4* p = reinterpret_cast<const uint4*>(bm + (int64_t)row * W);
    unsigned long long s = 0;
    for (int64_t w = threadIdx.x; w < W / 4; w += blockDim.x) {
        uint4 v = p[w];
        s += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
    }
    typedef cub::BlockReduce<unsigned long long, 256> BR;
    __shared__ typename BR::TempStorage t;
    unsigned long long b = BR(t).Sum(s);
    if (threadIdx.x == 0) out[row] = (int32_t)b;
}

int grid_for(int64_t n, int per = 256) {
    int64_t g = (n + per - 1) / per;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return (int)g;
}

}  // namespace

int compute_bit_supports(tfim_ctx* c) {
    // popcount of every bitmap row (the counted ones are the bitmap supports); their sum
    // equals the reduced transaction list's length exactly when no row repeats an id
    const int32_t rows = c->from_db ? c->info.n_dense : c->n_counted;
    std::vector<int32_t> all(std::max<int32_t>(rows, 0), 0);
    if (rows > 0) {
        TFIM_TRY(c->d_scratch[7].reserve((size_t)rows * 4));
        k_row_popc<<<rows, 256, 0, c->stream>>>(c->d_bitmap, c->W, rows, c->d_scratch[7].as<int32_t>());
        TFIM_CUDA(cudaGetLastError());
        TFIM_CUDA(cudaMemcpyAsync(all.data(), c->d_scratch[7].p, (size_t)rows * 4, cudaMemcpyDeviceToHost, c->stream));
        TFIM_CUDA(cudaStreamSynchronize(c->stream));
    }
    int64_t total = 0;
    for (int32_t v : all) total += v;
    c->csr_exact = c->from_db && c->d_red_off && total == c->n_red_items;
    if (c->sharded) {
        // row supports summed over the shards; the list counters are exact only if every shard's list is
        if (rows > 0) {
            TFIM_TRY(group_reduce(c, c->d_scratch[7].p, rows, TFIM_DT_I32, TFIM_RED_SUM, c->stream));
            TFIM_CUDA(cudaMemcpyAsync(all.data(), c->d_scratch[7].p, (size_t)rows * 4, cudaMemcpyDeviceToHost, c->stream));
            TFIM_CUDA(cudaStreamSynchronize(c->stream));
        }
        int64_t inexact = c->csr_exact ? 0 : 1;
        TFIM_TRY(group_reduce_host(c, &inexact, 1, TFIM_RED_MAX));
        c->csr_exact = inexact == 0;
    }
    c->bit_support.assign(all.begin(), all.begin() + std::min<int32_t>(rows, c->n_counted));
    return TFIM_OK;
}

int ingest_csr(tfim_ctx* c, const int64_t* h_off, const int32_t* h_items, int64_t n_rows, double thr) {
    cudaStream_t s = c->stream;
    const int64_t base = n_rows > 0 ? h_off[0] : 0;
    TFIM_CHECK(base == 0, TFIM_E_INVALID, "row_offsets[0] must be 0");
    const int64_t nnz = n_rows > 0 ? h_off[n_rows] : 0;
    TFIM_CHECK(nnz >= 0, TFIM_E_INVALID, "row_offsets[n_rows] is negative");
    DevBuf d_off, d_items;
    d_off.stream = d_items.stream = s;
    int rc = TFIM_OK;
    if (!(rc = d_off.reserve((size_t)(n_rows + 1) * 8)) && !(rc = d_items.reserve((size_t)std::max<int64_t>(nnz, 1) * 4))) {
        if (cudaMemcpyAsync(d_off.p, h_off, (size_t)(n_rows + 1) * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            (nnz > 0 && cudaMemcpyAsync(d_items.p, h_items, (size_t)nnz * 4, cudaMemcpyHostToDevice, s) != cudaSuccess)) {
            set_error("host-to-device copy of the transaction set failed");
            rc = TFIM_E_CUDA;
        } else {
            rc = ingest_device_csr(c, d_off.as<int64_t>(), d_items.as<int32_t>(), n_rows, nnz, thr);
        }
    }
    d_off.release();
    d_items.release();
    return rc;
}

int ingest_device_csr(tfim_ctx* c, const int64_t* d_off_p, const int32_t* d_items_p, int64_t n_rows, int64_t nnz,
                      double thr) {
    cudaStream_t s = c->stream;
    DevBuf d_stats, d_freq, d_map, d_flag, d_idx, d_tmp;
    for (DevBuf* b : {&d_stats, &d_freq, &d_map, &d_flag, &d_idx, &d_tmp}) b->stream = s;
    int rc = TFIM_OK;
    ScanStats hs{};
    std::vector<int32_t> freq;
    int64_t id_max = 0, id_min = INT_MAX;
    // all device scratch below is released at the end of this function
    auto done = [&](int r) {
        d_stats.release(); d_freq.release();
        d_map.release(); d_flag.release(); d_idx.release(); d_tmp.release();
        return r;
    };
    if ((rc = d_stats.reserve(sizeof(ScanStats)))) return done(rc);
    hs.id_min = INT_MAX; hs.id_max = INT_MIN; hs.len_min = LLONG_MAX; hs.red_min = LLONG_MAX;
    cudaMemcpyAsync(d_stats.p, &hs, sizeof hs, cudaMemcpyHostToDevice, s);
    if (nnz > 0) k_item_minmax<<<grid_for(nnz), 256, 0, s>>>(d_items_p, nnz, d_stats.as<ScanStats>());
    if (n_rows > 0) k_row_lengths<<<grid_for(n_rows), 256, 0, s>>>(d_off_p, n_rows, d_stats.as<ScanStats>());
    cudaMemcpyAsync(&hs, d_stats.p, sizeof hs, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { set_error("ingest statistics pass failed: %s", cudaGetErrorString(cudaGetLastError())); return done(TFIM_E_CUDA); }
    int64_t n_rows_all = n_rows;
    if (c->sharded) {
        // the whole database's statistics: errors, id range and row lengths (MIN as -MAX(-x))
        int64_t mx[6] = {hs.neg, hs.bad_off, nnz > 0 ? (int64_t)hs.id_max : -1, n_rows > 0 ? (int64_t)hs.len_max : 0,
                         nnz > 0 ? -(int64_t)hs.id_min : -(int64_t)INT_MAX, n_rows > 0 ? -(int64_t)hs.len_min : -(int64_t)LLONG_MAX};
        int64_t sm[3] = {n_rows, (int64_t)hs.len_sum, nnz};
        if ((rc = group_reduce_host(c, mx, 6, TFIM_RED_MAX)) || (rc = group_reduce_host(c, sm, 3, TFIM_RED_SUM))) return done(rc);
        hs.neg = (int32_t)mx[0];
        hs.bad_off = (int32_t)mx[1];
        n_rows_all = sm[0];
        hs.len_sum = (unsigned long long)sm[1];
        if (sm[2] > 0) { id_max = mx[2]; id_min = -mx[4]; }
        hs.len_max = mx[3];
        hs.len_min = -mx[5];
    } else if (nnz > 0) {
        id_min = hs.id_min;
        id_max = hs.id_max;
    }
    if (hs.neg) { set_error("negative item id in the transaction set"); return done(TFIM_E_INVALID); }
    if (hs.bad_off) { set_error("row_offsets must be non-decreasing"); return done(TFIM_E_INVALID); }

    // F1 histogram over ids 0..id_max (kernel_bitmap.cu:269-275)
    if ((rc = d_freq.reserve((size_t)(id_max + 1) * 4))) return done(rc);
    {
        const int32_t bins = (int32_t)(id_max + 1);
        if (nnz > 0 && bins <= kHistSmemBins) {
            const int32_t parts = (int32_t)std::min<int64_t>(148, (nnz + 65535) / 65536);
            if ((rc = d_tmp.reserve((size_t)parts * bins * 4))) return done(rc);
            static std::atomic<bool> configured[64];
            int dev = 0;
            cudaGetDevice(&dev);
            if (dev >= 0 && dev < 64 && !configured[dev].load()) {
                cudaFuncSetAttribute(k_hist_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, kHistSmemBins * 4);
                configured[dev].store(true);
            }
            k_hist_smem<<<parts, 1024, (size_t)bins * 4, s>>>(d_items_p, nnz, bins, d_tmp.as<int32_t>());
            k_hist_sum<<<(bins + 255) / 256, 256, 0, s>>>(d_tmp.as<int32_t>(), parts, bins, d_freq.as<int32_t>());
        } else {
            cudaMemsetAsync(d_freq.p, 0, (size_t)bins * 4, s);
            if (nnz > 0) k_hist<<<grid_for(nnz), 256, 0, s>>>(d_items_p, nnz, d_freq.as<int32_t>());
        }
    }
    if ((rc = group_reduce(c, d_freq.p, id_max + 1, TFIM_DT_I32, TFIM_RED_SUM, s))) return done(rc);
    freq.assign((size_t)id_max + 1, 0);
    cudaMemcpyAsync(freq.data(), d_freq.p, (size_t)(id_max + 1) * 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { set_error("F1 histogram failed: %s", cudaGetErrorString(cudaGetLastError())); return done(TFIM_E_CUDA); }

    tfim_db_info& I = c->info;
    memset(&I, 0, sizeof I);
    I.trans_num = n_rows_all;
    I.item_id_min = id_min;
    I.item_id_max = id_max;
    I.trans_len_min = n_rows_all > 0 ? hs.len_min : INT_MAX;
    I.trans_len_max = n_rows_all > 0 ? hs.len_max : 0;
    I.trans_len_mean = n_rows_all > 0 ? (double)hs.len_sum / (double)n_rows_all : 0.0;
    int64_t dim = 0;
    for (int64_t i = 0; i <= id_max; i++) dim += freq[i] != 0;
    I.dimension = dim;
    I.support_threshold = thr;
    const double fthr = (double)n_rows_all * thr;             // kernel_bitmap.cu:806
    I.frequency_threshold = fthr;
    I.min_count = (int32_t)std::max(0.0, std::ceil(fthr));     // v >= fthr  <=>  v >= ceil(fthr) for integer v
    int64_t dimred = 0;
    for (int64_t i = 0; i <= id_max; i++)                       // kernel_bitmap.cu:815-816
        if ((double)freq[i] / (double)n_rows_all > thr) dimred++;
    I.dimension_reduced = dimred;

    // dense ids (kernel_bitmap.cu:348-373)
    std::vector<int32_t> map((size_t)id_max + 1, -1);
    c->dense_to_orig.clear();
    c->dense_freq.clear();
    for (int64_t i = 1; i <= id_max; i++)
        if ((double)freq[i] >= fthr) {
            map[i] = (int32_t)c->dense_to_orig.size();
            c->dense_to_orig.push_back((int32_t)i);
            c->dense_freq.push_back(freq[i]);
        }
    const int32_t n_surv = (int32_t)c->dense_to_orig.size();
    if ((double)freq[0] >= fthr) {   // kernel_bitmap.cu:356 (true for an empty set: 0 >= 0.0)
        map[0] = n_surv;
        c->dense_to_orig.push_back(0);
        c->dense_freq.push_back(freq[0]);
    }
    const int32_t n_dense = (int32_t)c->dense_to_orig.size();
    I.n_survivors = n_surv;
    I.n_dense = n_dense;
    I.item_id_max_dense = n_dense - 1;
    c->n_counted = n_surv;
    c->items_in_freq_sort.resize(n_dense);
    std::iota(c->items_in_freq_sort.begin(), c->items_in_freq_sort.end(), 0);
    std::stable_sort(c->items_in_freq_sort.begin(), c->items_in_freq_sort.end(),
                     [&](int a, int b) { return c->dense_freq[a] > c->dense_freq[b]; });
    const int64_t n_roots = std::min<int64_t>(dimred, n_dense);
    c->roots.assign(c->items_in_freq_sort.begin(), c->items_in_freq_sort.begin() + n_roots);

    // reduced rows, their numbering, and the reduced transaction list in dense ids
    if ((rc = d_map.reserve((size_t)(id_max + 1) * 4)) || (rc = d_flag.reserve((size_t)std::max<int64_t>(n_rows, 1) * 4)) ||
        (rc = d_idx.reserve((size_t)std::max<int64_t>(n_rows, 1) * 16)))
        return done(rc);
    cudaMemcpyAsync(d_map.p, map.data(), (size_t)(id_max + 1) * 4, cudaMemcpyHostToDevice, s);
    int64_t n_red = 0, n_red_items = 0;
    int64_t* red_idx = d_idx.as<int64_t>();
    int64_t* item_off = red_idx + std::max<int64_t>(n_rows, 1);
    if (n_rows > 0) {
        int32_t* red_len = d_flag.as<int32_t>();
        k_reduced_rows<<<grid_for(n_rows), 256, 0, s>>>(d_off_p, d_items_p, n_rows,
                                                         d_map.as<int32_t>(), red_len, d_stats.as<ScanStats>());
        cub::TransformInputIterator<int32_t, IsPositive, const int32_t*> flags(red_len, IsPositive());
        size_t tb1 = 0, tb2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb1, flags, red_idx, n_rows, s);
        cub::DeviceScan::ExclusiveSum(nullptr, tb2, red_len, item_off, n_rows, s);
        if ((rc = d_tmp.reserve(std::max(tb1, tb2)))) return done(rc);
        cub::DeviceScan::ExclusiveSum(d_tmp.p, tb1, flags, red_idx, n_rows, s);
        cub::DeviceScan::ExclusiveSum(d_tmp.p, tb2, red_len, item_off, n_rows, s);
        int64_t last[2] = {0, 0};
        int32_t last_len = 0;
        cudaMemcpyAsync(&last[0], red_idx + (n_rows - 1), 8, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&last[1], item_off + (n_rows - 1), 8, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&last_len, red_len + (n_rows - 1), 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&hs, d_stats.p, sizeof hs, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) { set_error("row reduction failed: %s", cudaGetErrorString(cudaGetLastError())); return done(TFIM_E_CUDA); }
        n_red = last[0] + (last_len > 0);
        n_red_items = last[1] + last_len;
    }
    int64_t n_red_all = n_red;
    if (c->sharded) {
        int64_t mx[2] = {n_red > 0 ? (int64_t)hs.red_max : 0, n_red > 0 ? -(int64_t)hs.red_min : -(int64_t)LLONG_MAX};
        int64_t sm[3] = {n_red, (int64_t)hs.red_sum, (int64_t)hs.red_sq_sum};
        if ((rc = group_reduce_host(c, mx, 2, TFIM_RED_MAX)) || (rc = group_reduce_host(c, sm, 3, TFIM_RED_SUM))) return done(rc);
        hs.red_max = mx[0];
        hs.red_min = -mx[1];
        n_red_all = sm[0];
        hs.red_sum = (unsigned long long)sm[1];
        hs.red_sq_sum = (unsigned long long)sm[2];
    }
    I.trans_num_reduced = n_red_all;
    I.trans_len_red_min = n_red_all > 0 ? hs.red_min : INT_MAX;
    I.trans_len_red_max = n_red_all > 0 ? hs.red_max : 0;
    I.trans_len_red_mean = (double)hs.red_sum / (double)n_red_all;   // 0/0 -> nan, as the reference
    c->red_pair_work = (double)hs.red_sq_sum;
    if ((rc = dev_alloc((void**)&c->d_red_off, (size_t)(n_red + 1) * 8, s)) ||
        (rc = dev_alloc((void**)&c->d_red_items, (size_t)std::max<int64_t>(n_red_items, 1) * 4, s)))
        return done(rc);
    c->n_red_items = n_red_items;
    cudaMemcpyAsync(c->d_red_off + n_red, &n_red_items, 8, cudaMemcpyHostToDevice, s);
    if (n_red > 0)
        k_write_reduced<<<grid_for(n_rows), 256, 0, s>>>(d_off_p, d_items_p, n_rows, d_map.as<int32_t>(),
                                                          d_flag.as<int32_t>(), red_idx, item_off, c->d_red_off, c->d_red_items);

    // the bitmap: n_dense rows x W words, zero padded
    c->n_bits = n_red;
    c->n_bits_total = n_red_all;
    c->W = words_for_bits(n_red);
    if (c->sharded && c->W < kRowAlignWords) c->W = kRowAlignWords;   // an empty shard counts zeros
    I.words_per_row = (int32_t)c->W;
    const size_t bm_bytes = (size_t)std::max<int32_t>(n_dense, 1) * (size_t)std::max<int64_t>(c->W, 1) * 4;
    if ((rc = dev_alloc((void**)&c->d_bitmap, bm_bytes, s))) return done(rc);
    cudaMemsetAsync(c->d_bitmap, 0, bm_bytes, s);
    if (n_red > 0)
        k_scatter_bits<<<grid_for(n_red), 256, 0, s>>>(c->d_red_off, c->d_red_items, n_red, c->d_bitmap, c->W);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        set_error("bitmap scatter failed");
        return done(TFIM_E_CUDA);
    }
    c->from_db = true;
    rc = compute_bit_supports(c);
    return done(rc);
}

int ingest_bitmap(tfim_ctx* c, const uint32_t* rows, int32_t n_rows, int64_t n_bits, int32_t n_counted) {
    TFIM_CHECK(rows && n_rows > 0 && n_bits > 0 && n_counted >= 0 && n_counted <= n_rows, TFIM_E_INVALID,
               "tfim_open_bitmap: invalid arguments");
    const int64_t src_w = (n_bits + 31) / 32;
    c->n_bits = n_bits;
    c->n_bits_total = n_bits;
    if (c->sharded) TFIM_TRY(group_reduce_host(c, &c->n_bits_total, 1, TFIM_RED_SUM));
    c->W = words_for_bits(n_bits);
    c->n_counted = n_counted;
    memset(&c->info, 0, sizeof c->info);
    c->info.n_survivors = n_counted;
    c->info.n_dense = n_rows;
    c->info.trans_num_reduced = c->n_bits_total;
    c->info.words_per_row = (int32_t)c->W;
    const size_t bytes = (size_t)n_rows * (size_t)c->W * 4;
    TFIM_TRY(dev_alloc((void**)&c->d_bitmap, bytes, c->stream));
    TFIM_CUDA(cudaMemsetAsync(c->d_bitmap, 0, bytes, c->stream));
    TFIM_CUDA(cudaMemcpy2DAsync(c->d_bitmap, (size_t)c->W * 4, rows, (size_t)src_w * 4, (size_t)src_w * 4, n_rows,
                                cudaMemcpyHostToDevice, c->stream));
    // bits beyond n_bits in the last supplied word must not count: clear them
    if (n_bits % 32) {
        std::vector<uint32_t> last(n_rows);
        const uint32_t keep = (1u << (n_bits % 32)) - 1u;
        for (int32_t r = 0; r < n_rows; r++) last[r] = rows[(size_t)r * src_w + src_w - 1] & keep;
        TFIM_CUDA(cudaMemcpy2DAsync(c->d_bitmap + (src_w - 1), (size_t)c->W * 4, last.data(), 4, 4, n_rows,
                                    cudaMemcpyHostToDevice, c->stream));
    }
    TFIM_CUDA(cudaStreamSynchronize(c->stream));
    c->dense_to_orig.resize(n_rows);
    std::iota(c->dense_to_orig.begin(), c->dense_to_orig.end(), 0);
    return compute_bit_supports(c);
}

}  // namespace tfim
