// Projected counting for families whose prefix holds few transactions.
//
// A family's counts are popc(base & B[t] & B[e]) for t in its rows, e in its columns.
// When the base (the prefix mask) has few set bits, almost every word of those AND
// products is zero.  This counter walks only the base's set bits: for each transaction r
// in the prefix it reads r's items from the frequency-compacted transaction list and adds
// one for every (row item, column item) pair that r holds.  Work is
// sum over the prefix's transactions of (items in F)^2 instead of (rows + columns + 1) x N
// bits.  One block per job; the column list is hashed in shared memory and the job's count
// block is accumulated in shared memory when it fits.  Exact integer counts, the same as the
// bitmap counters'.
#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kProjHash = 4096;       // hash slots (column lists up to kProjMaxCols)
constexpr int kProjAcc = 4096;        // shared accumulator entries (rows x cols)

__device__ __forceinline__ uint32_t hash_item(int32_t x) { return ((uint32_t)x * 2654435761u) & (kProjHash - 1); }

__device__ __forceinline__ int32_t lookup(const int32_t* keys, const int32_t* vals, int32_t x) {
    uint32_t h = hash_item(x);
    for (int probe = 0; probe < kProjHash; probe++) {
        const int32_t k = keys[h];
        if (k == x) return vals[h];
        if (k == -1) return -1;
        h = (h + 1) & (kProjHash - 1);
    }
    return -1;
}

__global__ void __launch_bounds__(256) k_count_proj(CountArgs a, const int32_t* __restrict__ job_ids,
                                                    const int64_t* __restrict__ red_off,
                                                    const int32_t* __restrict__ red_items, int32_t r0_unused) {
    __shared__ int32_t keys[kProjHash];
    __shared__ int32_t vals[kProjHash];
    __shared__ int32_t acc[kProjAcc];
    const int32_t jid = job_ids[blockIdx.x];
    const JobDesc j = a.jobs[jid];
    const int nr = j.n_rows, nc = j.n_cols;
    // rows of the job are columns [row_first, row_first + nr) of its column list: the
    // family's rows are the first entries of its column list and row r of the job is
    // the column a.rows[j.row_off + r].item
    for (int q = threadIdx.x; q < kProjHash; q += blockDim.x) keys[q] = -1;
    const bool smem_acc = (int64_t)nr * nc <= kProjAcc;
    if (smem_acc)
        for (int q = threadIdx.x; q < nr * nc; q += blockDim.x) acc[q] = 0;
    __syncthreads();
    // column item -> column index
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        const int32_t x = c == j.self_col ? -2 : a.cols[j.col_off + c];
        if (x < 0) continue;
        uint32_t h = hash_item(x);
        while (true) {
            const int32_t prev = atomicCAS(&keys[h], -1, x);
            if (prev == -1 || prev == x) break;
            h = (h + 1) & (kProjHash - 1);
        }
        vals[h] = c;
    }
    __syncthreads();
    // the first row's column index: rows are consecutive columns of the list
    const int32_t first_item = a.rows[j.row_off].item;
    const int32_t row_first = lookup(keys, vals, first_item);
    const int64_t W = a.W;
    const uint32_t* base_m = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
    const uint32_t* base_i = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
    int32_t* out = a.out + j.out_off;
    for (int64_t w = threadIdx.x; w < W; w += blockDim.x) {
        uint32_t m = ~0u;
        if (base_m) m &= base_m[w];
        if (base_i) m &= __ldg(base_i + w);
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            const int64_t r = w * 32 + b;
            const int64_t b0 = red_off[r], b1 = red_off[r + 1];
            for (int64_t xa = b0; xa < b1; xa++) {
                const int32_t ca = lookup(keys, vals, red_items[xa]);
                const int32_t ra = ca - row_first;
                if (ca < 0 || ra < 0 || ra >= nr) continue;
                for (int64_t xb = b0; xb < b1; xb++) {
                    const int32_t cb = lookup(keys, vals, red_items[xb]);
                    if (cb < 0) continue;
                    if (smem_acc) atomicAdd(&acc[ra * nc + cb], 1);
                    else atomicAdd(out + (int64_t)ra * nc + cb, 1);
                }
                if (j.self_col >= 0) {   // the all-ones column counts the row's own support
                    if (smem_acc) atomicAdd(&acc[ra * nc + j.self_col], 1);
                    else atomicAdd(out + (int64_t)ra * nc + j.self_col, 1);
                }
            }
        }
    }
    __syncthreads();
    if (smem_acc)
        for (int q = threadIdx.x; q < nr * nc; q += blockDim.x) out[q] = acc[q];
}

}  // namespace

int launch_count_proj(const CountArgs& a, const int32_t* job_ids, int32_t n_jobs, const int64_t* red_off,
                      const int32_t* red_items, cudaStream_t s) {
    if (n_jobs <= 0) return TFIM_OK;
    k_count_proj<<<n_jobs, 256, 0, s>>>(a, job_ids, red_off, red_items, 0);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

}  // namespace tfim
