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

constexpr int kProjHash = 2048;       // hash slots (column lists up to kProjMaxCols = 1024)
constexpr int kProjAcc = 4096;        // shared accumulator entries (rows x cols)
constexpr int kProjWarps = 8;
constexpr int kProjTidBuf = 256;      // buffered transactions per warp

__device__ __forceinline__ uint32_t hash_item(int32_t x) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u;
    return (h ^ (h >> 15)) & (kProjHash - 1);
}

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

// One thread processes one transaction: it looks up the transaction's items, keeps the
// matched column indices in registers and adds one for every (row item, column item) pair.
constexpr int kProjRegMatch = 16;
__device__ void thread_transaction(int64_t r, const int64_t* __restrict__ red_off, const int32_t* __restrict__ red_items,
                                   const int32_t* keys, const int32_t* vals, int32_t row_first, int nr, int nc,
                                   bool smem_acc, int32_t* acc, int32_t* out) {
    const int64_t b0 = red_off[r], b1 = red_off[r + 1];
    int32_t mc[kProjRegMatch];
    int m = 0;
    bool overflow = false;
    for (int64_t x = b0; x < b1; x++) {
        const int32_t c = lookup(keys, vals, __ldg(red_items + x));
        if (c < 0) continue;
        if (m < kProjRegMatch) mc[m++] = c;
        else overflow = true;
    }
    if (!overflow) {
        for (int a = 0; a < m; a++) {
            const int32_t ra = mc[a] - row_first;
            if (ra < 0 || ra >= nr) continue;
            for (int b = 0; b < m; b++) {
                if (smem_acc) atomicAdd(&acc[ra * nc + mc[b]], 1);
                else atomicAdd(out + (int64_t)ra * nc + mc[b], 1);
            }
        }
        return;
    }
    for (int64_t xa = b0; xa < b1; xa++) {
        const int32_t ca = lookup(keys, vals, __ldg(red_items + xa));
        const int32_t ra = ca - row_first;
        if (ca < 0 || ra < 0 || ra >= nr) continue;
        for (int64_t xb = b0; xb < b1; xb++) {
            const int32_t cb = lookup(keys, vals, __ldg(red_items + xb));
            if (cb < 0) continue;
            if (smem_acc) atomicAdd(&acc[ra * nc + cb], 1);
            else atomicAdd(out + (int64_t)ra * nc + cb, 1);
        }
    }
}

struct ProjShared {
    int32_t keys[kProjHash];
    int32_t vals[kProjHash];
    int32_t acc[kProjAcc];
    int32_t tidbuf[kProjWarps][kProjTidBuf];
};

__device__ void proj_job(const CountArgs& a, int32_t jid, const int64_t* __restrict__ red_off,
                         const int32_t* __restrict__ red_items, ProjShared& sh) {
    int32_t* keys = sh.keys;
    int32_t* vals = sh.vals;
    int32_t* acc = sh.acc;
    int32_t (*tidbuf)[kProjTidBuf] = sh.tidbuf;
    const JobDesc j = a.jobs[jid];
    const int nr = j.n_rows, nc = j.n_cols;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < kProjHash; q += blockDim.x) keys[q] = -1;
    const bool smem_acc = (int64_t)nr * nc <= kProjAcc;
    if (smem_acc)
        for (int q = threadIdx.x; q < nr * nc; q += blockDim.x) acc[q] = 0;
    __syncthreads();
    // column item -> column index (the job's rows are the columns [row_first, row_first+nr))
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        const int32_t x = a.cols[j.col_off + c];
        uint32_t h = hash_item(x);
        while (true) {
            const int32_t prev = atomicCAS(&keys[h], -1, x);
            if (prev == -1 || prev == x) break;
            h = (h + 1) & (kProjHash - 1);
        }
        vals[h] = c;
    }
    __syncthreads();
    const int32_t row_first = lookup(keys, vals, a.rows[j.row_off].item);
    const int64_t W = a.W;
    const uint32_t* base_m = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
    const uint32_t* base_i = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
    int32_t* out = a.out + j.out_off;
    int32_t* tb = tidbuf[warp];
    int nb = 0;
    // each warp scans 32-word stripes of the base, buffering its transactions
    for (int64_t w0 = (int64_t)warp * 32; w0 < W; w0 += (int64_t)kProjWarps * 32) {
        const int64_t w = w0 + lane;
        uint32_t m = 0;
        if (w < W) {
            m = ~0u;
            if (base_m) m &= base_m[w];
            if (base_i) m &= __ldg(base_i + w);
        }
        int cnt = __popc(m);
        int excl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, excl, o);
            if (lane >= o) excl += v;
        }
        const int total = __shfl_sync(0xffffffffu, excl, 31);
        excl -= cnt;
        if (nb + total > kProjTidBuf) {
            // drain the buffer first: one transaction per lane
            __syncwarp();
            for (int q = lane; q < nb; q += 32)
                thread_transaction(tb[q], red_off, red_items, keys, vals, row_first, nr, nc, smem_acc, acc, out);
            __syncwarp();
            nb = 0;
        }
        if (total > kProjTidBuf) {
            // a stripe with more transactions than the buffer holds: each lane its own word
            while (m) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                thread_transaction(w * 32 + b, red_off, red_items, keys, vals, row_first, nr, nc, smem_acc, acc, out);
            }
            __syncwarp();
            continue;
        }
        int pos = nb + excl;
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            tb[pos++] = (int32_t)(w * 32 + b);
        }
        nb += total;
        __syncwarp();
    }
    __syncwarp();
    for (int q = lane; q < nb; q += 32)
        thread_transaction(tb[q], red_off, red_items, keys, vals, row_first, nr, nc, smem_acc, acc, out);
    __syncthreads();
    if (smem_acc)
        for (int q = threadIdx.x; q < nr * nc; q += blockDim.x) out[q] = acc[q];
    __syncthreads();   // the block's next job reuses the tables
}

__global__ void __launch_bounds__(kProjWarps * 32) k_count_proj(CountArgs a, const int32_t* __restrict__ job_ids,
                                                                const int64_t* __restrict__ red_off,
                                                                const int32_t* __restrict__ red_items) {
    __shared__ ProjShared sh;
    phase_begin(a.ph_s);
    proj_job(a, job_ids[blockIdx.x], red_off, red_items, sh);
    phase_end(a.ph_e);
}

__global__ void __launch_bounds__(kProjWarps * 32) k_count_proj_persistent(const CountArgs* __restrict__ args,
                                                                           const int32_t* n_jobs,
                                                                           const int64_t* __restrict__ red_off,
                                                                           const int32_t* __restrict__ red_items) {
    __shared__ ProjShared sh;
    const CountArgs a = *args;
    const int32_t n = *n_jobs;
    phase_begin(a.ph_s);
    for (int32_t q = blockIdx.x; q < n; q += gridDim.x) proj_job(a, a.job_list[q], red_off, red_items, sh);
    phase_end(a.ph_e);
}

}  // namespace

int occupancy_proj(int* blocks) {
    TFIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_count_proj_persistent, kProjWarps * 32, 0));
    return TFIM_OK;
}

int launch_count_proj_persistent(const CountArgs* d_args, const int32_t* d_n_jobs, int32_t grid, const int64_t* red_off,
                                 const int32_t* red_items, cudaStream_t s) {
    k_count_proj_persistent<<<grid, kProjWarps * 32, 0, s>>>(d_args, d_n_jobs, red_off, red_items);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_count_proj(const CountArgs& a, const int32_t* job_ids, int32_t n_jobs, const int64_t* red_off,
                      const int32_t* red_items, cudaStream_t s) {
    if (n_jobs <= 0) return TFIM_OK;
    k_count_proj<<<n_jobs, kProjWarps * 32, 0, s>>>(a, job_ids, red_off, red_items);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

}  // namespace tfim
