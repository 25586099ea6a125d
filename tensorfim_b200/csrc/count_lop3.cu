// CUDA-core support counting: AND + popc over 128-bit vector loads.
//
// Arithmetic of the reference counters getResFrequency / getResFrequencyCudaKernel
// (code/engine/src/kernel_bitmap.cu:390-442) and maskBuildKernelFast
// (code/engine/src/kernel_bmma.cu:619-634): a support is popc(prefix mask & item row)
// summed over the transaction words.  The layout differs: one tile stages up to
// kLop3Rows prefix rows of a word chunk in shared memory once, then streams each column
// row through all of them, so a column word is read from HBM once per tile instead of
// once per (node, item) pair, and partial sums over word chunks meet in an int32 atomic.
#include "tfim_internal.h"

namespace tfim {
namespace {

__device__ __forceinline__ uint4 and4(uint4 a, uint4 b) { return make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w); }
__device__ __forceinline__ uint32_t popc4(uint4 a) { return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w); }

// Block: 256 threads.  Shared memory: kLop3Rows x kLop3Chunk words.  A tile may span
// any word range; it is processed kLop3Chunk words at a time.
__global__ void __launch_bounds__(256) k_count_lop3(CountArgs a) {
    extern __shared__ uint4 sm4[];
    __shared__ const uint4* rsrc[kLop3Rows][2];
    const TileDesc t = a.tiles[blockIdx.x];
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    if (threadIdx.x < kLop3Rows && (int)threadIdx.x < t.nr) {
        const RowDesc rd = a.rows[j.row_off + t.r0 + threadIdx.x];
        rsrc[threadIdx.x][0] = rd.slot >= 0 ? reinterpret_cast<const uint4*>(a.masks + (int64_t)rd.slot * W) : nullptr;
        rsrc[threadIdx.x][1] = rd.item >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)rd.item * W) : nullptr;
    }
    const uint4* base_m = j.base_slot >= 0 ? reinterpret_cast<const uint4*>(a.masks + (int64_t)j.base_slot * W) : nullptr;
    const uint4* base_i = j.base_item >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)j.base_item * W) : nullptr;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int cw = t.w0; cw < t.w1; cw += kLop3Chunk) {
        const int w4b = cw >> 2;
        const int nw4 = (min(t.w1, cw + kLop3Chunk) - cw) >> 2;
        __syncthreads();   // rsrc visible; previous chunk's readers done
        // 1. stage the tile's row masks for this word chunk
        for (int r = 0; r < t.nr; r++) {
            const uint4* rs = rsrc[r][0];
            const uint4* ri = rsrc[r][1];
            for (int w = threadIdx.x; w < nw4; w += blockDim.x) {
                uint4 m = make_uint4(~0u, ~0u, ~0u, ~0u);
                if (base_m) m = and4(m, __ldg(base_m + w4b + w));
                if (base_i) m = and4(m, __ldg(base_i + w4b + w));
                if (rs) m = and4(m, __ldg(rs + w4b + w));
                if (ri) m = and4(m, __ldg(ri + w4b + w));
                sm4[r * nw4 + w] = m;
            }
        }
        __syncthreads();
        // 2. one warp per column: stream the column row through every staged row
        for (int c = t.c0 + warp; c < t.c1; c += 8) {
            const int32_t col = c == j.self_col ? -1 : a.cols[j.col_off + c];
            const uint4* cp = col >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)col * W) + w4b : nullptr;
            uint32_t acc[kLop3Rows];
#pragma unroll
            for (int r = 0; r < kLop3Rows; r++) acc[r] = 0;
            for (int w = lane; w < nw4; w += 32) {
                const uint4 v = cp ? __ldg(cp + w) : make_uint4(~0u, ~0u, ~0u, ~0u);
#pragma unroll
                for (int r = 0; r < kLop3Rows; r++)
                    if (r < t.nr) acc[r] += popc4(and4(sm4[r * nw4 + w], v));
            }
#pragma unroll
            for (int r = 0; r < kLop3Rows; r++) {
                if (r >= t.nr) break;
                uint32_t v = acc[r];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0 && v) atomicAdd(a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + c, (int32_t)v);
            }
        }
    }
}

// masks[dst] = (src >= 0 ? masks[src] : ~0) & AND of the listed item rows.
// grid = (word blocks, n descriptors)
__global__ void k_materialize(const uint32_t* __restrict__ B, int64_t W, uint32_t* __restrict__ masks,
                              const MatDesc* __restrict__ mats, const int32_t* __restrict__ items) {
    const MatDesc m = mats[blockIdx.y];
    const int64_t W4 = W >> 2;
    uint4* dst = reinterpret_cast<uint4*>(masks + (int64_t)m.dst * W);
    const uint4* src = m.src >= 0 ? reinterpret_cast<const uint4*>(masks + (int64_t)m.src * W) : nullptr;
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < W4; w += (int64_t)gridDim.x * blockDim.x) {
        uint4 v = src ? src[w] : make_uint4(~0u, ~0u, ~0u, ~0u);
        for (int q = 0; q < m.n; q++) v = and4(v, __ldg(reinterpret_cast<const uint4*>(B + (int64_t)items[m.off + q] * W) + w));
        dst[w] = v;
    }
}

// one warp per row
__global__ void k_nfreq(const int32_t* __restrict__ counts, int64_t n_rows, int32_t n_cols, int32_t min_count,
                        int32_t* __restrict__ nfreq) {
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= n_rows) return;
    const int32_t* row = counts + g * n_cols;
    int32_t c = 0;
    for (int e = lane; e < n_cols; e += 32) c += row[e] >= min_count;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if (lane == 0) nfreq[g] = c;
}

// one warp per job row: count the entries >= min_count, reserve space, then write them
__global__ void k_compact(const int32_t* __restrict__ counts, const JobDesc* __restrict__ jobs,
                          const int32_t* __restrict__ row_job, const int32_t* __restrict__ row_local, int64_t n_rows,
                          int32_t min_count, Entry* __restrict__ entries, int2* __restrict__ row_info,
                          int32_t* __restrict__ counter) {
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= n_rows) return;
    const JobDesc j = jobs[row_job[g]];
    const int32_t* row = counts + j.out_off + (int64_t)row_local[g] * j.n_cols;
    int32_t n = 0;
    for (int e = lane; e < j.n_cols; e += 32) n += row[e] >= min_count;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    int32_t start = 0;
    if (lane == 0 && n) start = atomicAdd(counter, n);
    start = __shfl_sync(0xffffffffu, start, 0);
    if (lane == 0) row_info[g] = make_int2(start, n);
    if (!n) return;
    int32_t pos = start;
    for (int e0 = 0; e0 < j.n_cols; e0 += 32) {
        const int e = e0 + lane;
        const int32_t v = e < j.n_cols ? row[e] : 0;
        const bool keep = e < j.n_cols && v >= min_count;
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int k = __popc(bal & ((1u << lane) - 1u));
            Entry en;
            en.col = e;
            en.count = v;
            entries[pos + k] = en;
        }
        pos += __popc(bal);
    }
}

}  // namespace

int launch_count_lop3(const CountArgs& a, cudaStream_t s) {
    if (a.n_tiles <= 0) return TFIM_OK;
    const size_t smem = (size_t)kLop3Rows * kLop3Chunk * 4;
    static bool configured = false;
    if (!configured) {
        TFIM_CUDA(cudaFuncSetAttribute(k_count_lop3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = true;
    }
    k_count_lop3<<<a.n_tiles, 256, smem, s>>>(a);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_materialize(const uint32_t* bitmap, int64_t W, uint32_t* masks, const MatDesc* mats, const int32_t* items,
                       int32_t n, cudaStream_t s) {
    if (n <= 0) return TFIM_OK;
    int64_t bx = (W / 4 + 255) / 256;
    if (bx > 64) bx = 64;
    dim3 grid((unsigned)bx, (unsigned)n);
    k_materialize<<<grid, 256, 0, s>>>(bitmap, W, masks, mats, items);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_nfreq(const int32_t* counts, int64_t n_rows, int32_t n_cols, int32_t min_count, int32_t* nfreq,
                 cudaStream_t s) {
    if (n_rows <= 0) return TFIM_OK;
    const int64_t threads = n_rows * 32;
    k_nfreq<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(counts, n_rows, n_cols, min_count, nfreq);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_compact(const int32_t* counts, const JobDesc* jobs, const int32_t* row_job, const int32_t* row_local,
                   int64_t n_rows, int32_t min_count, Entry* entries, int2* row_info, int32_t* counter,
                   cudaStream_t s) {
    if (n_rows <= 0) return TFIM_OK;
    const int64_t threads = n_rows * 32;
    k_compact<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(counts, jobs, row_job, row_local, n_rows, min_count,
                                                                 entries, row_info, counter);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

}  // namespace tfim
