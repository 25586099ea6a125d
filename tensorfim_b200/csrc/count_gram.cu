// CUDA-core counter for dense narrow family jobs: a register-tiled AND+popc Gram block.
//
// A family job counts popc(base & B[F[t]] & B[F[c]]) for its rows t (a run of F's entries)
// against every column c of F.  When the prefix is dense there is no zero word to skip, and
// the job is a small Gram block of X_c = base & B[F[c]] (at most kGramMaxCols columns).  The
// arithmetic is the reference's per-node count (code/engine/src/kernel_bitmap.cu:390-442:
// popc of ANDed bit rows summed over the transaction words); the schedule is a GEMM's:
//   * a tile is one job over a word slice; a CTA of 128 threads stages the job's column rows
//     and its base for a chunk of 32 to 256 128-bit positions (fewer rows, more positions) in
//     shared memory with cp.async, rows padded by 16 bytes, double-buffered (the next chunk's
//     copies run during this chunk's popc); the base is ANDed into the row operands;
//   * each thread owns a block of 16 (row, column) pairs -- 4 x 4, or 2 x 8 / 1 x 16 for tails
//     of 2 / 1 rows -- and a subset of the chunk's positions: per position 8 to 17 shared loads
//     of 16 bytes feed 64 popc, so the POPC pipe (16 per SM and clock) bounds it rather than
//     loads or staging;
//   * at the end of the tile the threads of a block add their sums in shared memory and one
//     thread adds each pair's count to the job's output (word slices of one job meet there).
// Measured on one B200 (one job, 4.2 Mbit rows, CUDA events): 86-91% of the POPC ceiling at
// 32 and 64 columns.
#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kGThreads = 128;
// staged rows: the job's columns, then the base's one or two sources
__host__ __device__ __forceinline__ int gram_rows(int nF, int nbase) { return nF + nbase; }
// positions (128-bit words) per chunk by the rows staged: about 2,048 staged words
__host__ __device__ __forceinline__ int gram_positions(int rows) {
    return rows <= 8 ? 256 : rows <= 16 ? 128 : rows <= 32 ? 64 : 32;
}
// one chunk of every staged row (a pair block at the edge reads its rows and columns clamped
// to the last column, and its results there are discarded); after the last chunk the first
// buffer holds the blocks' sums
constexpr int kGBuf = (kGramMaxCols + 2) * (32 * 16 + 16);
static_assert(8 * (256 * 16 + 16) <= kGBuf && 16 * (128 * 16 + 16) <= kGBuf && 32 * (64 * 16 + 16) <= kGBuf,
              "every chunk shape fits a buffer");
static_assert(kGThreads * 16 * 4 <= kGBuf, "the blocks' sums fit a buffer");
constexpr int kGSmem = 2 * kGBuf;

__device__ __forceinline__ uint32_t popc4and(uint4 a, uint4 b) {
    return __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
}
__device__ __forceinline__ uint4 and4g(uint4 a, uint4 b) { return make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Pair blocks of BR rows x BC columns (BR * BC = 16): a tail of 1 or 2 rows takes 1 x 16 or
// 2 x 8 blocks, longer tails 4 x 4, so few pairs of a block fall outside the job.
template <int BR>
__device__ void gram_tile_t(const CountArgs& a, const TileDesc t, uint8_t* smem, const uint32_t** rowp) {
    constexpr int BC = 16 / BR;
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x;
    const int nF = t.c1, nr = t.nr, s0 = t.pad;
    const int nbase = (j.base_slot >= 0 ? 1 : 0) + (j.base_item >= 0 ? 1 : 0);
    const int rows = gram_rows(nF, nbase);
    const int P = gram_positions(rows);
    const int stride = P * 16 + 16;
    // the staged rows' sources (shared: the columns, then the base's)
    for (int q = tid; q < rows; q += kGThreads) {
        const uint32_t* src;
        if (q < nF) src = a.bitmap + (int64_t)a.cols[j.col_off + q] * W;
        else if (q == nF && j.base_slot >= 0) src = a.masks + (int64_t)j.base_slot * W;
        else src = a.bitmap + (int64_t)j.base_item * W;
        rowp[q] = src;
    }
    __syncthreads();
    // pair blocks; G threads per block share its positions (G need not be a power of two)
    const int rb = (nr + BR - 1) / BR, cb = (nF + BC - 1) / BC, nb = rb * cb;   // nb <= kGThreads
    const int G = min(P, kGThreads / nb);
    const int b = tid / G, g = tid - b * G;
    const bool busy = b < nb;
    const int br = busy ? (b / cb) * BR : 0, bc = busy ? (b % cb) * BC : 0;
    uint32_t acc[BR][BC];
#pragma unroll
    for (int x = 0; x < BR; x++)
#pragma unroll
        for (int y = 0; y < BC; y++) acc[x][y] = 0;
    // byte offsets of the block's rows and columns within a staged chunk, clamped to the last
    // column (pairs outside the job are computed on valid rows and discarded)
    int rofs[BR], cofs[BC];
#pragma unroll
    for (int x = 0; x < BR; x++) rofs[x] = min(s0 + br + x, nF - 1) * stride;
#pragma unroll
    for (int y = 0; y < BC; y++) cofs[y] = min(bc + y, nF - 1) * stride;
    const int b0 = nF * stride, b1 = (nF + (nbase > 1 ? 1 : 0)) * stride;   // base rows

    const int64_t P0 = t.w0 >> 2, P1 = t.w1 >> 2;   // 128-bit positions of the slice
    const int n_ch = (int)((P1 - P0 + P - 1) / P);
    // chunk ch into buffer ch & 1: unit u = (row u / P, position u % P), 16 bytes each
    auto stage = [&](int ch) {
        if (ch < n_ch) {
            uint8_t* buf = smem + (ch & 1) * kGBuf;
            const int64_t c0 = P0 + (int64_t)ch * P;
            for (int u = tid; u < rows * P; u += kGThreads) {
                const int q = u / P, p = u - q * P;
                if (c0 + p < P1) cp_async16(buf + q * stride + p * 16, reinterpret_cast<const uint4*>(rowp[q]) + c0 + p);
            }
        }
        cp_async_commit();
    };
    stage(0);
    for (int ch = 0; ch < n_ch; ch++) {
        stage(ch + 1);           // the next chunk's copies run during this chunk's popc
        cp_async_wait<1>();      // this thread's copies of chunk ch have landed
        __syncthreads();         // ... and every thread's
        const uint8_t* buf = smem + (ch & 1) * kGBuf;
        const int64_t rem_p = P1 - (P0 + (int64_t)ch * P);
        const int np = rem_p < P ? (int)rem_p : P;
        if (busy) {
            for (int p = g; p < np; p += G) {
                const uint8_t* bp = buf + p * 16;
                uint4 base = make_uint4(~0u, ~0u, ~0u, ~0u);
                if (nbase > 0) base = *reinterpret_cast<const uint4*>(bp + b0);
                if (nbase > 1) base = and4g(base, *reinterpret_cast<const uint4*>(bp + b1));
                uint4 xr[BR], xc[BC];
#pragma unroll
                for (int x = 0; x < BR; x++) xr[x] = and4g(*reinterpret_cast<const uint4*>(bp + rofs[x]), base);
#pragma unroll
                for (int y = 0; y < BC; y++) xc[y] = *reinterpret_cast<const uint4*>(bp + cofs[y]);
#pragma unroll
                for (int x = 0; x < BR; x++)
#pragma unroll
                    for (int y = 0; y < BC; y++) acc[x][y] += popc4and(xr[x], xc[y]);
            }
        }
        __syncthreads();         // buffer ch & 1 is staged again two chunks on
    }
    cp_async_wait<0>();
    // sums over the G threads of each block in shared memory (the first buffer, free now),
    // then one atomic per pair
    int32_t* sums = reinterpret_cast<int32_t*>(smem);
    for (int q = tid; q < kGThreads * 16; q += kGThreads) sums[q] = 0;
    __syncthreads();
    if (busy) {
#pragma unroll
        for (int x = 0; x < BR; x++)
#pragma unroll
            for (int y = 0; y < BC; y++)
                if (acc[x][y]) atomicAdd(&sums[b * 16 + x * BC + y], (int32_t)acc[x][y]);
    }
    __syncthreads();
    for (int q = tid; q < nb * 16; q += kGThreads) {
        const int bb = q >> 4, x = (q & 15) / BC, y = (q & 15) % BC;
        const int r = (bb / cb) * BR + x, c = (bb % cb) * BC + y;
        const int32_t v = sums[q];
        if (r < nr && c < nF && v) atomicAdd(a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + c, v);
    }
    __syncthreads();   // the block's next tile reuses the buffers and the row table
}

__device__ __forceinline__ void gram_tile(const CountArgs& a, const TileDesc t, uint8_t* smem, const uint32_t** rowp) {
    if (t.nr <= 1) gram_tile_t<1>(a, t, smem, rowp);
    else if (t.nr <= 2) gram_tile_t<2>(a, t, smem, rowp);
    else gram_tile_t<4>(a, t, smem, rowp);
}

__global__ void __launch_bounds__(kGThreads, 3) k_count_gram(CountArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ const uint32_t* rowp[kGramMaxCols + 2];
    phase_begin(a.ph_s);
    gram_tile(a, a.tiles[blockIdx.x], smem, rowp);
    phase_end(a.ph_e);
}

// Persistent form: arguments and tile count from device memory, tiles from `next`.
__global__ void __launch_bounds__(kGThreads, 3) k_count_gram_persistent(const CountArgs* __restrict__ args,
                                                                        const int32_t* n_tiles, int32_t* next) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ const uint32_t* rowp[kGramMaxCols + 2];
    __shared__ int32_t s_t;
    const CountArgs a = *args;
    const int32_t n = *n_tiles;
    phase_begin(a.ph_s);
    while (true) {
        if (threadIdx.x == 0) s_t = atomicAdd(next, 1);
        __syncthreads();
        const int32_t t = s_t;
        __syncthreads();
        if (t >= n) break;
        gram_tile(a, a.tiles[t], smem, rowp);
    }
    phase_end(a.ph_e);
}

}  // namespace

int configure_gram_kernel() {
    static std::atomic<bool> configured[64];
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !configured[dev].load()) {
        TFIM_CUDA(cudaFuncSetAttribute(k_count_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
        TFIM_CUDA(cudaFuncSetAttribute(k_count_gram_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
        configured[dev].store(true);
    }
    return TFIM_OK;
}

int occupancy_gram(int* blocks) {
    TFIM_TRY(configure_gram_kernel());
    TFIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_count_gram_persistent, kGThreads, kGSmem));
    return TFIM_OK;
}

int launch_count_gram(const CountArgs& a, cudaStream_t s) {
    if (a.n_tiles <= 0) return TFIM_OK;
    TFIM_TRY(configure_gram_kernel());
    k_count_gram<<<a.n_tiles, kGThreads, kGSmem, s>>>(a);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_count_gram_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                                 cudaStream_t s) {
    TFIM_TRY(configure_gram_kernel());
    k_count_gram_persistent<<<grid, kGThreads, kGSmem, s>>>(d_args, d_n_tiles, d_next);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

}  // namespace tfim
