// CUDA-core counter for dense narrow family jobs: a register-tiled AND+popc Gram block.
//
// A family job counts popc(base & B[F[t]] & B[F[c]]) for its rows t (a run of F's entries)
// against every column c of F.  When the prefix is dense there is no zero word to skip, and
// the job is a small Gram block of X_c = base & B[F[c]] (at most kGramMaxCols columns).  The
// arithmetic is the reference's per-node count (code/engine/src/kernel_bitmap.cu:390-442:
// popc of ANDed bit rows summed over the transaction words); the schedule is a GEMM's:
//   * a tile is one job over a word slice; a CTA of 128 threads stages X for a chunk of 32
//     128-bit positions in shared memory (rows padded by 16 bytes), double-buffered, while
//     the next chunk's words are loaded into registers;
//   * each thread owns a 4 x 4 block of (row, column) pairs and a subset of the chunk's
//     positions: per position 8 shared loads of 16 bytes feed 64 popc, so the POPC pipe (16
//     per SM and clock) bounds it rather than loads or staging;
//   * at the end of the tile the threads of a block reduce their sums with shuffles and one
//     lane adds each pair's count to the job's output (word slices of one job meet there).
#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kGThreads = 128;
constexpr int kGPos = 32;                              // 128-bit positions per chunk
constexpr int kGRowStride = kGPos * 16 + 16;           // bytes per staged row (padded)
// one chunk of every column, plus 4 rows: a 4 x 4 pair block at the edge reads rows up to
// nF + 2 (its results are discarded), which stays inside the buffer
constexpr int kGBuf = (kGramMaxCols + 4) * kGRowStride;
constexpr int kGSmem = 2 * kGBuf;
constexpr int kGUnits = kGramMaxCols * kGPos / kGThreads;   // staged words per thread and chunk (16)

__device__ __forceinline__ uint32_t popc4and(uint4 a, uint4 b) {
    return __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
}

__device__ void gram_tile(const CountArgs& a, const TileDesc t, uint8_t* smem) {
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x;
    const int nF = t.c1, nr = t.nr, s0 = t.pad;
    const uint32_t* bm = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
    const uint32_t* bi = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
    // this thread's staged units: position p (fixed), columns c = tid / 32 + 4 * u
    const int p_ld = tid & (kGPos - 1), c_ld0 = tid >> 5;
    const int n_ld = (nF - c_ld0 + 3) >> 2;   // <= kGUnits
    const uint32_t* src[kGUnits];
#pragma unroll
    for (int u = 0; u < kGUnits; u++)
        src[u] = u < n_ld ? a.bitmap + (int64_t)a.cols[j.col_off + c_ld0 + 4 * u] * W : nullptr;
    // pair blocks of 4 rows x 4 columns; G threads per block share its positions
    const int rb = (nr + 3) >> 2, cb = (nF + 3) >> 2, nb = rb * cb;   // nb <= kGThreads
    int G = 1;
    while (G * 2 * nb <= kGThreads && G < kGPos) G *= 2;
    const int b = tid / G, g = tid % G;
    const bool busy = b < nb;
    const int br = busy ? (b / cb) * 4 : 0, bc = busy ? (b % cb) * 4 : 0;
    uint32_t acc[4][4];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = 0;

    const int64_t P0 = t.w0 >> 2, P1 = t.w1 >> 2;   // 128-bit positions of the slice
    const int n_ch = (int)((P1 - P0 + kGPos - 1) / kGPos);
    uint4 pre[kGUnits];
    uint4 pbase = make_uint4(~0u, ~0u, ~0u, ~0u);
    auto load = [&](int ch) {
        const int64_t p = P0 + (int64_t)ch * kGPos + p_ld;
        const bool in = ch < n_ch && p < P1;
        pbase = make_uint4(~0u, ~0u, ~0u, ~0u);
        if (in && bm) pbase = __ldg(reinterpret_cast<const uint4*>(bm) + p);
        if (in && bi) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(bi) + p);
            pbase = make_uint4(pbase.x & v.x, pbase.y & v.y, pbase.z & v.z, pbase.w & v.w);
        }
#pragma unroll
        for (int u = 0; u < kGUnits; u++)
            pre[u] = (in && u < n_ld) ? __ldg(reinterpret_cast<const uint4*>(src[u]) + p) : make_uint4(0, 0, 0, 0);
    };
    load(0);
    for (int ch = 0; ch < n_ch; ch++) {
        uint8_t* buf = smem + (ch & 1) * kGBuf;
#pragma unroll
        for (int u = 0; u < kGUnits; u++)
            if (u < n_ld) {
                const uint4 v = pre[u];
                *reinterpret_cast<uint4*>(buf + (c_ld0 + 4 * u) * kGRowStride + p_ld * 16) =
                    make_uint4(v.x & pbase.x, v.y & pbase.y, v.z & pbase.z, v.w & pbase.w);
            }
        __syncthreads();
        if (ch + 1 < n_ch) load(ch + 1);   // in flight during this chunk's popc
        const int64_t rem_p = P1 - (P0 + (int64_t)ch * kGPos);
        const int np = rem_p < kGPos ? (int)rem_p : kGPos;
        if (busy) {
            for (int p = g; p < np; p += G) {
                uint4 xr[4], xc[4];
#pragma unroll
                for (int x = 0; x < 4; x++) {
                    xr[x] = *reinterpret_cast<const uint4*>(buf + (s0 + br + x) * kGRowStride + p * 16);
                    xc[x] = *reinterpret_cast<const uint4*>(buf + (bc + x) * kGRowStride + p * 16);
                }
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] += popc4and(xr[x], xc[y]);
            }
        }
        // the next iteration writes the other buffer; the one after it, this one, only after
        // every thread passed the next iteration's barrier (and so finished this chunk)
    }
    // sums over the G threads of a block (consecutive lanes of one warp)
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++)
            for (int o = 1; o < G; o <<= 1) acc[x][y] += __shfl_xor_sync(0xffffffffu, acc[x][y], o);
    if (busy && g == 0) {
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) {
                const int r = br + x, c = bc + y;
                if (r < nr && c < nF && acc[x][y])
                    atomicAdd(a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + c, (int32_t)acc[x][y]);
            }
    }
    __syncthreads();   // the block's next tile reuses the buffers
}

__global__ void __launch_bounds__(kGThreads) k_count_gram(CountArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    phase_begin(a.ph_s);
    gram_tile(a, a.tiles[blockIdx.x], smem);
    phase_end(a.ph_e);
}

// Persistent form: arguments and tile count from device memory, tiles from `next`.
__global__ void __launch_bounds__(kGThreads) k_count_gram_persistent(const CountArgs* __restrict__ args,
                                                                     const int32_t* n_tiles, int32_t* next) {
    extern __shared__ __align__(16) uint8_t smem[];
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
        gram_tile(a, a.tiles[t], smem);
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
