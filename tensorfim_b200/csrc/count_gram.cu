// CUDA-core counter for dense narrow family jobs: a register-tiled AND+popc Gram block.
//
// A family job counts popc(base & B[F[t]] & B[F[c]]) for its rows t (a run of F's entries)
// against every column c of F.  When the prefix is dense there is no zero word to skip, and
// the job is a small Gram block of X_c = base & B[F[c]] (at most kGramMaxCols columns).  The
// arithmetic is the reference's per-node count (code/engine/src/kernel_bitmap.cu:390-442:
// popc of ANDed bit rows summed over the transaction words); the schedule is a GEMM's:
//   * a tile is one job over a word slice; a CTA of 128 threads stages X for a chunk of 32 to
//     256 128-bit positions (fewer columns, more positions) in shared memory, rows padded by
//     16 bytes, double-buffered, while the next chunk's words are loaded into registers;
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
constexpr int kGUnits = 16;                            // staged words per thread and chunk
// positions (128-bit words) per chunk by the family's width: kGUnits * kGThreads words of
// staging, every column of the chunk
__host__ __device__ __forceinline__ int gram_positions(int nF) {
    return nF <= 8 ? 256 : nF <= 16 ? 128 : nF <= 32 ? 64 : 32;
}
// one chunk of every column (a pair block at the edge reads its rows and columns clamped to
// the last column, and its results there are discarded)
constexpr int kGBuf = 64 * (32 * 16 + 16);
static_assert(8 * (256 * 16 + 16) <= kGBuf && 16 * (128 * 16 + 16) <= kGBuf && 32 * (64 * 16 + 16) <= kGBuf,
              "every chunk shape fits a buffer");
constexpr int kGSmem = 2 * kGBuf + kGThreads * 16 * 4;   // two buffers + the final sums

__device__ __forceinline__ uint32_t popc4and(uint4 a, uint4 b) {
    return __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
}

// Pair blocks of BR rows x BC columns (BR * BC = 16): a tail of 1 or 2 rows takes 1 x 16 or
// 2 x 8 blocks, longer tails 4 x 4, so few pairs of a block fall outside the job.
template <int BR>
__device__ void gram_tile_t(const CountArgs& a, const TileDesc t, uint8_t* smem) {
    constexpr int BC = 16 / BR;
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x;
    const int nF = t.c1, nr = t.nr, s0 = t.pad;
    const int P = gram_positions(nF);
    const int stride = P * 16 + 16;
    const uint32_t* bm = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
    const uint32_t* bi = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
    // staged unit u = tid + kGThreads * k: column u / P, position u % P (at most 2 positions
    // per thread, at 256 positions)
    const uint32_t* src[kGUnits];
    int ucol[kGUnits], upos[kGUnits];
#pragma unroll
    for (int k = 0; k < kGUnits; k++) {
        const int u = tid + kGThreads * k;
        ucol[k] = u / P;
        upos[k] = u % P;
        src[k] = ucol[k] < nF ? a.bitmap + (int64_t)a.cols[j.col_off + ucol[k]] * W : nullptr;
    }
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
    // byte offsets of the block's rows and columns within a staged chunk, clamped to the
    // last column (pairs outside the job are computed on valid rows and discarded)
    int rofs[BR], cofs[BC];
#pragma unroll
    for (int x = 0; x < BR; x++) rofs[x] = min(s0 + br + x, nF - 1) * stride;
#pragma unroll
    for (int y = 0; y < BC; y++) cofs[y] = min(bc + y, nF - 1) * stride;
    int32_t* sums = reinterpret_cast<int32_t*>(smem + 2 * kGBuf);   // (row, column) -> sum
    for (int q = tid; q < kGThreads * 16; q += kGThreads) sums[q] = 0;

    const int64_t P0 = t.w0 >> 2, P1 = t.w1 >> 2;   // 128-bit positions of the slice
    const int n_ch = (int)((P1 - P0 + P - 1) / P);
    uint4 pre[kGUnits];
    uint4 pb0 = make_uint4(~0u, ~0u, ~0u, ~0u), pb1 = pb0;   // base words of this thread's positions
    const int pa = upos[0], pbp = upos[kGUnits - 1];         // its (at most) two positions
    auto base_at = [&](int64_t p) {
        uint4 x = make_uint4(~0u, ~0u, ~0u, ~0u);
        if (bm) x = __ldg(reinterpret_cast<const uint4*>(bm) + p);
        if (bi) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(bi) + p);
            x = make_uint4(x.x & v.x, x.y & v.y, x.z & v.z, x.w & v.w);
        }
        return x;
    };
    auto load = [&](int ch) {
        const int64_t c0 = P0 + (int64_t)ch * P;
        if (ch < n_ch && c0 + pa < P1) pb0 = base_at(c0 + pa);
        if (ch < n_ch && c0 + pbp < P1 && pbp != pa) pb1 = base_at(c0 + pbp);
#pragma unroll
        for (int k = 0; k < kGUnits; k++) {
            const int64_t p = c0 + upos[k];
            pre[k] = (ch < n_ch && src[k] && p < P1) ? __ldg(reinterpret_cast<const uint4*>(src[k]) + p)
                                                     : make_uint4(0, 0, 0, 0);
        }
    };
    load(0);
    for (int ch = 0; ch < n_ch; ch++) {
        uint8_t* buf = smem + (ch & 1) * kGBuf;
#pragma unroll
        for (int k = 0; k < kGUnits; k++)
            if (ucol[k] < nF) {
                const uint4 v = pre[k];
                const uint4 bw = upos[k] == pa ? pb0 : pb1;
                *reinterpret_cast<uint4*>(buf + ucol[k] * stride + upos[k] * 16) =
                    make_uint4(v.x & bw.x, v.y & bw.y, v.z & bw.z, v.w & bw.w);
            }
        __syncthreads();
        if (ch + 1 < n_ch) load(ch + 1);   // in flight during this chunk's popc
        const int64_t rem_p = P1 - (P0 + (int64_t)ch * P);
        const int np = rem_p < P ? (int)rem_p : P;
        if (busy) {
            for (int p = g; p < np; p += G) {
                uint4 xr[BR], xc[BC];
#pragma unroll
                for (int x = 0; x < BR; x++) xr[x] = *reinterpret_cast<const uint4*>(buf + rofs[x] + p * 16);
#pragma unroll
                for (int y = 0; y < BC; y++) xc[y] = *reinterpret_cast<const uint4*>(buf + cofs[y] + p * 16);
#pragma unroll
                for (int x = 0; x < BR; x++)
#pragma unroll
                    for (int y = 0; y < BC; y++) acc[x][y] += popc4and(xr[x], xc[y]);
            }
        }
        // the next iteration writes the other buffer; the one after it, this one, only after
        // every thread passed the next iteration's barrier (and so finished this chunk)
    }
    // sums over the G threads of each block in shared memory, then one atomic per pair
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
    __syncthreads();   // the block's next tile reuses the buffers and the sums
}

__device__ __forceinline__ void gram_tile(const CountArgs& a, const TileDesc t, uint8_t* smem) {
    if (t.nr <= 1) gram_tile_t<1>(a, t, smem);
    else if (t.nr <= 2) gram_tile_t<2>(a, t, smem);
    else gram_tile_t<4>(a, t, smem);
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
