// Counting for the family of the empty prefix: the co-occurrence matrix of the frequent
// items, M[i][j] = sup({F[i], F[j]}).
//
// The reference counts these supports as the root nodes' rows of resFrequency
// (code/engine/src/kernel_bitmap.cu:390-408, one popc(bv[r] & bv[e]) per pair).  On a
// sparse database most of those bitmap words are zero, so this path reads the
// frequency-compacted transaction list instead (each reduced row holds only surviving
// items, as dense ids) and adds one for every pair of frequent items that a row holds:
// sum over rows of len^2/2 increments instead of d^2 x N/2 bit operations.  The engine
// picks it per database from those two work estimates.  Counts are exact integers either
// way.
#include <algorithm>

#include "tfim_internal.h"

namespace tfim {
namespace {

// Offset of row i of the packed triangle, less i + 1: pair (i, j) sits at tri_row(i) + j.
__device__ __forceinline__ int64_t tri_row(int32_t i, int32_t nF) {
    return (int64_t)i * (2 * (int64_t)nF - i - 1) / 2 - i - 1;
}

constexpr int kPairThreads = 256;
constexpr int kPairRow = 32;   // frequent items of a reduced row held in shared memory

// One thread per reduced row: every pair (a, b) of items of the row that are in F adds 1
// to the packed upper triangle T at (min(pos), max(pos)).  The triangle is half the square
// (76 MB at 6,162 items against 152 MB), so the scattered increments stay in L2.  A thread
// first gathers the row's positions in F into its own column of shared memory (at most
// kPairRow; a longer row takes the direct loop) and sorts them, so each pair costs one
// shared-memory read and one fire-and-forget add.
__global__ void __launch_bounds__(kPairThreads) k_pair_count(const int64_t* __restrict__ red_off,
                                                            const int32_t* __restrict__ red_items, int64_t n_red,
                                                            const int32_t* __restrict__ pos, int32_t nF,
                                                            int32_t* __restrict__ T) {
    __shared__ int32_t buf[kPairRow * kPairThreads];
    int32_t* my = buf + threadIdx.x;   // element k at my[k * kPairThreads]
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_red; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = red_off[r], e = red_off[r + 1];
        int n = 0;
        bool spill = false;
        for (int64_t x = b; x < e; x++) {
            const int32_t p = __ldg(pos + __ldg(red_items + x));
            if (p < 0) continue;
            if (n == kPairRow) { spill = true; break; }
            // insertion into the sorted column
            int k = n++;
            while (k > 0 && my[(k - 1) * kPairThreads] > p) {
                my[k * kPairThreads] = my[(k - 1) * kPairThreads];
                k--;
            }
            my[k * kPairThreads] = p;
        }
        if (!spill) {
            for (int a = 0; a + 1 < n; a++) {
                const int32_t i = my[a * kPairThreads];
                int32_t* row = T + tri_row(i, nF);
                for (int c = a + 1; c < n; c++) {
                    const int32_t j = my[c * kPairThreads];
                    if (j > i) atomicAdd(row + j, 1);
                }
            }
            continue;
        }
        for (int64_t x = b; x < e; x++) {
            const int32_t pa = __ldg(pos + red_items[x]);
            if (pa < 0) continue;
            for (int64_t y = x + 1; y < e; y++) {
                const int32_t pb = __ldg(pos + red_items[y]);
                if (pb < 0 || pb == pa) continue;
                const int32_t i = min(pa, pb), j = max(pa, pb);
                atomicAdd(T + tri_row(i, nF) + j, 1);
            }
        }
    }
}

// The full matrix from the packed triangle: M[r][c] = T(min, max) off the diagonal and
// M[r][r] = diag[r].  Block (bi, bj), bj <= bi, loads the upper tile (bj, bi) from T (rows
// contiguous in T), writes it to M directly and, transposed through shared memory, to the
// lower tile (bi, bj), so every write is coalesced and every entry of M is written once.
__global__ void __launch_bounds__(256) k_mirror_tri(const int32_t* __restrict__ T, int32_t* __restrict__ M, int32_t nF,
                                                    const int32_t* __restrict__ diag) {
    __shared__ int32_t tile[32][33];
    const int32_t bi = blockIdx.x, bj = blockIdx.y;
    if (bj > bi) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
    for (int k = ty; k < 32; k += 8) {
        const int64_t r = (int64_t)bj * 32 + k, c = (int64_t)bi * 32 + tx;   // upper tile
        int32_t v = 0;
        if (r < nF && c < nF) {
            if (r < c) v = T[tri_row((int32_t)r, nF) + c];
            else if (r == c) v = diag ? diag[r] : 0;
            if (r <= c) M[r * nF + c] = v;
        }
        tile[k][tx] = v;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int64_t r = (int64_t)bi * 32 + k, c = (int64_t)bj * 32 + tx;   // lower tile
        if (r < nF && c < nF && c < r) M[r * nF + c] = tile[tx][k];
    }
}

// M[j][i] = M[i][j] for i < j; M[i][i] = diag[i] (when given).  One 32 x 32 tile per block,
// transposed through shared memory so that both the upper-triangle reads and the
// lower-triangle writes are coalesced.  Blocks read only entries above the diagonal and
// write only entries on or below it, so no block reads what another writes.
__global__ void __launch_bounds__(256) k_mirror(int32_t* __restrict__ M, int32_t nF, const int32_t* __restrict__ diag) {
    __shared__ int32_t tile[32][33];
    const int32_t bi = blockIdx.x, bj = blockIdx.y;   // destination rows bi, columns bj
    if (bj > bi) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
    for (int k = ty; k < 32; k += 8) {
        const int64_t r = (int64_t)bj * 32 + k, c = (int64_t)bi * 32 + tx;   // source: upper triangle
        tile[k][tx] = r < nF && c < nF && r < c ? M[r * nF + c] : 0;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int64_t r = (int64_t)bi * 32 + k, c = (int64_t)bj * 32 + tx;
        if (r >= nF || c >= nF) continue;
        if (c < r) M[r * nF + c] = tile[tx][k];
        else if (c == r && diag) M[r * nF + c] = diag[r];
    }
}

}  // namespace

int64_t pair_triangle_entries(int32_t nF) { return nF > 1 ? (int64_t)nF * (nF - 1) / 2 : 0; }

int launch_pair_count(const int64_t* red_off, const int32_t* red_items, int64_t n_red, const int32_t* pos, int32_t nF,
                      int32_t* T, cudaStream_t s) {
    if (n_red <= 0 || nF <= 1) return TFIM_OK;
    int sms = 148, dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    TFIM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int per_sm = 0;
    TFIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_count, kPairThreads, 0));
    int64_t blocks = (n_red + kPairThreads - 1) / kPairThreads;
    if (blocks > (int64_t)sms * std::max(per_sm, 1)) blocks = (int64_t)sms * std::max(per_sm, 1);
    k_pair_count<<<(unsigned)blocks, kPairThreads, 0, s>>>(red_off, red_items, n_red, pos, nF, T);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_mirror_tri(const int32_t* T, int32_t* M, int32_t nF, const int32_t* diag, cudaStream_t s) {
    if (nF <= 0) return TFIM_OK;
    const unsigned nb = (unsigned)((nF + 31) / 32);
    TFIM_CHECK(nb <= 65535, TFIM_E_INVALID, "family of %d items exceeds the mirror grid", nF);
    k_mirror_tri<<<dim3(nb, nb), 256, 0, s>>>(T, M, nF, diag);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_mirror(int32_t* M, int32_t nF, const int32_t* diag, cudaStream_t s) {
    if (nF <= 0) return TFIM_OK;
    const unsigned nb = (unsigned)((nF + 31) / 32);
    TFIM_CHECK(nb <= 65535, TFIM_E_INVALID, "family of %d items exceeds the mirror grid", nF);
    k_mirror<<<dim3(nb, nb), 256, 0, s>>>(M, nF, diag);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

}  // namespace tfim
