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
#include "tfim_internal.h"

namespace tfim {
namespace {

// One thread per reduced row: every pair (a, b) of items of the row that are in F adds 1
// to M[min(pos)][max(pos)] (upper triangle; the diagonal is filled by the mirror pass).
__global__ void k_pair_count(const int64_t* __restrict__ red_off, const int32_t* __restrict__ red_items, int64_t n_red,
                             const int32_t* __restrict__ pos, int32_t nF, int32_t* __restrict__ M) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_red; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = red_off[r], e = red_off[r + 1];
        for (int64_t x = b; x < e; x++) {
            const int32_t pa = __ldg(pos + red_items[x]);
            if (pa < 0) continue;
            for (int64_t y = x + 1; y < e; y++) {
                const int32_t pb = __ldg(pos + red_items[y]);
                if (pb < 0) continue;
                const int32_t i = min(pa, pb), j = max(pa, pb);
                atomicAdd(M + (int64_t)i * nF + j, 1);
            }
        }
    }
}

// M[j][i] = M[i][j] for i < j; M[i][i] = diag[i].
__global__ void k_mirror(int32_t* __restrict__ M, int32_t nF, const int32_t* __restrict__ diag) {
    const int64_t n = (int64_t)nF * nF;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = (int32_t)(k / nF), j = (int32_t)(k % nF);
        if (j < i) M[k] = M[(int64_t)j * nF + i];
        else if (j == i && diag) M[k] = diag[i];
    }
}

}  // namespace

int launch_pair_count(const int64_t* red_off, const int32_t* red_items, int64_t n_red, const int32_t* pos, int32_t nF,
                      int32_t* M, cudaStream_t s) {
    if (n_red <= 0 || nF <= 0) return TFIM_OK;
    int64_t blocks = (n_red + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_pair_count<<<(unsigned)blocks, 256, 0, s>>>(red_off, red_items, n_red, pos, nF, M);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_mirror(int32_t* M, int32_t nF, const int32_t* diag, cudaStream_t s) {
    if (nF <= 0) return TFIM_OK;
    const int64_t n = (int64_t)nF * nF;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_mirror<<<(unsigned)blocks, 256, 0, s>>>(M, nF, diag);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

}  // namespace tfim
