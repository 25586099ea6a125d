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

// Every pair (a, b) of items of a reduced row that are in F adds 1 to M[min(pos)][max(pos)]
// (upper triangle; the diagonal is filled by the mirror pass).  A warp takes 32 consecutive
// rows: their offsets come in two coalesced loads, and each row's positions (rows of up to
// 32 items, one per lane) are requested while the previous row's pairs are added, so the
// offset -> item -> position load chain of a row overlaps the work of the one before.  The
// lanes pair lane x with lane x + d for d = 1, 2, ...; a row of more than 32 items pairs
// each lane's items with the rest of the row.  Measured on the 1M-row sparse workload (6,162
// frequent items, 37.2M increments): a warp per row without the overlap took 0.39 ms, a
// thread per row 0.44 ms, and the same increments into a packed upper triangle instead of
// the square matrix 0.62 ms.
__global__ void __launch_bounds__(256) k_pair_count(const int64_t* __restrict__ red_off,
                                                    const int32_t* __restrict__ red_items, int64_t n_red,
                                                    const int32_t* __restrict__ pos, int32_t nF,
                                                    int32_t* __restrict__ M) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t rb = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; rb < n_red;
         rb += warps * 32) {
        const int nrows = n_red - rb < 32 ? (int)(n_red - rb) : 32;
        const int64_t ob = lane <= nrows ? red_off[rb + lane] : 0;          // red_off holds n_red + 1
        const int64_t oe = lane < nrows ? red_off[rb + lane + 1] : 0;
        int64_t bn = __shfl_sync(0xffffffffu, ob, 0);
        int64_t ln = __shfl_sync(0xffffffffu, oe, 0) - bn;
        int32_t pn = ln <= 32 && lane < ln ? __ldg(pos + __ldg(red_items + bn + lane)) : -1;
        for (int j = 0; j < nrows; j++) {
            const int64_t b = bn, len = ln;
            const int32_t p = pn;
            if (j + 1 < nrows) {   // the next row's positions, in flight during this row's adds
                bn = __shfl_sync(0xffffffffu, ob, j + 1);
                ln = __shfl_sync(0xffffffffu, oe, j + 1) - bn;
                pn = ln <= 32 && lane < ln ? __ldg(pos + __ldg(red_items + bn + lane)) : -1;
            }
            if (len <= 32) {
                for (int d = 1; d < len; d++) {
                    const int32_t q = __shfl_down_sync(0xffffffffu, p, d);
                    if (lane + d < len && p >= 0 && q >= 0 && p != q)
                        atomicAdd(M + (int64_t)min(p, q) * nF + max(p, q), 1);
                }
                continue;
            }
            const int64_t e = b + len;
            for (int64_t x = b + lane; x < e; x += 32) {
                const int32_t pa = __ldg(pos + __ldg(red_items + x));
                if (pa < 0) continue;
                for (int64_t y = x + 1; y < e; y++) {
                    const int32_t pb = __ldg(pos + __ldg(red_items + y));
                    if (pb >= 0 && pb != pa) atomicAdd(M + (int64_t)min(pa, pb) * nF + max(pa, pb), 1);
                }
            }
        }
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

int launch_pair_count(const int64_t* red_off, const int32_t* red_items, int64_t n_red, const int32_t* pos, int32_t nF,
                      int32_t* M, cudaStream_t s) {
    if (n_red <= 0 || nF <= 1) return TFIM_OK;
    int sms = 148, dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    TFIM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int64_t blocks = (n_red + 255) / 256;   // 8 warps of 32 rows each
    if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
    k_pair_count<<<(unsigned)blocks, 256, 0, s>>>(red_off, red_items, n_red, pos, nF, M);
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
