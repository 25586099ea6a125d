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

// A tile is rows [r0, r0+nr) x columns [c0, c1) of one job over a word range.  Most of a
// prefix mask is zero, and the jobs of a sparse database are narrow (a few rows and
// columns), so the tile neither streams whole rows nor gives each column a warp.  Every
// warp works on its own 128-position (2048-bit) stripes, without block barriers:
//   (1) candidates: each lane tests 4 consecutive 128-bit positions of the base mask;
//   (2) rounds: each lane takes its next candidate, loads the tile's rows there and keeps
//       the position when any row survives the base; kept positions are compacted by
//       ballot into the warp's staging region with the masked row values;
//   (3) flush: lanes are spread over (staged position, column) pairs -- 32 / ncols
//       positions per pass -- gather the column words and accumulate
//       popc(staged row & column) in registers for the whole word range.
// The warps' partial sums meet in shared memory and one global atomic per (row, column)
// is issued per tile.  Row words are read only where the base is nonzero, column words
// only where a row of the tile survives.
constexpr int kL3Stage = 2048;   // staged 128-bit values (positions x rows), 32 KiB, 1/8 per warp
constexpr int kL3Pos = 1024;     // staged positions, 1/8 per warp
constexpr int kL3Step = 1024;    // positions per step (128 per warp, 4 per lane)

struct Lop3Shared {
    uint4 staged[kL3Stage];
    int32_t pos[kL3Pos];
    int32_t acc[kLop3Rows * 64];
    const uint4* rsrc[kLop3Rows][2];
};

__device__ __forceinline__ bool nonzero4(uint4 v) { return (v.x | v.y | v.z | v.w) != 0u; }

template <bool WIDE>
__device__ void lop3_tile_impl(const CountArgs& a, const TileDesc t, Lop3Shared& sh) {
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nr = t.nr;
    const int ncols = t.c1 - t.c0;
    if (tid < kLop3Rows && tid < nr) {
        const RowDesc rd = a.rows[j.row_off + t.r0 + tid];
        sh.rsrc[tid][0] = rd.slot >= 0 ? reinterpret_cast<const uint4*>(a.masks + (int64_t)rd.slot * W) : nullptr;
        sh.rsrc[tid][1] = rd.item >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)rd.item * W) : nullptr;
    }
    for (int q = tid; q < kLop3Rows * 64; q += blockDim.x) sh.acc[q] = 0;
    const uint4* base_m = j.base_slot >= 0 ? reinterpret_cast<const uint4*>(a.masks + (int64_t)j.base_slot * W) : nullptr;
    const uint4* base_i = j.base_item >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)j.base_item * W) : nullptr;
    // flush layout: G staged positions per pass, lane -> (position offset, column(s))
    constexpr bool wide = WIDE;
    constexpr int NC = WIDE ? 2 : 1;   // columns per lane
    const int G = wide ? 1 : 32 / ncols;
    const int koff = wide ? 0 : lane / ncols;
    const bool active = koff < G;
    const int cl[2] = {wide ? lane : lane % ncols, wide ? lane + 32 : -1};
    const uint4* cp[NC];
    int ck[NC];   // 0: column row, 1: all ones, 2: none
#pragma unroll
    for (int ci = 0; ci < NC; ci++) {
        const int c = t.c0 + cl[ci];
        ck[ci] = 2;
        cp[ci] = nullptr;
        if (cl[ci] >= 0 && cl[ci] < ncols && active) {
            const int32_t col = c == j.self_col ? -1 : a.cols[j.col_off + c];
            if (col < 0) ck[ci] = 1;   // the all-ones column
            else {
                ck[ci] = 0;
                cp[ci] = reinterpret_cast<const uint4*>(a.bitmap + (int64_t)col * W);
            }
        }
    }
    uint32_t acc[NC][kLop3Rows];
#pragma unroll
    for (int ci = 0; ci < NC; ci++)
#pragma unroll
        for (int r = 0; r < kLop3Rows; r++) acc[ci][r] = 0;
    __syncthreads();   // rsrc, acc
    uint4* wst = sh.staged + warp * (kL3Stage / 8);
    int32_t* wpos = sh.pos + warp * (kL3Pos / 8);
    const int wcap = min(kL3Pos / 8, (kL3Stage / 8) / nr);
    int ns = 0;   // staged positions of this warp (warp-uniform)

    // U staged positions per lane and pass: their column words are all requested before the
    // first is used, so a thin tile (one or two rows, each column word feeding one or two
    // popcounts) keeps several L2 reads in flight per lane instead of one.
    constexpr int U = WIDE ? 2 : 4;
    auto flush = [&]() {
        __syncwarp();
        for (int k0 = 0; k0 < ns; k0 += G * U) {
            uint4 v[U][NC];
            int kk[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int k = k0 + u * G + koff;
                kk[u] = active && k < ns ? k : -1;
                const int p = kk[u] >= 0 ? wpos[k] : 0;
#pragma unroll
                for (int ci = 0; ci < NC; ci++)
                    v[u][ci] = kk[u] < 0 || ck[ci] == 2 ? make_uint4(0, 0, 0, 0)
                               : ck[ci] == 0         ? __ldg(cp[ci] + p)
                                                     : make_uint4(~0u, ~0u, ~0u, ~0u);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (kk[u] < 0) continue;
                const uint4* st = wst + kk[u] * nr;
#pragma unroll
                for (int r = 0; r < kLop3Rows; r++) {
                    if (r >= nr) break;
                    const uint4 m = st[r];
#pragma unroll
                    for (int ci = 0; ci < NC; ci++) acc[ci][r] += popc4(and4(m, v[u][ci]));
                }
            }
        }
        __syncwarp();
        ns = 0;
    };
    auto base_at = [&](int64_t p) {
        uint4 x = make_uint4(~0u, ~0u, ~0u, ~0u);
        if (base_m) x = and4(x, __ldg(base_m + p));
        if (base_i) x = and4(x, __ldg(base_i + p));
        return x;
    };
    auto row_at = [&](int r, uint4 x, int64_t p) {
        const uint4* rs = sh.rsrc[r][0];
        const uint4* ri = sh.rsrc[r][1];
        if (rs) x = and4(x, __ldg(rs + p));
        if (ri) x = and4(x, __ldg(ri + p));
        return x;
    };

    const int64_t P0 = t.w0 >> 2, P1 = t.w1 >> 2;
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t s0 = P0 + warp * 128; s0 < P1; s0 += kL3Step) {
        // (1) candidates: nonzero base positions, 4 consecutive per lane
        const int64_t pl = s0 + 4 * lane;
        uint32_t valid = 0;
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (pl + q < P1 && nonzero4(base_at(pl + q))) valid |= 1u << q;
        // (2) rounds: each lane its next candidate.  The row words are read twice (to test,
        // then to stage); the second read hits L1.
        while (__any_sync(0xffffffffu, valid != 0)) {
            const int q_sel = valid ? __ffs(valid) - 1 : -1;
            valid &= valid - 1;
            const int64_t p = pl + q_sel;
            bool any = false;
            uint4 b = make_uint4(0, 0, 0, 0);
            if (q_sel >= 0) {
                b = base_at(p);
#pragma unroll
                for (int r = 0; r < kLop3Rows; r++)
                    if (r < nr) any |= nonzero4(row_at(r, b, p));
            }
            if (ns + 32 > wcap) flush();
            const unsigned bal = __ballot_sync(0xffffffffu, any);
            if (any) {
                const int k = ns + __popc(bal & lt);
                wpos[k] = (int32_t)p;
#pragma unroll
                for (int r = 0; r < kLop3Rows; r++)
                    if (r < nr) wst[k * nr + r] = row_at(r, b, p);
            }
            ns += __popc(bal);
        }
    }
    if (ns > 0) flush();
    // partial sums of the warps meet in shared memory; one global atomic per output
#pragma unroll
    for (int ci = 0; ci < NC; ci++)
#pragma unroll
        for (int r = 0; r < kLop3Rows; r++)
            if (r < nr && ck[ci] != 2 && acc[ci][r]) atomicAdd(&sh.acc[r * 64 + cl[ci]], (int32_t)acc[ci][r]);
    __syncthreads();
    for (int q = tid; q < nr * ncols; q += blockDim.x) {
        const int r = q / ncols, c = q - r * ncols;
        const int32_t v = sh.acc[r * 64 + c];
        if (v) atomicAdd(a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + t.c0 + c, v);
    }
    __syncthreads();   // shared state is reused by the block's next tile
}

// A tile of a dense family (flag bit 0 of TileDesc.pad, set by the resident pack when the
// prefix holds at least 1/16 of the transactions): no 128-bit position is zero there, so the
// skipping machinery above only costs L1 traffic (staged rows written and re-read, the base
// and rows read twice).  Instead every thread owns a block of BR rows x BC columns and a
// strided share of the slice's positions; per position it loads the base, its rows and its
// columns straight from L2 (16-byte loads, consecutive positions on consecutive lanes) and
// adds BR x BC popcounts held in registers -- (2 + BR + BC) loads per BR * BC popc4 instead of
// about 1 + nr per nr.  The G threads of a block meet in shared memory at the end, as above.
template <int BR>
__device__ void lop3_dense_impl(const CountArgs& a, const TileDesc t, int32_t* sacc) {
    constexpr int BC = BR == 1 ? 16 : BR == 2 ? 8 : BR == 3 ? 5 : 4;
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x;
    const int nr = t.nr, nc = t.c1 - t.c0;
    const int rb = (nr + BR - 1) / BR, cb = (nc + BC - 1) / BC, nb = rb * cb;   // at most 2 x 16
    const int G = blockDim.x / nb;
    const int b = tid / G, g = tid - b * G;
    const bool busy = b < nb;
    const int br = busy ? (b / cb) * BR : 0, bc = busy ? (b % cb) * BC : 0;
    for (int q = tid; q < kLop3Rows * 64; q += blockDim.x) sacc[q] = 0;
    const uint4* base_m = j.base_slot >= 0 ? reinterpret_cast<const uint4*>(a.masks + (int64_t)j.base_slot * W) : nullptr;
    const uint4* base_i = j.base_item >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)j.base_item * W) : nullptr;
    // sources of the block's rows and columns, clamped to the tile's last row / column (pairs
    // outside the tile are computed on valid rows and discarded); a null source is all ones
    const uint4* rsl[BR];
    const uint4* rit[BR];
    const uint4* csrc[BC];
#pragma unroll
    for (int x = 0; x < BR; x++) {
        const RowDesc rd = a.rows[j.row_off + t.r0 + min(br + x, nr - 1)];
        rsl[x] = rd.slot >= 0 ? reinterpret_cast<const uint4*>(a.masks + (int64_t)rd.slot * W) : nullptr;
        rit[x] = rd.item >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)rd.item * W) : nullptr;
    }
#pragma unroll
    for (int y = 0; y < BC; y++) {
        const int c = t.c0 + min(bc + y, nc - 1);
        const int32_t col = c == j.self_col ? -1 : a.cols[j.col_off + c];
        csrc[y] = col >= 0 ? reinterpret_cast<const uint4*>(a.bitmap + (int64_t)col * W) : nullptr;
    }
    uint32_t acc[BR][BC];
#pragma unroll
    for (int x = 0; x < BR; x++)
#pragma unroll
        for (int y = 0; y < BC; y++) acc[x][y] = 0;
    __syncthreads();   // sacc cleared
    const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
    const int64_t P0 = t.w0 >> 2, P1 = t.w1 >> 2;
    if (busy) {
        for (int64_t p = P0 + g; p < P1; p += G) {
            uint4 base = ones;
            if (base_m) base = and4(base, __ldg(base_m + p));
            if (base_i) base = and4(base, __ldg(base_i + p));
            uint4 xr[BR];
#pragma unroll
            for (int x = 0; x < BR; x++) {
                uint4 v = base;
                if (rsl[x]) v = and4(v, __ldg(rsl[x] + p));
                if (rit[x]) v = and4(v, __ldg(rit[x] + p));
                xr[x] = v;
            }
#pragma unroll
            for (int y = 0; y < BC; y++) {
                const uint4 cv = csrc[y] ? __ldg(csrc[y] + p) : ones;
#pragma unroll
                for (int x = 0; x < BR; x++) acc[x][y] += popc4(and4(xr[x], cv));
            }
        }
#pragma unroll
        for (int x = 0; x < BR; x++)
#pragma unroll
            for (int y = 0; y < BC; y++)
                if (br + x < nr && bc + y < nc && acc[x][y]) atomicAdd(&sacc[(br + x) * 64 + bc + y], (int32_t)acc[x][y]);
    }
    __syncthreads();
    for (int q = tid; q < nr * nc; q += blockDim.x) {
        const int r = q / nc, c = q - r * nc;
        const int32_t v = sacc[r * 64 + c];
        if (v) atomicAdd(a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + t.c0 + c, v);
    }
    __syncthreads();   // shared state is reused by the block's next tile
}

// Row blocks by the tile's rows: 1, 2, 3 (also 5, 6 as two blocks) or 4 (also 7, 8).
__device__ __forceinline__ void lop3_dense_tile(const CountArgs& a, const TileDesc t, int32_t* sacc) {
    switch (t.nr) {
        case 1: lop3_dense_impl<1>(a, t, sacc); break;
        case 2: lop3_dense_impl<2>(a, t, sacc); break;
        case 3: case 5: case 6: lop3_dense_impl<3>(a, t, sacc); break;
        default: lop3_dense_impl<4>(a, t, sacc); break;
    }
}

// Tiles of more than 32 columns give each lane two columns.  DENSE: the launch may hold
// dense tiles too (the persistent form); the plain launches hold one kind each.
template <bool DENSE>
__device__ __forceinline__ void lop3_tile(const CountArgs& a, const TileDesc t, Lop3Shared& sh) {
    if (DENSE && (t.pad & 1)) lop3_dense_tile(a, t, sh.acc);
    else if (t.c1 - t.c0 > 32) lop3_tile_impl<true>(a, t, sh);
    else lop3_tile_impl<false>(a, t, sh);
}

__global__ void __launch_bounds__(256, 4) k_count_lop3(CountArgs a) {
    __shared__ Lop3Shared sh;
    phase_begin(a.ph_s);
    lop3_tile<false>(a, a.tiles[blockIdx.x], sh);
    phase_end(a.ph_e);
}

// Dense tiles only (a separate launch, so that the register budget of the skipping tiles
// above stays as it is).
__global__ void __launch_bounds__(256, 4) k_count_lop3_dense(CountArgs a) {
    __shared__ int32_t sacc[kLop3Rows * 64];
    phase_begin(a.ph_s);
    lop3_dense_tile(a, a.tiles[blockIdx.x], sacc);
    phase_end(a.ph_e);
}

// Persistent form: arguments and tile count are read from device memory (a wave built on the
// GPU); blocks take tiles from a shared counter (`next`, zero at launch), so a block that
// drew light tiles takes more.
__global__ void __launch_bounds__(256, 4) k_count_lop3_persistent(const CountArgs* __restrict__ args,
                                                               const int32_t* n_tiles, int32_t* next) {
    __shared__ Lop3Shared sh;
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
        lop3_tile<true>(a, a.tiles[t], sh);
    }
    phase_end(a.ph_e);
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
    k_count_lop3<<<a.n_tiles, 256, 0, s>>>(a);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_count_lop3_dense(const CountArgs& a, cudaStream_t s) {
    if (a.n_tiles <= 0) return TFIM_OK;
    k_count_lop3_dense<<<a.n_tiles, 256, 0, s>>>(a);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int occupancy_lop3(int* blocks) {
    TFIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_count_lop3_persistent, 256, 0));
    return TFIM_OK;
}

int launch_count_lop3_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                                 cudaStream_t s) {
    k_count_lop3_persistent<<<grid, 256, 0, s>>>(d_args, d_n_tiles, d_next);
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
