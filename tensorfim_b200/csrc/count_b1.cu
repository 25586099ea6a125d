// Tensor-core support counting on the 0/1 bit matrices: C = popc(A AND B) per k-step of
// 256 bits, with `mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc`.
//
// This computes the same C as the reference's WMMA b1 kernels bmmaKernelNaive /
// bmmaKernelSmem / bmmaKernelSmemSplitK (code/engine/src/kernel_bmma.cu:636-758): row i
// of A is a prefix mask, row j of B an item bitmap, C[i][j] their AND-popcount.  The
// B200 design differs: A and B tiles of 64 rows x 2048 bits are staged with cp.async into
// a two-stage shared-memory ring, fragments come from ldmatrix over an XOR-swizzled
// layout (conflict-free), the per-job base mask along the transaction axis is ANDed into
// the A fragments in registers (so a family of children shares one staged parent mask),
// and split-k partial sums over transaction ranges meet in int32 atomics.
//
// Fragment layouts (PTX ISA, mma.m16n8k256 with .b1): A row-major 16x256, four .b32
// registers: a0 = row g, bits [32*tg, 32*tg+32) of k 0..127; a1 = row g+8, same bits;
// a2/a3 = the same rows for k 128..255 (g = lane/4, tg = lane%4).  B column-major
// 256x8: b0 = column g, bits [32*tg, +32) of k 0..127; b1 = the same for k 128..255.
// C: c0,c1 = row g, columns 2*tg, 2*tg+1; c2,c3 = row g+8.
#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kKcWords = 64;                     // words per K-chunk (2048 bits)
constexpr int kRowBytes = kKcWords * 4;          // 256 B per staged row
constexpr int kTileBytes = 64 * kRowBytes;       // 16 KiB per 64-row operand tile
constexpr int kStageBytes = 2 * kTileBytes + kRowBytes;   // A + B + base chunk
constexpr int kStages = 2;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void st_shared16(uint32_t dst, uint4 v) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};\n" ::"r"(dst), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void mma_b1(int32_t (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
        : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// byte offset of 16-byte chunk `ch` (0..15) of staged row `row` (0..63), swizzled
__device__ __forceinline__ uint32_t swz(int row, int ch) { return (uint32_t)(row * kRowBytes + ((ch ^ (row & 7)) << 4)); }

struct B1Shared {
    const uint32_t* row_src[64];
    const uint32_t* col_src[64];
    int32_t row_kind[64];   // 0 = source row, 1 = all ones, 2 = zeros
    int32_t col_kind[64];
};

// Block: 256 threads (8 warps as 2 x 4; each warp owns 32 rows x 16 columns).
__device__ void b1_tile(const CountArgs& a, const TileDesc t, unsigned char* smem, B1Shared& sh) {
    const uint32_t** row_src = sh.row_src;
    const uint32_t** col_src = sh.col_src;
    int32_t* row_kind = sh.row_kind;
    int32_t* col_kind = sh.col_kind;
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x;
    if (tid < 64) {
        const int r = tid;
        if (r < t.nr) {
            const RowDesc rd = a.rows[j.row_off + t.r0 + r];
            if (rd.slot >= 0) { row_src[r] = a.masks + (int64_t)rd.slot * W; row_kind[r] = 0; }
            else if (rd.item >= 0) { row_src[r] = a.bitmap + (int64_t)rd.item * W; row_kind[r] = 0; }
            else { row_src[r] = nullptr; row_kind[r] = 1; }
        } else {
            row_src[r] = nullptr;
            row_kind[r] = 2;
        }
    } else if (tid < 128) {
        const int c = tid - 64;
        if (t.c0 + c < t.c1) {
            const int32_t col = (t.c0 + c) == j.self_col ? -1 : a.cols[j.col_off + t.c0 + c];
            if (col >= 0) { col_src[c] = a.bitmap + (int64_t)col * W; col_kind[c] = 0; }
            else { col_src[c] = nullptr; col_kind[c] = 1; }
        } else {
            col_src[c] = nullptr;
            col_kind[c] = 2;
        }
    }
    const uint32_t* base_m = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
    const uint32_t* base_i = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
    const bool has_base = base_m || base_i;
    __syncthreads();

    const uint32_t sbase = smem_u32(smem);
    const int n_chunks = (t.w1 - t.w0) / kKcWords;

    // issue the copies of K-chunk `kc` (absolute word offset w) into stage `st`
    auto load_chunk = [&](int st, int w) {
        const uint32_t sa = sbase + st * kStageBytes;
        const uint32_t sb = sa + kTileBytes;
        const uint32_t sm = sb + kTileBytes;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int idx = tid + q * 256;        // 0..1023 = 64 rows x 16 chunks
            const int r = idx >> 4, ch = idx & 15;
            const int rk = row_kind[r];
            if (rk == 0) cp_async16(sa + swz(r, ch), row_src[r] + w + ch * 4);
            else st_shared16(sa + swz(r, ch), rk == 1 ? make_uint4(~0u, ~0u, ~0u, ~0u) : make_uint4(0, 0, 0, 0));
            const int ck = col_kind[r];
            if (ck == 0) cp_async16(sb + swz(r, ch), col_src[r] + w + ch * 4);
            else st_shared16(sb + swz(r, ch), ck == 1 ? make_uint4(~0u, ~0u, ~0u, ~0u) : make_uint4(0, 0, 0, 0));
        }
        if (has_base && tid < 16) {
            uint4 v = make_uint4(~0u, ~0u, ~0u, ~0u);
            if (base_m) {
                const uint4 x = __ldg(reinterpret_cast<const uint4*>(base_m + w) + tid);
                v.x &= x.x; v.y &= x.y; v.z &= x.z; v.w &= x.w;
            }
            if (base_i) {
                const uint4 x = __ldg(reinterpret_cast<const uint4*>(base_i + w) + tid);
                v.x &= x.x; v.y &= x.y; v.z &= x.z; v.w &= x.w;
            }
            st_shared16(sm + tid * 16, v);
        }
        cp_async_commit();
    };

    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp & 1, wn = warp >> 1;
    const int g = lane >> 2, tg = lane & 3;
    int32_t acc[2][2][4];
#pragma unroll
    for (int mf = 0; mf < 2; mf++)
#pragma unroll
        for (int nf = 0; nf < 2; nf++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[mf][nf][q] = 0;

    // ldmatrix row/chunk selection for this lane
    const int lm = lane >> 3, lr = lane & 7;
    if (n_chunks > 0) load_chunk(0, t.w0);
    for (int i = 0; i < n_chunks; i++) {
        if (i + 1 < n_chunks) {
            load_chunk((i + 1) & 1, t.w0 + (i + 1) * kKcWords);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const uint32_t sa = sbase + (i & 1) * kStageBytes;
        const uint32_t sb = sa + kTileBytes;
        const uint32_t* smask = reinterpret_cast<const uint32_t*>(smem + (i & 1) * kStageBytes + 2 * kTileBytes);
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            uint32_t af[2][4];
#pragma unroll
            for (int mf = 0; mf < 2; mf++) {
                const int row = wm * 32 + mf * 16 + lr + (lm & 1) * 8;
                const int ch = ks * 2 + (lm >> 1);
                ldsm_x4(sa + swz(row, ch), af[mf][0], af[mf][1], af[mf][2], af[mf][3]);
            }
            if (has_base) {
                const uint32_t mlo = smask[ks * 8 + tg], mhi = smask[ks * 8 + 4 + tg];
#pragma unroll
                for (int mf = 0; mf < 2; mf++) {
                    af[mf][0] &= mlo; af[mf][1] &= mlo;
                    af[mf][2] &= mhi; af[mf][3] &= mhi;
                }
            }
            uint32_t bf[4];
            {
                const int col = wn * 16 + lr + (lm >> 1) * 8;
                const int ch = ks * 2 + (lm & 1);
                ldsm_x4(sb + swz(col, ch), bf[0], bf[1], bf[2], bf[3]);
            }
#pragma unroll
            for (int mf = 0; mf < 2; mf++) {
                mma_b1(acc[mf][0], af[mf], bf[0], bf[1]);
                mma_b1(acc[mf][1], af[mf], bf[2], bf[3]);
            }
        }
        __syncthreads();
    }

    // epilogue: split-k partial sums meet in atomics
#pragma unroll
    for (int mf = 0; mf < 2; mf++)
#pragma unroll
        for (int nf = 0; nf < 2; nf++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int r = wm * 32 + mf * 16 + g + (q >> 1) * 8;
                const int c = wn * 16 + nf * 8 + tg * 2 + (q & 1);
                const int32_t v = acc[mf][nf][q];
                if (v && r < t.nr && t.c0 + c < t.c1)
                    atomicAdd(a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + (t.c0 + c), v);
            }
    __syncthreads();   // the block's next tile reuses the staging and the source tables
}

__global__ void __launch_bounds__(256) k_count_b1(CountArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ B1Shared sh;
    phase_begin(a.ph_s);
    b1_tile(a, a.tiles[blockIdx.x], smem, sh);
    phase_end(a.ph_e);
}

__global__ void __launch_bounds__(256) k_count_b1_persistent(const CountArgs* __restrict__ args, const int32_t* n_tiles,
                                                             int32_t* next) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ B1Shared sh;
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
        b1_tile(a, a.tiles[t], smem, sh);
    }
    phase_end(a.ph_e);
}

}  // namespace

int configure_count_kernels() {
    // dynamic shared memory above 48 KiB is opted into once per device
    static std::atomic<bool> done[64];
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev].load()) return TFIM_OK;
    const size_t smem = (size_t)kStages * kStageBytes;
    TFIM_CUDA(cudaFuncSetAttribute(k_count_b1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TFIM_CUDA(cudaFuncSetAttribute(k_count_b1_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (dev >= 0 && dev < 64) done[dev].store(true);
    return TFIM_OK;
}

int launch_count_b1(const CountArgs& a, cudaStream_t s) {
    if (a.n_tiles <= 0) return TFIM_OK;
    TFIM_TRY(configure_count_kernels());
    const size_t smem = (size_t)kStages * kStageBytes;
    k_count_b1<<<a.n_tiles, 256, smem, s>>>(a);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int occupancy_b1(int* blocks) {
    TFIM_TRY(configure_count_kernels());
    TFIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_count_b1_persistent, 256,
                                                             (size_t)kStages * kStageBytes));
    return TFIM_OK;
}

int launch_count_b1_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                               cudaStream_t s) {
    TFIM_TRY(configure_count_kernels());
    const size_t smem = (size_t)kStages * kStageBytes;
    k_count_b1_persistent<<<grid, 256, smem, s>>>(d_args, d_n_tiles, d_next);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int occupancy_lop3(int* blocks);
int occupancy_proj(int* blocks);

int persistent_occupancy(int* lop3, int* b1, int* proj) {
    TFIM_TRY(occupancy_lop3(lop3));
    TFIM_TRY(occupancy_b1(b1));
    TFIM_TRY(occupancy_proj(proj));
    return TFIM_OK;
}

}  // namespace tfim
