// Tensor-core counter for family jobs: tcgen05.mma kind::i8 on bits expanded to bytes.
//
// A family job counts popc(base & B[F[t]] & B[F[c]]) for the tail rows t (a run of F's
// first nT entries) against every column c of F; its rows are a subset of its columns.
// With the base ANDed into the columns, X_c = base & B[F[c]], the job is a Gram block of X:
// counts[t][c] = <X_t, X_c> over the transactions, an integer dot product of 0/1 vectors.
// This counter expands X's bits to bytes in shared memory once per stage and multiplies
// X (A operand: the F columns on the 128 accumulator lanes) by a window of X's own rows
// (B operand: the tail rows, N = 16..144 accumulator columns) with
// tcgen05.mma.cta_group::1.kind::i8 into tensor memory -- one expansion serves both
// operands, and narrow tails cost N, not 128.  The arithmetic is the reference's (a support
// is a popcount of ANDed bit rows, code/engine/src/kernel_bmma.cu:636-768, there with WMMA b1).
//
// Tile (TileDesc): one job over words [w0, w1); c1 = nF <= 128 columns; rows r0 .. r0+nr of
// the job, which are X rows s0 .. s0+nr with s0 = `pad`.  The B window starts at X row
// s0 & ~7 (8-row groups keep the 128-byte swizzle phase) and spans N = roundup16 of what
// it must cover, at most 144 rows, so the expanded stage holds 144 rows.
//
// Warp roles (288 threads, one CTA per SM, persistent over a tile counter):
//   warp 0     : one lane issues the stage's MMAs (K = 32 bytes each, 4 per K block of 128
//                bits, 2, 4 or 8 K blocks per stage by the family's width) once the stage is
//                full, and commits them to the stage's `empty` barrier; after the tile's last
//                stage it commits to `done`;
//   warps 1..8 : each lane owns one (X row, K block) unit of its warp's rows r = warp-1
//                (mod 8): it loads the unit's 128 raw bits and the base's with 16-byte
//                read-only loads four stages ahead into registers, ANDs them, expands them
//                (byte lane b of output word 8q+i is bit i+8b of input word q; any K order
//                shared by both operands works) into the K-major 128-byte-swizzle layout,
//                and the warp arrives on the stage's `full` barrier; warps 1..4 then read the
//                accumulator (tcgen05.ld, 32 lanes each) and add the counts to the job's output
//                with int32 atomics (word slices of one job meet there).
// The tensor core issues an i8 MMA of M = 128 in about 50 cycles up to N = 64 (64 at N = 128,
// 128 at N = 256), so this counter pays for families wide enough to fill it; narrow ones
// stay on the CUDA-core tiles.
// Every mbarrier wait is bounded; on expiry the kernel records an error, stops issuing,
// drains what it issued and frees its tensor memory.
#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kFM = 128;                               // accumulator lanes (F columns)
constexpr int kFXRows = 144;                           // expanded rows per K block
constexpr int kFKBytes = 128;                          // bytes (= bits) per row per K block
constexpr int kFStageBytes = 2 * kFXRows * kFKBytes;   // 36 KiB: 2 K blocks of 144 rows, or more of fewer
constexpr int kFStages = 5;
constexpr int kFExpWarps = 8;
constexpr int kFThreads = 32 * (1 + kFExpWarps);       // 288
constexpr int kFAhead = 4;                             // stages of raw words in flight per lane
// The A operand (M = 128 rows of 128 bytes) of a K block spans 16 KiB from the block's start
// whatever the family's width; when a K block holds fewer than 128 rows the window runs into
// the following blocks (rows the epilogue discards), so a guard of 16 KiB follows the last
// stage to keep every window inside the allocation.
constexpr int kFGuard = kFM * kFKBytes;
constexpr int kFSmem = kFStages * kFStageBytes + kFGuard + 1024;
static_assert(kFSmem <= 227 * 1024 - 256, "stages + guard + alignment fit the opt-in shared memory");
constexpr uint32_t kFTmemCols = 256;
constexpr uint32_t kFSpin = 1u << 22;

__device__ int g_fam_status;   // 0 ok, 1 an mbarrier wait expired

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ uint4 ldg4(const uint32_t* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

// K-major, 128-byte swizzle shared-memory matrix descriptor: start address, leading byte
// offset 16 (unused by swizzled K-major layouts), stride byte offset 1024 (8-row groups),
// version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor: D s32, A and B u8, both K-major, N columns, M = 128.
__device__ __forceinline__ uint32_t idesc_i8(int n) {
    return (2u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kFM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on phase `parity`; false when the limit expired.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t k = 0; k < kFSpin; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// The accumulator's registers are written asynchronously by tcgen05.ld and are valid only
// after tcgen05.wait::ld.  Both sit in one asm statement, so the compiler cannot read an
// output register (for example to test it before an atomic add) between the two.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {"
        "%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15"
        "}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        :
          "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}

struct FamShared {
    uint64_t full[kFStages], empty[kFStages], done;
    uint32_t tmem;
    int32_t tile, abort;
};

// a_dev (device copy of the arguments, read when non-null: a graph's launches outlive pool
// growth) or a_val; n_tiles from n_tiles_p when non-null; tiles from `next` when non-null
// (persistent), else tile blockIdx.x.
__global__ void __launch_bounds__(kFThreads, 1) k_count_fam(CountArgs a_val, const CountArgs* __restrict__ a_dev,
                                                            const int32_t* n_tiles_p, int32_t n_tiles_h, int32_t* next) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ FamShared sh;
    const CountArgs a = a_dev ? *a_dev : a_val;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const int32_t n_tiles = n_tiles_p ? *n_tiles_p : n_tiles_h;
    const int64_t W = a.W;

    phase_begin(a.ph_s);
    if (tid == 0) {
        for (int s = 0; s < kFStages; s++) {
            mbar_init(smem_u32(&sh.full[s]), kFExpWarps);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        mbar_init(smem_u32(&sh.done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sh.abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem)),
                     "r"(kFTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sh.tmem;

    uint32_t g = 0;        // stages of the CTA before the current tile (phases of full / empty)
    uint32_t n_done = 0;   // tiles finished (phase of `done`)
    bool first = true;
    while (true) {
        if (tid == 0) {
            int32_t t;
            if (next) t = atomicAdd(next, 1);
            else t = first ? (int32_t)blockIdx.x : n_tiles;
            sh.tile = sh.abort ? n_tiles : t;
        }
        first = false;
        __syncthreads();
        const int32_t ti = sh.tile;
        if (ti >= n_tiles) break;
        const TileDesc t = a.tiles[ti];
        const JobDesc j = a.jobs[t.job];
        const int nF = t.c1;                       // columns 0 .. nF of the job (nF <= 128)
        const int s0 = t.pad;                      // X row of the tile's first row
        const int b8 = s0 & ~7;
        const int ncov = s0 + t.nr - b8;
        const int N = (ncov + 15) & ~15;           // 16 .. 144
        // rows of a K block (a multiple of 8, so K blocks stay 1024-byte aligned) and K blocks
        // per stage: a narrow family takes more K per synchronisation; a warp's units (rows x
        // K blocks) never exceed its 32 lanes
        const int rows_alloc = max((nF + 7) & ~7, b8 + N);   // <= 136
        const int KB = (nF <= 32 && rows_alloc * kFKBytes * 8 <= kFStageBytes) ? 8
                       : (nF <= 64 && rows_alloc * kFKBytes * 4 <= kFStageBytes) ? 4 : 2;
        // the last A window of a stage, (KB - 1) * kb_bytes + 16 KiB from the stage, stays
        // inside stage + guard: KB * kb_bytes <= kFStageBytes and the guard is 16 KiB
        const uint32_t kb_bytes = (uint32_t)rows_alloc * kFKBytes;
        const int stage_words = KB * 4;            // raw 32-bit words per row per stage
        const int n_st = (t.w1 - t.w0) / stage_words;

        if (warp == 0) {
            if (lane == 0) {
                bool ok = true;
                const uint32_t idesc = idesc_i8(N);
                for (int st = 0; st < n_st && ok; st++) {
                    const uint32_t it = g + (uint32_t)st;
                    const int s = (int)(it % kFStages);
                    if (!mbar_wait(smem_u32(&sh.full[s]), (it / kFStages) & 1u)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t stage = base + (uint32_t)s * kFStageBytes;
                    for (int kb = 0; kb < KB; kb++) {
                        const uint32_t blk = stage + (uint32_t)kb * kb_bytes;
#pragma unroll
                        for (int k = 0; k < kFKBytes / 32; k++) {
                            const uint64_t da = smem_desc(blk + k * 32);
                            const uint64_t db = smem_desc(blk + (uint32_t)b8 * kFKBytes + k * 32);
                            mma_i8(tmem, da, db, idesc, (st > 0 || kb > 0 || k > 0) ? 1u : 0u);
                        }
                    }
                    tc_commit(smem_u32(&sh.empty[s]));
                }
                if (!ok) {
                    atomicExch(&sh.abort, 1);
                    atomicExch(&g_fam_status, 1);
                }
                // tracks every MMA issued so far
                tc_commit(smem_u32(&sh.done));
            }
            __syncwarp();
        } else {
            // ---- expansion: lane -> unit (row q of the warp's rows, K block kb)
            const int e = warp - 1;
            const int nrw = nF > e ? (nF - e + kFExpWarps - 1) / kFExpWarps : 0;
            const int kb_log = KB == 8 ? 3 : KB == 4 ? 2 : 1;
            const bool active = lane < (nrw << kb_log);
            const int q = lane >> kb_log, kb = lane & (KB - 1);
            const int r = e + q * kFExpWarps;
            const uint32_t* src = active ? a.bitmap + (int64_t)a.cols[j.col_off + r] * W : nullptr;
            const uint32_t* bm = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
            const uint32_t* bi = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
            const int64_t w_unit = t.w0 + (int64_t)kb * 4;   // + st * stage_words
            const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
            uint4 pr[kFAhead], pm[kFAhead], pi[kFAhead];
            auto load = [&](int st, uint4& xr, uint4& xm, uint4& xi) {
                xr = xm = xi = ones;
                if (active && st < n_st) {
                    const int64_t w = w_unit + (int64_t)st * stage_words;
                    xr = ldg4(src + w);
                    if (bm) xm = ldg4(bm + w);
                    if (bi) xi = ldg4(bi + w);
                }
            };
#pragma unroll
            for (int d = 0; d < kFAhead; d++) load(d, pr[d], pm[d], pi[d]);
            const uint32_t row_off = (uint32_t)r * kFKBytes + (uint32_t)kb * kb_bytes;
            const int rs = r & 7;
            bool ok = true;
            for (int st0 = 0; st0 < n_st && ok; st0 += kFAhead) {
#pragma unroll
                for (int d = 0; d < kFAhead; d++) {
                    const int st = st0 + d;
                    if (st >= n_st) break;
                    const uint32_t it = g + (uint32_t)st;
                    const int s = (int)(it % kFStages);
                    if (ok && it >= (uint32_t)kFStages)
                        ok = mbar_wait(smem_u32(&sh.empty[s]), ((it / kFStages) - 1u) & 1u);
                    ok = __all_sync(0xffffffffu, ok);
                    if (!ok) break;
                    const uint4 x = make_uint4(pr[d].x & pm[d].x & pi[d].x, pr[d].y & pm[d].y & pi[d].y,
                                               pr[d].z & pm[d].z & pi[d].z, pr[d].w & pm[d].w & pi[d].w);
                    load(st + kFAhead, pr[d], pm[d], pi[d]);
                    if (active) {
                        const uint32_t row = base + (uint32_t)s * kFStageBytes + row_off;
                        const uint32_t ws[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                        for (int c = 0; c < 8; c++) {
                            const uint32_t v = ws[c >> 1] >> (4 * (c & 1));
                            st_shared_v4(row + (uint32_t)((c ^ rs) << 4), v & 0x01010101u, (v >> 1) & 0x01010101u,
                                         (v >> 2) & 0x01010101u, (v >> 3) & 0x01010101u);
                        }
                    }
                    // generic-proxy stores -> visible to the tensor cores' async proxy
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&sh.full[s]));
                }
            }
            if (!ok && lane == 0) {
                atomicExch(&sh.abort, 1);
                atomicExch(&g_fam_status, 1);
            }
            // ---- epilogue: warps 1..4 read lanes 32*(warp%4) .. +32 (columns of F)
            if (warp <= 4) {
                const bool fin = mbar_wait(smem_u32(&sh.done), n_done & 1u);
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const bool all_fin = __all_sync(0xffffffffu, fin);
                if (!all_fin && lane == 0) {
                    atomicExch(&sh.abort, 1);
                    atomicExch(&g_fam_status, 1);
                }
                if (all_fin && !sh.abort && n_st > 0) {
                    const int lq = warp & 3;
                    const int col = 32 * lq + lane;
                    for (int n0 = 0; n0 < N; n0 += 16) {
                        uint32_t v[16];
                        tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + (uint32_t)n0, v);
                        if (col < nF) {
#pragma unroll
                            for (int u = 0; u < 16; u++) {
                                const int xr = b8 + n0 + u;   // X row of accumulator column n0+u
                                if (xr >= s0 && xr < s0 + t.nr && v[u]) {
                                    const int jr = t.r0 + (xr - s0);
                                    atomicAdd(a.out + j.out_off + (int64_t)jr * j.n_cols + col, (int32_t)v[u]);
                                }
                            }
                        }
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();   // accumulator read, stages free for the next tile
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        g += (uint32_t)max(n_st, 0);
        n_done++;
    }
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kFTmemCols));
    phase_end(a.ph_e);
}

}  // namespace

int configure_fam_kernel() {
    static std::atomic<bool> configured[64];
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !configured[dev].load()) {
        TFIM_CUDA(cudaFuncSetAttribute(k_count_fam, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
        configured[dev].store(true);
    }
    return TFIM_OK;
}

int launch_count_fam(const CountArgs& a, cudaStream_t s) {
    if (a.n_tiles <= 0) return TFIM_OK;
    TFIM_TRY(configure_fam_kernel());
    k_count_fam<<<a.n_tiles, kFThreads, kFSmem, s>>>(a, nullptr, nullptr, a.n_tiles, nullptr);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int launch_count_fam_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                                cudaStream_t s) {
    TFIM_TRY(configure_fam_kernel());
    CountArgs none;
    k_count_fam<<<grid, kFThreads, kFSmem, s>>>(none, d_args, d_n_tiles, 0, d_next);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int count_fam_status(bool reset) {
    int v = 0;
    TFIM_CUDA(cudaMemcpyFromSymbol(&v, g_fam_status, sizeof v));
    if (reset && v) {
        const int z = 0;
        TFIM_CUDA(cudaMemcpyToSymbol(g_fam_status, &z, sizeof z));
    }
    TFIM_CHECK(v == 0, TFIM_E_TIMEOUT, "tensor-memory family counter: an mbarrier wait expired");
    return TFIM_OK;
}

}  // namespace tfim
