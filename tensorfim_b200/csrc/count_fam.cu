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
// Warp roles (320 threads, one CTA per SM, persistent over a tile counter):
//   warp 0     : one lane issues the stage's 8 MMAs (K = 32 bytes each, 2 K blocks of
//                128 bits) once the stage is full, and commits them to the stage's `empty`
//                barrier; after the tile's last stage it commits to `done`;
//   warp 9     : the loader: the raw bit words of a chunk of stages -- every X row's item
//                row and the base's one or two sources, C stages of 256 bits each -- come
//                into a three-slot ring with one bulk copy (cp.async.bulk, the TMA engine's
//                untiled copy of this GPU's own memory) per row and chunk, completing on
//                the slot's transaction-count barrier.  A chunk is about 24 KiB whatever
//                the family's width (C = 5 stages at 130 rows, 42 at 18), so about 72 KiB
//                are in flight per SM;
//   warps 1..8 : X rows r = warp-1 (mod 8): the stage's raw words, ANDed with the base, are
//                expanded (byte lane b of output word 8q+i is bit i+8b of input word q; any K
//                order shared by both operands works) and stored in the K-major
//                128-byte-swizzle layout; each warp arrives on the stage's `full` barrier and,
//                after a chunk's last stage, on the slot's `rempty` barrier; warps 1..4 then
//                read the accumulator (tcgen05.ld, 32 lanes each) and add the counts to the
//                job's output with int32 atomics (word slices of one job meet there).
// Every mbarrier wait is bounded; on expiry the kernel records an error, stops issuing,
// drains what it issued and frees its tensor memory.
#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kFM = 128;                               // accumulator lanes (F columns)
constexpr int kFXRows = 144;                           // expanded rows per K block
constexpr int kFKBytes = 128;                          // bytes (= bits) per row per K block
constexpr int kFMaxKBlocks = 8;                        // K blocks per stage: 2, 4 or 8 (1024 bits)
constexpr int kFStageBytes = 2 * kFXRows * kFKBytes;   // 36 KiB: 2 K blocks of 144 rows, or more of fewer
constexpr int kFStages = 4;
constexpr int kFExpWarps = 8;
constexpr int kFLoadWarp = 1 + kFExpWarps;             // warp 9
constexpr int kFThreads = 32 * (2 + kFExpWarps);       // 320
constexpr int kFRawSlots = 3;
constexpr int kFRawSlotBytes = 24 * 1024;              // one chunk of raw rows
constexpr int kFMaxEntries = kFM + 2;                  // rows + up to two base sources
constexpr int kFSmem = kFStages * kFStageBytes + kFRawSlots * kFRawSlotBytes + 1024;
constexpr uint32_t kFTmemCols = 256;
constexpr uint32_t kFSpin = 1u << 22;
static_assert(kFRawSlotBytes / (kFMaxEntries * 2 * 16) >= 1, "a chunk holds at least one stage");

__device__ int g_fam_status;   // 0 ok, 1 an mbarrier wait expired

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from this GPU's
// global memory into shared memory, completing on the barrier's transaction count.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar), "r"(bytes)
                 : "memory");
}

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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct FamShared {
    uint64_t full[kFStages], empty[kFStages], done, rfull[kFRawSlots], rempty[kFRawSlots];
    uint32_t tmem;
    int32_t tile, abort;
    const uint32_t* src[kFMaxEntries];   // raw sources of the tile: X rows, then the base's
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
    const uint32_t raw_base = base + kFStages * kFStageBytes;
    const int32_t n_tiles = n_tiles_p ? *n_tiles_p : n_tiles_h;
    const int64_t W = a.W;

    phase_begin(a.ph_s);
    if (tid == 0) {
        for (int s = 0; s < kFStages; s++) {
            mbar_init(smem_u32(&sh.full[s]), kFExpWarps);
            mbar_init(smem_u32(&sh.empty[s]), 1);
        }
        for (int s = 0; s < kFRawSlots; s++) {
            mbar_init(smem_u32(&sh.rfull[s]), 1);
            mbar_init(smem_u32(&sh.rempty[s]), kFExpWarps);
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
    uint32_t gc = 0;       // raw chunks of the CTA before the current tile (phases of rfull / rempty)
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
        // per stage: a narrow family takes more K per synchronisation
        const int rows_alloc = max((nF + 7) & ~7, b8 + N);   // <= 144
        const int KB = rows_alloc * kFKBytes * 8 <= kFStageBytes ? 8 : rows_alloc * kFKBytes * 4 <= kFStageBytes ? 4 : 2;
        const uint32_t kb_bytes = (uint32_t)rows_alloc * kFKBytes;
        const int stage_words = KB * 4;            // raw 32-bit words per row per stage
        const int stage_raw = stage_words * 4;     // raw bytes per row per stage
        const int n_st = (t.w1 - t.w0) / stage_words;
        const int nbase = (j.base_slot >= 0 ? 1 : 0) + (j.base_item >= 0 ? 1 : 0);
        const int n_ent = nF + nbase;
        // stages per raw chunk: a chunk of every entry fits one ring slot
        const int C = max(1, kFRawSlotBytes / (n_ent * stage_raw));
        const int n_chunks = (n_st + C - 1) / C;
        // the tile's raw sources
        for (int q = tid; q < n_ent; q += kFThreads) {
            const uint32_t* p;
            if (q < nF) p = a.bitmap + (int64_t)a.cols[j.col_off + q] * W;
            else if (q == nF && j.base_slot >= 0) p = a.masks + (int64_t)j.base_slot * W;
            else p = a.bitmap + (int64_t)j.base_item * W;
            sh.src[q] = p;
        }
        __syncthreads();

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
        } else if (warp == kFLoadWarp) {
            // ---- loader: chunk k of the tile into slot (gc + k) % kFRawSlots
            bool ok = true;
            for (int k = 0; k < n_chunks; k++) {
                const uint32_t ck = gc + (uint32_t)k;
                const int slot = (int)(ck % kFRawSlots);
                if (ck >= (uint32_t)kFRawSlots) ok = mbar_wait(smem_u32(&sh.rempty[slot]), ((ck / kFRawSlots) - 1u) & 1u);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
                const int st0 = k * C, ns = min(C, n_st - st0);
                const uint32_t bytes = (uint32_t)(ns * stage_raw);   // per entry, a multiple of 32
                const uint32_t bar = smem_u32(&sh.rfull[slot]);
                if (lane == 0) mbar_expect_tx(bar, bytes * (uint32_t)n_ent);
                __syncwarp();
                const uint32_t dst0 = raw_base + (uint32_t)slot * kFRawSlotBytes;
                const int64_t w = t.w0 + (int64_t)st0 * stage_words;
                for (int q = lane; q < n_ent; q += 32)
                    bulk_load(dst0 + (uint32_t)(q * C * stage_raw), sh.src[q] + w, bytes, bar);
            }
            if (!ok && lane == 0) {
                atomicExch(&sh.abort, 1);
                atomicExch(&g_fam_status, 1);
            }
        } else {
            // ---- expansion: X rows r = e, e + 8, ... (< nF); a task is one 16-byte output chunk
            // (row, K block, chunk c): 8 chunks per K block, KB * 8 per row
            const int e = warp - 1;
            const int nrw = nF > e ? (nF - e + kFExpWarps - 1) / kFExpWarps : 0;
            const int tpr_log = KB == 8 ? 6 : KB == 4 ? 5 : 4;   // log2(KB * 8)
            const int ntask = nrw << tpr_log;
            const uint32_t ent = (uint32_t)(C * stage_raw);
            bool ok = true;
            int k = 0, within = 0;   // chunk of the tile and stage within it
            for (int st = 0; st < n_st; st++) {
                const uint32_t ck = gc + (uint32_t)k;
                const int slot = (int)(ck % kFRawSlots);
                if (within == 0 && ok) ok = mbar_wait(smem_u32(&sh.rfull[slot]), (ck / kFRawSlots) & 1u);
                const uint32_t it = g + (uint32_t)st;
                const int s = (int)(it % kFStages);
                if (ok && it >= (uint32_t)kFStages)
                    ok = mbar_wait(smem_u32(&sh.empty[s]), ((it / kFStages) - 1u) & 1u);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) break;
                const uint32_t rs = raw_base + (uint32_t)slot * kFRawSlotBytes + (uint32_t)(within * stage_raw);
                const uint32_t stage = base + (uint32_t)s * kFStageBytes;
                for (int tk = lane; tk < ntask; tk += 32) {
                    const int qi = tk >> tpr_log, rem = tk & ((1 << tpr_log) - 1);
                    const int kb = rem >> 3, c = rem & 7;
                    const uint32_t off = (uint32_t)((kb * 4 + (c >> 1)) * 4);   // raw word of the chunk
                    const int r = e + qi * kFExpWarps;
                    uint32_t x;
                    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(x) : "r"(rs + (uint32_t)r * ent + off));
                    for (int b = 0; b < nbase; b++) {
                        uint32_t y;
                        asm volatile("ld.shared.b32 %0, [%1];" : "=r"(y) : "r"(rs + (uint32_t)(nF + b) * ent + off));
                        x &= y;
                    }
                    x >>= 4 * (c & 1);
                    st_shared_v4(stage + (uint32_t)kb * kb_bytes + (uint32_t)r * kFKBytes + (uint32_t)((c ^ (r & 7)) << 4),
                                 x & 0x01010101u, (x >> 1) & 0x01010101u, (x >> 2) & 0x01010101u, (x >> 3) & 0x01010101u);
                }
                // generic-proxy stores -> visible to the tensor cores' async proxy
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                const bool chunk_end = within == C - 1 || st == n_st - 1;
                if (lane == 0) {
                    mbar_arrive(smem_u32(&sh.full[s]));
                    if (chunk_end) mbar_arrive(smem_u32(&sh.rempty[slot]));
                }
                if (++within == C) {
                    within = 0;
                    k++;
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
        __syncthreads();   // accumulator read, stages, ring and tables free for the next tile
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        g += (uint32_t)max(n_st, 0);
        gc += (uint32_t)n_chunks;
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
