// Tensor-core family counter on the 5th-generation tensor cores: tcgen05.mma kind::i8.
//
// The AND+popc Gram of a count job, popc(base & A_r & B_c), is the integer dot product of
// the rows' 0/1 bit vectors.  This counter expands each tile's bits to bytes (0 or 1) in
// shared memory and multiplies them with tcgen05.mma.cta_group::1.kind::i8 (u8 x u8 ->
// s32) into a 128 x 128 accumulator in tensor memory.  The arithmetic is the reference's
// (a support is a popcount of ANDed bit rows, code/engine/src/kernel_bmma.cu:636-768, there
// computed by WMMA b1); the expansion trades 8x more shared-memory bytes for the i8 tensor
// rate.
//
// Tile: 128 rows x 128 columns of one job over a word slice [w0, w1) (TileDesc), 512
// threads.  Per stage (256 bits of K): every thread loads one 128-bit word group of an A row
// (ANDed with the base) or of a B row -- the next stage's while the current one is
// expanded -- expands it to 128 bytes and stores them in the canonical K-major
// 128-byte-swizzle layout (row r, 16-byte chunk c at r*128 + ((c ^ (r & 7)) << 4), 8-row
// groups 1024 bytes apart); one thread then issues the stage's 8 MMAs (K = 32 bytes each)
// and commits them to the stage's mbarrier, which the threads wait on before overwriting
// that stage.  Three stages.  Epilogue: tcgen05.ld of the accumulator (warp w reads lanes
// 32*(w%4).., columns 32*(w/4)..), one int32 atomic per nonzero count (tiles over word
// slices of one job meet in the atomics).
//
// Every mbarrier wait is bounded; on expiry the kernel records an error, stops issuing, and
// frees its tensor memory.
#include <atomic>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr int kTcM = 128, kTcN = 128;
constexpr int kTcKBytes = 128;                         // one K block: 128 bytes = 128 bits per row
constexpr int kTcBlocks = 2;                           // K blocks per stage (256 bits)
constexpr int kTcTileBytes = kTcM * kTcKBytes;         // 16 KiB (A or B, one K block)
constexpr int kTcStageBytes = 2 * kTcBlocks * kTcTileBytes;   // A + B: 64 KiB
constexpr int kTcStages = 3;
constexpr int kTcThreads = 512;
constexpr int kTcSmem = kTcStages * kTcStageBytes + 1024;   // + alignment slack
constexpr uint32_t kTcSpin = 1u << 22;                 // try_wait attempts before giving up

__device__ int g_tc_status;   // 0 ok, 1 an mbarrier wait expired

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }


__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

// Expand 4 words (128 bits) into one swizzled 128-byte row of 0/1 bytes.  A dot product
// does not depend on the order of K, so any order shared by A and B works; this one is
// cheap: byte lane b of output word 8q + i holds bit i + 8b of word q, i.e. output word
// 8q + i = (w_q >> i) & 0x01010101.
__device__ __forceinline__ void store_row_bytes(uint32_t tile, int r, uint4 w) {
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
    const uint32_t row = tile + r * 128;
    const int rs = r & 7;
#pragma unroll
    for (int q = 0; q < 4; q++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t x = ws[q] >> (4 * h);
            const int c = 2 * q + h;   // 16-byte chunk: output words 8q + 4h .. 8q + 4h + 3
            st_shared_v4(row + ((c ^ rs) << 4), x & 0x01010101u, (x >> 1) & 0x01010101u, (x >> 2) & 0x01010101u,
                         (x >> 3) & 0x01010101u);
        }
    }
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (tcgen05 format): start address,
// leading byte offset 16 (unused by swizzled K-major layouts), stride byte offset 1024
// (between 8-row groups), version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor: D s32 (2 << 4), A and B u8 (format 0), both K-major, N = 128
// (N >> 3 at bit 17), M = 128 (M >> 4 at bit 24).
constexpr uint32_t kTcIdesc = (2u << 4) | ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kTcIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
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
    for (uint32_t k = 0; k < kTcSpin; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// The accumulator's registers are written asynchronously by tcgen05.ld and are valid only
// after tcgen05.wait::ld.  Both sit in one asm statement, so the compiler cannot read an
// output register (for example to test it before an atomic add) between the two.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {"
        "%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31"
        "}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        :
          "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1) k_count_i8(CountArgs a) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[kTcStages + 1];   // stage "free" barriers + "done"
    __shared__ uint32_t s_tmem;
    __shared__ const uint32_t* row_src[kTcM][2];
    __shared__ const uint32_t* col_src[kTcN];
    __shared__ int32_t col_kind[kTcN];   // 0 column row, 1 all ones, 2 zeros
    __shared__ int32_t s_abort;

    const TileDesc t = a.tiles[blockIdx.x];
    const JobDesc j = a.jobs[t.job];
    const int64_t W = a.W;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;

    // operand rows of the tile
    if (tid < kTcM) {
        const int r = tid;
        row_src[r][0] = row_src[r][1] = nullptr;
        if (r < t.nr) {
            const RowDesc rd = a.rows[j.row_off + t.r0 + r];
            if (rd.slot >= 0) row_src[r][0] = a.masks + (int64_t)rd.slot * W;
            if (rd.item >= 0) row_src[r][1] = a.bitmap + (int64_t)rd.item * W;
        }
    } else if (tid < kTcM + kTcN) {
        const int c = tid - kTcM;
        col_src[c] = nullptr;
        col_kind[c] = 2;
        if (t.c0 + c < t.c1) {
            const int32_t col = t.c0 + c == j.self_col ? -1 : a.cols[j.col_off + t.c0 + c];
            if (col < 0) col_kind[c] = 1;   // the all-ones column
            else {
                col_kind[c] = 0;
                col_src[c] = a.bitmap + (int64_t)col * W;
            }
        }
    }
    if (tid == 0) {
        for (int s = 0; s <= kTcStages; s++) mbar_init(smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"((uint32_t)kTcN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    const uint32_t* base_m = j.base_slot >= 0 ? a.masks + (int64_t)j.base_slot * W : nullptr;
    const uint32_t* base_i = j.base_item >= 0 ? a.bitmap + (int64_t)j.base_item * W : nullptr;
    // this thread's unit: matrix my_b (0 A, 1 B), row my_r, K block my_kb of each stage
    const int my_b = tid >> 8, my_r = (tid & 255) >> 1, my_kb = tid & 1;
    const uint32_t* ra = my_b ? nullptr : row_src[my_r][0];
    const uint32_t* ri = my_b ? nullptr : row_src[my_r][1];
    const bool a_zero = my_r >= t.nr;
    const uint32_t* cb = col_src[my_r];
    const int ck = col_kind[my_r];

    const int n_stages = (t.w1 - t.w0) / (kTcBlocks * 4);   // word slices are multiples of 64 words
    // this thread's words of stage `it`: A row my_r (ANDed with the base) and B row my_r
    auto load_stage = [&](int it, uint4& v) {
        const int64_t w = t.w0 + (int64_t)it * (kTcBlocks * 4) + my_kb * 4;
        v = make_uint4(0, 0, 0, 0);
        if (my_b == 0) {
            if (!a_zero) {
                v = make_uint4(~0u, ~0u, ~0u, ~0u);
                auto andv = [&](const uint32_t* p) {
                    const uint4 x = __ldg(reinterpret_cast<const uint4*>(p + w));
                    v.x &= x.x; v.y &= x.y; v.z &= x.z; v.w &= x.w;
                };
                if (ra) andv(ra);
                if (ri) andv(ri);
                if (base_m) andv(base_m);
                if (base_i) andv(base_i);
            }
        } else if (ck == 0) {
            v = __ldg(reinterpret_cast<const uint4*>(cb + w));
        } else if (ck == 1) {
            v = make_uint4(~0u, ~0u, ~0u, ~0u);
        }
    };
    const uint32_t my_tile_off = (uint32_t)((my_b * kTcBlocks + my_kb) * kTcTileBytes);
    bool ok = true;
    uint4 v, nv = make_uint4(0, 0, 0, 0);
    if (n_stages > 0) load_stage(0, v);
    for (int it = 0; it < n_stages; it++) {
        const int s = it % kTcStages;
        const uint32_t stage = base + s * kTcStageBytes;
        // the next stage's words are in flight while this one is expanded and multiplied
        if (it + 1 < n_stages) load_stage(it + 1, nv);
        if (it >= kTcStages) {
            // the MMAs that read this stage kTcStages iterations ago must be done
            if (!mbar_wait(smem_u32(&bars[s]), (uint32_t)((it / kTcStages - 1) & 1))) ok = false;
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                s_abort = 1;
                atomicExch(&g_tc_status, 1);
            }
            break;
        }
        store_row_bytes(stage + my_tile_off, my_r, v);
        // generic-proxy stores -> visible to the tensor cores' async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kb = 0; kb < kTcBlocks; kb++)
#pragma unroll
                for (int k = 0; k < kTcKBytes / 32; k++) {
                    const uint64_t da = smem_desc(stage + kb * kTcTileBytes + k * 32);
                    const uint64_t db = smem_desc(stage + (kTcBlocks + kb) * kTcTileBytes + k * 32);
                    mma_i8(tmem, da, db, (it > 0 || kb > 0 || k > 0) ? 1u : 0u);
                }
            tc_commit(smem_u32(&bars[s]));
        }
        v = nv;
    }
    // all MMAs issued by thread 0 are tracked by one more commit
    if (tid == 0) tc_commit(smem_u32(&bars[kTcStages]));
    const bool done = mbar_wait(smem_u32(&bars[kTcStages]), 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool failed = __syncthreads_or(!done) != 0;   // block-uniform: tcgen05.ld is warp-collective
    if (failed && tid == 0) atomicExch(&g_tc_status, 1);
    if (!failed && !s_abort && n_stages > 0) {
        const int lane_base = 32 * (warp & 3), col_base = 32 * (warp >> 2);   // 16 warps: 4 x 4
        const int r = lane_base + (tid & 31);
        uint32_t acc[32];
        tmem_ld32(tmem + ((uint32_t)lane_base << 16) + (uint32_t)col_base, acc);
        if (r < t.nr) {
            int32_t* out = a.out + j.out_off + (int64_t)(t.r0 + r) * j.n_cols + t.c0;
#pragma unroll
            for (int q = 0; q < 32; q++) {
                const int c = col_base + q;
                if (acc[q] && t.c0 + c < t.c1) atomicAdd(out + c, (int32_t)acc[q]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcN));
}

}  // namespace

int launch_count_i8(const CountArgs& a, cudaStream_t s) {
    if (a.n_tiles <= 0) return TFIM_OK;
    static std::atomic<bool> configured[64];
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !configured[dev].load()) {
        TFIM_CUDA(cudaFuncSetAttribute(k_count_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
        configured[dev].store(true);
    }
    k_count_i8<<<a.n_tiles, kTcThreads, kTcSmem, s>>>(a);
    TFIM_CUDA(cudaGetLastError());
    return TFIM_OK;
}

int count_i8_status(bool reset) {
    int v = 0;
    TFIM_CUDA(cudaMemcpyFromSymbol(&v, g_tc_status, sizeof v));
    if (reset && v) {
        const int z = 0;
        TFIM_CUDA(cudaMemcpyToSymbol(g_tc_status, &z, sizeof z));
    }
    TFIM_CHECK(v == 0, TFIM_E_TIMEOUT, "tensor-memory counter: an mbarrier wait expired");
    return TFIM_OK;
}

}  // namespace tfim
