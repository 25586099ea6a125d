// Allocation-free counting: tfim_count_wave_noalloc.
//
// Some callers cannot allocate GPU memory at all: code that runs inside a memory
// budget owned by someone else (an allocator that hands out every byte of a device up
// front, so a cudaMalloc from a library would fail or steal from it), and callers that
// only hold device pointers they were given.  For them this entry
// point does the counting contract of tfim_count_wave_device without a context and
// without any allocation: the caller passes the bitmap, the item lists and the output
// buffers, and the per-node prefix masks (the only scratch the count needs) live in a
// fixed file-scope device array.
//
// That array is a static __device__ object: every GPU that loads the library holds its
// kTfimStaticScratchBytes until the process exits, all calls on a device share it, and
// it keeps whatever the last call wrote.  Calls whose work overlaps on the GPU (for
// example on two streams) race on it.  Host code cannot use the array's name as a
// device address; its address is looked up with cudaGetSymbolAddress once per device,
// by the first call made with that device current.
#include <algorithm>
#include <mutex>

#include "tfim_internal.h"

namespace tfim {
namespace {

constexpr size_t kTfimStaticScratchBytes = 16u << 20;   // 16 MiB of prefix masks per device

__device__ __align__(256) uint32_t g_static_scratch[kTfimStaticScratchBytes / 4];

std::mutex g_static_mu;
uint32_t* g_static_ptr[64] = {};
int g_static_sms[64] = {};

// The scratch array's device address and the SM count of device `dev` (current), looked
// up once per device.
int static_scratch(int dev, uint32_t** out, int* sms) {
    TFIM_CHECK(dev >= 0 && dev < 64, TFIM_E_INVALID, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[dev]) {
        int n_sm = 0;
        TFIM_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error("cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev, cudaGetErrorString(e));
            return TFIM_E_CUDA;
        }
        g_static_sms[dev] = n_sm > 0 ? n_sm : 1;
        g_static_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_static_ptr[dev];
    *sms = g_static_sms[dev];
    return TFIM_OK;
}

__device__ __forceinline__ uint4 and4s(uint4 a, uint4 b) { return make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w); }
__device__ __forceinline__ uint32_t popc4s(uint4 a) { return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w); }

// masks[i] = AND of the rows listed for node i (all ones for an empty list).
// grid = (word blocks, b)
__global__ void k_static_masks(const uint32_t* __restrict__ B, int64_t W, const int32_t* __restrict__ items,
                               const int64_t* __restrict__ offs, uint32_t* __restrict__ masks) {
    const int i = blockIdx.y;
    const int64_t q0 = offs[i], q1 = offs[i + 1];
    const int64_t W4 = W >> 2;
    uint4* dst = reinterpret_cast<uint4*>(masks + (int64_t)i * W);
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < W4; w += (int64_t)gridDim.x * blockDim.x) {
        uint4 v = make_uint4(~0u, ~0u, ~0u, ~0u);
        for (int64_t q = q0; q < q1; q++) v = and4s(v, __ldg(reinterpret_cast<const uint4*>(B + (int64_t)items[q] * W) + w));
        dst[w] = v;
    }
}

constexpr int kStaticRows = 8;     // nodes per block
constexpr int kStaticChunk = 1024; // words staged per step

// grid = (ceil(d/64), ceil(b/8), word slices); counts[i*d + e] += popc(mask_i & B[e]) over
// the block's word slice.  Shared memory: kStaticRows x kStaticChunk words (32 KiB).
__global__ void __launch_bounds__(256) k_static_count(const uint32_t* __restrict__ B, int64_t W,
                                                      const uint32_t* __restrict__ masks, int32_t b, int32_t d,
                                                      int64_t wslice, int32_t* __restrict__ counts) {
    __shared__ uint4 sm4[kStaticRows * kStaticChunk / 4];
    const int c0 = blockIdx.x * 64, c1 = min(d, c0 + 64);
    const int n0 = blockIdx.y * kStaticRows, nr = min(kStaticRows, b - n0);
    const int64_t w0 = blockIdx.z * wslice, w1 = min(W, w0 + wslice);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t cw = w0; cw < w1; cw += kStaticChunk) {
        const int64_t w4b = cw >> 2;
        const int nw4 = (int)((min(w1, cw + kStaticChunk) - cw) >> 2);
        __syncthreads();
        for (int r = 0; r < nr; r++) {
            const uint4* src = reinterpret_cast<const uint4*>(masks + (int64_t)(n0 + r) * W) + w4b;
            for (int w = threadIdx.x; w < nw4; w += blockDim.x) sm4[r * nw4 + w] = src[w];
        }
        __syncthreads();
        for (int c = c0 + warp; c < c1; c += 8) {
            const uint4* cp = reinterpret_cast<const uint4*>(B + (int64_t)c * W) + w4b;
            uint32_t acc[kStaticRows];
#pragma unroll
            for (int r = 0; r < kStaticRows; r++) acc[r] = 0;
            for (int w = lane; w < nw4; w += 32) {
                const uint4 v = __ldg(cp + w);
#pragma unroll
                for (int r = 0; r < kStaticRows; r++)
                    if (r < nr) acc[r] += popc4s(and4s(sm4[r * nw4 + w], v));
            }
#pragma unroll
            for (int r = 0; r < kStaticRows; r++) {
                if (r >= nr) break;
                uint32_t v = acc[r];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0 && v) atomicAdd(counts + (int64_t)(n0 + r) * d + c, (int32_t)v);
            }
        }
    }
}

}  // namespace
}  // namespace tfim

using namespace tfim;

extern "C" int tfim_count_wave_noalloc(const uint32_t* d_bitmap, int64_t words_per_row, int32_t n_counted,
                                       const int32_t* d_item_lists, const int64_t* d_list_offsets, int32_t b,
                                       int32_t min_count, int32_t* d_counts_out, int32_t* d_nfreq_out, void* stream) {
    TFIM_CHECK(d_bitmap && d_list_offsets && d_counts_out && d_nfreq_out && b >= 0 && n_counted >= 0, TFIM_E_INVALID,
               "tfim_count_wave_noalloc: invalid arguments");
    TFIM_CHECK(words_per_row > 0 && words_per_row % 4 == 0, TFIM_E_INVALID,
               "tfim_count_wave_noalloc: words_per_row must be a positive multiple of 4 (got %lld)", (long long)words_per_row);
    TFIM_CHECK(((uintptr_t)d_bitmap & 15) == 0, TFIM_E_INVALID, "tfim_count_wave_noalloc: bitmap must be 16-byte aligned");
    if (b == 0) return TFIM_OK;
    TFIM_CHECK(b <= 65535, TFIM_E_INVALID, "tfim_count_wave_noalloc: at most 65535 nodes per call (got %d)", b);
    const size_t need = (size_t)b * (size_t)words_per_row * 4;
    TFIM_CHECK(need <= kTfimStaticScratchBytes, TFIM_E_INVALID,
               "tfim_count_wave_noalloc: %d nodes x %lld words need %zu bytes of prefix masks; the static scratch holds %zu "
               "(split the wave)", b, (long long)words_per_row, need, kTfimStaticScratchBytes);
    int dev = 0;
    TFIM_CUDA(cudaGetDevice(&dev));
    uint32_t* scratch = nullptr;
    int sms = 1;
    TFIM_TRY(static_scratch(dev, &scratch, &sms));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t W = words_per_row;
    if (n_counted > 0) TFIM_CUDA(cudaMemsetAsync(d_counts_out, 0, (size_t)b * n_counted * 4, s));
    {
        int64_t bx = (W / 4 + 255) / 256;
        if (bx > 64) bx = 64;
        k_static_masks<<<dim3((unsigned)bx, (unsigned)b), 256, 0, s>>>(d_bitmap, W, d_item_lists, d_list_offsets, scratch);
        TFIM_CUDA(cudaGetLastError());
    }
    if (n_counted > 0) {
        const int64_t gx = (n_counted + 63) / 64, gy = (b + kStaticRows - 1) / kStaticRows;
        // about 8 blocks per SM over the word slices
        int64_t slices = std::max<int64_t>(1, (8LL * sms + gx * gy - 1) / (gx * gy));
        slices = std::min<int64_t>(slices, std::max<int64_t>(1, W / 256));
        const int64_t wslice = ((W / 4 + slices - 1) / slices) * 4;
        const int64_t gz = (W + wslice - 1) / wslice;
        k_static_count<<<dim3((unsigned)gx, (unsigned)gy, (unsigned)gz), 256, 0, s>>>(d_bitmap, W, scratch, b, n_counted,
                                                                                   wslice, d_counts_out);
        TFIM_CUDA(cudaGetLastError());
    }
    return launch_nfreq(d_counts_out, b, n_counted, min_count, d_nfreq_out, s);
}
