// All frequent itemsets, level by level, on the counting contract.
//
// The reference's level-wise prototype (code/batch_proto/batch_proto.cu:257-409) mines every
// frequent itemset (not only the maximal ones): F1 from the item rows' popcounts, then per
// level every frequent (k-1)-itemset is a prefix whose mask is counted against all items,
// and the extensions j > its last item with support >= minsup are the frequent k-itemsets
// (canonical extension, each itemset generated once).  This is the same search on the
// library's counting pipeline: prefix masks from the item lists, the automatically chosen
// counter (LOP3 / b1 / tcgen05 kind::i8), and a device-side compaction that returns only the
// frequent extensions of each prefix.
#include <algorithm>
#include <chrono>
#include <cstring>

#include "tfim_internal.h"

namespace tfim {
namespace {

// One warp per prefix row: the number of columns j > last item of the prefix with
// counts[row][j] >= min_count.
__global__ void k_ext_count(const int32_t* __restrict__ counts, int32_t b, int32_t d, int32_t min_count,
                            const MatDesc* __restrict__ mats, const int32_t* __restrict__ items, int32_t* __restrict__ n_ext) {
    const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= b) return;
    const MatDesc m = mats[row];
    const int32_t last = m.n > 0 ? items[m.off + m.n - 1] : -1;
    const int32_t* cr = counts + row * (int64_t)d;
    int n = 0;
    for (int32_t j = last + 1 + lane; j < d; j += 32) n += cr[j] >= min_count;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if (lane == 0) n_ext[row] = n;
}

// Second pass: the (column, support) entries of each row at its offset, in column order.
__global__ void k_ext_write(const int32_t* __restrict__ counts, int32_t b, int32_t d, int32_t min_count,
                            const MatDesc* __restrict__ mats, const int32_t* __restrict__ items,
                            const int64_t* __restrict__ off, int2* __restrict__ out) {
    const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= b) return;
    const MatDesc m = mats[row];
    const int32_t last = m.n > 0 ? items[m.off + m.n - 1] : -1;
    const int32_t* cr = counts + row * (int64_t)d;
    int64_t pos = off[row];
    for (int32_t j0 = last + 1; j0 < d; j0 += 32) {
        const int32_t j = j0 + lane;
        const int32_t v = j < d ? cr[j] : 0;
        const bool e = j < d && v >= min_count;
        const unsigned bal = __ballot_sync(0xffffffffu, e);
        if (e) out[pos + __popc(bal & ((1u << lane) - 1u))] = make_int2(j, v);
        pos += __popc(bal);
    }
}

}  // namespace
}  // namespace tfim

using namespace tfim;

extern "C" {

int tfim_mine_all(tfim_ctx* c, int32_t min_count, int32_t max_len, int64_t max_itemsets, tfim_mine_stats* stats) {
    TFIM_CHECK(c, TFIM_E_INVALID, "null context");
    TFIM_CHECK(min_count >= 1, TFIM_E_INVALID, "min_count must be at least 1");
    TFIM_CHECK(max_len >= 1 && max_len <= kMaxListLen + 1, TFIM_E_DEPTH, "max_len %d outside 1..%d", max_len,
               kMaxListLen + 1);
    TFIM_CHECK(max_itemsets >= 1, TFIM_E_INVALID, "max_itemsets must be at least 1");
    TFIM_CUDA(cudaSetDevice(c->device));
    const auto t0 = std::chrono::steady_clock::now();
    tfim_mine_stats st;
    memset(&st, 0, sizeof st);
    cudaStream_t s = c->stream;
    const int32_t d = c->n_counted;
    MfiSet& A = c->all_fis;
    A.clear();
    c->all_mined = false;
    // level 1: the counted items frequent by bitmap support
    std::vector<int32_t> cur;   // flat (k-1)-itemsets of the current level, ascending dense ids
    for (int32_t e = 0; e < d; e++)
        if (c->bit_support[e] >= min_count) {
            A.add(&e, 1, c->bit_support[e]);
            cur.push_back(e);
        }
    TFIM_CHECK((int64_t)A.size() <= max_itemsets, TFIM_E_NOMEM, "more than %lld frequent itemsets", (long long)max_itemsets);
    // prefixes per wave: at most 4096, and their masks within 1 GiB
    const int64_t mask_bytes = c->W * 4;
    const int32_t wave_cap = (int32_t)std::max<int64_t>(1, std::min<int64_t>(4096, (1LL << 30) / std::max<int64_t>(mask_bytes, 1)));
    DevBuf &d_items = c->d_scratch[3], &d_counts = c->d_scratch[4], &d_aux = c->d_scratch[5], &d_ent = c->d_scratch[6];
    HostBuf &h_in = c->h_scratch[2], &h_out = c->h_scratch[3];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TFIM_CUDA(cudaEventCreate(&e0));
    TFIM_CUDA(cudaEventCreate(&e1));
    int rc = TFIM_OK;
    bool any_i8 = false;
    for (int32_t k = 2; k <= max_len && !cur.empty() && rc == TFIM_OK; k++) {
        const int32_t plen = k - 1;
        const int64_t n_pref = (int64_t)cur.size() / plen;
        std::vector<int32_t> next;
        for (int64_t p0 = 0; p0 < n_pref && rc == TFIM_OK; p0 += wave_cap) {
            const int32_t b = (int32_t)std::min<int64_t>(wave_cap, n_pref - p0);
            // items and mask descriptors, one pinned upload
            const size_t o_mats = (((size_t)b * plen * 4) + 15) & ~size_t(15);
            const size_t up = o_mats + (size_t)b * sizeof(MatDesc);
            if ((rc = h_in.reserve(up)) || (rc = d_items.reserve(up))) break;
            unsigned char* hp = h_in.as<unsigned char>();
            memcpy(hp, cur.data() + p0 * plen, (size_t)b * plen * 4);
            MatDesc* hm = (MatDesc*)(hp + o_mats);
            for (int32_t i = 0; i < b; i++) hm[i] = MatDesc{i, -1, i * plen, plen};
            const int32_t* di = d_items.as<int32_t>();
            const MatDesc* dm = (const MatDesc*)(d_items.as<unsigned char>() + o_mats);
            if (cudaMemcpyAsync(d_items.p, hp, up, cudaMemcpyHostToDevice, s) != cudaSuccess) { rc = TFIM_E_CUDA; break; }
            if ((rc = d_counts.reserve((size_t)b * d * 4)) || (rc = d_aux.reserve((size_t)b * 4 + (size_t)(b + 1) * 8 + 16))) break;
            int32_t* dc = d_counts.as<int32_t>();
            int32_t* dn = d_aux.as<int32_t>();   // nfreq of the count call, then the extension counts
            int64_t* doff = (int64_t*)(d_aux.as<unsigned char>() + (((size_t)b * 4 + 15) & ~size_t(15)));
            cudaEventRecord(e0, s);
            if ((rc = count_wave_impl(c, b, min_count, di, dm, dc, dn, s))) break;
            any_i8 |= c->used_i8;
            cudaEventRecord(e1, s);
            const unsigned grid = (unsigned)(((int64_t)b * 32 + 255) / 256);
            k_ext_count<<<grid, 256, 0, s>>>(dc, b, d, min_count, dm, di, dn);
            // extension counts -> offsets (host scan) -> entries
            if ((rc = h_out.reserve((size_t)(b + 1) * 8))) break;
            int32_t* hn = h_out.as<int32_t>();
            if (cudaMemcpyAsync(hn, dn, (size_t)b * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) { rc = TFIM_E_CUDA; break; }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            st.kernel_ms += ms;
            std::vector<int64_t> off((size_t)b + 1, 0);
            for (int32_t i = 0; i < b; i++) off[i + 1] = off[i] + hn[i];
            const int64_t n_new = off[b];
            if ((int64_t)A.size() + n_new > max_itemsets) {
                set_error("more than %lld frequent itemsets (level %d)", (long long)max_itemsets, k);
                rc = TFIM_E_NOMEM;
                break;
            }
            st.waves++;
            st.count_launches++;
            st.nodes += b;
            st.supports += (int64_t)b * d;
            if (n_new == 0) continue;
            if ((rc = d_ent.reserve((size_t)n_new * sizeof(int2))) || (rc = h_out.reserve((size_t)n_new * sizeof(int2)))) break;
            if (cudaMemcpyAsync(doff, off.data(), off.size() * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) { rc = TFIM_E_CUDA; break; }
            k_ext_write<<<grid, 256, 0, s>>>(dc, b, d, min_count, dm, di, doff, d_ent.as<int2>());
            const int2* he = h_out.as<int2>();
            if (cudaMemcpyAsync((void*)he, d_ent.p, (size_t)n_new * sizeof(int2), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) { rc = TFIM_E_CUDA; break; }
            std::vector<int32_t> buf((size_t)k);
            for (int32_t i = 0; i < b; i++) {
                const int32_t* pre = cur.data() + (p0 + i) * plen;
                for (int64_t q = off[i]; q < off[i + 1]; q++) {
                    memcpy(buf.data(), pre, (size_t)plen * 4);
                    buf[plen] = he[q].x;
                    A.add(buf.data(), (size_t)k, he[q].y);
                    next.insert(next.end(), buf.begin(), buf.end());
                }
            }
        }
        cur.swap(next);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == TFIM_OK && any_i8) rc = count_i8_status(true);
    if (rc != TFIM_OK) {
        if (rc == TFIM_E_CUDA) set_error("all-itemset mining: %s", cudaGetErrorString(cudaGetLastError()));
        A.clear();
        return rc;
    }
    st.n_mfi = (int64_t)A.size();
    st.bit_ops = st.supports * c->n_bits;
    st.mine_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    st.device_ms = st.mine_seconds * 1e3;
    c->all_mined = true;
    if (stats) *stats = st;
    return TFIM_OK;
}

int64_t tfim_num_all(const tfim_ctx* c) { return c && c->all_mined ? (int64_t)c->all_fis.size() : -1; }

int64_t tfim_all_item_total(const tfim_ctx* c) { return c && c->all_mined ? (int64_t)c->all_fis.items.size() : -1; }

int tfim_get_all(const tfim_ctx* c, int32_t* items, int64_t* offsets, int32_t* supports) {
    TFIM_CHECK(c && items && offsets && supports, TFIM_E_INVALID, "null argument");
    TFIM_CHECK(c->all_mined, TFIM_E_STATE, "tfim_get_all before tfim_mine_all");
    const MfiSet& A = c->all_fis;
    const int32_t* map = c->dense_to_orig.data();
    for (size_t q = 0; q < A.items.size(); q++) items[q] = map[A.items[q]];
    std::copy(A.off.begin(), A.off.end(), offsets);
    std::copy(A.sup.begin(), A.sup.end(), supports);
    return TFIM_OK;
}

}  // extern "C"
