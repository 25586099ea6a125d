// MFI search drivers.
//
// PLAIN: the reference's search exactly (code/engine/src/kernel_bitmap.cu:841-894):
//   roots = the first dimensionReduced items in frequency order, a LIFO of nodes, and
//   per node one count of every survivor; a node X is an MFI iff the number of
//   survivors e with sup(X+e) >= threshold equals |X|, else X+{i} is pushed for every
//   dense i < progress(X) with sup >= threshold.  One node is counted per launch, like
//   getResFrequencyCuda (:451-536).
//
// BATCHED: a pruned search whose output set is provably the reference's:
//   The reference outputs {X : X maximal among frequent itemsets over the counted
//   items, and max dense id of X is a root} (its MFI test is a local maximality test,
//   and X is visited iff X is frequent and its largest dense id is a root).  This engine
//   enumerates all maximal frequent itemsets over the counted items with
//     * candidate restriction: a node counts only F(parent) (items frequent with its
//       parent); an item outside F(parent) cannot extend any descendant, so the local
//       maximality test over F(parent) equals the reference's test over all survivors;
//     * dynamic tail order (increasing support);
//     * equal-support pruning: if sup(X+e) == sup(X), e belongs to every maximal
//       superset of X: e joins X when e is in X's tail, otherwise X's subtree holds no
//       maximal set;
//     * head-union-tail lookahead: if X + tail(X) is frequent it is the only candidate of
//       the subtree and one count decides it;
//   then keeps those whose largest dense id is a root.  Counting happens in waves: the
//   children of a node X form a family whose counts are one masked Gram block
//   popc(mask(X) & B[t] & B[e]) for t in tail(X), e in F(X); many families, split into
//   tiles, go into one launch per counter.
//   The reference quirk for a frequent original id 0 (parked dense id, a root whose MFI
//   test counts it differently) is reproduced by running the PLAIN search on that one root.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <numeric>

#include "tfim_internal.h"

namespace tfim {
namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// packs descriptor sections into one pinned host buffer and one device buffer
struct Packer {
    std::vector<unsigned char> h;
    size_t add(const void* p, size_t bytes) {
        size_t off = (h.size() + 15) & ~size_t(15);
        h.resize(off + bytes);
        if (bytes) memcpy(h.data() + off, p, bytes);
        return off;
    }
};

struct SlotPool {
    std::vector<int32_t> free_list;
    std::vector<int32_t> deferred;   // freed this wave; reusable after the next launch batch
    int32_t n = 0;
    int32_t cap = 0;
    int grow(tfim_ctx* c, int32_t need) {
        if (need <= cap) return TFIM_OK;
        int32_t ncap = std::max<int32_t>(need, std::max<int32_t>(64, cap * 2));
        DevBuf nb;
        nb.stream = c->stream;
        TFIM_TRY(nb.reserve((size_t)ncap * (size_t)c->W * 4));
        if (c->d_masks.p && cap > 0)
            TFIM_CUDA(cudaMemcpyAsync(nb.p, c->d_masks.p, (size_t)cap * (size_t)c->W * 4, cudaMemcpyDeviceToDevice, c->stream));
        c->d_masks.release();   // stream-ordered: after the copy
        c->d_masks = nb;
        cap = ncap;
        return TFIM_OK;
    }
    int alloc(tfim_ctx* c, int32_t* out) {
        if (!free_list.empty()) { *out = free_list.back(); free_list.pop_back(); return TFIM_OK; }
        TFIM_TRY(grow(c, n + 1));
        *out = n++;
        return TFIM_OK;
    }
    void reset(tfim_ctx* c) {
        free_list.clear();
        deferred.clear();
        n = 0;
        cap = c->W > 0 ? (int32_t)std::min<size_t>(c->d_masks.bytes / ((size_t)c->W * 4), INT32_MAX) : 0;
    }
    void release(int32_t s) { if (s >= 0) deferred.push_back(s); }
    void flush() { free_list.insert(free_list.end(), deferred.begin(), deferred.end()); deferred.clear(); }
};

}  // namespace

// Tile builders --------------------------------------------------------------------------
// `upper`: the job's rows and columns are the same list; only tiles holding some (i, j>=i)
// are emitted and the mirror pass fills the rest.
void tiles_lop3(int32_t job, int32_t nr, int32_t nc, int64_t W, int64_t wslice, std::vector<TileDesc>& out,
                bool upper) {
    for (int32_t r0 = 0; r0 < nr; r0 += kLop3Rows)
        for (int32_t c0 = 0; c0 < nc; c0 += 64)
            for (int64_t w0 = 0; w0 < W; w0 += wslice) {
                if (upper && std::min(nc, c0 + 64) <= r0) continue;
                TileDesc t;
                t.job = job; t.r0 = r0; t.nr = std::min(kLop3Rows, nr - r0);
                t.c0 = c0; t.c1 = std::min(nc, c0 + 64);
                t.w0 = (int32_t)w0; t.w1 = (int32_t)std::min<int64_t>(W, w0 + wslice);
                t.pad = 0;
                out.push_back(t);
            }
}
void tiles_b1(int32_t job, int32_t nr, int32_t nc, int64_t W, int64_t kslice, std::vector<TileDesc>& out,
              bool upper) {
    for (int64_t w0 = 0; w0 < W; w0 += kslice)
        for (int32_t r0 = 0; r0 < nr; r0 += kB1Rows)
            for (int32_t c0 = 0; c0 < nc; c0 += kB1Cols) {
                if (upper && std::min(nc, c0 + kB1Cols) <= r0) continue;
                TileDesc t;
                t.job = job; t.r0 = r0; t.nr = std::min(kB1Rows, nr - r0);
                t.c0 = c0; t.c1 = std::min(nc, c0 + kB1Cols);
                t.w0 = (int32_t)w0; t.w1 = (int32_t)std::min<int64_t>(W, w0 + kslice);
                t.pad = 0;
                out.push_back(t);
            }
}

namespace {

// A wave of count jobs, ready to upload.
struct Wave {
    std::vector<JobDesc> jobs;
    std::vector<RowDesc> rows;
    std::vector<int32_t> cols;
    std::vector<int32_t> row_job, row_local;
    std::vector<MatDesc> mats;
    std::vector<int32_t> mat_items;
    std::vector<char> use_b1;    // per job
    int64_t out_total = 0;
    int64_t supports = 0;
    // the family of the empty prefix (rows == columns): counted as a symmetric bitmap Gram
    // (top_mode 1) or by pair co-occurrence over the reduced transaction list (top_mode 2)
    int32_t top_job = -1;
    int32_t top_mode = 0;
    std::vector<int32_t> top_pos;    // dense id -> position in the family's list, or -1
    std::vector<int32_t> top_diag;   // the diagonal: bitmap supports in list order
    void clear() {
        jobs.clear(); rows.clear(); cols.clear(); row_job.clear(); row_local.clear();
        mats.clear(); mat_items.clear(); use_b1.clear(); out_total = 0; supports = 0;
        top_job = -1; top_mode = 0; top_pos.clear(); top_diag.clear();
    }
    int32_t add_job(int32_t base_slot, int32_t base_item, const std::vector<RowDesc>& rs, const std::vector<int32_t>& cs, bool b1) {
        JobDesc j;
        j.base_slot = base_slot; j.base_item = base_item;
        j.n_rows = (int32_t)rs.size(); j.n_cols = (int32_t)cs.size();
        j.row_off = (int32_t)rows.size(); j.col_off = (int32_t)cols.size();
        j.out_off = out_total;
        j.self_col = -1;   // a -1 column id is the all-ones column: tell the counters its index
        for (int32_t q = 0; q < j.n_cols; q++)
            if (cs[q] < 0) { j.self_col = q; break; }
        j.pad = 0;
        const int32_t id = (int32_t)jobs.size();
        jobs.push_back(j);
        use_b1.push_back(b1);
        rows.insert(rows.end(), rs.begin(), rs.end());
        cols.insert(cols.end(), cs.begin(), cs.end());
        for (int32_t r = 0; r < j.n_rows; r++) { row_job.push_back(id); row_local.push_back(r); }
        out_total += (int64_t)j.n_rows * j.n_cols;
        supports += (int64_t)j.n_rows * j.n_cols;
        return id;
    }
};

// Device-side execution of a wave: materialise masks, count, compact.  On return the
// host holds row_info (per global row: start,len) and the compacted entries.
struct WaveRunner {
    tfim_ctx* c;
    DevBuf d_desc, d_counts, d_entries, d_rowinfo;
    HostBuf h_desc, h_rowinfo, h_entries;
    std::vector<int2> row_info;
    std::vector<Entry> entries;
    int64_t launches = 0;
    int64_t count_launches = 0;
    int64_t bytes_alg = 0;
    double kernel_ms = 0;
    double sync_ms = 0;
    int32_t counter = TFIM_COUNTER_AUTO;
    int sm_count = 148;
    // per counting path (TFIM_PATH_*): device time, algorithmic bytes, bit-ops, supports, launches
    double path_ms[6] = {};
    int64_t path_bytes[6] = {}, path_bitops[6] = {}, path_supports[6] = {}, path_launches[6] = {};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};   // before pairs, lop3, b1; after b1

    void reset_counters() {
        launches = 0;
        count_launches = 0;
        bytes_alg = 0;
        kernel_ms = 0;
        sync_ms = 0;
        for (int q = 0; q < 6; q++) {
            path_ms[q] = 0;
            path_bytes[q] = path_bitops[q] = path_supports[q] = path_launches[q] = 0;
        }
    }
    void add_to(tfim_mine_stats* st) const {
        for (int q = 0; q < 6; q++) {
            st->path_ms[q] += path_ms[q];
            st->path_bytes[q] += path_bytes[q];
            st->path_bitops[q] += path_bitops[q];
            st->path_supports[q] += path_supports[q];
            st->path_launches[q] += path_launches[q];
        }
    }
    // device time of the wave's counting launches per path (the events of this wave are done)
    void read_path_times(bool pairs, bool l3, bool b1) {
        float ms = 0;
        if (pairs && cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) path_ms[TFIM_PATH_PAIRS] += ms;
        if (l3 && cudaEventElapsedTime(&ms, ev[1], ev[2]) == cudaSuccess) path_ms[TFIM_PATH_LOP3] += ms;
        if (b1 && cudaEventElapsedTime(&ms, ev[2], ev[3]) == cudaSuccess) path_ms[TFIM_PATH_B1] += ms;
        if (cudaEventElapsedTime(&ms, ev[0], ev[3]) == cudaSuccess) kernel_ms += ms;
    }

    int run(Wave& w, int32_t min_count, bool want_full_counts, std::vector<int32_t>* full_counts) {
        const int64_t W = c->W;
        const tfim_tuning tn = tuning();
        std::vector<TileDesc> t_l3, t_b1;
        // split-k factor for tensor tiles: enough tiles to cover the SMs a few times
        int64_t base_b1 = 0;
        for (size_t j = 0; j < w.jobs.size(); j++)
            if (w.use_b1[j] && !((int32_t)j == w.top_job && w.top_mode == 2))
                base_b1 += (int64_t)((w.jobs[j].n_rows + kB1Rows - 1) / kB1Rows) * ((w.jobs[j].n_cols + kB1Cols - 1) / kB1Cols);
        // word slices of CUDA-core tiles: whole rows when the wave has many tiles already
        int64_t base_l3 = 0;
        for (size_t j = 0; j < w.jobs.size(); j++)
            if (!w.use_b1[j] && !((int32_t)j == w.top_job && w.top_mode == 2))
                base_l3 += (int64_t)((w.jobs[j].n_rows + kLop3Rows - 1) / kLop3Rows) * ((w.jobs[j].n_cols + 63) / 64);
        int64_t wslice = W;
        if (base_l3 > 0) {
            const int64_t want = (int64_t)(tn.l3_slices_per_sm * sm_count);
            int64_t ks = std::max<int64_t>(1, (want + base_l3 - 1) / base_l3);
            ks = std::min<int64_t>(ks, std::max<int64_t>(1, W / 256));
            wslice = ((W / 64 + ks - 1) / ks) * 64;
        }
        int64_t kslice = W;
        if (base_b1 > 0) {
            const int64_t want = (int64_t)(tn.b1_tiles_per_sm * sm_count);
            int64_t ks = std::max<int64_t>(1, (want + base_b1 - 1) / base_b1);
            ks = std::min<int64_t>(ks, W / 64);
            kslice = ((W / 64 + ks - 1) / ks) * 64;
        }
        const int64_t row_bytes = (c->n_bits + 7) / 8;
        for (size_t j = 0; j < w.jobs.size(); j++) {
            const JobDesc& jd = w.jobs[j];
            const int64_t sup = (int64_t)jd.n_rows * jd.n_cols;
            if ((int32_t)j == w.top_job && w.top_mode == 2) {
                // pair counting reads the reduced transaction list and writes the matrix
                const int64_t by = (c->d_red_off ? (c->n_bits + 1) * 8 + c->n_red_items * 4 : 0) + 4LL * sup;
                bytes_alg += by;
                path_bytes[TFIM_PATH_PAIRS] += by;
                path_supports[TFIM_PATH_PAIRS] += sup;
                continue;
            }
            const int64_t base_rows = (jd.base_slot >= 0) + (jd.base_item >= 0);
            const int64_t by = row_bytes * (jd.n_rows + jd.n_cols + base_rows) + 4LL * sup;
            const int q = w.use_b1[j] ? TFIM_PATH_B1 : TFIM_PATH_LOP3;
            bytes_alg += by;
            path_bytes[q] += by;
            path_bitops[q] += sup * c->n_bits;
            path_supports[q] += sup;
        }
        for (size_t j = 0; j < w.jobs.size(); j++) {
            const bool top = (int32_t)j == w.top_job;
            if (top && w.top_mode == 2) continue;
            if (w.use_b1[j]) tiles_b1((int32_t)j, w.jobs[j].n_rows, w.jobs[j].n_cols, W, kslice, t_b1, top);
            else tiles_lop3((int32_t)j, w.jobs[j].n_rows, w.jobs[j].n_cols, W, wslice, t_l3, top);
        }
        Packer pk;
        const size_t o_jobs = pk.add(w.jobs.data(), w.jobs.size() * sizeof(JobDesc));
        const size_t o_rows = pk.add(w.rows.data(), w.rows.size() * sizeof(RowDesc));
        const size_t o_cols = pk.add(w.cols.data(), w.cols.size() * 4);
        const size_t o_tl3 = pk.add(t_l3.data(), t_l3.size() * sizeof(TileDesc));
        const size_t o_tb1 = pk.add(t_b1.data(), t_b1.size() * sizeof(TileDesc));
        const size_t o_rj = pk.add(w.row_job.data(), w.row_job.size() * 4);
        const size_t o_rl = pk.add(w.row_local.data(), w.row_local.size() * 4);
        const size_t o_mat = pk.add(w.mats.data(), w.mats.size() * sizeof(MatDesc));
        const size_t o_mi = pk.add(w.mat_items.data(), w.mat_items.size() * 4);
        const size_t o_tpos = pk.add(w.top_pos.data(), w.top_pos.size() * 4);
        const size_t o_tdiag = pk.add(w.top_diag.data(), w.top_diag.size() * 4);
        const size_t o_ctr = pk.add(nullptr, 16);
        memset(pk.h.data() + o_ctr, 0, 16);
        TFIM_TRY(h_desc.reserve(pk.h.size()));
        TFIM_TRY(d_desc.reserve(pk.h.size()));
        memcpy(h_desc.p, pk.h.data(), pk.h.size());
        cudaStream_t s = c->stream;
        unsigned char* db = d_desc.as<unsigned char>();
        TFIM_CUDA(cudaMemcpyAsync(db, h_desc.p, pk.h.size(), cudaMemcpyHostToDevice, s));
        if (!w.mats.empty()) {
            TFIM_TRY(launch_materialize(c->d_bitmap, W, c->d_masks.as<uint32_t>(), (const MatDesc*)(db + o_mat),
                                        (const int32_t*)(db + o_mi), (int32_t)w.mats.size(), s));
            launches++;
        }
        const int64_t n_rows = (int64_t)w.row_job.size();
        if (w.jobs.empty()) {
            TFIM_CUDA(cudaStreamSynchronize(s));
            row_info.clear(); entries.clear();
            return TFIM_OK;
        }
        TFIM_TRY(d_counts.reserve((size_t)std::max<int64_t>(w.out_total, 1) * 4));
        TFIM_CUDA(cudaMemsetAsync(d_counts.p, 0, (size_t)w.out_total * 4, s));
        CountArgs a;
        a.bitmap = c->d_bitmap; a.W = W; a.masks = c->d_masks.as<uint32_t>();
        a.jobs = (const JobDesc*)(db + o_jobs); a.rows = (const RowDesc*)(db + o_rows);
        a.cols = (const int32_t*)(db + o_cols); a.out = d_counts.as<int32_t>();
        for (int q = 0; q < 4; q++)
            if (!ev[q]) TFIM_CUDA(cudaEventCreate(&ev[q]));
        const bool run_pairs = w.top_job >= 0 && w.top_mode == 2;
        TFIM_CUDA(cudaEventRecord(ev[0], s));
        if (run_pairs) {
            const JobDesc& tj = w.jobs[w.top_job];
            TFIM_TRY(launch_pair_count(c->d_red_off, c->d_red_items, c->n_bits, (const int32_t*)(db + o_tpos), tj.n_rows,
                                       d_counts.as<int32_t>() + tj.out_off, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_PAIRS]++;
        }
        TFIM_CUDA(cudaEventRecord(ev[1], s));
        if (!t_l3.empty()) {
            a.tiles = (const TileDesc*)(db + o_tl3); a.n_tiles = (int32_t)t_l3.size();
            TFIM_TRY(launch_count_lop3(a, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_LOP3]++;
        }
        TFIM_CUDA(cudaEventRecord(ev[2], s));
        if (!t_b1.empty()) {
            a.tiles = (const TileDesc*)(db + o_tb1); a.n_tiles = (int32_t)t_b1.size();
            TFIM_TRY(launch_count_b1(a, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_B1]++;
        }
        TFIM_CUDA(cudaEventRecord(ev[3], s));
        // a transaction-sharded context sums the partial counts of the whole wave over the group
        TFIM_TRY(group_reduce(c, d_counts.p, w.out_total, TFIM_DT_I32, TFIM_RED_SUM, s));
        if (w.top_job >= 0) {
            const JobDesc& tj = w.jobs[w.top_job];
            TFIM_TRY(launch_mirror(d_counts.as<int32_t>() + tj.out_off, tj.n_rows,
                                   w.top_mode == 2 ? (const int32_t*)(db + o_tdiag) : nullptr, s));
            launches++;
        }
        if (want_full_counts) {
            full_counts->resize(w.out_total);
            TFIM_CUDA(cudaMemcpyAsync(full_counts->data(), d_counts.p, (size_t)w.out_total * 4, cudaMemcpyDeviceToHost, s));
            const double ts0 = now_s();
            TFIM_CUDA(cudaStreamSynchronize(s));
            sync_ms += (now_s() - ts0) * 1e3;
            read_path_times(run_pairs, !t_l3.empty(), !t_b1.empty());
            return TFIM_OK;
        }
        // compact: entries >= min_count per row
        TFIM_TRY(d_entries.reserve((size_t)std::max<int64_t>(w.out_total, 1) * sizeof(Entry)));
        TFIM_TRY(d_rowinfo.reserve((size_t)(n_rows + 2) * sizeof(int2)));
        int32_t* d_ctr = (int32_t*)(d_rowinfo.as<int2>() + n_rows);
        TFIM_CUDA(cudaMemsetAsync(d_ctr, 0, 8, s));
        TFIM_TRY(launch_compact(d_counts.as<int32_t>(), a.jobs, (const int32_t*)(db + o_rj), (const int32_t*)(db + o_rl),
                                n_rows, min_count, d_entries.as<Entry>(), d_rowinfo.as<int2>(), d_ctr, s));
        launches++;
        TFIM_TRY(h_rowinfo.reserve((size_t)(n_rows + 2) * sizeof(int2)));
        TFIM_CUDA(cudaMemcpyAsync(h_rowinfo.p, d_rowinfo.p, (size_t)(n_rows + 1) * sizeof(int2), cudaMemcpyDeviceToHost, s));
        const double ts0 = now_s();
        TFIM_CUDA(cudaStreamSynchronize(s));
        sync_ms += (now_s() - ts0) * 1e3;
        read_path_times(run_pairs, !t_l3.empty(), !t_b1.empty());
        const int2* ri = h_rowinfo.as<int2>();
        const int32_t total = *(const int32_t*)(ri + n_rows);
        row_info.assign(ri, ri + n_rows);
        entries.resize(total);
        if (total > 0) {
            TFIM_TRY(h_entries.reserve((size_t)total * sizeof(Entry)));
            TFIM_CUDA(cudaMemcpyAsync(h_entries.p, d_entries.p, (size_t)total * sizeof(Entry), cudaMemcpyDeviceToHost, s));
            const double ts1 = now_s();
            TFIM_CUDA(cudaStreamSynchronize(s));
            sync_ms += (now_s() - ts1) * 1e3;
            memcpy(entries.data(), h_entries.p, (size_t)total * sizeof(Entry));
        }
        return TFIM_OK;
    }
    void release() {
        d_desc.release(); d_counts.release(); d_entries.release(); d_rowinfo.release();
        h_desc.release(); h_rowinfo.release(); h_entries.release();
        for (cudaEvent_t& e : ev)
            if (e) {
                cudaEventDestroy(e);
                e = nullptr;
            }
    }
};

struct MfiSink {
    tfim_ctx* c;
    std::vector<char> is_root;
    void emit(std::vector<int32_t> items, int32_t sup) {
        int32_t mx = -1;
        for (int32_t x : items) mx = std::max(mx, x);
        if (mx < 0 || !is_root[mx]) return;
        std::sort(items.begin(), items.end(), std::greater<int32_t>());
        if (items.size() == 1) sup = c->dense_freq[items[0]];   // a root's own frequency is its F1 count
        c->mfis.add(items.data(), items.size(), sup);
    }
};

}  // namespace

// Buffers that persist across tfim_mine calls on one context.
struct EngineState {
    WaveRunner wr;
    SlotPool pool;
};

void free_engine(EngineState* e) {
    if (!e) return;
    e->wr.release();
    delete e;
}

namespace {

// Features of a lookahead candidate (the learned proposal's input, 32 floats).
void lookahead_features(float* f, int head_n, const std::vector<std::pair<int32_t, int32_t>>& tail, int nF, int32_t supc,
                        int32_t minc, int64_t nbits, int n_eq, double pair_frac, int parent_tail, int row, bool top_child) {
    for (int q = 0; q < 32; q++) f[q] = 0.f;
    const int k = (int)tail.size();
    double mn = 1e30, mn2 = 1e30, mx = 0, sum = 0, sum2 = 0, logprod = 0;
    int gt90 = 0, gt99 = 0;
    for (auto& pr : tail) {
        const double r = (double)pr.second / (double)supc;
        if (r < mn) { mn2 = mn; mn = r; } else if (r < mn2) mn2 = r;
        mx = std::max(mx, r);
        sum += r;
        sum2 += r * r;
        logprod += std::log(std::max(r, 1e-12));
        gt90 += r > 0.9;
        gt99 += r > 0.99;
    }
    const double mean = k ? sum / k : 0, var = k ? std::max(0.0, sum2 / k - mean * mean) : 0;
    const double minc_d = std::max<int32_t>(1, minc);
    f[0] = head_n / 16.f;
    f[1] = k / 32.f;
    f[2] = nF / 64.f;
    f[3] = (float)((double)supc / (double)std::max<int64_t>(1, nbits));
    f[4] = (float)(std::log2(1.0 + supc) / 24.0);
    f[5] = (float)mn;
    f[6] = (float)mean;
    f[7] = (float)mx;
    f[8] = (float)(std::min(mn * supc / minc_d, 8.0) / 8.0);
    f[9] = (float)std::exp(logprod);
    f[10] = (float)(std::max(-8.0, std::min(8.0, logprod + std::log(supc / minc_d))) / 8.0);
    f[11] = (float)pair_frac;
    f[12] = (nF - k) / 64.f;
    f[13] = (float)(minc_d / (double)std::max<int64_t>(1, nbits));
    f[14] = (float)(std::min(supc / minc_d, 64.0) / 64.0);
    f[15] = (float)std::sqrt(var);
    f[16] = (float)(k > 1 ? mn2 : mn);
    f[17] = k ? (float)gt90 / k : 0.f;
    f[18] = k ? (float)gt99 / k : 0.f;
    f[19] = (float)(std::log2(1.0 + k) / 6.0);
    f[20] = n_eq / 8.f;
    f[21] = parent_tail / 64.f;
    f[22] = (float)row / (float)std::max(1, parent_tail);
    f[23] = top_child ? 1.f : 0.f;
}

EngineState& engine_state(tfim_ctx* c) {
    if (!c->engine) {
        c->engine = new EngineState();
        for (DevBuf* b : {&c->engine->wr.d_desc, &c->engine->wr.d_counts, &c->engine->wr.d_entries, &c->engine->wr.d_rowinfo})
            b->stream = c->stream;
    }
    c->engine->wr.c = c;
    c->engine->wr.reset_counters();
    c->engine->pool.reset(c);
    return *c->engine;
}

// The reference search for the given roots (pushed in the given order onto a LIFO).
int run_plain(tfim_ctx* c, const std::vector<int32_t>& roots, WaveRunner& wr, SlotPool& pool, tfim_mine_stats* st) {
    struct Node { std::vector<int32_t> items; int32_t freq; int32_t progress; };
    const int32_t d = c->n_counted;
    const int32_t minc = c->info.min_count;
    std::vector<Node> stack;
    for (int32_t r : roots) stack.push_back({{r}, c->dense_freq[r], r});
    std::vector<int32_t> counts;
    std::vector<int32_t> all_cols(d);
    std::iota(all_cols.begin(), all_cols.end(), 0);
    TFIM_TRY(pool.grow(c, 1));
    Wave w;
    while (!stack.empty()) {
        Node nd = std::move(stack.back());
        stack.pop_back();
        st->nodes++;
        w.clear();
        TFIM_CHECK(nd.items.size() <= (size_t)kMaxListLen, TFIM_E_DEPTH, "itemset depth %zu exceeds %d", nd.items.size(), kMaxListLen);
        MatDesc m;
        m.dst = 0; m.src = -1; m.off = 0; m.n = (int32_t)nd.items.size();
        w.mats.push_back(m);
        w.mat_items = nd.items;
        w.add_job(-1, -1, {RowDesc{0, -1}}, all_cols, false);
        TFIM_TRY(wr.run(w, minc, true, &counts));
        st->waves++;
        st->supports += d;
        int32_t cnt = 0;
        for (int32_t e = 0; e < d; e++) cnt += counts[e] >= minc;
        if ((size_t)cnt == nd.items.size()) {
            std::vector<int32_t> items = nd.items;
            std::sort(items.begin(), items.end(), std::greater<int32_t>());
            c->mfis.add(items.data(), items.size(), nd.freq);
            continue;
        }
        for (int32_t i = 0; i <= nd.progress - 1; i++) {
            if (counts[i] >= minc) {
                Node ch;
                ch.items = nd.items;
                ch.items.push_back(i);
                ch.freq = counts[i];
                ch.progress = i;
                stack.push_back(std::move(ch));
            }
        }
    }
    return TFIM_OK;
}

}  // namespace

int mine_plain(tfim_ctx* c, const tfim_mine_opts* o, tfim_mine_stats* st) {
    EngineState& es = engine_state(c);
    WaveRunner& wr = es.wr;
    wr.counter = TFIM_COUNTER_LOP3;
    int rc = run_plain(c, c->roots, wr, es.pool, st);
    st->launches += wr.launches;
    st->count_launches += wr.count_launches;
    st->bytes_alg += wr.bytes_alg;
    st->kernel_ms += wr.kernel_ms;
    st->sync_ms += wr.sync_ms;
    wr.add_to(st);
    return rc;
}

int mine_plain_roots(tfim_ctx* c, const std::vector<int32_t>& roots, tfim_mine_stats* st) {
    EngineState& es = engine_state(c);
    WaveRunner& wr = es.wr;
    wr.counter = TFIM_COUNTER_LOP3;
    int rc = run_plain(c, roots, wr, es.pool, st);
    st->launches += wr.launches;
    st->count_launches += wr.count_launches;
    st->bytes_alg += wr.bytes_alg;
    st->kernel_ms += wr.kernel_ms;
    st->sync_ms += wr.sync_ms;
    wr.add_to(st);
    return rc;
}

int mine_batched(tfim_ctx* c, const tfim_mine_opts* o, tfim_mine_stats* st) {
    const int32_t d = c->n_counted;
    const int32_t minc = c->info.min_count;
    const int64_t W = c->W;
    EngineState& es = engine_state(c);
    WaveRunner& wr = es.wr;
    SlotPool& pool = es.pool;
    wr.counter = o->counter;
    {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n > 0) wr.sm_count = n;
    }
    MfiSink sink;
    sink.c = c;
    sink.is_root.assign((size_t)c->info.n_dense + 1, 0);
    for (int32_t r : c->roots) sink.is_root[r] = 1;

    // the reference quirk for a frequent id 0 used as a root: run its search as-is
    int rc = TFIM_OK;
    if (c->info.n_dense > d) {
        const int32_t parked = d;
        if (sink.is_root[parked]) {
            rc = run_plain(c, {parked}, wr, pool, st);
            if (rc) return rc;
            pool.reset(c);
        }
    }

    struct Fam {
        int32_t slot = -1, item = -1;       // base mask
        std::vector<int32_t> head;
        std::vector<int32_t> F;             // columns
        std::vector<int32_t> T;             // tail rows, ordered
        int32_t next_row = 0;               // rows handed out so far
        int32_t rows_done = 0;              // rows whose results were processed
        bool waiting = false;               // a lookahead is pending
        bool dead = false;
    };
    // Invariant: F begins with T in the same order, so tail item T[i] is column i and an
    // item at column j is in the tail of row i's child iff i < j < |T|.
    struct Look {
        int32_t fam;                        // family it decides
        int32_t slot;                       // mask of head + tail
        std::vector<int32_t> cols;          // F \ T, then -1 (self)
        int64_t log = -1;                   // index into the outcome log
    };
    struct Cand {                           // a family that may get a lookahead
        int32_t fam;
        int32_t src_slot, src_item, t;      // its mask = masks[src_slot] & B[src_item] & B[t]
        float feat[32];
    };
    std::vector<Cand> cands;
    std::vector<float> probs;
    c->la_feats.clear();
    c->la_labels.clear();
    std::deque<Fam> fams;   // stable references while children are appended
    std::vector<int32_t> stack;             // family ids, top = back
    std::vector<Look> looks_pending;        // issued with the next wave
    const tfim_tuning tn = tuning();
    const int32_t wave_cap = o->wave_cap > 0 ? o->wave_cap : tn.wave_rows;
    const int32_t la_mode = o->lookahead;   // 0 off, 1 filtered, 2 learned, 3 every node
    const bool lookahead = la_mode != 0;
    TFIM_CHECK(la_mode != 2 || c->proposal, TFIM_E_STATE, "lookahead mode 2 needs a proposal network (tfim_set_proposal)");

    // top-level family: P = {}, F = T = counted items that are frequent by bitmap support
    {
        Fam f;
        for (int32_t e = 0; e < d; e++)
            if (c->bit_support[e] >= minc) f.F.push_back(e);
        std::stable_sort(f.F.begin(), f.F.end(), [&](int32_t a, int32_t b) { return c->bit_support[a] < c->bit_support[b]; });
        f.T = f.F;
        if (!f.T.empty()) {
            fams.push_back(std::move(f));
            stack.push_back(0);
        }
    }
    // how the family of the empty prefix is counted (whole, in the first wave)
    int32_t top_mode = 0;
    if (!fams.empty()) {
        const double nF = (double)fams[0].F.size();
        const bool fits = nF * nF * 4.0 <= (double)(1LL << 32);
        const bool b1 = wr.counter != TFIM_COUNTER_LOP3 &&
                        (wr.counter == TFIM_COUNTER_TENSOR || (nF >= tn.b1_min_rows && nF >= tn.b1_min_cols));
        const double bit_rate = b1 ? tn.rate_b1_bitops : tn.rate_lop3_bitops;
        const double bitmap_s = nF * nF * (double)c->n_bits_total / 2.0 / bit_rate;
        const double pairs_s = c->red_pair_work / 2.0 / tn.rate_pair_incr + nF * nF * 4.0 / kTuneHbmBytes;
        if (fits) {
            if (o->top_counter == 1) top_mode = 1;
            else if (o->top_counter == 2) top_mode = c->csr_exact ? 2 : 1;
            else top_mode = (c->csr_exact && pairs_s < bitmap_s) ? 2 : 1;
        }
    }
    auto use_b1_for = [&](int32_t nr, int32_t nc) {
        if (wr.counter == TFIM_COUNTER_LOP3) return false;
        if (wr.counter == TFIM_COUNTER_TENSOR) return true;
        return nr >= tn.b1_min_rows && nc >= tn.b1_min_cols;
    };

    Wave w;
    struct Piece { int32_t fam; int32_t r0, r1; int32_t job; };
    std::vector<Piece> pieces;
    std::vector<std::pair<int32_t, int32_t>> look_jobs;   // (look index into `looks`, job)
    std::vector<Look> looks;
    std::vector<MatDesc> pending_mats;
    std::vector<int32_t> pending_mat_items;

    while (!stack.empty() || !looks_pending.empty()) {
        w.clear();
        pieces.clear();
        look_jobs.clear();
        looks.swap(looks_pending);
        looks_pending.clear();
        w.mats.swap(pending_mats);
        w.mat_items.swap(pending_mat_items);
        pending_mats.clear();
        pending_mat_items.clear();
        for (size_t li = 0; li < looks.size(); li++) {
            const int32_t job = w.add_job(-1, -1, {RowDesc{looks[li].slot, -1}}, looks[li].cols,
                                          use_b1_for(1, (int32_t)looks[li].cols.size()) && wr.counter == TFIM_COUNTER_TENSOR);
            look_jobs.push_back({(int32_t)li, job});
            st->lookaheads++;
        }
        // families from the top of the stack, skipping those that wait on a lookahead
        int64_t rows_taken = (int64_t)looks.size();
        for (int64_t si = (int64_t)stack.size() - 1; si >= 0 && rows_taken < wave_cap; si--) {
            Fam& f = fams[stack[si]];
            if (f.waiting || f.dead) continue;
            const int32_t nT = (int32_t)f.T.size();
            if (f.next_row >= nT) continue;
            const bool whole_top = stack[si] == 0 && top_mode != 0 && f.next_row == 0;
            const int32_t take = whole_top ? nT : (int32_t)std::min<int64_t>(nT - f.next_row, wave_cap - rows_taken);
            std::vector<RowDesc> rs(take);
            for (int32_t r = 0; r < take; r++) rs[r] = RowDesc{-1, f.T[f.next_row + r]};
            const int32_t job = w.add_job(f.slot, f.item, rs, f.F, use_b1_for(take, (int32_t)f.F.size()));
            if (whole_top) {
                w.top_job = job;
                w.top_mode = top_mode;
                w.top_pos.assign((size_t)std::max<int32_t>(c->info.n_dense, 1), -1);
                w.top_diag.resize(f.F.size());
                for (size_t q = 0; q < f.F.size(); q++) {
                    w.top_pos[f.F[q]] = (int32_t)q;
                    w.top_diag[q] = c->bit_support[f.F[q]];
                }
            }
            pieces.push_back({stack[si], f.next_row, f.next_row + take, job});
            f.next_row += take;
            rows_taken += take;
        }
        // remove fully handed-out families from the stack (they stay alive until processed)
        stack.erase(std::remove_if(stack.begin(), stack.end(),
                                   [&](int32_t id) { return fams[id].dead || (!fams[id].waiting && fams[id].next_row >= (int32_t)fams[id].T.size()); }),
                    stack.end());
        if (w.jobs.empty()) {
            TFIM_CHECK(stack.empty(), TFIM_E_STATE, "batched search stalled with %zu families", stack.size());
            break;
        }
        TFIM_TRY(wr.run(w, minc, false, nullptr));
        pool.flush();
        st->waves++;
        st->supports += w.supports;
        st->nodes += (int64_t)w.row_job.size();

        // lookahead results
        for (auto& lj : look_jobs) {
            Look& L = looks[lj.first];
            Fam& f = fams[L.fam];
            const JobDesc& jd = w.jobs[lj.second];
            const int2 ri = wr.row_info[lj.second];   // lookahead jobs come first, one row each
            int32_t self = -1;
            bool ext = false;
            for (int32_t k = 0; k < ri.y; k++) {
                const Entry& en = wr.entries[ri.x + k];
                if (en.col == jd.n_cols - 1) self = en.count;
                else ext = true;
            }
            pool.release(L.slot);
            if (L.log >= 0) c->la_labels[L.log] = self >= 0 ? 1.f : 0.f;
            if (self >= 0) {   // head + tail is frequent: it decides the whole subtree
                st->lookahead_hits++;
                if (!ext) {
                    std::vector<int32_t> items = f.head;
                    items.insert(items.end(), f.T.begin(), f.T.end());
                    sink.emit(items, self);
                }
                f.dead = true;
                pool.release(f.slot);
            } else {
                f.waiting = false;
                stack.push_back(L.fam);   // ready; explore next
            }
        }

        // family results -> children
        std::vector<int64_t> job_row_base(w.jobs.size() + 1, 0);
        for (size_t q = 0; q < w.jobs.size(); q++) job_row_base[q + 1] = job_row_base[q] + w.jobs[q].n_rows;
        std::vector<int32_t> new_fams;
        for (auto& pc : pieces) {
            Fam& P = fams[pc.fam];
            const int32_t nT = (int32_t)P.T.size();
            for (int32_t i = pc.r0; i < pc.r1; i++) {
                const int32_t t = P.T[i];
                const int2 ri = wr.row_info[job_row_base[pc.job] + (i - pc.r0)];
                int32_t supc = -1;
                std::vector<std::pair<int32_t, int32_t>> ext;   // (F index, count) of the child X = head + t
                for (int32_t k = 0; k < ri.y; k++) {
                    const Entry& en = wr.entries[ri.x + k];
                    if (en.col == i) supc = en.count;
                    else ext.push_back({en.col, en.count});
                }
                TFIM_CHECK(supc >= minc, TFIM_E_STATE, "family row lost its own support");
                auto in_tail = [&](int32_t col) { return col > i && col < nT; };
                std::vector<int32_t> head = P.head;
                head.push_back(t);
                if (ext.empty()) { sink.emit(head, supc); continue; }
                bool prune = false;
                std::vector<int32_t> eq;
                for (auto& pr : ext)
                    if (pr.second == supc) {
                        if (!in_tail(pr.first)) { prune = true; break; }
                        eq.push_back(pr.first);
                    }
                if (prune) { st->pruned_pep++; continue; }
                for (int32_t fx : eq) head.push_back(P.F[fx]);
                std::vector<std::pair<int32_t, int32_t>> rest, tail;
                for (auto& pr : ext) {
                    if (pr.second == supc) continue;
                    rest.push_back(pr);
                    if (in_tail(pr.first)) tail.push_back(pr);
                }
                if (rest.empty()) { sink.emit(head, supc); continue; }
                if (tail.empty()) continue;
                std::stable_sort(tail.begin(), tail.end(), [&](const std::pair<int32_t, int32_t>& a, const std::pair<int32_t, int32_t>& b) {
                    return a.second < b.second;
                });
                Fam ch;
                ch.head = std::move(head);
                for (auto& pr : tail) ch.T.push_back(P.F[pr.first]);
                // columns: tail first (in order), then the other candidates
                ch.F = ch.T;
                for (auto& pr : rest)
                    if (!in_tail(pr.first)) ch.F.push_back(P.F[pr.first]);
                // base mask of the child: P's base AND B[t]
                if (P.slot < 0 && P.item < 0) {
                    ch.slot = -1;
                    ch.item = t;
                } else {
                    int32_t s = 0;
                    TFIM_TRY(pool.alloc(c, &s));
                    MatDesc m;
                    m.dst = s; m.src = P.slot; m.off = (int32_t)pending_mat_items.size(); m.n = 0;
                    if (P.item >= 0) { pending_mat_items.push_back(P.item); m.n++; }
                    pending_mat_items.push_back(t); m.n++;
                    pending_mats.push_back(m);
                    ch.slot = s;
                    ch.item = -1;
                }
                // lookahead on head + tail.  Filter: every pair of tail items must be frequent
                // with P (a necessary condition, read from P's counted rows).
                const int32_t list_len = (int32_t)ch.T.size() + 1 + (P.item >= 0 ? 1 : 0);
                if (lookahead && ch.T.size() >= 2 && list_len <= kMaxListLen) {
                    int64_t pairs = 0, pairs_ok = 0;
                    bool filtered = false;
                    for (size_t a = 0; a < tail.size(); a++) {
                        const int32_t ra = tail[a].first;   // F index < |T(P)|: a row of P's family
                        if (ra < pc.r0 || ra >= pc.r1) continue;   // row not in this wave: unknown
                        const int2 rinfo = wr.row_info[job_row_base[pc.job] + (ra - pc.r0)];
                        const Entry* eb = wr.entries.data() + rinfo.x;
                        const Entry* ee = eb + rinfo.y;
                        for (size_t b = a + 1; b < tail.size(); b++) {
                            const int32_t cb = tail[b].first;
                            const Entry* it = std::lower_bound(eb, ee, cb, [](const Entry& x, int32_t v) { return x.col < v; });
                            pairs++;
                            if (it != ee && it->col == cb) pairs_ok++;
                            else filtered = true;
                        }
                    }
                    if (filtered && la_mode != 3) {
                        st->lookaheads_skipped++;
                    } else {
                        Cand cd;
                        cd.fam = (int32_t)fams.size();
                        cd.src_slot = P.slot;
                        cd.src_item = P.item;
                        cd.t = t;
                        lookahead_features(cd.feat, (int)ch.head.size(), tail, (int)ch.F.size(), supc, minc, c->n_bits_total,
                                           (int)eq.size(), pairs ? (double)pairs_ok / (double)pairs : 1.0, nT, i,
                                           P.slot < 0 && P.item < 0);
                        cands.push_back(cd);
                    }
                }
                new_fams.push_back((int32_t)fams.size());
                fams.push_back(std::move(ch));
            }
            Fam& P2 = fams[pc.fam];
            P2.rows_done += pc.r1 - pc.r0;
            if (P2.rows_done >= (int32_t)P2.T.size()) {
                pool.release(P2.slot);
                P2.dead = true;
                P2.F.clear(); P2.F.shrink_to_fit();
                P2.T.clear(); P2.T.shrink_to_fit();
                P2.head.clear(); P2.head.shrink_to_fit();
            }
        }
        // lookahead decisions for this wave's candidates
        if (!cands.empty()) {
            probs.assign(cands.size(), 1.f);
            if (la_mode == 2) {
                std::vector<float> feats(cands.size() * 32);
                for (size_t q = 0; q < cands.size(); q++) memcpy(&feats[q * 32], cands[q].feat, 32 * sizeof(float));
                if (tfim_mlp_predict(c->proposal, feats.data(), (int64_t)cands.size(), probs.data()) != TFIM_OK) return TFIM_E_CUDA;
            }
            for (size_t q = 0; q < cands.size(); q++) {
                const Cand& cd = cands[q];
                if (la_mode == 2 && probs[q] < c->proposal_threshold) {
                    st->lookaheads_skipped++;
                    continue;
                }
                Fam& ch = fams[cd.fam];
                int32_t ls = 0;
                TFIM_TRY(pool.alloc(c, &ls));
                MatDesc m;
                m.dst = ls; m.src = cd.src_slot; m.off = (int32_t)pending_mat_items.size(); m.n = 0;
                if (cd.src_item >= 0) { pending_mat_items.push_back(cd.src_item); m.n++; }
                pending_mat_items.push_back(cd.t); m.n++;
                for (int32_t x : ch.T) { pending_mat_items.push_back(x); m.n++; }
                pending_mats.push_back(m);
                Look L;
                L.fam = cd.fam;
                L.slot = ls;
                for (size_t q2 = ch.T.size(); q2 < ch.F.size(); q2++) L.cols.push_back(ch.F[q2]);
                L.cols.push_back(-1);
                if (o->log_lookahead) {
                    L.log = (int64_t)c->la_labels.size();
                    c->la_feats.insert(c->la_feats.end(), cd.feat, cd.feat + 32);
                    c->la_labels.push_back(0.f);
                }
                looks_pending.push_back(std::move(L));
                ch.waiting = true;
            }
            cands.clear();
        }
        // children explored first-in-order: push in reverse
        for (auto it = new_fams.rbegin(); it != new_fams.rend(); ++it)
            if (!fams[*it].waiting) stack.push_back(*it);
        // waiting families re-enter the stack when their lookahead resolves
    }
    st->launches += wr.launches;
    st->count_launches += wr.count_launches;
    st->bytes_alg += wr.bytes_alg;
    st->kernel_ms += wr.kernel_ms;
    st->sync_ms += wr.sync_ms;
    wr.add_to(st);
    st->bit_ops = st->supports * c->n_bits;
    (void)W;
    return TFIM_OK;
}

}  // namespace tfim
