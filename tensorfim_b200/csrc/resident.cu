// RESIDENT engine: the batched search with its state on the device.
//
// Same search and pruning as mine_batched (mine.cu) -- families of children counted as
// masked Gram blocks, candidate restriction, equal-support pruning, head-union-tail
// lookahead with the tail-pair filter or the learned proposal, dynamic tail order, root
// filter -- but the family records, the DFS stack, the lookahead queue, the mask-slot
// free list and the MFI output live in device memory, and two kernels drive it:
//   k_res_pack    (one block) pops families from the top of the device stack into a wave:
//                 count-job descriptors, counted rows, tiles and output offsets;
//   k_res_expand  (one warp per counted row) turns a counted row into the child's MFI
//                 test, equal-support pruning, tail (sorted by support in the warp),
//                 child mask, lookahead decision (tail-pair filter, or the proposal MLP
//                 evaluated in the warp) and pushes the child onto the stack.
// Between them the counting kernels of count_lop3.cu / count_b1.cu run on the wave.  The
// host reads one small status record per wave (to size the launches and grow pools) and
// copies the MFIs back once at the end.
#include <cub/cub.cuh>
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>

#include "tfim_internal.h"

namespace tfim {
namespace {

struct DFam {
    int32_t slot, item;        // base mask = masks[slot] & B[item] (either optional)
    int32_t head_off, head_len;
    int32_t F_off, nF, nT;     // F list in the item pool, tail = its first nT entries
    int32_t sup;
    int32_t next_row;          // rows handed to waves
    int32_t rows_done;         // rows expanded
    int32_t state;             // 0 ready, 1 waiting on its lookahead, 2 finished
    int32_t top;               // 1: the family of the empty prefix
};

struct DLook {
    int32_t fam, slot, log, pad;
};

// A prefix mask to build after an expand: masks[dst] = (slot >= 0 ? masks[slot] : ~0) &
// (item >= 0 ? B[item] : ~0) & (t >= 0 ? B[t] : ~0) & AND of B[items[off + q]], q < n.
struct MaskJob {
    int32_t dst, slot, item, t, off, n, pad0, pad1;
};

enum { kJobFam = 0, kJobLook = 1 };
struct DJob {
    int32_t fam, kind, r0, nr, slot, log;
    int32_t b3, b1;            // exclusive prefix of CUDA-core / tensor-core tiles over the wave's jobs
    int32_t cls, sl3;          // counter class (kCls*); word slices of its CUDA-core tiles
    int32_t b3l, heavy;        // CUDA-core tiles: heavy jobs' tiles come first (prefix b3), then the light
                               // jobs' (prefix b3l after all heavy tiles)
    int32_t btc;               // exclusive prefix of the tcgen05 family counter's jobs
    int32_t bgr;               // exclusive prefix of the CUDA-core Gram counter's jobs
    int32_t b3d;               // CUDA-core tiles of dense families (heavy == 2): they come before all
                               // others (prefix b3d), for the register-blocked dense launch
};

// Phases of a wave (device-time stamps) and counter classes of a count job.
enum { kPhPack = 0, kPhZero, kPhLop3, kPhB1, kPhTc, kPhProj, kPhGram, kPhExpand, kPhMasks, kPhases };
enum { kClsLop3 = 0, kClsB1 = 1, kClsProj = 2, kClsTc = 3, kClsGram = 4, kClasses = 5 };

struct ResStatus {
    int32_t stack_n, look_n, fam_n, item_n, head_n, mfi_n, mfi_item_n, slot_n, free_n, free_taken, defer_n, log_n;
    int32_t jobs, rows, tiles_l3, tiles_b1, n_proj, n_mjobs;   // n_mjobs: masks the last expand asked for
    int64_t out_total;
    int32_t max_cols, max_head, starved, error;
    // grow: the wave the pack built does not fit the pools; nothing was consumed and the
    // g_* fields hold its size, for the host to grow the pools and pack again
    int32_t grow, g_rows, g_jobs, g_max_head, g_max_cols, waves;
    int64_t g_out, g_tiles;
    int32_t launch_id, next3, next1;         // next3 / next1: tile counters of the persistent counters
    int32_t tiles_l3d;                       // the first tiles_l3d CUDA-core tiles are dense families'
    int32_t tiles_tc, next_tc;               // tcgen05 family counter: tiles, tile counter
    int32_t tiles_gr, next_gr;               // CUDA-core Gram counter: tiles, tile counter
    unsigned long long launch_t0;
    unsigned long long supports, nodes, lookaheads, hits, skipped, pep;
    // superset check: MFIs [0, sup_done) are in the item -> MFI index the expand reads
    int32_t sup_done, pad2;
    unsigned long long sup_pruned;
    // phase stamps of the current wave (first block start, last block end; %globaltimer ns)
    // and their durations summed over the search; the pack folds and resets them
    unsigned long long ph_s[kPhases], ph_e[kPhases], ph_ns[kPhases];
    // committed count jobs per counter class: algorithmic bytes (every operand row read once,
    // every count written once), bit-ops (supports x transactions), supports, jobs
    unsigned long long cls_bytes[kClasses], cls_bitops[kClasses], cls_sup[kClasses], cls_jobs[kClasses];
};

// Pool capacities, in entries.  A wave is packed only when the worst case of its expand fits.
struct Caps {
    int64_t fam, item, head, mfi, mfi_items, looks, slots, log, rows;
};
__host__ __device__ __forceinline__ bool wave_fits(const Caps& c, const ResStatus& st, int64_t rows, int64_t jobs,
                                                   int64_t out_total, int64_t max_head, int64_t max_cols, bool log_on) {
    const int64_t list = max_head + 2 + max_cols;
    return st.fam_n + rows + 1 <= c.fam && st.item_n + 2 * out_total + rows + 1 <= c.item &&
           st.head_n + rows * list + 1 <= c.head && st.mfi_n + rows + jobs + 1 <= c.mfi &&
           st.mfi_item_n + (rows + jobs) * list + 1 <= c.mfi_items && rows + 1 <= c.looks &&
           st.slot_n + 2 * rows + 2 <= c.slots && (!log_on || st.log_n + rows + 1 <= c.log) && rows <= c.rows;
}

struct ResPtrs {
    // pools
    DFam* fams;
    int32_t* items;
    int32_t* heads;
    int32_t* stack;
    DLook* looks;
    int32_t* free_slots;
    int32_t* defer;
    int32_t* mfi_off;
    int32_t* mfi_len;
    int32_t* mfi_sup;
    int32_t* mfi_items;
    float* log_feat;
    float* log_label;
    // wave
    DJob* djobs;
    MaskJob* mjobs;
    JobDesc* jobs;
    RowDesc* rows;
    int32_t* row_job;
    int32_t* row_local;
    TileDesc* tiles_l3;
    TileDesc* tiles_b1;
    TileDesc* tiles_tc;
    TileDesc* tiles_gr;
    int32_t* counts;
    // constants
    const uint32_t* bitmap;
    uint32_t* masks;
    const int32_t* dense_freq;
    const uint8_t* is_root;
    const __nv_bfloat16* mlp_w;   // BF16 weights of the proposal (nullptr: none)
    const float* mlp_p;           // FP32 parameters (biases read from here)
    ResStatus* st;
    int64_t W, n_bits;
    int32_t min_count;
    int32_t wave_rows;            // cap on rows per wave
    int64_t cap_out, cap_tiles;
    int32_t counter;              // TFIM_COUNTER_*
    int32_t la_mode;              // 0 off, 1 filtered, 2 learned, 3 every node
    int32_t log_on;
    float proposal_threshold;
    int64_t kslice_min;           // b1 word slice when tiles are few (multiple of 64)
    int32_t sm_count;
    int32_t* proj_list;           // family jobs counted by the projected counter
    float avg_len;                // mean reduced transaction length
    int32_t csr_ok;               // the reduced transaction list repeats no id within a row
    int32_t proj_auto;            // let the automatic counter choice pick the projected counter
    int32_t b1_min_rows, b1_min_cols;   // automatic choice: tensor path from this job shape
    float l3_slices_per_sm, b1_tiles_per_sm;   // work split targets per wave
    float l3_dense_slices_per_sm;               // ... of dense families' CUDA-core tiles
    int32_t tc_min_work;                       // automatic choice of the tcgen05 family counter
    float tc_min_density, tc_tiles_per_sm;
    int32_t gram_min_rows;                     // ... and of the CUDA-core Gram counter
    Caps caps;
    int64_t row_bytes;            // bytes of one bitmap row (algorithmic traffic accounting)
    const struct RowSum* row_sum; // first pass of the expand precomputed per wave row (or nullptr)
    // graph-driven wave loop: stop after wave_limit waves or max_launch_ns of device time
    int32_t wave_limit, launch_id;
    unsigned long long max_launch_ns;
    // superset check (nullptr: off): bit k of word sup_index[x * sup_words + k / 32] is set
    // when MFI k holds item x, for items x < sup_items and MFIs k < sup_words * 32
    uint32_t* sup_index;
    int32_t sup_words, sup_items;
};

// The first pass of the expand over one counted row: extensions (count >= min_count, own
// column excluded), equal-support extensions, tail extensions, whether an equal-support
// extension lies outside the tail (the subtree is pruned), and the column blocks of
// `column_block(nF)` columns that hold an extension.
struct RowSum {
    int32_t n_ext, n_eq, n_tail, prune;
    unsigned long long blocks;
    int64_t pad;
};
__host__ __device__ __forceinline__ int column_block(int nF) { return max(128, (((nF + 63) >> 6) + 31) & ~31); }

// Arguments of the graph-driven wave loop, kept in device memory so that growing a pool
// only rewrites this record (the captured launches stay valid).
struct ResArgs {
    ResPtrs p;
    CountArgs a3, a1, ap, atc, agr;   // CUDA-core, b1, projected, tcgen05 family and Gram counters
};

__device__ __forceinline__ unsigned long long globaltimer() { return dev_globaltimer(); }

// Projected counting pays when the prefix holds few transactions: it walks the base's set
// bits (W words) and looks up about 6 entries per item of each of its sup transactions,
// against the bitmap counters' (rows + columns + 1) x W words.
__device__ __forceinline__ bool use_proj(const ResPtrs& p, const JobDesc& jd, int32_t sup) {
    if (!p.csr_ok || jd.n_cols > kProjMaxCols || (jd.base_slot >= 0 && jd.base_item >= 0)) return false;
    if (jd.base_slot < 0 && jd.base_item < 0) return false;
    if (p.counter == TFIM_COUNTER_PROJ) return true;
    if (p.counter != TFIM_COUNTER_AUTO || !p.proj_auto) return false;
    const double proj = (double)p.W + (double)sup * 6.0 * (double)p.avg_len;
    const double bitmap = (double)(jd.n_rows + jd.n_cols + 1) * (double)p.W;
    return proj < bitmap;
}

__host__ __device__ __forceinline__ int64_t lmin(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t lmax(int64_t a, int64_t b) { return a > b ? a : b; }

constexpr int kPackThreads = 1024;
constexpr int kPackItems = 4;
constexpr int kPackCand = kPackThreads * kPackItems;

// The tcgen05 family counter takes a family job (its rows are a run of its columns) of at
// most kFamMaxCols columns: always when that counter is asked for, and in the automatic choice
// when the job is large enough and its prefix dense enough that skipping zero words (which
// the CUDA-core tiles do and the tensor tiles do not) saves little.
__device__ __forceinline__ bool use_tc(const ResPtrs& p, const JobDesc& jd, int32_t sup) {
    if (jd.n_cols < 1 || jd.n_cols > kFamMaxCols || jd.n_rows < 1) return false;
    if (p.counter == TFIM_COUNTER_I8) return true;
    if (p.counter != TFIM_COUNTER_AUTO) return false;
    // families up to kGramMaxCols columns are the Gram counter's (measured faster at every
    // shape there); wider ones take the tensor tiles when large enough to fill their MMAs
    if (jd.n_cols <= kGramMaxCols) return false;
    if ((int64_t)jd.n_rows * jd.n_cols < p.tc_min_work) return false;
    const float d = p.n_bits > 0 ? fminf(1.f, 128.f * (float)sup / (float)p.n_bits) : 1.f;
    return d >= p.tc_min_density;
}

// The CUDA-core Gram counter takes a dense family job of at most kGramMaxCols columns (and at
// most 128 blocks of 4 x 4 pairs): a dense prefix has no zero word for the general tiles to
// skip, and at these widths the register-tiled Gram block (86-91% of the POPC ceiling at 32
// and 64 columns) beats the tensor tiles, whose narrow MMAs cost about 50 cycles each.
__device__ __forceinline__ bool use_gram(const ResPtrs& p, const JobDesc& jd, int32_t sup) {
    // tails of 1 or 2 rows are memory-bound in any kernel (8 bit-ops per byte and row); the
    // general tiles handle them as well, and measured faster on the dense benchmark
    if (jd.n_cols < 1 || jd.n_cols > kGramMaxCols || jd.n_rows < p.gram_min_rows) return false;
    if (((jd.n_rows + 3) / 4) * ((jd.n_cols + 3) / 4) > 128) return false;
    if (p.counter != TFIM_COUNTER_AUTO) return false;
    const float d = p.n_bits > 0 ? fminf(1.f, 128.f * (float)sup / (float)p.n_bits) : 1.f;
    return d >= p.tc_min_density;
}

__device__ __forceinline__ bool use_b1_shape(const ResPtrs& p, int nr, int nc) {
    if (p.counter == TFIM_COUNTER_LOP3) return false;
    if (p.counter == TFIM_COUNTER_TENSOR) return true;
    return nr >= p.b1_min_rows && nc >= p.b1_min_cols;
}
__device__ __forceinline__ int64_t l3_tiles(int nr, int nc) { return (int64_t)((nr + kLop3Rows - 1) / kLop3Rows) * ((nc + 63) / 64); }
__device__ __forceinline__ int64_t b1_tiles(int nr, int nc) { return (int64_t)((nr + kB1Rows - 1) / kB1Rows) * ((nc + kB1Cols - 1) / kB1Cols); }

// ---------------------------------------------------------------------------------- pack
// One block.  Phases: (0) recycle the mask slots released by the last expand; (1) one job
// per queued lookahead; (2) families from the top of the stack, 4096 candidates per pass,
// with block scans deciding how many fit the wave's row and output budgets; (3) the counted
// rows and row->job maps; (4) tiles (split-k slices chosen from the wave's base tile count).
// Every phase is block-parallel; jobs are ordered by their row offsets, which the row and
// tile writers binary-search.
__device__ __forceinline__ int find_job_by_row(const JobDesc* jobs, int nj, int32_t g) {
    int lo = 0, hi = nj - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].row_off <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}
// The last job whose prefix (0: b3, 1: b1, 2: b3l) is <= t: the job owning tile t, since a
// job with no tiles of that kind shares its prefix with the next job that has some.
template <int K>
__device__ __forceinline__ int find_job_by_tile(const DJob* dj, int nj, int64_t t) {
    int lo = 0, hi = nj - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int32_t v = K == 0   ? dj[mid].b3
                          : K == 1 ? dj[mid].b1
                          : K == 2 ? dj[mid].b3l
                          : K == 3 ? dj[mid].btc
                          : K == 4 ? dj[mid].bgr
                                   : dj[mid].b3d;
        if (v <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void res_pack(const ResPtrs& p) {
    typedef cub::BlockScan<int64_t, kPackThreads> Scan;
    typedef cub::BlockReduce<int64_t, kPackThreads> Red;
    __shared__ union {
        typename Scan::TempStorage scan;
        typename Red::TempStorage red;
    } tmp;
    __shared__ int32_t s_fam[kPackCand];
    __shared__ int32_t s_n_jobs, s_rows_total, s_done, s_max_cols, s_max_head, s_stack_after, s_kstop, s_fit;
    __shared__ int64_t s_out_total, s_agg;
    ResStatus* st = p.st;
    const int tid = threadIdx.x;
    // (0) recycle
    const int32_t taken = min(st->free_taken, st->free_n);
    const int32_t fn = st->free_n - taken, dn = st->defer_n;
    for (int k = tid; k < dn; k += kPackThreads) p.free_slots[fn + k] = p.defer[k];
    if (tid == 0) {
        s_n_jobs = 0; s_rows_total = 0; s_out_total = 0; s_max_cols = 0; s_max_head = 0; s_done = 0;
        s_stack_after = st->stack_n;
        st->n_proj = 0;
        st->n_mjobs = 0;
        st->grow = 0;
        st->starved = 0;
        // MFIs of the finished waves are indexed (k_index_mfis ran after the last expand)
        if (p.sup_index) st->sup_done = min(st->mfi_n, p.sup_words * 32);
        if (st->launch_id != p.launch_id) {
            st->launch_id = p.launch_id;
            st->launch_t0 = globaltimer();
        }
        // the last wave's phases: add their durations, clear the stamps, stamp this pack
        for (int k = 0; k < kPhases; k++) {
            const unsigned long long s0 = st->ph_s[k], e0 = st->ph_e[k];
            if (s0 != ~0ull && e0 > s0) st->ph_ns[k] += e0 - s0;
            st->ph_s[k] = ~0ull;
            st->ph_e[k] = 0;
        }
        st->ph_s[kPhPack] = globaltimer();
    }
    __syncthreads();
    if (tid == 0) {
        st->free_n = fn + dn;
        st->free_taken = 0;
        st->defer_n = 0;
    }
    // (1) lookahead jobs
    const int32_t n_look = st->look_n;
    for (int base = 0; base < n_look; base += kPackCand) {
        int64_t v[kPackItems], ex[kPackItems];
        int64_t mc = 0;
        for (int q = 0; q < kPackItems; q++) {
            const int k = base + tid * kPackItems + q;
            v[q] = 0;
            if (k < n_look) {
                const DFam f = p.fams[p.looks[k].fam];
                v[q] = f.nF - f.nT + 1;
                mc = max(mc, v[q]);
            }
        }
        Scan(tmp.scan).ExclusiveSum(v, ex, s_agg);
        __syncthreads();
        const int64_t agg = s_agg;
        const int64_t mcb = Red(tmp.red).Reduce(mc, cub::Max());
        for (int q = 0; q < kPackItems; q++) {
            const int k = base + tid * kPackItems + q;
            if (k >= n_look) continue;
            const DLook L = p.looks[k];
            const DFam f = p.fams[L.fam];
            DJob dj;
            dj.fam = L.fam; dj.kind = kJobLook; dj.r0 = 0; dj.nr = 1; dj.slot = L.slot; dj.log = L.log; dj.b3 = 0; dj.b1 = 0;
            dj.cls = 0; dj.sl3 = 1; dj.b3l = 0; dj.heavy = 0; dj.btc = 0; dj.bgr = 0; dj.b3d = 0;
            p.djobs[k] = dj;
            JobDesc jd;
            jd.base_slot = -1; jd.base_item = -1; jd.n_rows = 1; jd.n_cols = f.nF - f.nT + 1;
            jd.row_off = k; jd.col_off = f.F_off + f.nT; jd.out_off = s_out_total + ex[q]; jd.self_col = f.nF - f.nT; jd.pad = 0;
            p.jobs[k] = jd;
        }
        __syncthreads();
        if (tid == 0) {
            s_out_total += agg;
            s_max_cols = max(s_max_cols, (int32_t)mcb);
        }
        __syncthreads();
    }
    if (tid == 0) {
        s_rows_total = n_look;
        s_n_jobs = n_look;
    }
    __syncthreads();
    // (2) families from the top of the stack
    while (!s_done) {
        const int32_t avail = s_stack_after;
        const int32_t n_c = min(avail, kPackCand);
        if (n_c == 0) break;
        const int64_t rows_left = (int64_t)p.wave_rows - s_rows_total;
        const int64_t out_left = p.cap_out - s_out_total;
        const bool wave_empty = s_n_jobs == 0;
        int64_t rv[kPackItems], ov[kPackItems], rc[kPackItems], oc[kPackItems];
        int32_t nf[kPackItems], hl[kPackItems];
        for (int q = 0; q < kPackItems; q++) {
            const int k = tid * kPackItems + q;
            rv[q] = ov[q] = 0;
            nf[q] = 0;
            hl[q] = 0;
            if (k < n_c) {
                const int32_t fid = p.stack[avail - 1 - k];
                const DFam f = p.fams[fid];
                s_fam[k] = fid;
                const int32_t rem = f.state == 0 ? f.nT - f.next_row : 0;
                rv[q] = rem;
                ov[q] = (int64_t)rem * f.nF;
                nf[q] = f.nF;
                hl[q] = f.head_len;
            }
        }
        Scan(tmp.scan).InclusiveSum(rv, rc);
        __syncthreads();
        Scan(tmp.scan).InclusiveSum(ov, oc);
        __syncthreads();
        // take per candidate and the first stop point
        int32_t take[kPackItems];
        int64_t kstop_local = n_c;
        for (int q = 0; q < kPackItems; q++) {
            const int k = tid * kPackItems + q;
            take[q] = -1;
            if (k >= n_c) continue;
            const int64_t r_before = rc[q] - rv[q], o_before = oc[q] - ov[q];
            if (rc[q] <= rows_left && oc[q] <= out_left) {
                take[q] = (int32_t)rv[q];
            } else if (r_before < rows_left && o_before < out_left) {
                int64_t t_rows = min(rows_left - r_before, (out_left - o_before) / max(1, nf[q]));
                take[q] = (int32_t)min(t_rows, rv[q]);
                if (take[q] == 0 && r_before == 0 && o_before == 0 && wave_empty) atomicExch(&st->starved, 1);
            }
            const bool stop = take[q] < 0 || (rv[q] > 0 && take[q] < rv[q]);
            if (stop) kstop_local = min(kstop_local, (int64_t)k);
        }
        const int64_t kstop = Red(tmp.red).Reduce(kstop_local, cub::Min());
        if (tid == 0) s_kstop = (int32_t)kstop;
        __syncthreads();
        const int32_t ks = s_kstop;
        // jobs: candidates before the stop point with rows left, and the stop point if it takes rows
        int64_t hj[kPackItems], hx[kPackItems], tr[kPackItems];
        int64_t mcol = 0, mhead = 0;
        for (int q = 0; q < kPackItems; q++) {
            const int k = tid * kPackItems + q;
            hj[q] = 0;
            tr[q] = 0;
            if (k < n_c && ((k < ks && rv[q] > 0) || (k == ks && take[q] > 0))) {
                hj[q] = 1;
                tr[q] = take[q];
                mcol = max(mcol, (int64_t)nf[q]);
                mhead = max(mhead, (int64_t)hl[q]);
            }
        }
        Scan(tmp.scan).ExclusiveSum(hj, hx, s_agg);
        __syncthreads();
        const int64_t n_new = s_agg;
        int64_t trx[kPackItems];
        Scan(tmp.scan).ExclusiveSum(tr, trx, s_agg);
        __syncthreads();
        const int64_t rows_new = s_agg;
        const int64_t mcb = Red(tmp.red).Reduce(mcol, cub::Max());
        __syncthreads();
        const int64_t mhb = Red(tmp.red).Reduce(mhead, cub::Max());
        for (int q = 0; q < kPackItems; q++) {
            const int k = tid * kPackItems + q;
            if (!hj[q]) continue;
            const int32_t fid = s_fam[k];
            DFam* fp = p.fams + fid;
            const DFam f = *fp;
            const int32_t jid = s_n_jobs + (int32_t)hx[q];
            DJob dj;
            dj.fam = fid; dj.kind = kJobFam; dj.r0 = f.next_row; dj.nr = take[q]; dj.slot = -1; dj.log = -1; dj.b3 = 0; dj.b1 = 0;
            dj.cls = 0; dj.sl3 = 1; dj.b3l = 0; dj.heavy = 0; dj.btc = 0; dj.bgr = 0; dj.b3d = 0;
            p.djobs[jid] = dj;
            JobDesc jd;
            jd.base_slot = f.slot; jd.base_item = f.item; jd.n_rows = take[q]; jd.n_cols = f.nF;
            jd.row_off = s_rows_total + (int32_t)trx[q];
            jd.col_off = f.F_off;
            // outputs: every candidate before this one contributed rv * nF, this one take * nF
            jd.out_off = s_out_total + (oc[q] - ov[q]);
            jd.self_col = -1; jd.pad = 0;
            p.jobs[jid] = jd;
            (void)fp;   // next_row advances when the wave is committed
        }
        __syncthreads();
        // outputs of this pass: every job's taken rows x its columns
        int64_t contrib = 0;
        for (int q = 0; q < kPackItems; q++) contrib += (int64_t)(hj[q] ? (int64_t)tr[q] * nf[q] : 0);
        const int64_t out_pass = Red(tmp.red).Sum(contrib);
        if (tid == 0) {
            s_n_jobs += (int32_t)n_new;
            s_rows_total += (int32_t)rows_new;
            s_out_total += out_pass;
            s_max_cols = max(s_max_cols, (int32_t)mcb);
            s_max_head = max(s_max_head, (int32_t)mhb);
            s_stack_after -= ks;   // candidates before the stop point are consumed
            if (ks < n_c || s_rows_total >= p.wave_rows || n_c < kPackCand || s_stack_after == 0) s_done = 1;
        }
        __syncthreads();
    }
    __syncthreads();
    const int32_t nj = s_n_jobs, rows_total = s_rows_total;
    // (3) rows
    for (int32_t g = tid; g < rows_total; g += kPackThreads) {
        const int j = find_job_by_row(p.jobs, nj, g);
        const JobDesc jd = p.jobs[j];
        const DJob dj = p.djobs[j];
        const int32_t r = g - jd.row_off;
        if (dj.kind == kJobFam) p.rows[g] = RowDesc{-1, p.items[jd.col_off + dj.r0 + r]};
        else p.rows[g] = RowDesc{dj.slot, -1};
        p.row_job[g] = j;
        p.row_local[g] = r;
    }
    // (4) tiles.  Pass 1 picks each job's counter and sums the estimated cost of its
    // CUDA-core tiles; pass 2 gives every CUDA-core job its own number of word slices (a
    // heavy job -- dense prefix, many rows and columns -- is split so that no tile runs
    // far longer than the wave's average) and forms the prefix sums the tile writers
    // search.  Tensor-core jobs share one split-k factor.
    const int64_t W = p.W;
    const float P4 = (float)(W >> 2);
    auto l3_cost = [&](const JobDesc& jd, const DJob& dj) -> float {
        float d = 1.f;   // fraction of 128-bit base positions that are nonzero
        if (dj.kind == kJobFam && (jd.base_slot >= 0 || jd.base_item >= 0) && p.n_bits > 0)
            d = fminf(1.f, 128.f * (float)p.fams[dj.fam].sup / (float)p.n_bits);
        const float nr = (float)min(jd.n_rows, kLop3Rows), nc = (float)min(jd.n_cols, 64);
        return P4 * (1.f + d * (2.f + nr + nr * nc / 32.f));
    };
    float cost_local = 0.f;
    int64_t tot1 = 0, tottc = 0, totgr = 0;
    for (int base = 0; base < nj; base += kPackCand) {
        int64_t a1[kPackItems], x1[kPackItems], at[kPackItems], xt[kPackItems], ag[kPackItems], xg[kPackItems];
        for (int q = 0; q < kPackItems; q++) {
            const int j = base + tid * kPackItems + q;
            a1[q] = 0;
            at[q] = 0;
            ag[q] = 0;
            if (j < nj) {
                const JobDesc jd = p.jobs[j];
                DJob* djp = p.djobs + j;
                const bool fam = djp->kind == kJobFam;
                const int32_t fsup = p.fams[djp->fam].sup;
                int cls = kClsLop3;
                if (fam && use_proj(p, jd, fsup)) {
                    cls = kClsProj;
                    const int32_t k = atomicAdd(&p.st->n_proj, 1);
                    p.proj_list[k] = j;
                } else if (fam && use_gram(p, jd, fsup)) {
                    cls = kClsGram;
                    ag[q] = 1;
                } else if (fam && use_tc(p, jd, fsup)) {
                    cls = kClsTc;
                    at[q] = 1;
                } else if (use_b1_shape(p, jd.n_rows, jd.n_cols) && fam) {
                    cls = kClsB1;
                    a1[q] = b1_tiles(jd.n_rows, jd.n_cols);
                } else {
                    cost_local += (float)l3_tiles(jd.n_rows, jd.n_cols) * l3_cost(jd, *djp);
                }
                djp->cls = cls;
            }
        }
        Scan(tmp.scan).ExclusiveSum(a1, x1, s_agg);
        __syncthreads();
        const int64_t g1 = s_agg;
        Scan(tmp.scan).ExclusiveSum(at, xt, s_agg);
        __syncthreads();
        const int64_t gt = s_agg;
        Scan(tmp.scan).ExclusiveSum(ag, xg, s_agg);
        __syncthreads();
        const int64_t gg = s_agg;
        for (int q = 0; q < kPackItems; q++) {
            const int j = base + tid * kPackItems + q;
            if (j < nj) {
                p.djobs[j].b1 = (int32_t)(tot1 + x1[q]);
                p.djobs[j].btc = (int32_t)(tottc + xt[q]);
                p.djobs[j].bgr = (int32_t)(totgr + xg[q]);
            }
        }
        tot1 += g1;
        tottc += gt;
        totgr += gg;
        __syncthreads();
    }
    __shared__ float s_cost;
    {
        typedef cub::BlockReduce<float, kPackThreads> RedF;
        __shared__ typename RedF::TempStorage redf;
        const float c = RedF(redf).Sum(cost_local);
        if (tid == 0) s_cost = c;
        __syncthreads();
    }
    // the wave's estimated CUDA-core cost over (slices per SM x SMs): the cost of one tile
    // slice; dense families are split more finely (their own target), which shortens the
    // launch's tail on large dense databases
    const float target = fmaxf(s_cost / (p.l3_slices_per_sm * (float)p.sm_count), 1.f);
    const float target_d = fmaxf(s_cost / (p.l3_dense_slices_per_sm * (float)p.sm_count), 1.f);
    const int64_t max_sl = lmax(1, W / 256);
    // Tiles of dense families and of their lookaheads (the family's prefix holds at least 1/16
    // of the transactions, so no 128-bit position is zero to skip) come first, for the
    // register-blocked dense launch;
    // then heavy jobs (cost at least half the slice target), so that the longest tiles are
    // dispatched first and the light ones fill in behind them.
    int64_t tot3d = 0, tot3h = 0, tot3l = 0;
    for (int base = 0; base < nj; base += kPackCand) {
        int64_t ad[kPackItems], ah[kPackItems], al[kPackItems], xd[kPackItems], xh[kPackItems], xl[kPackItems];
        for (int q = 0; q < kPackItems; q++) {
            const int j = base + tid * kPackItems + q;
            ad[q] = ah[q] = al[q] = 0;
            if (j < nj) {
                const JobDesc jd = p.jobs[j];
                DJob* djp = p.djobs + j;
                if (djp->cls == 0) {
                    const float cost = l3_cost(jd, *djp);
                    // a family job, or the lookahead of a family (its head-union-tail mask is a subset
                    // of the family's prefix, and on a dense family almost never zero per 128 bits)
                    const bool dense = 16 * (int64_t)p.fams[djp->fam].sup >= p.n_bits;
                    int64_t sl = lmin(max_sl, lmax(1, (int64_t)ceilf(cost / (dense ? target_d : target))));
                    const int64_t wsl = ((W / 64 + sl - 1) / sl) * 64;
                    sl = wsl > 0 ? (W + wsl - 1) / wsl : 1;
                    djp->sl3 = (int32_t)sl;
                    djp->heavy = dense ? 2 : cost >= 0.5f * target ? 1 : 0;
                    const int64_t nt = l3_tiles(jd.n_rows, jd.n_cols) * sl;
                    if (djp->heavy == 2) ad[q] = nt;
                    else if (djp->heavy) ah[q] = nt;
                    else al[q] = nt;
                }
            }
        }
        Scan(tmp.scan).ExclusiveSum(ad, xd, s_agg);
        __syncthreads();
        const int64_t gd = s_agg;
        Scan(tmp.scan).ExclusiveSum(ah, xh, s_agg);
        __syncthreads();
        const int64_t gh = s_agg;
        Scan(tmp.scan).ExclusiveSum(al, xl, s_agg);
        __syncthreads();
        const int64_t gl = s_agg;
        for (int q = 0; q < kPackItems; q++) {
            const int j = base + tid * kPackItems + q;
            if (j < nj) {
                p.djobs[j].b3d = (int32_t)(tot3d + xd[q]);
                p.djobs[j].b3 = (int32_t)(tot3h + xh[q]);
                p.djobs[j].b3l = (int32_t)(tot3l + xl[q]);
            }
        }
        tot3d += gd;
        tot3h += gh;
        tot3l += gl;
        __syncthreads();
    }
    const int64_t tot3 = tot3d + tot3h + tot3l;
    const int64_t want1 = lmax(1, (int64_t)(p.b1_tiles_per_sm * (float)p.sm_count));
    int64_t ks1 = tot1 > 0 ? lmax(1, (want1 + tot1 - 1) / tot1) : 1;
    ks1 = lmin(ks1, lmax(1, W / 64));
    int64_t kslice = ((W / 64 + ks1 - 1) / ks1) * 64;
    if (kslice <= 0) kslice = 64;
    const int64_t nk = W > 0 ? (W + kslice - 1) / kslice : 1;
    const int64_t T3 = tot3, T1 = tot1 * nk;
    // tcgen05 family tiles: every job whole, over `sltc` word slices (multiples of 64 words)
    const int64_t want_tc = lmax(1, (int64_t)(p.tc_tiles_per_sm * (float)p.sm_count));
    int64_t sltc = tottc > 0 ? lmax(1, (want_tc + tottc - 1) / tottc) : 1;
    sltc = lmin(sltc, lmax(1, W / 64));
    int64_t wsltc = ((W / 64 + sltc - 1) / sltc) * 64;
    if (wsltc <= 0) wsltc = 64;
    const int64_t ntc = W > 0 ? (W + wsltc - 1) / wsltc : 1;
    const int64_t TT = tottc * ntc;
    // CUDA-core Gram tiles: every job whole, over `slgr` word slices (multiples of 64 words)
    const int64_t want_gr = lmax(1, (int64_t)(p.l3_slices_per_sm * (float)p.sm_count));
    int64_t slgr = totgr > 0 ? lmax(1, (want_gr + totgr - 1) / totgr) : 1;
    slgr = lmin(slgr, lmax(1, W / 64));
    int64_t wslgr = ((W / 64 + slgr - 1) / slgr) * 64;
    if (wslgr <= 0) wslgr = 64;
    const int64_t ngr = W > 0 ? (W + wslgr - 1) / wslgr : 1;
    const int64_t TG = totgr * ngr;
    // the wave is committed only when the worst case of its expand fits the pools
    if (tid == 0) {
        const bool fit = s_out_total <= p.cap_out && T1 <= p.cap_tiles && T3 <= p.cap_tiles && TT <= p.cap_tiles &&
                         TG <= p.cap_tiles &&
                         wave_fits(p.caps, *st, rows_total, nj, s_out_total, s_max_head, s_max_cols, p.log_on != 0);
        s_fit = fit;
        if (!fit) {
            st->grow = 1;
            st->g_rows = rows_total;
            st->g_jobs = nj;
            st->g_out = s_out_total;
            st->g_max_head = s_max_head;
            st->g_max_cols = s_max_cols;
            st->g_tiles = lmax(lmax(lmax(T1, T3), TT), TG);
        }
    }
    __syncthreads();
    if (!s_fit) {
        if (tid == 0) {
            st->jobs = 0; st->rows = 0; st->tiles_l3 = 0; st->tiles_l3d = 0; st->tiles_b1 = 0; st->tiles_tc = 0;
            st->tiles_gr = 0; st->n_proj = 0;
            st->out_total = 0;
            st->ph_e[kPhPack] = globaltimer();
        }
        return;
    }
    // commit: the families hand out their rows
    for (int j = n_look + tid; j < nj; j += kPackThreads) {
        const DJob dj = p.djobs[j];
        p.fams[dj.fam].next_row = dj.r0 + dj.nr;
    }
    // the wave's work per counter class (warp sums, one atomic per warp and class)
    {
        unsigned long long cb[kClasses], cbo[kClasses], cs[kClasses], cj[kClasses];
#pragma unroll
        for (int k = 0; k < kClasses; k++) cb[k] = cbo[k] = cs[k] = cj[k] = 0;
        for (int j = tid; j < nj; j += kPackThreads) {
            const JobDesc jd = p.jobs[j];
            const int cls = p.djobs[j].cls;
            const unsigned long long nbase = (jd.base_slot >= 0) + (jd.base_item >= 0);
            const unsigned long long sup = (unsigned long long)jd.n_rows * (unsigned long long)jd.n_cols;
            const unsigned long long by =
                (unsigned long long)p.row_bytes * ((unsigned long long)jd.n_rows + jd.n_cols + nbase) + 4ull * sup;
#pragma unroll
            for (int k = 0; k < kClasses; k++)
                if (cls == k) {
                    cb[k] += by;
                    cbo[k] += sup * (unsigned long long)p.n_bits;
                    cs[k] += sup;
                    cj[k] += 1;
                }
        }
#pragma unroll
        for (int k = 0; k < kClasses; k++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cb[k] += __shfl_xor_sync(0xffffffffu, cb[k], o);
                cbo[k] += __shfl_xor_sync(0xffffffffu, cbo[k], o);
                cs[k] += __shfl_xor_sync(0xffffffffu, cs[k], o);
                cj[k] += __shfl_xor_sync(0xffffffffu, cj[k], o);
            }
            if ((tid & 31) == 0 && cj[k]) {
                atomicAdd(&st->cls_bytes[k], cb[k]);
                atomicAdd(&st->cls_bitops[k], cbo[k]);
                atomicAdd(&st->cls_sup[k], cs[k]);
                atomicAdd(&st->cls_jobs[k], cj[k]);
            }
        }
    }
    if (T3 <= p.cap_tiles)
        for (int64_t t = tid; t < T3; t += kPackThreads) {
            const int grp = t < tot3d ? 0 : t < tot3d + tot3h ? 1 : 2;   // dense, heavy, light
            const int j = grp == 0   ? find_job_by_tile<5>(p.djobs, nj, t)
                          : grp == 1 ? find_job_by_tile<0>(p.djobs, nj, t - tot3d)
                                     : find_job_by_tile<2>(p.djobs, nj, t - tot3d - tot3h);
            const JobDesc jd = p.jobs[j];
            const DJob dj = p.djobs[j];
            const int64_t local = grp == 0 ? t - dj.b3d : grp == 1 ? t - tot3d - dj.b3 : t - tot3d - tot3h - dj.b3l;
            const int64_t bt = l3_tiles(jd.n_rows, jd.n_cols);
            const int64_t slice = local / bt, within = local % bt;
            const int64_t wsl = ((W / 64 + dj.sl3 - 1) / dj.sl3) * 64;
            const int cg = (jd.n_cols + 63) / 64;
            const int rg = (int)(within / cg), cc = (int)(within % cg);
            const int64_t w0 = slice * wsl;
            p.tiles_l3[t] = TileDesc{j, rg * kLop3Rows, min(kLop3Rows, jd.n_rows - rg * kLop3Rows), cc * 64,
                                     min(jd.n_cols, cc * 64 + 64), (int32_t)w0, (int32_t)lmin(W, w0 + wsl), grp == 0 ? 1 : 0};
        }
    if (T1 <= p.cap_tiles)
        for (int64_t t = tid; t < T1; t += kPackThreads) {
            const int64_t slice = t / tot1, local = t % tot1;
            const int j = find_job_by_tile<1>(p.djobs, nj, local);
            const JobDesc jd = p.jobs[j];
            const int64_t within = local - p.djobs[j].b1;
            const int cg = (jd.n_cols + kB1Cols - 1) / kB1Cols;
            const int rg = (int)(within / cg), cc = (int)(within % cg);
            const int64_t w0 = slice * kslice;
            p.tiles_b1[t] = TileDesc{j, rg * kB1Rows, min(kB1Rows, jd.n_rows - rg * kB1Rows), cc * kB1Cols,
                                     min(jd.n_cols, cc * kB1Cols + kB1Cols), (int32_t)w0, (int32_t)lmin(W, w0 + kslice), 0};
        }
    if (TT <= p.cap_tiles)
        for (int64_t t = tid; t < TT; t += kPackThreads) {
            const int64_t slice = t / tottc, local = t % tottc;
            const int j = find_job_by_tile<3>(p.djobs, nj, local);
            const JobDesc jd = p.jobs[j];
            const int64_t w0 = slice * wsltc;
            // rows 0 .. n_rows of the job are its columns dj.r0 .. dj.r0 + n_rows
            p.tiles_tc[t] = TileDesc{j, 0, jd.n_rows, 0, jd.n_cols, (int32_t)w0, (int32_t)lmin(W, w0 + wsltc),
                                     p.djobs[j].r0};
        }
    if (TG <= p.cap_tiles)
        for (int64_t t = tid; t < TG; t += kPackThreads) {
            const int64_t slice = t / totgr, local = t % totgr;
            const int j = find_job_by_tile<4>(p.djobs, nj, local);
            const JobDesc jd = p.jobs[j];
            const int64_t w0 = slice * wslgr;
            p.tiles_gr[t] = TileDesc{j, 0, jd.n_rows, 0, jd.n_cols, (int32_t)w0, (int32_t)lmin(W, w0 + wslgr),
                                     p.djobs[j].r0};
        }
    if (tid == 0) {
        st->jobs = nj;
        st->rows = rows_total;
        st->tiles_l3 = (int32_t)T3;
        st->tiles_l3d = (int32_t)tot3d;
        st->tiles_b1 = (int32_t)T1;
        st->tiles_tc = (int32_t)TT;
        st->tiles_gr = (int32_t)TG;
        st->out_total = s_out_total;
        st->max_cols = s_max_cols;
        st->max_head = s_max_head;
        st->stack_n = s_stack_after;
        st->look_n = 0;
        st->nodes += rows_total;
        st->supports += s_out_total;
        st->ph_e[kPhPack] = globaltimer();
    }
}

__global__ void __launch_bounds__(kPackThreads) k_res_pack(ResPtrs p) { res_pack(p); }
__global__ void __launch_bounds__(kPackThreads) k_res_pack_g(const ResArgs* __restrict__ args) {
    const ResPtrs p = args->p;
    res_pack(p);
}

// ---------------------------------------------------------------------------------- expand helpers
__device__ __forceinline__ int32_t pop_slot(const ResPtrs& p) {
    const int32_t k = atomicAdd(&p.st->free_taken, 1);
    const int32_t fn = p.st->free_n;
    if (k < fn) return p.free_slots[fn - 1 - k];
    return atomicAdd(&p.st->slot_n, 1);
}
__device__ __forceinline__ void release_slot(const ResPtrs& p, int32_t s) {
    if (s < 0) return;
    const int32_t k = atomicAdd(&p.st->defer_n, 1);
    p.defer[k] = s;
}

// Record a mask for k_build_masks (lane 0 of the calling warp).
__device__ __forceinline__ void emit_mask(const ResPtrs& p, int32_t dst, int32_t slot, int32_t item, int32_t t, int32_t off,
                                          int32_t n, int lane) {
    if (lane == 0) {
        const int32_t k = atomicAdd(&p.st->n_mjobs, 1);
        p.mjobs[k] = MaskJob{dst, slot, item, t, off, n, 0, 0};
    }
}

// Sort an emitted MFI's item list (distinct dense ids) in descending order in place: a rank
// sort with two items per lane when it holds at most 64 items (longer lists are sorted by the
// host, which checks every list).
__device__ void warp_sort_desc(int32_t* a, int n, int lane) {
    if (n > 64 || n < 2) return;
    __syncwarp();
    const int32_t v0 = lane < n ? a[lane] : INT_MIN, v1 = lane + 32 < n ? a[lane + 32] : INT_MIN;
    int r0 = 0, r1 = 0;
    for (int j = 0; j < n; j++) {
        const int32_t x = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        r0 += x > v0;
        r1 += x > v1;
    }
    __syncwarp();
    if (lane < n) a[r0] = v0;
    if (lane + 32 < n) a[r1] = v1;
    __syncwarp();
}

__device__ void warp_emit_mfi(const ResPtrs& p, const int32_t* head, int head_len, int32_t t, const int32_t* extra_cols,
                              int n_extra, const int32_t* F, int32_t sup, int lane) {
    // max dense id decides the root rule
    int32_t mx = t;
    for (int q = lane; q < head_len; q += 32) mx = max(mx, head[q]);
    for (int q = lane; q < n_extra; q += 32) mx = max(mx, F[extra_cols[q]]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (!p.is_root[mx]) return;
    const int len = head_len + 1 + n_extra;
    int32_t k = 0, off = 0;
    if (lane == 0) {
        k = atomicAdd(&p.st->mfi_n, 1);
        off = atomicAdd(&p.st->mfi_item_n, len);
    }
    k = __shfl_sync(0xffffffffu, k, 0);
    off = __shfl_sync(0xffffffffu, off, 0);
    for (int q = lane; q < head_len; q += 32) p.mfi_items[off + q] = head[q];
    if (lane == 0) p.mfi_items[off + head_len] = t;
    for (int q = lane; q < n_extra; q += 32) p.mfi_items[off + head_len + 1 + q] = F[extra_cols[q]];
    warp_sort_desc(p.mfi_items + off, len, lane);
    if (lane == 0) {
        p.mfi_off[k] = off;
        p.mfi_len[k] = len;
        p.mfi_sup[k] = len == 1 ? p.dense_freq[t] : sup;   // a root's own frequency is its F1 count
    }
}

// Whether some indexed MFI (ids below `done`) holds every item of head[0, nh) and tail[0, nt):
// one index word per lane, ANDed over the items until every lane's word is zero.  Items
// beyond the index hold no indexed MFI.
__device__ bool warp_covered(const ResPtrs& p, int32_t done, const int32_t* head, int nh, const int32_t* tail, int nt,
                             int lane) {
    const int nw = (done + 31) >> 5;
    const int n = nh + nt;
    for (int w0 = 0; w0 < nw; w0 += 32) {
        const int w = w0 + lane;
        uint32_t acc = w < nw ? ~0u : 0u;
        if (w == nw - 1 && (done & 31)) acc = (1u << (done & 31)) - 1u;
        for (int q = 0; q < n; q++) {
            if (!__any_sync(0xffffffffu, acc != 0u)) break;
            const int32_t x = q < nh ? head[q] : tail[q - nh];
            if (x < 0 || x >= p.sup_items) acc = 0u;
            else if (acc) acc &= p.sup_index[(int64_t)x * p.sup_words + w];
        }
        if (__any_sync(0xffffffffu, acc != 0u)) return true;
    }
    return false;
}

__device__ void finish_row(const ResPtrs& p, DFam* f, int lane) {
    if (lane == 0) {
        const int32_t done = atomicAdd(&f->rows_done, 1) + 1;
        if (done == f->nT) {
            release_slot(p, f->slot);
            f->state = 2;
        }
    }
}

// The proposal network on one warp: lane i holds feature i.
__device__ float warp_mlp(const ResPtrs& p, float x, int lane) {
    const __nv_bfloat16* w = p.mlp_w;
    const float* P = p.mlp_p;
    constexpr int kIn = 32, kH = 64;
    constexpr int oW1 = 0, oB1 = kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
    float h1a = P[oB1 + lane], h1b = P[oB1 + lane + 32];
    for (int i = 0; i < kIn; i++) {
        const float xi = __shfl_sync(0xffffffffu, x, i);
        h1a = fmaf(__bfloat162float(w[oW1 + lane * kIn + i]), xi, h1a);
        h1b = fmaf(__bfloat162float(w[oW1 + (lane + 32) * kIn + i]), xi, h1b);
    }
    h1a = fmaxf(h1a, 0.f);
    h1b = fmaxf(h1b, 0.f);
    float h2a = P[oB2 + lane], h2b = P[oB2 + lane + 32];
    for (int j = 0; j < kH; j++) {
        const float hj = __shfl_sync(0xffffffffu, j < 32 ? h1a : h1b, j & 31);
        h2a = fmaf(__bfloat162float(w[oW2 + lane * kH + j]), hj, h2a);
        h2b = fmaf(__bfloat162float(w[oW2 + (lane + 32) * kH + j]), hj, h2b);
    }
    float z = __bfloat162float(w[oW3 + lane]) * fmaxf(h2a, 0.f) + __bfloat162float(w[oW3 + lane + 32]) * fmaxf(h2b, 0.f);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    z += P[oB3];
    return 1.f / (1.f + expf(-z));
}

// ---------------------------------------------------------------------------------- expand
// One warp per counted row of the wave.
__device__ void expand_row(const ResPtrs& p, int64_t g, int lane) {
    ResStatus* st = p.st;
    const int32_t jid = p.row_job[g];
    const int32_t r = p.row_local[g];
    const DJob dj = p.djobs[jid];
    const JobDesc jd = p.jobs[jid];
    const int32_t* crow = p.counts + jd.out_off + (int64_t)r * jd.n_cols;
    const int32_t minc = p.min_count;
    DFam* fp = p.fams + dj.fam;
    const DFam f = *fp;
    const int32_t* F = p.items + f.F_off;

    if (dj.kind == kJobLook) {
        const int32_t self = crow[jd.n_cols - 1];
        bool ext = false;
        for (int c = lane; c < jd.n_cols - 1; c += 32) ext |= crow[c] >= minc;
        ext = __any_sync(0xffffffffu, ext);
        if (lane == 0) {
            release_slot(p, dj.slot);
            if (dj.log >= 0) p.log_label[dj.log] = self >= minc ? 1.f : 0.f;
        }
        if (self >= minc) {
            if (lane == 0) atomicAdd(&st->hits, 1ull);
            if (!ext) {
                // head + whole tail: the tail is F[0..nT)
                const int32_t* head = p.heads + f.head_off;
                // emit head + F[0] ... F[nT-1]: treat F[0] as "t" and the rest as extra columns
                int32_t mx = -1;
                for (int q = lane; q < f.head_len; q += 32) mx = max(mx, head[q]);
                for (int q = lane; q < f.nT; q += 32) mx = max(mx, F[q]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                if (mx >= 0 && p.is_root[mx]) {
                    const int len = f.head_len + f.nT;
                    int32_t k = 0, off = 0;
                    if (lane == 0) {
                        k = atomicAdd(&st->mfi_n, 1);
                        off = atomicAdd(&st->mfi_item_n, len);
                    }
                    k = __shfl_sync(0xffffffffu, k, 0);
                    off = __shfl_sync(0xffffffffu, off, 0);
                    for (int q = lane; q < f.head_len; q += 32) p.mfi_items[off + q] = head[q];
                    for (int q = lane; q < f.nT; q += 32) p.mfi_items[off + f.head_len + q] = F[q];
                    warp_sort_desc(p.mfi_items + off, len, lane);
                    if (lane == 0) {
                        p.mfi_off[k] = off;
                        p.mfi_len[k] = len;
                        p.mfi_sup[k] = len == 1 ? p.dense_freq[F[0]] : self;
                    }
                }
            }
            if (lane == 0) {
                release_slot(p, f.slot);
                fp->state = 2;
            }
        } else if (lane == 0) {
            fp->state = 0;
            const int32_t k = atomicAdd(&st->stack_n, 1);
            p.stack[k] = dj.fam;
        }
        return;
    }

    // a family row: the child X = head(P) + t
    const int32_t i = dj.r0 + r;
    const int32_t nT = f.nT, nF = f.nF;
    const int32_t t = F[i];
    const int32_t supc = crow[i];
    if (supc < minc) {   // cannot happen: t is in F(P)
        if (lane == 0) atomicExch(&st->error, 1);
        finish_row(p, fp, lane);
        return;
    }
    // scan the row: extensions, equal-support items, tail.  Four loads in flight per lane;
    // `blocks` marks the column blocks of `bs` columns that hold an extension, so that the
    // later passes read only those.
    bool prune = false;
    int n_ext = 0, n_eq = 0, n_tail = 0;
    const int bs = column_block(nF);   // nF / bs <= 64, a multiple of 32
    unsigned long long blocks = 0;
    if (p.row_sum) {
        const RowSum rs = p.row_sum[g];
        n_ext = rs.n_ext; n_eq = rs.n_eq; n_tail = rs.n_tail; prune = rs.prune != 0; blocks = rs.blocks;
    }
    for (int c0 = 0; c0 < (p.row_sum ? 0 : nF); c0 += 128) {
        int32_t v4[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int c = c0 + 32 * u + lane;
            v4[u] = c < nF && c != i ? crow[c] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int c = c0 + 32 * u + lane;
            const int32_t v = v4[u];
            const bool e = v >= minc;
            const bool in_tail = c > i && c < nT;
            const bool eq = e && v == supc;
            prune |= eq && !in_tail;
            if (e) blocks |= 1ull << (c / bs);
            n_ext += __popc(__ballot_sync(0xffffffffu, e));
            n_eq += __popc(__ballot_sync(0xffffffffu, eq));
            n_tail += __popc(__ballot_sync(0xffffffffu, e && !eq && in_tail));
        }
    }
    prune = __any_sync(0xffffffffu, prune);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) blocks |= __shfl_xor_sync(0xffffffffu, blocks, o);
    if (prune) {
        if (lane == 0) atomicAdd(&st->pep, 1ull);
        finish_row(p, fp, lane);
        return;
    }
    const int32_t* head = p.heads + f.head_off;
    const int n_rest = n_ext - n_eq;
    if (n_rest == 0 || n_tail == 0) {
        if (n_rest == 0) {
            // MFI: head + t + the equal-support items.  Gather their columns into the item
            // pool's scratch (the emit reads F[col]).
            int32_t eoff = 0;
            if (lane == 0 && n_eq) eoff = atomicAdd(&st->item_n, n_eq);
            eoff = __shfl_sync(0xffffffffu, eoff, 0);
            int32_t* ecols = p.items + eoff;
            int pos = 0;
            for (unsigned long long bm = n_eq ? blocks : 0ull; bm; bm &= bm - 1) {
                const int b0 = (__ffsll((long long)bm) - 1) * bs;
                for (int c0 = b0; c0 < min(nF, b0 + bs); c0 += 32) {
                    const int c = c0 + lane;
                    const int32_t v = c < nF && c != i ? crow[c] : -1;
                    const bool eq = v >= minc && v == supc;
                    const unsigned bal = __ballot_sync(0xffffffffu, eq);
                    if (eq) ecols[pos + __popc(bal & ((1u << lane) - 1u))] = c;
                    pos += __popc(bal);
                }
            }
            __syncwarp();
            warp_emit_mfi(p, head, f.head_len, t, ecols, n_eq, F, supc, lane);
        }
        finish_row(p, fp, lane);
        return;
    }
    // the child family: head' = head + t + eq; F' = sorted tail, then the other extensions
    const int head_len = f.head_len + 1 + n_eq;
    int32_t fid = 0, foff = 0, hoff = 0;
    if (lane == 0) {
        fid = atomicAdd(&st->fam_n, 1);
        foff = atomicAdd(&st->item_n, n_rest + n_tail);   // + staging for the unsorted tail
        hoff = atomicAdd(&st->head_n, head_len);
    }
    fid = __shfl_sync(0xffffffffu, fid, 0);
    foff = __shfl_sync(0xffffffffu, foff, 0);
    hoff = __shfl_sync(0xffffffffu, hoff, 0);
    int32_t* Fc = p.items + foff;              // n_rest entries
    int32_t* stage = p.items + foff + n_rest;  // n_tail tail columns in column order
    int32_t* hc = p.heads + hoff;
    for (int q = lane; q < f.head_len; q += 32) hc[q] = head[q];
    if (lane == 0) hc[f.head_len] = t;
    int pos_eq = 0, pos_tail = 0, pos_rest = 0;
    for (unsigned long long bm = blocks; bm; bm &= bm - 1) {
        const int b0 = (__ffsll((long long)bm) - 1) * bs;
        for (int c0 = b0; c0 < min(nF, b0 + bs); c0 += 32) {
            const int c = c0 + lane;
            const int32_t v = c < nF && c != i ? crow[c] : -1;
            const bool e = v >= minc;
            const bool eq = e && v == supc;
            const bool tl = e && !eq && c > i && c < nT;
            const bool rs = e && !eq && !tl;
            const unsigned lt = (1u << lane) - 1u;
            const unsigned bq = __ballot_sync(0xffffffffu, eq), bt = __ballot_sync(0xffffffffu, tl),
                           br = __ballot_sync(0xffffffffu, rs);
            if (eq) hc[f.head_len + 1 + pos_eq + __popc(bq & lt)] = F[c];
            if (tl) stage[pos_tail + __popc(bt & lt)] = c;
            if (rs) Fc[n_tail + pos_rest + __popc(br & lt)] = F[c];
            pos_eq += __popc(bq);
            pos_tail += __popc(bt);
            pos_rest += __popc(br);
        }
    }
    __syncwarp();
    // tail sorted by (support, column), written as items to Fc[0 .. n_tail)
    if (n_tail <= 32) {
        unsigned long long key = ~0ull;
        if (lane < n_tail) {
            const int32_t c = stage[lane];
            key = ((unsigned long long)(uint32_t)crow[c] << 32) | (uint32_t)c;
        }
        // bitonic sort across the warp, ascending
        for (int k = 2; k <= 32; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, j);
                const bool up = (lane & k) == 0;
                const bool lower = (lane & j) == 0;
                const bool take_min = (lower == up);
                key = take_min ? min(key, other) : max(key, other);
            }
        if (lane < n_tail) Fc[lane] = F[(int32_t)(key & 0xffffffffu)];
    } else if (n_tail <= 4096) {
        for (int a = lane; a < n_tail; a += 32) {
            const int32_t ca = stage[a];
            const unsigned long long ka = ((unsigned long long)(uint32_t)crow[ca] << 32) | (uint32_t)ca;
            int rank = 0;
            for (int b = 0; b < n_tail; b++) {
                const int32_t cb = stage[b];
                const unsigned long long kb = ((unsigned long long)(uint32_t)crow[cb] << 32) | (uint32_t)cb;
                rank += kb < ka;
            }
            Fc[rank] = F[ca];
        }
    } else {
        for (int a = lane; a < n_tail; a += 32) Fc[a] = F[stage[a]];
    }
    __syncwarp();
    // superset check: every itemset of the child's subtree lies inside head' + tail; when an
    // MFI of an earlier wave holds them all, none of those itemsets is a new maximal set
    if (p.sup_index && warp_covered(p, p.st->sup_done, hc, head_len, Fc, n_tail, lane)) {
        if (lane == 0) atomicAdd(&st->sup_pruned, 1ull);
        finish_row(p, fp, lane);
        return;
    }
    // base mask of the child
    int32_t cslot = -1, citem = -1;
    if (f.slot < 0 && f.item < 0) {
        citem = t;
    } else {
        if (lane == 0) cslot = pop_slot(p);
        cslot = __shfl_sync(0xffffffffu, cslot, 0);
        emit_mask(p, cslot, f.slot, f.item, t, 0, 0, lane);
    }
    // lookahead decision
    bool issue = false;
    float feat = 0.f;
    int log_idx = -1;
    const int list_len = n_tail + 1 + (f.item >= 0 ? 1 : 0);
    if (p.la_mode != 0 && n_tail >= 2 && list_len <= kMaxListLen) {
        // tail-pair filter: rows of tail items that are in this job's row range
        int pairs = 0, pairs_ok = 0;
        for (int a = 0; a < n_tail; a++) {
            const int32_t ra = stage[a];
            if (ra < dj.r0 || ra >= dj.r0 + dj.nr) continue;
            const int32_t* rowa = p.counts + jd.out_off + (int64_t)(ra - dj.r0) * jd.n_cols;
            for (int b = a + 1 + lane; b < n_tail; b += 32) {
                pairs++;
                pairs_ok += rowa[stage[b]] >= minc;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
            pairs_ok += __shfl_xor_sync(0xffffffffu, pairs_ok, o);
        }
        const bool filtered = pairs_ok < pairs;
        if (filtered && p.la_mode != 3) {
            if (lane == 0) atomicAdd(&st->skipped, 1ull);
        } else {
            issue = true;
            if (p.la_mode == 2 || p.log_on) {
                // features (same definitions as the host engine's)
                double mn = 1e30, mn2 = 1e30, mx = 0, sum = 0, sum2 = 0, logprod = 0;
                int gt90 = 0, gt99 = 0;
                for (int a = 0; a < n_tail; a++) {
                    const double rr = (double)crow[stage[a]] / (double)supc;
                    if (rr < mn) { mn2 = mn; mn = rr; } else if (rr < mn2) mn2 = rr;
                    mx = fmax(mx, rr);
                    sum += rr;
                    sum2 += rr * rr;
                    logprod += log(fmax(rr, 1e-12));
                    gt90 += rr > 0.9;
                    gt99 += rr > 0.99;
                }
                const int k = n_tail;
                const double mean = sum / k, var = fmax(0.0, sum2 / k - mean * mean);
                const double minc_d = max(1, minc);
                const bool top_child = f.slot < 0 && f.item < 0;
                const double pf = pairs ? (double)pairs_ok / (double)pairs : 1.0;
                double v = 0.0;
                switch (lane) {
                    case 0: v = head_len / 16.0; break;
                    case 1: v = k / 32.0; break;
                    case 2: v = n_rest / 64.0; break;
                    case 3: v = (double)supc / (double)lmax(1, p.n_bits); break;
                    case 4: v = log2(1.0 + supc) / 24.0; break;
                    case 5: v = mn; break;
                    case 6: v = mean; break;
                    case 7: v = mx; break;
                    case 8: v = fmin(mn * supc / minc_d, 8.0) / 8.0; break;
                    case 9: v = exp(logprod); break;
                    case 10: v = fmax(-8.0, fmin(8.0, logprod + log(supc / minc_d))) / 8.0; break;
                    case 11: v = pf; break;
                    case 12: v = (n_rest - k) / 64.0; break;
                    case 13: v = minc_d / (double)lmax(1, p.n_bits); break;
                    case 14: v = fmin(supc / minc_d, 64.0) / 64.0; break;
                    case 15: v = sqrt(var); break;
                    case 16: v = k > 1 ? mn2 : mn; break;
                    case 17: v = (double)gt90 / k; break;
                    case 18: v = (double)gt99 / k; break;
                    case 19: v = log2(1.0 + k) / 6.0; break;
                    case 20: v = n_eq / 8.0; break;
                    case 21: v = nT / 64.0; break;
                    case 22: v = (double)i / (double)max(1, nT); break;
                    case 23: v = top_child ? 1.0 : 0.0; break;
                    default: v = 0.0;
                }
                feat = (float)v;
                if (p.la_mode == 2 && p.mlp_w) {
                    const float prob = warp_mlp(p, feat, lane);
                    if (prob < p.proposal_threshold) {
                        issue = false;
                        if (lane == 0) atomicAdd(&st->skipped, 1ull);
                    }
                }
            }
        }
    }
    if (issue && p.log_on) {
        if (lane == 0) log_idx = atomicAdd(&st->log_n, 1);
        log_idx = __shfl_sync(0xffffffffu, log_idx, 0);
        p.log_feat[(int64_t)log_idx * 32 + lane] = feat;
        if (lane == 0) p.log_label[log_idx] = 0.f;
    }
    // the child record
    if (lane == 0) {
        DFam ch;
        ch.slot = cslot; ch.item = citem; ch.head_off = hoff; ch.head_len = head_len;
        ch.F_off = foff; ch.nF = n_rest; ch.nT = n_tail; ch.sup = supc;
        ch.next_row = 0; ch.rows_done = 0; ch.state = issue ? 1 : 0; ch.top = 0;
        p.fams[fid] = ch;
    }
    if (issue) {
        int32_t ls = 0;
        if (lane == 0) ls = pop_slot(p);
        ls = __shfl_sync(0xffffffffu, ls, 0);
        // mask of head + tail: the child's base (the parent's sources and t) & the tail rows
        emit_mask(p, ls, f.slot, f.item, t, foff, n_tail, lane);
        if (lane == 0) {
            const int32_t q = atomicAdd(&st->look_n, 1);
            p.looks[q] = DLook{fid, ls, log_idx, 0};
            atomicAdd(&st->lookaheads, 1ull);
        }
    } else if (lane == 0) {
        const int32_t k = atomicAdd(&st->stack_n, 1);
        p.stack[k] = fid;
    }
    __syncwarp();
    finish_row(p, fp, lane);
}

__global__ void __launch_bounds__(256) k_res_expand(ResPtrs p) {
    phase_begin(&p.st->ph_s[kPhExpand]);
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (g < p.st->rows) expand_row(p, g, threadIdx.x & 31);
    phase_end(&p.st->ph_e[kPhExpand]);
}

// The masks the expand asked for, with the whole grid: units of 1,024 128-bit words of one
// mask, strided over the blocks (one warp building a 1,000,000-bit mask alone would take a
// chain of ~250 dependent load rounds).
__device__ __forceinline__ void build_masks(const ResPtrs& p) {
    const int32_t n = p.st->n_mjobs;
    const int64_t W4 = p.W >> 2;
    const int64_t chunks = (W4 + 1023) / 1024;
    const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
    for (int64_t u = blockIdx.x; u < (int64_t)n * chunks; u += gridDim.x) {
        const MaskJob mj = p.mjobs[u / chunks];
        const int64_t c0 = (u % chunks) * 1024, c1 = lmin(W4, c0 + 1024);
        uint4* d = reinterpret_cast<uint4*>(p.masks + (int64_t)mj.dst * p.W);
        const uint4* sm = mj.slot >= 0 ? reinterpret_cast<const uint4*>(p.masks + (int64_t)mj.slot * p.W) : nullptr;
        const uint4* si = mj.item >= 0 ? reinterpret_cast<const uint4*>(p.bitmap + (int64_t)mj.item * p.W) : nullptr;
        const uint4* st = mj.t >= 0 ? reinterpret_cast<const uint4*>(p.bitmap + (int64_t)mj.t * p.W) : nullptr;
        for (int64_t w = c0 + threadIdx.x; w < c1; w += blockDim.x) {
            uint4 v = ones;
            auto andv = [&](uint4 x) { v.x &= x.x; v.y &= x.y; v.z &= x.z; v.w &= x.w; };
            if (sm) andv(sm[w]);
            if (si) andv(__ldg(si + w));
            if (st) andv(__ldg(st + w));
            for (int q = 0; q < mj.n; q++)
                andv(__ldg(reinterpret_cast<const uint4*>(p.bitmap + (int64_t)p.items[mj.off + q] * p.W) + w));
            d[w] = v;
        }
    }
}
__global__ void __launch_bounds__(256) k_build_masks(ResPtrs p) {
    phase_begin(&p.st->ph_s[kPhMasks]);
    build_masks(p);
    phase_end(&p.st->ph_e[kPhMasks]);
}

// Add the MFIs emitted since the last pack to the superset index: one warp per MFI, one
// atomicOr per item.  An MFI holding an item beyond the index is left out (it then prunes
// nothing); so are MFIs beyond the index's capacity.
__device__ void index_mfis(const ResPtrs& p) {
    if (!p.sup_index) return;
    const int32_t lo = p.st->sup_done;
    const int32_t hi = min(p.st->mfi_n, p.sup_words * 32);
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t k = lo + (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; k < hi; k += warps) {
        const int32_t off = p.mfi_off[k], len = p.mfi_len[k];
        bool ok = true;
        for (int q = lane; q < len; q += 32) {
            const int32_t x = p.mfi_items[off + q];
            ok &= x >= 0 && x < p.sup_items;
        }
        if (!__all_sync(0xffffffffu, ok)) continue;
        const uint32_t bit = 1u << (k & 31);
        for (int q = lane; q < len; q += 32)
            atomicOr(&p.sup_index[(int64_t)p.mfi_items[off + q] * p.sup_words + (k >> 5)], bit);
    }
}
__global__ void __launch_bounds__(256) k_index_mfis(ResPtrs p) {
    phase_begin(&p.st->ph_s[kPhMasks]);
    index_mfis(p);
    phase_end(&p.st->ph_e[kPhMasks]);
}

// Families waiting on the stack that an MFI found since their creation covers: a fresh
// family (no row handed out, not waiting on a lookahead) whose head and whole tail lie inside
// an indexed MFI is marked finished and its mask slot released; the pack then pops it without
// a job.  One warp per stack entry, from the top, over the entries the next waves take first.
__device__ void prune_stack(const ResPtrs& p) {
    if (!p.sup_index) return;
    ResStatus* st = p.st;
    const int32_t done = min(st->mfi_n, p.sup_words * 32);   // k_index_mfis has indexed these
    const int32_t n = st->stack_n;
    const int32_t depth = min(n, 4 * p.wave_rows);
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; k < depth; k += warps) {
        const int32_t fid = p.stack[n - 1 - k];
        DFam* fp = p.fams + fid;
        const DFam f = *fp;
        if (f.state != 0 || f.next_row != 0 || f.rows_done != 0 || f.top) continue;
        if (warp_covered(p, done, p.heads + f.head_off, f.head_len, p.items + f.F_off, f.nT, lane) && lane == 0) {
            fp->state = 2;
            release_slot(p, f.slot);
            atomicAdd(&st->sup_pruned, 1ull);
        }
    }
}
__global__ void __launch_bounds__(256) k_prune_stack(ResPtrs p) {
    phase_begin(&p.st->ph_s[kPhMasks]);
    prune_stack(p);
    phase_end(&p.st->ph_e[kPhMasks]);
}

// The expand's first pass for the family of the empty prefix (an n x n count block whose
// rows are its tail, nT = nF = n): one block per row streams the row with four loads in
// flight per thread and writes the row's summary.
__global__ void __launch_bounds__(256) k_top_summary(const int32_t* __restrict__ M, int32_t n, int32_t minc,
                                                     RowSum* __restrict__ out) {
    const int32_t i = blockIdx.x;
    const int32_t* row = M + (int64_t)i * n;
    const int32_t supc = row[i];
    const int bs = column_block(n);
    int n_ext = 0, n_eq = 0, n_tail = 0, prune = 0;
    unsigned long long blocks = 0;
    for (int c0 = threadIdx.x; c0 < n; c0 += 4 * 256) {
        int32_t v4[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int c = c0 + u * 256;
            v4[u] = c < n && c != i ? __ldg(row + c) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int c = c0 + u * 256;
            const bool e = v4[u] >= minc;
            const bool eq = e && v4[u] == supc;
            const bool in_tail = c > i;
            n_ext += e;
            n_eq += eq;
            n_tail += e && !eq && in_tail;
            prune |= eq && !in_tail;
            if (e) blocks |= 1ull << (c / bs);
        }
    }
    typedef cub::BlockReduce<int, 256> RedI;
    __shared__ typename RedI::TempStorage ti;
    __shared__ unsigned long long s_blocks;
    if (threadIdx.x == 0) s_blocks = 0;
    __syncthreads();
    if (blocks) atomicOr(&s_blocks, blocks);
    const int a = RedI(ti).Sum(n_ext);
    __syncthreads();
    const int b = RedI(ti).Sum(n_eq);
    __syncthreads();
    const int t = RedI(ti).Sum(n_tail);
    __syncthreads();
    const int pr = RedI(ti).Reduce(prune, cub::Max());
    __syncthreads();
    if (threadIdx.x == 0) out[i] = RowSum{a, b, t, pr, s_blocks, 0};
}

// ---------------------------------------------------------------------------------- graph loop
// The wave loop as a graph: a conditional WHILE node whose body is
//   pack -> zero the count block -> persistent counters -> persistent expand -> control.
// Every kernel reads its arguments from the ResArgs record and its sizes from the status
// record, so the launch shapes are fixed.  The control kernel ends the loop when the search
// is done, when the pack asks for larger pools or reports an error, or after the slice's
// wave / time limit; the host then reads the status once.

// Zero the wave's count block and the persistent counters' tile counters.
__global__ void __launch_bounds__(256) k_res_zero(const ResArgs* __restrict__ args) {
    ResStatus* st = args->p.st;
    int32_t* counts = args->p.counts;
    phase_begin(&st->ph_s[kPhZero]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->next3 = 0;
        st->next1 = 0;
        st->next_tc = 0;
        st->next_gr = 0;
    }
    const int64_t n = st->out_total;
    const int64_t n4 = n >> 2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int4* c4 = reinterpret_cast<int4*>(counts);
    for (int64_t i = i0; i < n4; i += stride) c4[i] = make_int4(0, 0, 0, 0);
    for (int64_t i = (n4 << 2) + i0; i < n; i += stride) counts[i] = 0;
    phase_end(&st->ph_e[kPhZero]);
}

__global__ void __launch_bounds__(256) k_res_expand_g(const ResArgs* __restrict__ args) {
    const ResPtrs p = args->p;
    const int lane = threadIdx.x & 31;
    phase_begin(&p.st->ph_s[kPhExpand]);
    const int32_t rows = p.st->rows;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < rows; g += warps) expand_row(p, g, lane);
    phase_end(&p.st->ph_e[kPhExpand]);
}

__global__ void __launch_bounds__(256) k_build_masks_g(const ResArgs* __restrict__ args) {
    const ResPtrs p = args->p;
    phase_begin(&p.st->ph_s[kPhMasks]);
    build_masks(p);
    phase_end(&p.st->ph_e[kPhMasks]);
}

__global__ void __launch_bounds__(256) k_index_mfis_g(const ResArgs* __restrict__ args) {
    phase_begin(&args->p.st->ph_s[kPhMasks]);
    index_mfis(args->p);
    phase_end(&args->p.st->ph_e[kPhMasks]);
}
__global__ void __launch_bounds__(256) k_prune_stack_g(const ResArgs* __restrict__ args) {
    phase_begin(&args->p.st->ph_s[kPhMasks]);
    prune_stack(args->p);
    phase_end(&args->p.st->ph_e[kPhMasks]);
}

__global__ void k_res_control(const ResArgs* __restrict__ args, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    ResStatus* st = args->p.st;
    const bool progressed = st->jobs > 0;
    if (progressed) st->waves += 1;
    const bool go = progressed && !st->error && !st->grow && !st->starved && st->waves < args->p.wave_limit &&
                    globaltimer() - st->launch_t0 < args->p.max_launch_ns;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ------------------------------------------------------------------------ output order
// The MFIs leave the device in their output order: descending support, then item lists
// (each in descending order) compared lexicographically, larger first.  The sort key packs
// the support and the two largest items, complemented so that an ascending radix sort gives
// that order.  Narrow keys (support below 2^24, item ids below 2^20 - 1) hold both items;
// wide ones only the first.  Lists whose keys are equal are finished on the host.
__global__ void __launch_bounds__(256) k_mfi_keys(const int32_t* __restrict__ off, const int32_t* __restrict__ len,
                                                  const int32_t* __restrict__ sup, const int32_t* __restrict__ items,
                                                  int32_t n, int wide, uint64_t* __restrict__ keys,
                                                  int32_t* __restrict__ idx) {
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int32_t o = off[k], l = len[k];
        int32_t a = -1, b = -1;   // the two largest items
        for (int32_t q = 0; q < l; q++) {
            const int32_t x = items[o + q];
            if (x > a) {
                b = a;
                a = x;
            } else if (x > b) {
                b = x;
            }
        }
        const uint32_t s = (uint32_t)sup[k];
        uint64_t key;
        if (wide) key = ((uint64_t)(0xFFFFFFFFu - s) << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)(a + 1));
        else
            key = ((uint64_t)(0xFFFFFFu - s) << 40) | ((uint64_t)(0xFFFFFu - (uint32_t)(a + 1)) << 20) |
                  (uint64_t)(0xFFFFFu - (uint32_t)(b + 1));
        keys[k] = key;
        idx[k] = k;
    }
}

// Lengths and supports in sorted order.
__global__ void __launch_bounds__(256) k_mfi_permute(const int32_t* __restrict__ idx, const int32_t* __restrict__ len,
                                                     const int32_t* __restrict__ sup, int32_t n,
                                                     int32_t* __restrict__ len_o, int32_t* __restrict__ sup_o) {
    for (int32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int32_t k = idx[q];
        len_o[q] = len[k];
        sup_o[q] = sup[k];
    }
}

// Item lists in sorted order: one warp per MFI.
__global__ void __launch_bounds__(256) k_mfi_gather(const int32_t* __restrict__ idx, const int32_t* __restrict__ off,
                                                    const int32_t* __restrict__ items, const int32_t* __restrict__ off_o,
                                                    const int32_t* __restrict__ len_o, int32_t n,
                                                    int32_t* __restrict__ items_o) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t q = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); q < n; q += warps) {
        const int32_t* src = items + off[idx[q]];
        int32_t* dst = items_o + off_o[q];
        for (int32_t x = lane; x < len_o[q]; x += 32) dst[x] = src[x];
    }
}

// ---------------------------------------------------------------------------------- host
struct Pool {
    void* p = nullptr;
    size_t bytes = 0;
};

int grow(Pool& b, size_t need, cudaStream_t s, size_t min_bytes = 1 << 16) {
    if (need <= b.bytes && b.p) return TFIM_OK;
    size_t cap = std::max<size_t>(need + need / 2, min_bytes);
    void* np = nullptr;
    TFIM_TRY(dev_alloc(&np, cap, s));
    if (b.p && b.bytes) TFIM_CUDA(cudaMemcpyAsync(np, b.p, b.bytes, cudaMemcpyDeviceToDevice, s));
    dev_free(b.p, s);
    b.p = np;
    b.bytes = cap;
    return TFIM_OK;
}

// The captured wave loop.  Its launches read ResArgs at `args` and sizes from the status
// record at `status`; it is rebuilt when either moves or the set of counters changes.
struct WaveGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* args = nullptr;
    const void* status = nullptr;
    int with_proj = -1;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        args = status = nullptr;
        with_proj = -1;
    }
};

int build_wave_graph(WaveGraph& G, const ResArgs* d_args, ResStatus* d_status, bool with_proj, const int64_t* red_off,
                     const int32_t* red_items, cudaStream_t s) {
    G.release();
    int sm = 148, dev = 0, occ3 = 1, occ1 = 1, occp = 1, occe = 1, occg = 1;
    TFIM_CUDA(cudaGetDevice(&dev));
    TFIM_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));
    TFIM_TRY(persistent_occupancy(&occ3, &occ1, &occp));
    TFIM_TRY(configure_fam_kernel());
    TFIM_TRY(occupancy_gram(&occg));
    TFIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occe, k_res_expand_g, 256, 0));
    TFIM_CUDA(cudaGraphCreate(&G.graph, 0));
    cudaGraphConditionalHandle h;
    TFIM_CUDA(cudaGraphConditionalHandleCreate(&h, G.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TFIM_CUDA(cudaGraphAddNode(&node, G.graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    TFIM_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int rc = TFIM_OK;
    do {
        k_res_pack_g<<<1, kPackThreads, 0, s>>>(d_args);
        k_res_zero<<<sm * 4, 256, 0, s>>>(d_args);
        if ((rc = launch_count_lop3_persistent(&d_args->a3, &d_status->tiles_l3, &d_status->next3, sm * std::max(1, occ3), s)))
            break;
        if ((rc = launch_count_b1_persistent(&d_args->a1, &d_status->tiles_b1, &d_status->next1, sm * std::max(1, occ1), s)))
            break;
        if (with_proj &&
            (rc = launch_count_proj_persistent(&d_args->ap, &d_status->n_proj, sm * std::max(1, occp), red_off, red_items, s)))
            break;
        if ((rc = launch_count_fam_persistent(&d_args->atc, &d_status->tiles_tc, &d_status->next_tc, sm, s))) break;
        if ((rc = launch_count_gram_persistent(&d_args->agr, &d_status->tiles_gr, &d_status->next_gr, sm * std::max(1, occg),
                                               s)))
            break;
        k_res_expand_g<<<sm * std::max(1, occe), 256, 0, s>>>(d_args);
        k_build_masks_g<<<sm * 8, 256, 0, s>>>(d_args);
        k_index_mfis_g<<<sm, 256, 0, s>>>(d_args);
        k_prune_stack_g<<<sm, 256, 0, s>>>(d_args);
        k_res_control<<<1, 32, 0, s>>>(d_args, h);
    } while (0);
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(s, &captured);
    if (rc != TFIM_OK) return rc;
    TFIM_CUDA(ec);
    TFIM_CUDA(cudaGetLastError());
    TFIM_CUDA(cudaGraphInstantiate(&G.exec, G.graph, 0));
    G.args = d_args;
    G.status = d_status;
    G.with_proj = with_proj ? 1 : 0;
    return TFIM_OK;
}

}  // namespace

struct ResidentState {
    Pool fams, items, heads, stack, looks, free_slots, defer, mfi_off, mfi_len, mfi_sup, mfi_items, log_feat, log_label;
    Pool djobs, jobs, rows, row_job, row_local, tiles_l3, tiles_b1, tiles_tc, tiles_gr, counts, status, is_root, dense_freq, top_pos,
        top_diag, proj_list, args, top_sum, mjobs, sup_index;
    Pool ord_keys, ord_idx, ord_meta, ord_items, ord_tmp;   // output order of the MFIs
    HostBuf h_status, h_args, h_res, h_setup;
    // the database's part of the search's initial state (root flags, the top family in
    // increasing support order), computed at a context's first resident mine and its pinned
    // staging reused by later mines; setup_uid names the context it belongs to
    uint64_t setup_uid = 0;
    std::vector<char> is_root_h;
    std::vector<int32_t> F0;
    size_t setup_total = 0;
    WaveGraph graph;
    int32_t launch_id = 0;
    void release(cudaStream_t s) {
        graph.release();
        for (Pool* b : {&fams, &items, &heads, &stack, &looks, &free_slots, &defer, &mfi_off, &mfi_len, &mfi_sup, &mfi_items,
                        &log_feat, &log_label, &djobs, &jobs, &rows, &row_job, &row_local, &tiles_l3, &tiles_b1, &tiles_tc, &tiles_gr, &counts,
                        &status, &is_root, &dense_freq, &top_pos, &top_diag, &proj_list, &args, &top_sum, &mjobs,
                        &sup_index, &ord_keys, &ord_idx, &ord_meta, &ord_items, &ord_tmp}) {
            dev_free(b->p, s);
            b->p = nullptr;
            b->bytes = 0;
        }
        h_status.release();
        h_args.release();
        h_res.release();
        h_setup.release();
    }
};

void free_resident(ResidentState* r, cudaStream_t s) {
    if (!r) return;
    r->release(s);
    delete r;
}

// Resident-engine pools and mask pools of closed contexts, one of each per device.  A
// context that closes after its work has finished hands them over (its stream is idle); the
// next context's first resident mine on that device adopts them, so a database opened again
// starts from pools already grown to the last search's size instead of growing (and copying)
// them from their minimum.  tfim_release_cached frees them.
namespace {
std::mutex g_cache_mu;
ResidentState* g_cached_res[64] = {};
DevBuf g_cached_masks[64];
}  // namespace

void stash_resident(tfim_ctx* c) {
    const int dev = c->device;
    if (dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (c->resident) {
        c->resident->graph.release();   // its launches hold this context's transaction list
        if (g_cached_res[dev]) free_resident(g_cached_res[dev], c->stream);
        g_cached_res[dev] = c->resident;
        c->resident = nullptr;
    }
    if (c->d_masks.p && c->d_masks.bytes > g_cached_masks[dev].bytes) {
        g_cached_masks[dev].release();
        g_cached_masks[dev] = c->d_masks;
        // the closing context's stream is idle and about to be destroyed: a cached buffer
        // holds no stream (freed on the default stream, adopted onto the adopter's)
        g_cached_masks[dev].stream = nullptr;
        c->d_masks.p = nullptr;
        c->d_masks.bytes = 0;
    }
}

void adopt_resident(tfim_ctx* c) {
    const int dev = c->device;
    if (dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (!c->resident && g_cached_res[dev]) {
        c->resident = g_cached_res[dev];
        g_cached_res[dev] = nullptr;
    }
    if (g_cached_masks[dev].p && g_cached_masks[dev].bytes > c->d_masks.bytes) {
        c->d_masks.release();
        c->d_masks = g_cached_masks[dev];
        c->d_masks.stream = c->stream;
        g_cached_masks[dev].p = nullptr;
        g_cached_masks[dev].bytes = 0;
    }
}

int release_cached(int dev) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (int d = 0; d < 64; d++) {
        if (dev >= 0 && d != dev) continue;
        if (!g_cached_res[d] && !g_cached_masks[d].p) continue;
        TFIM_CUDA(cudaSetDevice(d));
        if (g_cached_res[d]) free_resident(g_cached_res[d], nullptr);
        g_cached_res[d] = nullptr;
        g_cached_masks[d].stream = nullptr;
        g_cached_masks[d].release();
        TFIM_CUDA(cudaDeviceSynchronize());
    }
    return TFIM_OK;
}

namespace {
// Sorts the n MFIs of the pool (ni items) into output order on the device and queues the
// copies of their sort keys (hkey[n]), lengths then supports (hmeta[2n]) and items
// (hitems[ni]) into pinned host memory; they are valid once the stream has finished.
int order_mfis(ResidentState& R, const tfim_ctx* c, const ResPtrs& P, int32_t n, int64_t ni, int sm_count,
               cudaStream_t s, uint64_t* hkey, int32_t* hmeta, int32_t* hitems) {
    int32_t max_sup = 0;
    for (int32_t f : c->dense_freq) max_sup = std::max(max_sup, f);
    const int wide = c->n_bits > 0xFFFFFF || max_sup > 0xFFFFFF || c->info.n_dense > 0xFFFFF ? 1 : 0;
    size_t t_sort = 0, t_scan = 0;
    TFIM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                              (const int32_t*)nullptr, (int32_t*)nullptr, n, 0, 64, s));
    TFIM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, (const int32_t*)nullptr, (int32_t*)nullptr, n, s));
    TFIM_TRY(grow(R.ord_keys, (size_t)n * 16, s));
    TFIM_TRY(grow(R.ord_idx, (size_t)n * 8, s));
    TFIM_TRY(grow(R.ord_meta, ((size_t)n * 3 + 1) * 4, s));
    TFIM_TRY(grow(R.ord_items, (size_t)std::max<int64_t>(ni, 1) * 4, s));
    TFIM_TRY(grow(R.ord_tmp, std::max<size_t>(std::max(t_sort, t_scan), 16), s));
    uint64_t* k_in = (uint64_t*)R.ord_keys.p;
    uint64_t* k_out = k_in + n;
    int32_t* i_in = (int32_t*)R.ord_idx.p;
    int32_t* i_out = i_in + n;
    int32_t* len_o = (int32_t*)R.ord_meta.p;
    int32_t* sup_o = len_o + n;
    int32_t* off_o = sup_o + n;
    int32_t* items_o = (int32_t*)R.ord_items.p;
    const unsigned grid = (unsigned)std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)sm_count * 8);
    k_mfi_keys<<<grid, 256, 0, s>>>(P.mfi_off, P.mfi_len, P.mfi_sup, P.mfi_items, n, wide, k_in, i_in);
    TFIM_CUDA(cudaGetLastError());
    size_t t = R.ord_tmp.bytes;
    TFIM_CUDA(cub::DeviceRadixSort::SortPairs(R.ord_tmp.p, t, k_in, k_out, i_in, i_out, n, 0, 64, s));
    k_mfi_permute<<<grid, 256, 0, s>>>(i_out, P.mfi_len, P.mfi_sup, n, len_o, sup_o);
    TFIM_CUDA(cudaGetLastError());
    t = R.ord_tmp.bytes;
    TFIM_CUDA(cub::DeviceScan::ExclusiveSum(R.ord_tmp.p, t, len_o, off_o, n, s));
    const unsigned ggrid = (unsigned)std::min<int64_t>(((int64_t)n + 7) / 8, (int64_t)sm_count * 8);
    k_mfi_gather<<<ggrid, 256, 0, s>>>(i_out, P.mfi_off, P.mfi_items, off_o, len_o, n, items_o);
    TFIM_CUDA(cudaGetLastError());
    TFIM_CUDA(cudaMemcpyAsync(hkey, k_out, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    TFIM_CUDA(cudaMemcpyAsync(hmeta, len_o, (size_t)n * 8, cudaMemcpyDeviceToHost, s));   // len_o, sup_o
    if (ni) TFIM_CUDA(cudaMemcpyAsync(hitems, items_o, (size_t)ni * 4, cudaMemcpyDeviceToHost, s));
    return TFIM_OK;
}

// Finishes the output order on the host: item lists longer than 64 (the device sorts
// shorter ones as it emits them) are sorted, then each run of equal sort keys is ordered by
// the full comparison of item lists.
void finish_mfi_order(MfiSet& M, const uint64_t* key) {
    const size_t n = M.size();
    for (size_t k = 0; k < n; k++)
        if (M.off[k + 1] - M.off[k] > 64)
            std::sort(M.items.begin() + M.off[k], M.items.begin() + M.off[k + 1], std::greater<int32_t>());
    std::vector<int32_t> idx, items;
    for (size_t a = 0; a < n;) {
        size_t b = a + 1;
        while (b < n && key[b] == key[a]) b++;
        if (b - a > 1) {
            idx.resize(b - a);
            for (size_t q = a; q < b; q++) idx[q - a] = (int32_t)q;
            std::sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) {
                return std::lexicographical_compare(M.items.begin() + M.off[y], M.items.begin() + M.off[y + 1],
                                                    M.items.begin() + M.off[x], M.items.begin() + M.off[x + 1]);
            });
            items.assign(M.items.begin() + M.off[a], M.items.begin() + M.off[b]);
            const int64_t base = M.off[a];
            int64_t o = base;
            for (int32_t q : idx) {
                const int64_t l = M.off[q + 1] - M.off[q];
                std::copy(items.begin() + (M.off[q] - base), items.begin() + (M.off[q] - base) + l, M.items.begin() + o);
                o += l;
            }
            // supports are equal within the run; the offsets follow the new lengths
            std::vector<int64_t> lens(b - a);
            for (size_t q = 0; q < idx.size(); q++) lens[q] = M.off[idx[q] + 1] - M.off[idx[q]];
            for (size_t q = 0; q < idx.size(); q++) M.off[a + q + 1] = M.off[a + q] + lens[q];
        }
        a = b;
    }
}
}  // namespace

int mine_resident(tfim_ctx* c, const tfim_mine_opts* o, tfim_mine_stats* stt) {
    const auto t_entry = std::chrono::steady_clock::now();
    cudaStream_t s = c->stream;
    const int32_t d = c->n_counted;
    const int32_t minc = c->info.min_count;
    const int64_t W = c->W;
    const int32_t la_mode = o->lookahead;
    TFIM_CHECK(la_mode != 2 || c->proposal, TFIM_E_STATE, "lookahead mode 2 needs a proposal network (tfim_set_proposal)");
    if (!c->resident) adopt_resident(c);
    if (!c->resident) c->resident = new ResidentState();
    ResidentState& R = *c->resident;
    c->la_feats.clear();
    c->la_labels.clear();

    const bool fresh_setup = R.setup_uid != c->uid;
    if (fresh_setup) {
        R.is_root_h.assign((size_t)c->info.n_dense + 1, 0);
        for (int32_t r : c->roots) R.is_root_h[r] = 1;
        // top family: the counted items frequent by bitmap support, increasing support
        R.F0.clear();
        for (int32_t e = 0; e < d; e++)
            if (c->bit_support[e] >= minc) R.F0.push_back(e);
        std::stable_sort(R.F0.begin(), R.F0.end(),
                         [&](int32_t a, int32_t b) { return c->bit_support[a] < c->bit_support[b]; });
    }
    const std::vector<char>& is_root = R.is_root_h;
    const std::vector<int32_t>& F0 = R.F0;
    // the parked id 0 used as a root: the reference's search for that root (host driver)
    if (c->info.n_dense > d && is_root[d]) TFIM_TRY(mine_plain_roots(c, {d}, stt));
    const int32_t n0 = (int32_t)F0.size();
    if (n0 == 0) return TFIM_OK;

    int sm_count = 148;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
    }
    const tfim_tuning tn = tuning();
    const int32_t wave_rows = o->wave_cap > 0 ? o->wave_cap : tn.wave_rows;
    const int64_t top_out = (int64_t)n0 * n0;
    const bool small = o->small_pools != 0;
    const size_t gmin = small ? 64 : (1 << 16);
    auto grow = [&](Pool& b, size_t need, cudaStream_t st) { return tfim::grow(b, need, st, gmin); };
    int64_t cap_out = small ? top_out : std::max<int64_t>(top_out, 64LL << 20);
    int64_t cap_tiles = small ? 64 : 1LL << 21;
    int64_t cap_rows = std::max<int64_t>(wave_rows, n0) + 64;

    // initial capacities (the first wave's ensure grows them to what its expand needs)
    int64_t cap_fam = small ? 1 : std::max<int64_t>(4 * n0, 1 << 16);
    int64_t cap_item = small ? n0 : std::max<int64_t>(4 * top_out + 2 * n0, 1 << 20);   // holds the top family's list
    int64_t cap_head = 1 << 20, cap_mfi = 1 << 16, cap_mfi_items = 1 << 20, cap_slots = 1 << 12, cap_log = 1 << 16;
    if (small) cap_head = cap_mfi = cap_mfi_items = cap_slots = cap_log = 1;
    TFIM_TRY(grow(R.status, sizeof(ResStatus), s));
    TFIM_TRY(grow(R.fams, cap_fam * sizeof(DFam), s));
    TFIM_TRY(grow(R.items, cap_item * 4, s));
    TFIM_TRY(grow(R.heads, cap_head * 4, s));
    TFIM_TRY(grow(R.stack, cap_fam * 4, s));
    TFIM_TRY(grow(R.looks, cap_rows * sizeof(DLook), s));
    TFIM_TRY(grow(R.free_slots, cap_slots * 4, s));
    TFIM_TRY(grow(R.defer, cap_slots * 4, s));
    TFIM_TRY(grow(R.mfi_off, cap_mfi * 4, s));
    TFIM_TRY(grow(R.mfi_len, cap_mfi * 4, s));
    TFIM_TRY(grow(R.mfi_sup, cap_mfi * 4, s));
    TFIM_TRY(grow(R.mfi_items, cap_mfi_items * 4, s));
    if (o->log_lookahead) {
        TFIM_TRY(grow(R.log_feat, cap_log * 32 * 4, s));
        TFIM_TRY(grow(R.log_label, cap_log * 4, s));
    }
    TFIM_TRY(grow(R.djobs, cap_rows * sizeof(DJob), s));
    TFIM_TRY(grow(R.jobs, cap_rows * sizeof(JobDesc), s));
    TFIM_TRY(grow(R.rows, cap_rows * sizeof(RowDesc), s));
    TFIM_TRY(grow(R.row_job, cap_rows * 4, s));
    TFIM_TRY(grow(R.row_local, cap_rows * 4, s));
    TFIM_TRY(grow(R.proj_list, cap_rows * 4, s));
    TFIM_TRY(grow(R.mjobs, (2 * cap_rows + 2) * sizeof(MaskJob), s));   // at most two masks per expanded row
    TFIM_TRY(grow(R.tiles_l3, cap_tiles * sizeof(TileDesc), s));
    TFIM_TRY(grow(R.tiles_b1, cap_tiles * sizeof(TileDesc), s));
    TFIM_TRY(grow(R.tiles_tc, cap_tiles * sizeof(TileDesc), s));
    TFIM_TRY(grow(R.tiles_gr, cap_tiles * sizeof(TileDesc), s));
    TFIM_TRY(grow(R.counts, cap_out * 4, s));
    TFIM_TRY(grow(R.is_root, is_root.size(), s));
    TFIM_TRY(grow(R.dense_freq, (size_t)std::max<int32_t>(c->info.n_dense, 1) * 4, s));
    TFIM_TRY(grow(R.top_pos, (size_t)std::max<int32_t>(c->info.n_dense, 1) * 4, s));
    TFIM_TRY(grow(R.top_diag, (size_t)n0 * 4, s));
    // superset index (opts.superset): d items x sup_words words (about 32 MiB; MFIs past its
    // capacity are not indexed and prune nothing), cleared for every mine
    const bool sup_on = o->superset != 0;
    const int32_t sup_words = (int32_t)std::min<int64_t>(65536, std::max<int64_t>(32, (8LL << 20) / std::max(d, 1)));
    if (sup_on) {
        const size_t sup_bytes = (size_t)d * (size_t)sup_words * 4;
        TFIM_TRY(grow(R.sup_index, sup_bytes, s));
        TFIM_CUDA(cudaMemsetAsync(R.sup_index.p, 0, sup_bytes, s));
    }
    // mask slots (grown on demand)
    int64_t slot_cap = c->d_masks.bytes / ((size_t)W * 4);

    // the search's initial state, staged in pinned memory and copied asynchronously:
    // root flags, F1 counts, the top family record, its F list and its single job, rows,
    // F positions and row supports, the status record
    DFam top;
    top.slot = -1; top.item = -1; top.head_off = 0; top.head_len = 0; top.F_off = 0; top.nF = n0; top.nT = n0;
    top.sup = 0; top.next_row = n0; top.rows_done = 0; top.state = 0; top.top = 1;
    ResStatus hs;
    memset(&hs, 0, sizeof hs);
    for (int k = 0; k < kPhases; k++) hs.ph_s[k] = ~0ull;
    hs.fam_n = 1;
    hs.item_n = n0;
    hs.jobs = 1;
    hs.rows = n0;
    hs.out_total = top_out;
    hs.max_cols = n0;
    hs.nodes = n0;
    hs.supports = (unsigned long long)top_out;
    {
        // the staging blob is the same for every mine of this database: built once, and the
        // parts (whose device pools may have moved) copied again on every mine
        const size_t nd = (size_t)std::max<int32_t>(c->info.n_dense, 1);
        struct Part { void* dst; size_t off, bytes; };
        std::vector<Part> parts;
        size_t total = 0;
        auto part = [&](void* dst, size_t bytes) {
            parts.push_back(Part{dst, total, bytes});
            total += (bytes + 15) & ~size_t(15);
            return parts.size() - 1;
        };
        const size_t p_root = part(R.is_root.p, is_root.size()), p_freq = part(R.dense_freq.p, c->dense_freq.size() * 4),
                     p_fam = part(R.fams.p, sizeof(DFam)), p_F = part(R.items.p, (size_t)n0 * 4),
                     p_dj = part(R.djobs.p, sizeof(DJob)), p_jd = part(R.jobs.p, sizeof(JobDesc)),
                     p_rows = part(R.rows.p, (size_t)n0 * sizeof(RowDesc)), p_rj = part(R.row_job.p, (size_t)n0 * 4),
                     p_rl = part(R.row_local.p, (size_t)n0 * 4), p_pos = part(R.top_pos.p, nd * 4),
                     p_diag = part(R.top_diag.p, (size_t)n0 * 4), p_st = part(R.status.p, sizeof(ResStatus));
        unsigned char* h = nullptr;
        if (fresh_setup || !R.h_setup.p || R.setup_total != total) {
            TFIM_TRY(R.h_setup.reserve(total));
            h = R.h_setup.as<unsigned char>();
            auto at = [&](size_t k) { return (void*)(h + parts[k].off); };
            memcpy(at(p_root), is_root.data(), is_root.size());
            memcpy(at(p_freq), c->dense_freq.data(), c->dense_freq.size() * 4);
            memcpy(at(p_fam), &top, sizeof top);
            memcpy(at(p_F), F0.data(), (size_t)n0 * 4);
            *(DJob*)at(p_dj) = DJob{0, kJobFam, 0, n0, -1, -1, 0, 0, 0, 1, 0, 0, 0, 0};
            *(JobDesc*)at(p_jd) = JobDesc{-1, -1, n0, n0, 0, 0, 0, -1, 0};
            RowDesc* rows = (RowDesc*)at(p_rows);
            int32_t* rj = (int32_t*)at(p_rj);
            int32_t* rl = (int32_t*)at(p_rl);
            int32_t* pos = (int32_t*)at(p_pos);
            int32_t* diag = (int32_t*)at(p_diag);
            std::fill(pos, pos + nd, -1);
            for (int32_t k = 0; k < n0; k++) {
                rows[k] = RowDesc{-1, F0[k]};
                rj[k] = 0;
                rl[k] = k;
                pos[F0[k]] = k;
                diag[k] = c->bit_support[F0[k]];
            }
            memcpy(at(p_st), &hs, sizeof hs);
            R.setup_uid = c->uid;
            R.setup_total = total;
        }
        h = R.h_setup.as<unsigned char>();
        for (const Part& q : parts)
            if (q.bytes) TFIM_CUDA(cudaMemcpyAsync(q.dst, h + q.off, q.bytes, cudaMemcpyHostToDevice, s));
    }
    TFIM_TRY(R.h_status.reserve(sizeof(ResStatus)));
    ResStatus* hst = R.h_status.as<ResStatus>();

    // top family counting: pair co-occurrence or the symmetric bitmap Gram (cost model)
    int top_mode;
    {
        const double nF = n0;
        const bool b1 = o->counter != TFIM_COUNTER_LOP3 &&
                        (o->counter == TFIM_COUNTER_TENSOR || (nF >= tn.b1_min_rows && nF >= tn.b1_min_cols));
        const bool i8 = b1 && o->counter != TFIM_COUNTER_TENSOR && nF >= tn.i8_min_rows && nF >= tn.i8_min_cols;
        const double rate = i8 ? tn.rate_i8_bitops : b1 ? tn.rate_b1_bitops : tn.rate_lop3_bitops;
        const double bitmap_s = nF * nF * (double)c->n_bits / 2.0 / rate;
        const double pairs_s = c->red_pair_work / 2.0 / tn.rate_pair_incr + nF * nF * 4.0 / kTuneHbmBytes;
        if (o->top_counter == 1) top_mode = 1;
        else if (o->top_counter == 2) top_mode = c->csr_exact ? 2 : 1;
        else top_mode = (c->csr_exact && pairs_s < bitmap_s) ? 2 : 1;
    }
    const bool top_b1 = o->counter == TFIM_COUNTER_TENSOR ||
                        (o->counter != TFIM_COUNTER_LOP3 && n0 >= tn.b1_min_rows && n0 >= tn.b1_min_cols);
    // large families of the empty prefix: the tcgen05 kind::i8 counter, 128 x 128 tiles
    const bool top_i8 = top_b1 && o->counter != TFIM_COUNTER_TENSOR && n0 >= tn.i8_min_rows && n0 >= tn.i8_min_cols;

    double sync_ms = 0, kernel_ms = 0;
    int64_t launches = 0, count_launches = 0, bytes_alg = 0, waves = 0;
    int64_t path_launches[6] = {0, 0, 0, 0, 0, 0};
    bool used_tc = false;   // the tcgen05 family counter ran (its error flag is read at the end)
    const int64_t row_bytes = (c->n_bits + 7) / 8;
    ResStatus* d_st = (ResStatus*)R.status.p;

    ResPtrs P;
    auto refresh_ptrs = [&]() {
        P.fams = (DFam*)R.fams.p; P.items = (int32_t*)R.items.p; P.heads = (int32_t*)R.heads.p;
        P.stack = (int32_t*)R.stack.p; P.looks = (DLook*)R.looks.p; P.free_slots = (int32_t*)R.free_slots.p;
        P.defer = (int32_t*)R.defer.p; P.mfi_off = (int32_t*)R.mfi_off.p; P.mfi_len = (int32_t*)R.mfi_len.p;
        P.mfi_sup = (int32_t*)R.mfi_sup.p; P.mfi_items = (int32_t*)R.mfi_items.p;
        P.log_feat = (float*)R.log_feat.p; P.log_label = (float*)R.log_label.p;
        P.djobs = (DJob*)R.djobs.p; P.jobs = (JobDesc*)R.jobs.p; P.rows = (RowDesc*)R.rows.p;
        P.mjobs = (MaskJob*)R.mjobs.p;
        P.row_job = (int32_t*)R.row_job.p; P.row_local = (int32_t*)R.row_local.p;
        P.tiles_l3 = (TileDesc*)R.tiles_l3.p; P.tiles_b1 = (TileDesc*)R.tiles_b1.p; P.tiles_tc = (TileDesc*)R.tiles_tc.p;
        P.tiles_gr = (TileDesc*)R.tiles_gr.p;
        P.counts = (int32_t*)R.counts.p;
        P.bitmap = c->d_bitmap; P.masks = c->d_masks.as<uint32_t>(); P.dense_freq = (const int32_t*)R.dense_freq.p;
        P.is_root = (const uint8_t*)R.is_root.p; P.st = (ResStatus*)R.status.p;
        P.W = W; P.n_bits = c->n_bits; P.min_count = minc; P.wave_rows = wave_rows;
        P.cap_out = cap_out; P.cap_tiles = cap_tiles; P.counter = o->counter; P.la_mode = la_mode;
        P.log_on = o->log_lookahead; P.proposal_threshold = c->proposal_threshold; P.kslice_min = 64; P.sm_count = sm_count;
        P.mlp_w = nullptr; P.mlp_p = nullptr;
        P.proj_list = (int32_t*)R.proj_list.p;
        P.avg_len = c->n_bits > 0 ? (float)((double)c->n_red_items / (double)c->n_bits) : 0.f;
        P.csr_ok = c->csr_exact ? 1 : 0;
        P.proj_auto = o->proj_auto >= 0 ? o->proj_auto : tn.proj_auto;
        P.b1_min_rows = tn.b1_min_rows;
        P.b1_min_cols = tn.b1_min_cols;
        P.l3_slices_per_sm = tn.l3_slices_per_sm;
        P.l3_dense_slices_per_sm = tn.l3_dense_slices_per_sm;
        P.b1_tiles_per_sm = tn.b1_tiles_per_sm;
        P.tc_min_work = tn.tc_min_work;
        P.tc_min_density = tn.tc_min_density;
        P.tc_tiles_per_sm = tn.tc_tiles_per_sm;
        P.gram_min_rows = tn.gram_min_rows;
        if (la_mode == 2 && c->proposal) {
            const void* wb = nullptr;
            const float* pp = nullptr;
            mlp_device_params(c->proposal, &wb, &pp);
            P.mlp_w = (const __nv_bfloat16*)wb;
            P.mlp_p = pp;
        }
        Caps& k = P.caps;
        k.fam = (int64_t)std::min(R.fams.bytes / sizeof(DFam), R.stack.bytes / 4);
        k.item = (int64_t)(R.items.bytes / 4);
        k.head = (int64_t)(R.heads.bytes / 4);
        k.mfi = (int64_t)std::min({R.mfi_off.bytes, R.mfi_len.bytes, R.mfi_sup.bytes}) / 4;
        k.mfi_items = (int64_t)(R.mfi_items.bytes / 4);
        k.looks = (int64_t)(R.looks.bytes / sizeof(DLook));
        k.slots = std::min<int64_t>(slot_cap, (int64_t)std::min(R.free_slots.bytes, R.defer.bytes) / 4);
        k.log = o->log_lookahead ? (int64_t)std::min(R.log_feat.bytes / 128, R.log_label.bytes / 4) : 0;
        k.rows = cap_rows;
        P.row_bytes = row_bytes;
        P.row_sum = nullptr;
        P.wave_limit = 0x7fffffff;
        P.launch_id = 0;
        P.max_launch_ns = 2000000000ull;
        P.sup_index = sup_on ? (uint32_t*)R.sup_index.p : nullptr;
        P.sup_words = sup_words;
        P.sup_items = d;
    };
    // capacity for the worst case of one expand over `rows` rows of at most `max_cols`
    // columns each and `out_total` counts
    auto ensure = [&](const ResStatus& h, int64_t rows, int64_t jobs, int64_t out_total, int64_t max_head,
                      int64_t max_cols) -> int {
        const int64_t list = max_head + 2 + max_cols;
        const int64_t need_fam = h.fam_n + rows + 1;
        const int64_t need_item = h.item_n + 2 * out_total + rows + 1;
        const int64_t need_head = h.head_n + rows * list + 1;
        const int64_t need_mfi = h.mfi_n + rows + jobs + 1;
        const int64_t need_mfi_items = h.mfi_item_n + (rows + jobs) * list + 1;
        const int64_t need_slots = h.slot_n + 2 * rows + 2;
        const int64_t need_log = h.log_n + rows + 1;
        TFIM_TRY(grow(R.fams, need_fam * sizeof(DFam), s));
        TFIM_TRY(grow(R.stack, need_fam * 4, s));
        TFIM_TRY(grow(R.items, need_item * 4, s));
        TFIM_TRY(grow(R.heads, need_head * 4, s));
        TFIM_TRY(grow(R.mfi_off, need_mfi * 4, s));
        TFIM_TRY(grow(R.mfi_len, need_mfi * 4, s));
        TFIM_TRY(grow(R.mfi_sup, need_mfi * 4, s));
        TFIM_TRY(grow(R.mfi_items, need_mfi_items * 4, s));
        TFIM_TRY(grow(R.looks, (rows + 1) * sizeof(DLook), s));
        TFIM_TRY(grow(R.free_slots, need_slots * 4, s));
        TFIM_TRY(grow(R.defer, need_slots * 4, s));
        if (o->log_lookahead) {
            TFIM_TRY(grow(R.log_feat, need_log * 32 * 4, s));
            TFIM_TRY(grow(R.log_label, need_log * 4, s));
        }
        if (need_slots > slot_cap) {
            DevBuf nb;
            nb.stream = s;
            const int64_t ncap = std::max<int64_t>(need_slots + need_slots / 2, 64);
            TFIM_TRY(nb.reserve((size_t)ncap * (size_t)W * 4));
            if (c->d_masks.p && slot_cap > 0)
                TFIM_CUDA(cudaMemcpyAsync(nb.p, c->d_masks.p, (size_t)slot_cap * (size_t)W * 4, cudaMemcpyDeviceToDevice, s));
            c->d_masks.release();
            c->d_masks = nb;
            slot_cap = ncap;
        }
        refresh_ptrs();
        return TFIM_OK;
    };
    // the pack declined a wave: grow what it asked for
    auto grow_for = [&](const ResStatus& h) -> int {
        if (h.starved) {
            // a single row does not fit the count buffer
            cap_out *= 4;
            TFIM_TRY(grow(R.counts, cap_out * 4, s));
        }
        if (h.grow) {
            if (h.g_out > cap_out) {
                cap_out = std::max<int64_t>(2 * cap_out, h.g_out);
                TFIM_TRY(grow(R.counts, cap_out * 4, s));
            }
            if (h.g_tiles > cap_tiles) {
                cap_tiles = std::max<int64_t>(2 * cap_tiles, h.g_tiles);
                TFIM_TRY(grow(R.tiles_l3, cap_tiles * sizeof(TileDesc), s));
                TFIM_TRY(grow(R.tiles_b1, cap_tiles * sizeof(TileDesc), s));
                TFIM_TRY(grow(R.tiles_tc, cap_tiles * sizeof(TileDesc), s));
    TFIM_TRY(grow(R.tiles_gr, cap_tiles * sizeof(TileDesc), s));
            }
            TFIM_TRY(ensure(h, h.g_rows, h.g_jobs, h.g_out, h.g_max_head, h.g_max_cols));
        }
        refresh_ptrs();   // the next pack clears the request
        return TFIM_OK;
    };

    // wave 1: the top family, counted whole
    *hst = hs;
    TFIM_TRY(ensure(hs, hs.rows, hs.jobs, hs.out_total, 0, hs.max_cols));
    {
        std::vector<TileDesc> tl;
        if (top_mode == 1) {
            if (top_i8) {
                const int64_t g = (n0 + 127) / 128;
                const int64_t base = g * (g + 1) / 2;   // upper-triangle tiles
                int64_t ks = std::min<int64_t>(std::max<int64_t>(1, (2LL * sm_count + base - 1) / base), W / 64);
                const int64_t kslice = ((W / 64 + ks - 1) / ks) * 64;
                for (int64_t w0 = 0; w0 < W; w0 += kslice)
                    for (int32_t r0 = 0; r0 < n0; r0 += 128)
                        for (int32_t c0 = r0; c0 < n0; c0 += 128)
                            tl.push_back(TileDesc{0, r0, std::min(128, n0 - r0), c0, std::min(n0, c0 + 128), (int32_t)w0,
                                                  (int32_t)std::min<int64_t>(W, w0 + kslice), 0});
            } else if (top_b1) {
                const int64_t base = (int64_t)((n0 + kB1Rows - 1) / kB1Rows) * ((n0 + kB1Cols - 1) / kB1Cols);
                const int64_t want = (int64_t)(tn.b1_tiles_per_sm * sm_count);
                int64_t ks = std::min<int64_t>(std::max<int64_t>(1, (want + base - 1) / base), W / 64);
                const int64_t kslice = ((W / 64 + ks - 1) / ks) * 64;
                tiles_b1(0, n0, n0, W, kslice, tl, true);
            } else {
                const int64_t base = (int64_t)((n0 + kLop3Rows - 1) / kLop3Rows) * ((n0 + 63) / 64);
                const int64_t want = (int64_t)(tn.l3_slices_per_sm * sm_count);
                int64_t ws = std::min<int64_t>(std::max<int64_t>(1, (want + base - 1) / base), std::max<int64_t>(1, W / 256));
                const int64_t wslice = ((W / 64 + ws - 1) / ws) * 64;
                tiles_lop3(0, n0, n0, W, wslice, tl, true);
            }
        }
        if ((int64_t)tl.size() > cap_tiles) {
            cap_tiles = (int64_t)tl.size();
            TFIM_TRY(grow(R.tiles_l3, cap_tiles * sizeof(TileDesc), s));
            TFIM_TRY(grow(R.tiles_b1, cap_tiles * sizeof(TileDesc), s));
            TFIM_TRY(grow(R.tiles_tc, cap_tiles * sizeof(TileDesc), s));
    TFIM_TRY(grow(R.tiles_gr, cap_tiles * sizeof(TileDesc), s));
            refresh_ptrs();
        }
        if (!tl.empty())
            TFIM_CUDA(cudaMemcpyAsync(top_b1 ? R.tiles_b1.p : R.tiles_l3.p, tl.data(), tl.size() * sizeof(TileDesc),
                                      cudaMemcpyHostToDevice, s));
        TFIM_CUDA(cudaMemsetAsync(R.counts.p, 0, (size_t)top_out * 4, s));
        CountArgs a;
        a.bitmap = c->d_bitmap; a.W = W; a.masks = c->d_masks.as<uint32_t>(); a.jobs = P.jobs; a.rows = P.rows;
        a.cols = P.items; a.out = P.counts;
        stt->setup_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_entry).count();
        TFIM_CUDA(cudaEventRecord(c->ev0, s));
        if (top_mode == 2) {
            TFIM_TRY(launch_pair_count(c->d_red_off, c->d_red_items, c->n_bits, (const int32_t*)R.top_pos.p, n0, P.counts, s));
            bytes_alg += (c->n_bits + 1) * 8 + c->n_red_items * 4 + 4 * top_out;
        } else {
            a.tiles = top_b1 ? P.tiles_b1 : P.tiles_l3;
            a.n_tiles = (int32_t)tl.size();
            TFIM_TRY(top_i8 ? launch_count_i8(a, s) : top_b1 ? launch_count_b1(a, s) : launch_count_lop3(a, s));
            bytes_alg += row_bytes * 2 * n0 + 4 * top_out;
        }
        TFIM_CUDA(cudaEventRecord(c->ev1, s));
        TFIM_TRY(launch_mirror(P.counts, n0, top_mode == 2 ? (const int32_t*)R.top_diag.p : nullptr, s));
        TFIM_TRY(grow(R.top_sum, (size_t)n0 * sizeof(RowSum), s));
        k_top_summary<<<n0, 256, 0, s>>>(P.counts, n0, minc, (RowSum*)R.top_sum.p);
        TFIM_CUDA(cudaGetLastError());
        launches += 3;
        count_launches++;
        const int64_t threads = (int64_t)n0 * 32;
        ResPtrs Ptop = P;
        Ptop.row_sum = (const RowSum*)R.top_sum.p;
        k_res_expand<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(Ptop);
        TFIM_CUDA(cudaGetLastError());
        k_build_masks<<<sm_count * 8, 256, 0, s>>>(P);
        TFIM_CUDA(cudaGetLastError());
        if (sup_on) {
            k_index_mfis<<<sm_count, 256, 0, s>>>(P);
            k_prune_stack<<<sm_count, 256, 0, s>>>(P);
            TFIM_CUDA(cudaGetLastError());
            launches += 2;
        }
        launches++;
        launches++;
        waves++;
    }
    // the counting path of the empty-prefix family, its work and (read at the end) its time
    const int top_path = top_mode == 2 ? TFIM_PATH_PAIRS : top_i8 ? TFIM_PATH_TC : top_b1 ? TFIM_PATH_B1 : TFIM_PATH_LOP3;
    path_launches[top_path]++;
    // following waves
    const bool use_graph = o->use_graphs != 0;
    int64_t host_waves = 0;
    if (use_graph) {
        TFIM_TRY(grow(R.args, sizeof(ResArgs), s));
        TFIM_TRY(R.h_args.reserve(sizeof(ResArgs)));
        const bool with_proj = c->csr_exact && (o->counter == TFIM_COUNTER_PROJ || (o->counter == TFIM_COUNTER_AUTO && P.proj_auto));
        ResArgs* d_args = (ResArgs*)R.args.p;
        if (!R.graph.exec || R.graph.args != R.args.p || R.graph.status != R.status.p || R.graph.with_proj != (int)with_proj)
            TFIM_TRY(build_wave_graph(R.graph, d_args, (ResStatus*)R.status.p, with_proj, c->d_red_off, c->d_red_items, s));
        int64_t slices = 0;
        while (true) {
            ResArgs* ha = R.h_args.as<ResArgs>();
            ha->p = P;
            ha->p.launch_id = ++R.launch_id;
            ha->p.wave_limit = 0x7fffffff;
            CountArgs a;
            a.bitmap = c->d_bitmap; a.W = W; a.masks = P.masks; a.jobs = P.jobs; a.rows = P.rows;
            a.cols = P.items; a.out = P.counts; a.n_tiles = 0; a.job_list = P.proj_list;
            a.tiles = P.tiles_l3;
            a.ph_s = &d_st->ph_s[kPhLop3]; a.ph_e = &d_st->ph_e[kPhLop3];
            ha->a3 = a;
            a.tiles = P.tiles_b1;
            a.ph_s = &d_st->ph_s[kPhB1]; a.ph_e = &d_st->ph_e[kPhB1];
            ha->a1 = a;
            a.tiles = P.tiles_l3;
            a.ph_s = &d_st->ph_s[kPhProj]; a.ph_e = &d_st->ph_e[kPhProj];
            ha->ap = a;
            a.tiles = P.tiles_tc;
            a.ph_s = &d_st->ph_s[kPhTc]; a.ph_e = &d_st->ph_e[kPhTc];
            ha->atc = a;
            a.tiles = P.tiles_gr;
            a.ph_s = &d_st->ph_s[kPhGram]; a.ph_e = &d_st->ph_e[kPhGram];
            ha->agr = a;
            TFIM_CUDA(cudaMemcpyAsync(d_args, ha, sizeof(ResArgs), cudaMemcpyHostToDevice, s));
            TFIM_CUDA(cudaGraphLaunch(R.graph.exec, s));
            launches++;
            slices++;
            TFIM_CUDA(cudaMemcpyAsync(hst, R.status.p, sizeof(ResStatus), cudaMemcpyDeviceToHost, s));
            const double ts = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
            TFIM_CUDA(cudaStreamSynchronize(s));
            sync_ms += (std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count() - ts) * 1e3;
            TFIM_CHECK(hst->error == 0, TFIM_E_STATE, "resident search invariant failed (code %d)", hst->error);
            if (hst->starved || hst->grow) {
                TFIM_TRY(grow_for(*hst));
                continue;
            }
            if (hst->jobs == 0) break;   // the stack and the lookahead queue are empty
            TFIM_CHECK(slices < (1LL << 40), TFIM_E_STATE, "resident search did not finish");
        }
        // per wave: pack, zero, lop3, b1, [proj], tc, gram, expand, masks, index, prune, control
        launches += (int64_t)hst->waves * (11 + (with_proj ? 1 : 0));
        count_launches += (int64_t)hst->waves * (4 + (with_proj ? 1 : 0));
        path_launches[TFIM_PATH_GRAM] += hst->waves;
        path_launches[TFIM_PATH_LOP3] += hst->waves;
        path_launches[TFIM_PATH_B1] += hst->waves;
        path_launches[TFIM_PATH_TC] += hst->waves;
        used_tc = true;
        if (with_proj) path_launches[TFIM_PATH_PROJ] += hst->waves;
    }
    while (!use_graph) {
        k_res_pack<<<1, kPackThreads, 0, s>>>(P);
        TFIM_CUDA(cudaGetLastError());
        launches++;
        TFIM_CUDA(cudaMemcpyAsync(hst, R.status.p, sizeof(ResStatus), cudaMemcpyDeviceToHost, s));
        const double ts = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
        TFIM_CUDA(cudaStreamSynchronize(s));
        sync_ms += (std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count() - ts) * 1e3;
        TFIM_CHECK(hst->error == 0, TFIM_E_STATE, "resident search invariant failed (code %d)", hst->error);
        if (hst->starved || hst->grow) {
            TFIM_TRY(grow_for(*hst));
            continue;
        }
        if (hst->jobs == 0) break;
        TFIM_CUDA(cudaMemsetAsync(R.counts.p, 0, (size_t)hst->out_total * 4, s));
        CountArgs a;
        a.bitmap = c->d_bitmap; a.W = W; a.masks = c->d_masks.as<uint32_t>(); a.jobs = P.jobs; a.rows = P.rows;
        a.cols = P.items; a.out = P.counts; a.job_list = P.proj_list;
        if (hst->tiles_l3) {
            // dense families' tiles (the first tiles_l3d), then the zero-skipping ones
            a.ph_s = &d_st->ph_s[kPhLop3]; a.ph_e = &d_st->ph_e[kPhLop3];
            if (hst->tiles_l3d) {
                a.tiles = P.tiles_l3;
                a.n_tiles = hst->tiles_l3d;
                TFIM_TRY(launch_count_lop3_dense(a, s));
                launches++;
                count_launches++;
            }
            if (hst->tiles_l3 > hst->tiles_l3d) {
                a.tiles = P.tiles_l3 + hst->tiles_l3d;
                a.n_tiles = hst->tiles_l3 - hst->tiles_l3d;
                TFIM_TRY(launch_count_lop3(a, s));
                launches++;
                count_launches++;
            }
            path_launches[TFIM_PATH_LOP3]++;
        }
        if (hst->tiles_b1) {
            a.tiles = P.tiles_b1;
            a.n_tiles = hst->tiles_b1;
            a.ph_s = &d_st->ph_s[kPhB1]; a.ph_e = &d_st->ph_e[kPhB1];
            TFIM_TRY(launch_count_b1(a, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_B1]++;
        }
        if (hst->tiles_tc) {
            a.tiles = P.tiles_tc;
            a.n_tiles = hst->tiles_tc;
            a.ph_s = &d_st->ph_s[kPhTc]; a.ph_e = &d_st->ph_e[kPhTc];
            TFIM_TRY(launch_count_fam(a, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_TC]++;
            used_tc = true;
        }
        if (hst->tiles_gr) {
            a.tiles = P.tiles_gr;
            a.n_tiles = hst->tiles_gr;
            a.ph_s = &d_st->ph_s[kPhGram]; a.ph_e = &d_st->ph_e[kPhGram];
            TFIM_TRY(launch_count_gram(a, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_GRAM]++;
        }
        if (hst->n_proj) {
            a.ph_s = &d_st->ph_s[kPhProj]; a.ph_e = &d_st->ph_e[kPhProj];
            TFIM_TRY(launch_count_proj(a, P.proj_list, hst->n_proj, c->d_red_off, c->d_red_items, s));
            launches++;
            count_launches++;
            path_launches[TFIM_PATH_PROJ]++;
        }
        const int64_t threads = (int64_t)hst->rows * 32;
        k_res_expand<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(P);
        TFIM_CUDA(cudaGetLastError());
        k_build_masks<<<sm_count * 8, 256, 0, s>>>(P);
        TFIM_CUDA(cudaGetLastError());
        if (sup_on) {
            k_index_mfis<<<sm_count, 256, 0, s>>>(P);
            k_prune_stack<<<sm_count, 256, 0, s>>>(P);
            TFIM_CUDA(cudaGetLastError());
            launches += 2;
        }
        launches++;
        launches++;
        host_waves++;
    }
    waves += use_graph ? (int64_t)hst->waves : host_waves;
    // results
    const auto t_read0 = std::chrono::steady_clock::now();
    const ResStatus fin = *hst;
    // the MFIs in output order (sorted on the device) through one pinned staging buffer:
    // sort keys, lengths, supports, items
    const int32_t nm = fin.mfi_n;
    const int64_t ni = fin.mfi_item_n;
    TFIM_TRY(R.h_res.reserve(((size_t)nm * 4 + (size_t)ni + 2) * 4));
    uint64_t* hkey = R.h_res.as<uint64_t>();
    int32_t* hlen = (int32_t*)(hkey + nm);
    int32_t* hsup = hlen + nm;
    int32_t* hitems = hsup + nm;
    if (nm) {
        refresh_ptrs();
        TFIM_TRY(order_mfis(R, c, P, nm, ni, sm_count, s, hkey, hlen, hitems));
    }
    if (o->log_lookahead && fin.log_n) {
        c->la_feats.resize((size_t)fin.log_n * 32);
        c->la_labels.resize(fin.log_n);
        TFIM_CUDA(cudaMemcpyAsync(c->la_feats.data(), R.log_feat.p, (size_t)fin.log_n * 32 * 4, cudaMemcpyDeviceToHost, s));
        TFIM_CUDA(cudaMemcpyAsync(c->la_labels.data(), R.log_label.p, (size_t)fin.log_n * 4, cudaMemcpyDeviceToHost, s));
    }
    TFIM_CUDA(cudaStreamSynchronize(s));
    if (top_i8 && top_mode == 1) TFIM_TRY(count_i8_status(true));
    if (used_tc) TFIM_TRY(count_fam_status(true));
    {
        MfiSet& M = c->mfis;
        const bool fresh = M.size() == 0;
        const size_t kbase = M.size();
        M.items.insert(M.items.end(), hitems, hitems + ni);
        M.sup.insert(M.sup.end(), hsup, hsup + nm);
        M.off.resize(kbase + 1 + (size_t)nm);
        for (int32_t k = 0; k < nm; k++) M.off[kbase + k + 1] = M.off[kbase + k] + hlen[k];
        if (fresh) {
            finish_mfi_order(M, hkey);
            M.ordered = true;
        } else {
            // appended to earlier results: long lists sorted here, the whole set by the caller
            for (size_t k = kbase; k < M.size(); k++)
                if (M.off[k + 1] - M.off[k] > 64)
                    std::sort(M.items.begin() + M.off[k], M.items.begin() + M.off[k + 1], std::greater<int32_t>());
            M.ordered = false;
        }
    }
    stt->nodes += (int64_t)fin.nodes;
    stt->supports += (int64_t)fin.supports;
    stt->lookaheads += (int64_t)fin.lookaheads;
    stt->lookahead_hits += (int64_t)fin.hits;
    stt->lookaheads_skipped += (int64_t)fin.skipped;
    stt->pruned_pep += (int64_t)fin.pep;
    stt->pruned_superset += (int64_t)fin.sup_pruned;
    // device times: the empty-prefix family's counting (events) and every later wave's phases
    // (stamps folded by the pack)
    {
        float top_ms = 0;
        cudaEventElapsedTime(&top_ms, c->ev0, c->ev1);
        stt->top_ms += top_ms;
        kernel_ms += top_ms;
        stt->path_ms[top_path] += top_ms;
        stt->path_bytes[top_path] += bytes_alg;
        stt->path_bitops[top_path] += top_mode == 2 ? 0 : (int64_t)n0 * (n0 + 1) / 2 * c->n_bits;
        stt->path_supports[top_path] += top_out;
        const double ns = 1e-6;
        const int ph_of_path[6] = {kPhLop3, kPhB1, kPhTc, -1, kPhProj, kPhGram};
        const int cls_of_path[6] = {kClsLop3, kClsB1, kClsTc, -1, kClsProj, kClsGram};
        for (int q = 0; q < 6; q++) {
            if (ph_of_path[q] >= 0) {
                const double ms = (double)fin.ph_ns[ph_of_path[q]] * ns;
                stt->path_ms[q] += ms;
                kernel_ms += ms;
            }
            if (cls_of_path[q] >= 0) {
                stt->path_bytes[q] += (int64_t)fin.cls_bytes[cls_of_path[q]];
                stt->path_bitops[q] += (int64_t)fin.cls_bitops[cls_of_path[q]];
                stt->path_supports[q] += (int64_t)fin.cls_sup[cls_of_path[q]];
                bytes_alg += (int64_t)fin.cls_bytes[cls_of_path[q]];
            }
            stt->path_launches[q] += path_launches[q];
        }
        stt->pack_ms += (double)fin.ph_ns[kPhPack] * ns;
        stt->zero_ms += (double)fin.ph_ns[kPhZero] * ns;
        stt->expand_ms += (double)fin.ph_ns[kPhExpand] * ns;
        stt->mask_ms += (double)fin.ph_ns[kPhMasks] * ns;
    }
    stt->waves += waves;
    stt->launches += launches;
    stt->count_launches += count_launches;
    stt->kernel_ms += kernel_ms;
    stt->sync_ms += sync_ms;
    stt->bytes_alg += bytes_alg;
    stt->bit_ops = stt->supports * c->n_bits;
    stt->readback_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_read0).count();
    return TFIM_OK;
}

}  // namespace tfim
