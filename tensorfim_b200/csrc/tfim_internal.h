// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "tfim.h"

namespace tfim {

// ------------------------------------------------------------------ errors
void set_error(const char* fmt, ...);
const char* get_error();

#define TFIM_CUDA(call)                                                                    \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) {                                                          \
            ::tfim::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e__)); \
            return TFIM_E_CUDA;                                                            \
        }                                                                                  \
    } while (0)

#define TFIM_CHECK(cond, code, ...)                                                        \
    do {                                                                                   \
        if (!(cond)) {                                                                     \
            ::tfim::set_error(__VA_ARGS__);                                                \
            return (code);                                                                 \
        }                                                                                  \
    } while (0)

#define TFIM_TRY(call)                                                                     \
    do {                                                                                   \
        int s__ = (call);                                                                  \
        if (s__ != TFIM_OK) return s__;                                                    \
    } while (0)

// ------------------------------------------------------------------ layout
// Bitmap rows are padded to a multiple of 64 uint32 words (2048 bits, 256 bytes), so
// every row starts 256-byte aligned and any 2048-bit K-chunk is whole.
constexpr int kRowAlignWords = 64;
inline int64_t words_for_bits(int64_t bits) {
    int64_t w = (bits + 31) / 32;
    return (w + kRowAlignWords - 1) / kRowAlignWords * kRowAlignWords;
}

constexpr int kMaxListLen = 64;   // longest item list one counted row may AND

// Device memory comes from one stream-ordered pool per device that keeps freed blocks
// cached (up to a release threshold), so opening and closing contexts or growing
// buffers does not go back to the driver; pinned host staging comes from a process-wide
// cache of blocks.
int dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);
void* pinned_alloc(size_t bytes, size_t* got);
void pinned_free(void* p, size_t bytes);

// A device buffer that grows on demand (stream-ordered on `stream`), freed with its owner.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    int reserve(size_t need);
    void release();
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};
struct HostBuf {   // pinned host staging
    void* p = nullptr;
    size_t bytes = 0;
    int reserve(size_t need);
    void release();
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

// ------------------------------------------------------------------ count jobs
// A count job: a base mask along the transaction axis (a mask-pool row AND an item row,
// either optional), a set of counted rows and a set of columns (item rows):
//   out[out_off + r*n_cols + c] = popc(base & A_r & B[col c])
//   A_r = (row.slot >= 0 ? masks[row.slot] : ~0) & (row.item >= 0 ? B[row.item] : ~0)
// A column id of -1 stands for the all-ones column (so the count is popc(base & A_r)).
struct JobDesc {
    int32_t base_slot;    // mask-pool row, or -1
    int32_t base_item;    // bitmap row, or -1
    int32_t n_rows;
    int32_t n_cols;
    int32_t row_off;      // into the RowDesc table
    int32_t col_off;      // into the column table
    int64_t out_off;      // into the counts buffer
    int32_t self_col;     // column index that stands for all ones (not read from the table), or -1
    int32_t pad;
};
struct RowDesc {
    int32_t slot;
    int32_t item;
};
// One tile: rows [r0, r0+nr) x columns [c0, c1) of job `job` over words [w0, w1).
struct TileDesc {
    int32_t job;
    int32_t r0, nr;
    int32_t c0, c1;
    int32_t w0, w1;
    int32_t pad;
};
// Mask build: masks[dst] = (src >= 0 ? masks[src] : ~0) & AND of items[off .. off+n).
struct MatDesc {
    int32_t dst, src, off, n;
};
// One entry of a compacted count row: column index and its count.
struct Entry {
    int32_t col, count;
};

// Throughput figures of the counting paths on B200 (measured; used by the engine's cost
// model to choose how the family of the empty prefix is counted).
constexpr double kTuneB1BitOps = 1.9e14;       // b1 tensor-core tiles, bit-ops/s
constexpr double kTuneLop3BitOps = 1.0e14;     // AND+popc tiles, bit-ops/s
constexpr double kTunePairIncrements = 2.0e10; // pair co-occurrence increments/s
constexpr double kTuneHbmBytes = 6.5e12;       // bytes/s
constexpr int kTuneProjAuto = 0;               // projected counter in the automatic choice

constexpr int kLop3Rows = 8;        // rows per CUDA-core tile
constexpr int kLop3Chunk = 4096;    // word slice of a CUDA-core tile in tfim_count_wave
constexpr int kB1Rows = 64;         // rows per tensor-core tile
constexpr int kB1Cols = 64;         // columns per tensor-core tile

struct CountArgs {
    const uint32_t* bitmap;
    int64_t W;
    const uint32_t* masks;
    const JobDesc* jobs;
    const RowDesc* rows;
    const int32_t* cols;
    const TileDesc* tiles;
    int32_t n_tiles;
    int32_t* out;
    const int32_t* job_list;   // projected counter: the jobs it counts
    // phase stamps of the launch (or nullptr): the earliest block start and the latest block
    // end, in %globaltimer nanoseconds (phase_begin / phase_end)
    unsigned long long* ph_s = nullptr;
    unsigned long long* ph_e = nullptr;
};

__device__ __forceinline__ unsigned long long dev_globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Device time of a launch without any barrier: thread 0 of every block folds its start time
// into *s (minimum) and its finish time into *e (maximum), so the phase runs from the first
// block's start to the last block's end.  One atomic per block; a null pointer records nothing.
__device__ __forceinline__ void phase_begin(unsigned long long* s) {
    if (s && threadIdx.x == 0) atomicMin(s, dev_globaltimer());
}
__device__ __forceinline__ void phase_end(unsigned long long* e) {
    if (e && threadIdx.x == 0) atomicMax(e, dev_globaltimer());
}

int launch_count_lop3(const CountArgs& a, cudaStream_t s);
// tiles flagged dense (TileDesc.pad bit 0): register-blocked, no zero-position skipping
int launch_count_lop3_dense(const CountArgs& a, cudaStream_t s);
int launch_count_b1(const CountArgs& a, cudaStream_t s);
// Persistent forms for waves built on the GPU: the arguments and the tile / job count are
// read from device memory and a fixed grid strides over the tiles, so the launches do not
// depend on the wave and can be captured once in a graph.
int launch_count_lop3_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                                 cudaStream_t s);
int launch_count_b1_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                               cudaStream_t s);
int launch_count_proj_persistent(const CountArgs* d_args, const int32_t* d_n_jobs, int32_t grid, const int64_t* red_off,
                                 const int32_t* red_items, cudaStream_t s);
// blocks of each persistent kernel resident per SM
int persistent_occupancy(int* lop3, int* b1, int* proj);
int configure_count_kernels();
// tcgen05 kind::i8 counter (count_tc.cu): 128 x 128 tiles; the status reads (and with
// `reset` clears) the device flag the kernel sets when an mbarrier wait expired.
int launch_count_i8(const CountArgs& a, cudaStream_t s);
int count_i8_status(bool reset);
// tcgen05 kind::i8 family counter (count_fam.cu): a tile is one family job (rows a run of its
// columns, at most kFamMaxCols columns) over a word slice, TileDesc.pad = the F position of
// the tile's first row; one CTA per SM.  The persistent form reads its arguments and tile
// count from device memory and takes tiles from `d_next` (zero at launch).
constexpr int kFamMaxCols = 128;
int launch_count_fam(const CountArgs& a, cudaStream_t s);
int launch_count_fam_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                                cudaStream_t s);
int count_fam_status(bool reset);
int configure_fam_kernel();   // opt into its shared memory (once per device, before any capture)
// CUDA-core Gram counter for dense family jobs (count_gram.cu): a tile is one family job of at
// most kGramMaxCols columns and at most 128 blocks of 4 x 4 (row, column) pairs, over a word
// slice; TileDesc.pad = the F position of the job's first row.
constexpr int kGramMaxCols = 64;
int launch_count_gram(const CountArgs& a, cudaStream_t s);
int launch_count_gram_persistent(const CountArgs* d_args, const int32_t* d_n_tiles, int32_t* d_next, int32_t grid,
                                 cudaStream_t s);
int occupancy_gram(int* blocks);
int configure_gram_kernel();
// The tuning table in force (common.cu): built-in values, or the table loaded / set.
tfim_tuning tuning();
int launch_pair_count(const int64_t* red_off, const int32_t* red_items, int64_t n_red, const int32_t* pos,
                      int32_t nF, int32_t* M, cudaStream_t s);
int launch_mirror(int32_t* M, int32_t nF, const int32_t* diag, cudaStream_t s);
// Projected counting of family jobs (count_proj.cu): one block per listed job.
int launch_count_proj(const CountArgs& a, const int32_t* job_ids, int32_t n_jobs, const int64_t* red_off,
                      const int32_t* red_items, cudaStream_t s);
constexpr int kProjMaxCols = 1024;  // longest column list the projected counter hashes
int launch_materialize(const uint32_t* bitmap, int64_t W, uint32_t* masks, const MatDesc* mats,
                       const int32_t* items, int32_t n, cudaStream_t s);
// nfreq[g] = #{c < n_cols : counts[g*n_cols + c] >= min_count} for g < n_rows
int launch_nfreq(const int32_t* counts, int64_t n_rows, int32_t n_cols, int32_t min_count,
                 int32_t* nfreq, cudaStream_t s);
// For each job row g (global row index over all jobs, row_job[g] = its job):
// entries >= min_count are appended to `entries` (one atomic reservation per row) and
// row_info[g] = (start, len).  counter[0] ends as the total entry count.
int launch_compact(const int32_t* counts, const JobDesc* jobs, const int32_t* row_job,
                   const int32_t* row_local, int64_t n_rows, int32_t min_count, Entry* entries,
                   int2* row_info, int32_t* counter, cudaStream_t s);

}  // namespace tfim

namespace tfim {
struct EngineState;
struct ResidentState;
// The MFIs of a mine, flat: MFI k holds items[off[k] .. off[k+1]) (dense ids, descending)
// and has support sup[k].
struct MfiSet {
    std::vector<int32_t> items;
    std::vector<int64_t> off{0};
    std::vector<int32_t> sup;
    bool ordered = false;   // already in output order (descending support, then item lists)
    size_t size() const { return sup.size(); }
    void clear() {
        items.clear();
        off.assign(1, 0);
        sup.clear();
        ordered = false;
    }
    void add(const int32_t* x, size_t n, int32_t s) {
        items.insert(items.end(), x, x + n);
        off.push_back((int64_t)items.size());
        sup.push_back(s);
    }
};
}  // namespace tfim

// ------------------------------------------------------------------ context
struct tfim_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t uid = 0;                      // unique per context opened in this process
    cudaEvent_t ev_span0 = nullptr, ev_span1 = nullptr;   // the span of a tfim_mine
    tfim_db_info info{};
    bool from_db = false;
    // host-side item tables (dense id space)
    std::vector<int32_t> dense_to_orig;
    std::vector<int32_t> dense_freq;       // occurrence counts (F1)
    std::vector<int32_t> items_in_freq_sort;
    std::vector<int32_t> roots;            // first dimension_reduced of items_in_freq_sort
    // device bitmap: n_dense rows x W words
    uint32_t* d_bitmap = nullptr;
    int64_t W = 0;
    int64_t n_bits = 0;
    int32_t n_counted = 0;
    std::vector<int32_t> bit_support;      // popc of each counted row (bitmap supports)
    // reduced transaction list (dense ids): row rr = red_items[red_off[rr] .. red_off[rr+1])
    int64_t* d_red_off = nullptr;
    int32_t* d_red_items = nullptr;
    int64_t n_red_items = 0;
    double red_pair_work = 0;              // sum over reduced rows of length^2
    bool csr_exact = false;                // the reduced list repeats no id within a row: the
                                           // list-based counters (pairs, projected) are exact
    // scratch
    tfim::DevBuf d_scratch[8];
    tfim::HostBuf h_scratch[4];
    tfim::DevBuf d_masks;                   // mask pool (rows of W words)
    int64_t mask_slots = 0;
    // results
    tfim::MfiSet mfis;                      // dense ids
    tfim::MfiSet all_fis;                   // all frequent itemsets of tfim_mine_all (dense ids)
    bool all_mined = false;
    bool mined = false;
    int32_t counter_pref = TFIM_COUNTER_AUTO;   // counter used by tfim_count_wave
    bool used_i8 = false;                       // the last counting wave ran the tcgen05 i8 counter
    tfim_mine_stats last_stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    tfim::EngineState* engine = nullptr;
    tfim::ResidentState* resident = nullptr;
    // learned lookahead proposal (not owned) and the outcome log of the last mine
    tfim_mlp* proposal = nullptr;
    float proposal_threshold = 0.5f;
    std::vector<float> la_feats;    // n x 32
    std::vector<float> la_labels;   // n
    // transaction sharding (tfim_open_*_sharded): the group, and the transaction count over
    // all shards (equal to n_bits for an unsharded context); decisions use the latter
    tfim_group group{0, 1, nullptr, nullptr};
    bool sharded = false;
    int64_t n_bits_total = 0;
    tfim::DevBuf d_group;                   // staging of host values reduced over the group
};

namespace tfim {
// Tile lists of one count job (mine.cu).  `upper`: rows and columns are the same list and
// only tiles holding some (i, j >= i) are emitted.
void tiles_lop3(int32_t job, int32_t nr, int32_t nc, int64_t W, int64_t wslice, std::vector<TileDesc>& out,
                bool upper = false);
void tiles_b1(int32_t job, int32_t nr, int32_t nc, int64_t W, int64_t kslice, std::vector<TileDesc>& out,
              bool upper = false);
struct EngineState;                        // persistent buffers of the search drivers (mine.cu)
void free_engine(EngineState* e);
int mine_plain(tfim_ctx* ctx, const tfim_mine_opts* o, tfim_mine_stats* st);
int mine_batched(tfim_ctx* ctx, const tfim_mine_opts* o, tfim_mine_stats* st);
int mine_resident(tfim_ctx* ctx, const tfim_mine_opts* o, tfim_mine_stats* st);
int mine_plain_roots(tfim_ctx* ctx, const std::vector<int32_t>& roots, tfim_mine_stats* st);
void free_resident(ResidentState* r, cudaStream_t s);
// Per-device cache of the resident pools and mask pool of closed contexts (resident.cu).
void stash_resident(tfim_ctx* c);
void adopt_resident(tfim_ctx* c);
int release_cached(int device);
int mlp_device_params(tfim_mlp* h, const void** wbf, const float** params);
int compute_bit_supports(tfim_ctx* ctx);
// ingest from a CSR already in device memory (row_offsets[0] == 0, ids >= 0 checked)
int ingest_device_csr(tfim_ctx* c, const int64_t* d_off, const int32_t* d_items, int64_t n_rows, int64_t nnz, double thr);
// A transaction file's bytes as a source: either a host buffer or an open file descriptor
// (read with pread), copied to the device in chunks through pinned staging.
struct TextSource {
    const char* host = nullptr;   // host bytes (pageable or pinned), or
    int fd = -1;                  // a readable file descriptor
    int64_t n_bytes = 0;
};
// Parse the file bytes on the device (reference readTransSetFile) into a device CSR:
// *d_off (n_rows + 1 int64) and *d_items (max(nnz, 1) int32), both from dev_alloc on `s`.
int parse_text_device(const TextSource& src, cudaStream_t s, int64_t** d_off, int32_t** d_items, int64_t* n_rows,
                      int64_t* nnz);
// Per-node prefix masks from item lists and one count job over every counted row (abi.cu):
// counts[i][e] = popc(AND of node i's items & B[e]), nfreq[i] = #{e : counts >= min_count}.
int count_wave_impl(tfim_ctx* c, int32_t b, int32_t min_count, const int32_t* d_items, const MatDesc* d_mats,
                    int32_t* d_counts, int32_t* d_nfreq, cudaStream_t s);
// In-place all-reduce of `count` device elements over a sharded context's group, ordered on
// `s`; nothing for an unsharded context (shard.cu).
int group_reduce(tfim_ctx* c, void* d_buf, int64_t count, int32_t dtype, int32_t op, cudaStream_t s);
// The same for n host int64 values (staged through the context's device buffer).
int group_reduce_host(tfim_ctx* c, int64_t* vals, int32_t n, int32_t op);
}  // namespace tfim
