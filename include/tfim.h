/*
 * tfim.h -- C ABI of the TensorFIM-B200 exact maximal-frequent-itemset engine.
 *
 * Plain C types only (pointers, sizes, status codes); no torch or CUDA types cross
 * this boundary except an opaque `void* stream` (a cudaStream_t, or NULL for the
 * engine's own stream).  Every call returns a status code; none exits the process.
 * On failure, tfim_last_error() returns a message for the calling thread.
 *
 * The reference (hap04210384/TensorFIM) has no plugin or FFI layer: its boundaries are
 * the engine's command line and two internal C++ counting functions.  Each entry point
 * below names the reference interface it replaces.
 *
 * Threading: a tfim_ctx may be used by one host thread at a time.  Distinct contexts
 * are independent.
 */
#ifndef TFIM_H
#define TFIM_H

#include <stdint.h>

#if defined(__GNUC__)
#define TFIM_API __attribute__((visibility("default")))
#else
#define TFIM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define TFIM_OK            0
#define TFIM_E_INVALID     1   /* bad argument (null pointer, size, threshold outside (0,1]) */
#define TFIM_E_CUDA        2   /* a CUDA runtime call failed */
#define TFIM_E_NOMEM       3   /* host or device allocation failed */
#define TFIM_E_DEPTH       4   /* an item list longer than the counter supports */
#define TFIM_E_TIMEOUT     5   /* a bounded device-side wait expired */
#define TFIM_E_STATE       6   /* call order violated (e.g. results before tfim_mine) */
#define TFIM_E_IO          7   /* a transaction file could not be read, or a results file written */
#define TFIM_E_COMM        8   /* a sharded context's all-reduce callback reported failure */

typedef struct tfim_ctx tfim_ctx;

/* counting paths */
#define TFIM_COUNTER_AUTO    0   /* chosen per job from its shape */
#define TFIM_COUNTER_LOP3    1   /* AND + popc on CUDA cores */
#define TFIM_COUNTER_TENSOR  2   /* b1 AND+POPC tensor-core MMA */
#define TFIM_COUNTER_I8      4   /* tcgen05.mma kind::i8 on the bits expanded to bytes
                                    (tfim_count_wave only) */
#define TFIM_COUNTER_PROJ    3   /* resident engine: projected counting (prefix transactions x
                                    the reduced transaction list) wherever it applies, else auto */

TFIM_API const char* tfim_version(void);
TFIM_API const char* tfim_last_error(void);

/* Statistics the reference prints in its results header
 * (code/engine/src/kernel_bitmap.cu:651-679). */
typedef struct {
    int64_t trans_num;            /* transactions, empty lines included */
    int64_t dimension;            /* distinct item ids */
    int64_t item_id_min;
    int64_t item_id_max;          /* largest original id */
    int64_t item_id_max_dense;    /* the header's itemIDmax: dense ids after compaction */
    int64_t trans_len_min, trans_len_max;
    double  trans_len_mean;
    int64_t trans_num_reduced;    /* rows left after dropping infrequent items and empty rows */
    int64_t trans_len_red_min, trans_len_red_max;
    double  trans_len_red_mean;
    int64_t dimension_reduced;    /* ids with freq/transNum > threshold (strict): the root count */
    double  support_threshold;
    double  frequency_threshold;  /* trans_num * support_threshold */
    int32_t min_count;            /* smallest integer support >= frequency_threshold */
    int32_t n_survivors;          /* dense ids 0..n_survivors-1 are counted */
    int32_t n_dense;              /* n_survivors, plus one when id 0 is frequent (parked) */
    int32_t words_per_row;        /* uint32 words per bitmap row in HBM (multiple of 64) */
} tfim_db_info;

/*
 * Build the device database from a transaction set given in host memory as CSR
 * (row r holds items[row_offsets[r] .. row_offsets[r+1])), with the reference's
 * semantics: F1 occurrence counts, frequencyThreshold = n_rows * support_threshold,
 * removal of infrequent items and then empty rows, dense ids for survivors in
 * ascending original-id order, and a vertical bitmap with one 128-byte-aligned row
 * per dense id.  Ids must be >= 0.
 *
 * Replaces readTransSetFile's successors getItemsFrequenc, reduceTransSet, buildBitmap
 * and uploadBitmapToGPU (code/engine/src/kernel_bitmap.cu:269-298, 692-703, 342-388;
 * code/engine/src/kernel_bmma.cu:388-444).
 */
TFIM_API int tfim_open_db(const int64_t* row_offsets, const int32_t* items, int64_t n_rows,
                 double support_threshold, int32_t device, tfim_ctx** out);

/*
 * Build the device database from the bytes of a transaction file, parsed on the GPU.
 * The bytes are copied to device memory (in chunks through pinned staging, or in one copy
 * from a pinned buffer) and two passes over them produce the CSR that tfim_open_db takes,
 * with the reference's parse rules: every '\n' ends a row (empty rows included), a maximal
 * run of digits is an id, a run right after '-' is dropped, every other byte separates,
 * and a last row without '\n' counts only when it holds an id.  Ingest then continues as in
 * tfim_open_db.  Ids accumulate modulo 2^32 (the reference's value for runs of up to 18
 * digits); an id above INT32_MAX reads as negative and is rejected (TFIM_E_INVALID).
 *
 * Replaces readTransSetFile (code/engine/src/kernel_bitmap.cu:205-267) and its successors.
 */
TFIM_API int tfim_open_text(const char* bytes, int64_t n_bytes, double support_threshold, int32_t device,
                            tfim_ctx** out);
/* tfim_open_text over a file's contents, read with worker threads straight into the pinned
 * staging (TFIM_E_IO when it cannot be opened or read).  Used by the `tfim` command. */
TFIM_API int tfim_open_file(const char* path, double support_threshold, int32_t device, tfim_ctx** out);
/*
 * The parse alone: the CSR of a transaction file's bytes, built on `device` and copied to
 * the caller's arrays.  Always sets *n_rows and *n_items; with null row_offsets and items
 * it only measures, and with arrays smaller than n_rows + 1 offsets or n_items ids it
 * returns TFIM_E_NOMEM and writes neither.  Replaces readTransSetFile's scanner
 * (code/engine/src/kernel_bitmap.cu:205-233) for callers that keep their own ingest.
 */
TFIM_API int tfim_parse_text(const char* bytes, int64_t n_bytes, int32_t device, int64_t* row_offsets, int64_t rows_cap,
                             int32_t* items, int64_t items_cap, int64_t* n_rows, int64_t* n_items);

/*
 * Open a context over a vertical bitmap supplied directly: n_rows rows of
 * ceil(n_bits/32) uint32 words each (row-major, bit t of word t/32 = transaction t).
 * Rows [0, n_counted) are the counted survivors.  Used by the counting interface and
 * its tests; tfim_mine needs a context from tfim_open_db.
 */
TFIM_API int tfim_open_bitmap(const uint32_t* rows, int32_t n_rows, int64_t n_bits, int32_t n_counted,
                     int32_t device, tfim_ctx** out);

/*
 * Transaction sharding across a process group (one process per GPU).  Each rank holds a
 * slice of the transactions and opens its context with the group; every per-transaction
 * statistic the search decides on (id range, row lengths, F1 counts, row supports, wave
 * counts) is summed (or min/max-reduced) over the group through `allreduce`, so all ranks
 * see the whole database's numbers, take the same search steps and find the same MFIs.
 * Integer sums make the result exact.  No counterpart in the reference's engines, which
 * run on one GPU; this shards a database larger than one GPU's memory by transactions.
 *
 * allreduce(buf, count, dtype, op, stream, user): reduce `count` elements at device address
 * `buf` in place over all ranks (dtype TFIM_DT_*, op TFIM_RED_*), ordered on `stream` (a
 * cudaStream_t): work enqueued on `stream` after the call returns must see the result.
 * Return 0 on success.  With NCCL:
 *   ncclAllReduce(buf, buf, count, dtype ? ncclInt64 : ncclInt32,
 *                 op == TFIM_RED_SUM ? ncclSum : op == TFIM_RED_MIN ? ncclMin : ncclMax,
 *                 comm, (cudaStream_t)stream)
 * Every rank calls the library's entry points in the same order with the same arguments
 * (apart from its own transactions); the library then issues the same sequence of
 * collectives on every rank.
 */
#define TFIM_DT_I32 0
#define TFIM_DT_I64 1
#define TFIM_RED_SUM 0
#define TFIM_RED_MIN 1
#define TFIM_RED_MAX 2
typedef int (*tfim_allreduce_fn)(void* buf, int64_t count, int32_t dtype, int32_t op, void* stream, void* user);
typedef struct {
    int32_t rank;                 /* this process's index, 0 .. world-1 */
    int32_t world;                /* number of shards */
    tfim_allreduce_fn allreduce;  /* required when world > 1 */
    void* user;                   /* passed to allreduce */
} tfim_group;

/*
 * tfim_open_db over this rank's rows of a transaction-sharded database.  The threshold
 * applies to the total row count over the group; info fields describe the whole database
 * except words_per_row (this shard's bitmap).  tfim_mine on the context runs the batched or
 * plain engine (the default for a sharded context is batched; the resident engine keeps its
 * counts on the device between waves and is refused with TFIM_E_STATE); tfim_count_wave,
 * tfim_count_wave_device and tfim_mine_all return whole-database counts.
 */
TFIM_API int tfim_open_db_sharded(const int64_t* row_offsets, const int32_t* items, int64_t n_rows,
                                  double support_threshold, int32_t device, const tfim_group* group, tfim_ctx** out);
/*
 * tfim_open_bitmap over this rank's transactions (bit columns) of a sharded bitmap; n_bits
 * is this shard's transaction count (> 0).  Row supports are summed over the group.
 */
TFIM_API int tfim_open_bitmap_sharded(const uint32_t* rows, int32_t n_rows, int64_t n_bits, int32_t n_counted,
                                      int32_t device, const tfim_group* group, tfim_ctx** out);

TFIM_API int tfim_db_info_get(const tfim_ctx* ctx, tfim_db_info* out);
/* dense id -> original id (n_dense entries; out may be null when there are none) */
TFIM_API int tfim_dense_to_orig(const tfim_ctx* ctx, int32_t* out);
/* occurrence count per dense id (n_dense entries; out may be null when there are none) */
TFIM_API int tfim_dense_freq(const tfim_ctx* ctx, int32_t* out);

/*
 * Counting interface: a wave of b nodes, node i given by its dense item list
 * item_lists[list_offsets[i] .. list_offsets[i+1]) (at most 64 items; an empty list
 * is the all-ones prefix).  Writes counts_out[i*n_counted + e] =
 * popc(AND of the listed rows & row e) for every counted row e, and
 * nfreq_out[i] = #{e : counts_out[i*n_counted+e] >= min_count}.
 * Host buffers; the call returns when the results are in them.
 *
 * Replaces getResFrequencyCuda(FI, vector<int>*) (code/engine/src/kernel_bitmap.cu:451-536)
 * and batchCountBMMA(nodes, out) (code/engine/src/kernel_bmma.cu:772-872): the same
 * per-node vector minus the trailing slot, which is nfreq_out here.
 */
TFIM_API int tfim_count_wave(tfim_ctx* ctx, const int32_t* item_lists, const int64_t* list_offsets,
                    int32_t b, int32_t min_count, int32_t* counts_out, int32_t* nfreq_out);

/* Choose the counter tfim_count_wave uses: TFIM_COUNTER_AUTO (default), _LOP3, _TENSOR or _I8. */
TFIM_API int tfim_set_counter(tfim_ctx* ctx, int32_t counter);

/*
 * Same contract with every buffer in device memory, ordered on `stream`
 * (NULL = the context's stream); returns when the counts are in d_counts_out and
 * d_nfreq_out.  max_len bounds the list lengths (<= 64).
 */
TFIM_API int tfim_count_wave_device(tfim_ctx* ctx, const int32_t* d_item_lists, const int64_t* d_list_offsets,
                           int32_t b, int32_t max_len, int32_t min_count,
                           int32_t* d_counts_out, int32_t* d_nfreq_out, void* stream);

/*
 * Allocation-free form of tfim_count_wave_device, for callers that cannot allocate GPU
 * memory: code running inside a memory budget that another allocator owns (it hands out
 * the whole device up front, so a library cudaMalloc would fail or take memory the
 * owner has counted on), and code that only holds device pointers it was handed.  It
 * needs no context: the caller passes a device bitmap, the device item lists and
 * offsets, and the outputs; the result contract is tfim_count_wave's.
 *   bitmap: rows of words_per_row uint32 words, 16-byte aligned, words_per_row a multiple
 *     of 4, bits past the last transaction zero.  Rows 0 .. n_counted-1 are the counted
 *     items (the columns of counts_out); the bitmap must hold a row for every item id
 *     that appears in the lists, which may go beyond n_counted.  Item ids are read on the
 *     device and not range-checked: an id without a row reads outside the bitmap.
 * The per-node prefix masks go to a fixed 16 MiB device array inside the library (held
 * on every device that loads it, until exit): a call needing more than
 * b * words_per_row * 4 = 16 MiB is rejected with TFIM_E_INVALID, and so is b > 65535.
 * The array is shared by all calls and keeps the last call's contents, so calls that
 * overlap on the GPU race.  The first call on a device looks the array's address and
 * the SM count up (cudaGetSymbolAddress, cudaDeviceGetAttribute) with that device
 * current; make that first call before any stream capture.  Enqueued on `stream`
 * (NULL = the legacy default stream); returns after enqueueing.
 * No counterpart in the reference.
 */
TFIM_API int tfim_count_wave_noalloc(const uint32_t* d_bitmap, int64_t words_per_row, int32_t n_counted,
                                     const int32_t* d_item_lists, const int64_t* d_list_offsets, int32_t b,
                                     int32_t min_count, int32_t* d_counts_out, int32_t* d_nfreq_out, void* stream);

/* mining engines */
#define TFIM_ENGINE_PLAIN    0   /* the reference's search, one counted node per launch */
#define TFIM_ENGINE_BATCHED  1   /* pruned search counted in waves of families (host-driven) */
#define TFIM_ENGINE_RESIDENT 2   /* the same search with its state on the device: pack and
                                    expand kernels, one status read per wave */

typedef struct {
    int32_t engine;        /* TFIM_ENGINE_* */
    int32_t counter;       /* TFIM_COUNTER_* */
    int32_t wave_cap;      /* max family rows per wave; 0 = tuned default */
    int32_t lookahead;     /* 0 off, 1 every node that passes the tail-pair filter,
                              2 learned proposal (tfim_set_proposal), 3 every node (no filter) */
    int32_t use_graphs;    /* resident engine: run the wave loop as one captured CUDA graph
                              (conditional WHILE node: pack, count, expand repeat on the
                              device; the host reads the status when the search ends or a
                              pool must grow) */
    int32_t top_counter;   /* family of the empty prefix: 0 by cost model, 1 bitmap Gram,
                              2 pair co-occurrence over the reduced transaction list */
    int32_t log_lookahead; /* 1: log features and outcomes of every lookahead issued */
    int32_t proj_auto;     /* resident engine, automatic counter choice may pick the projected
                              counter: -1 tuned default, 0 no, 1 yes */
    int32_t small_pools;   /* resident engine: start from minimal pool capacities so that
                              every pool grows during the search (exercises the growth path) */
    int32_t superset;      /* resident engine: 1 drops a family whose head and whole tail lie
                              inside an MFI already found (none of its itemsets can be a new
                              maximal set), at creation and again before it leaves the stack;
                              0 (default) off.  Speed only: the MFI set is the same either way */
    int32_t reserved[6];
} tfim_mine_opts;

typedef struct {
    double  mine_seconds;      /* search + counting, bitmap resident (computation_time) */
    double  device_ms;         /* CUDA-event span of the whole search on the engine's stream */
    double  kernel_ms;         /* CUDA-event time of the counting launches */
    int64_t nodes;             /* itemsets counted */
    int64_t supports;          /* individual supports counted (sum over counted rows) */
    int64_t bit_ops;           /* supports x transactions (the roofline unit) */
    int64_t bytes_alg;         /* algorithmic bytes of the counting launches: every operand
                                  row read once, every count written once */
    int64_t waves;
    int64_t launches;          /* kernels launched by the engine */
    int64_t count_launches;    /* ... of which counting kernels */
    int64_t lookaheads;        /* head-union-tail checks issued */
    int64_t lookahead_hits;    /* ... that were frequent and closed a subtree */
    int64_t pruned_pep;        /* subtrees closed by equal-support pruning */
    int64_t n_mfi;
    double  host_ms;           /* host time spent building waves and processing results */
    double  sync_ms;           /* host time blocked on device results */
    int64_t lookaheads_skipped;/* lookaheads ruled out because a tail pair is infrequent */
    double  top_ms;            /* CUDA-event time of counting the empty-prefix family (resident) */
    int64_t pruned_superset;   /* families dropped by the superset check (resident) */
    /* per counting path (index TFIM_PATH_*): device time of its launches, algorithmic bytes
       (every operand row read once as a dense row, every count written once), bit-ops
       (supports x transactions), supports and launches.  Device times come from CUDA events
       around the host-driven launches and from %globaltimer stamps at the start of each
       kernel of a wave (the time from one phase's start to the next phase's start). */
    double  path_ms[6];
    int64_t path_bytes[6];
    int64_t path_bitops[6];
    int64_t path_supports[6];
    int64_t path_launches[6];
    /* device time of the other phases of the search (same stamps): wave packing, row
       expansion, prefix-mask building, and the count-block zeroing */
    double  pack_ms;
    double  expand_ms;
    double  mask_ms;
    double  zero_ms;
    /* host time before the first search launch (pool growth, initial state) and after the
       last one (MFI read-back and assembly, result ordering) */
    double  setup_ms;
    double  readback_ms;
} tfim_mine_stats;

/* counting paths of tfim_mine_stats.path_* */
#define TFIM_PATH_LOP3   0   /* AND + popc tiles on CUDA cores */
#define TFIM_PATH_B1     1   /* b1 AND+POPC mma.sync tiles */
#define TFIM_PATH_TC     2   /* tcgen05.mma kind::i8 tiles (bits expanded to bytes) */
#define TFIM_PATH_PAIRS  3   /* pair co-occurrence over the reduced transaction list */
#define TFIM_PATH_PROJ   4   /* projected counting over the prefix's transactions */
#define TFIM_PATH_GRAM   5   /* register-tiled AND+popc Gram blocks of dense narrow families */

/* ------------------------------------------------------------------ tuning table
 * Launch shapes and counter selection of the engines.  The reference fixes these as
 * constants (wave cap clamp(96 MiB / row bytes, 64, 1024) and split-k <= 32 in
 * code/engine/src/kernel_bmma.cu:636-768,896-910; no selection between counters); here
 * they form a table whose built-in values were measured on B200 and which
 * `python -m tensorfim_b200.autotune` re-measures by sweeping the benchmark databases and
 * writes to tensorfim_b200/tuning.json.  The library loads that file (the `tuning.json`
 * in the parent directory of libtfim.so) the first time a tuning value is needed.
 * Set or load a table before mining; a mine in flight reads the table once at its start. */
typedef struct {
    int32_t wave_rows;          /* family rows per wave (resident and batched engines) */
    float   l3_slices_per_sm;   /* CUDA-core work split: tile slices per SM and wave */
    float   b1_tiles_per_sm;    /* tensor-core split-k target: tiles per SM and wave */
    int32_t b1_min_rows;        /* automatic counter choice: the tensor path for count jobs */
    int32_t b1_min_cols;        /*   of at least b1_min_rows rows x b1_min_cols columns */
    int32_t proj_auto;          /* automatic choice may pick the projected counter (0/1) */
    double  rate_b1_bitops;     /* cost model of the empty-prefix family: b1 bit-ops/s, */
    double  rate_lop3_bitops;   /*   LOP3 bit-ops/s, */
    double  rate_pair_incr;     /*   pair co-occurrence increments/s */
    int32_t i8_min_rows;        /* automatic choice: the tcgen05 kind::i8 counter for count jobs */
    int32_t i8_min_cols;        /*   of at least i8_min_rows x i8_min_cols (tfim_count_wave and
                                     the empty-prefix family's bitmap Gram) */
    double  rate_i8_bitops;     /* cost model: tcgen05 kind::i8 bit-ops/s */
    int32_t tc_min_work;        /* automatic choice: the tcgen05 family counter for family jobs of
                                   at most 128 columns with rows x columns >= tc_min_work and a */
    float   tc_min_density;     /*   prefix holding at least this fraction of 128-bit positions */
    float   tc_tiles_per_sm;    /* tcgen05 family counter: word-slice tiles per SM and wave */
    int32_t gram_min_rows;      /* automatic choice: the CUDA-core Gram counter for dense family
                                   jobs of at most 64 columns and at least this many rows */
    float   l3_dense_slices_per_sm; /* CUDA-core work split of dense families' tiles (resident
                                   engine): tile slices per SM and wave */
} tfim_tuning;

/* The table in force (built-in values, or the loaded / set table). */
TFIM_API void tfim_tuning_get(tfim_tuning* out);
/* Replace the table; values out of range give TFIM_E_INVALID and change nothing. */
TFIM_API int tfim_tuning_set(const tfim_tuning* t);
/* Load a flat JSON object {"wave_rows": 4096, ...}; keys not given keep their value. */
TFIM_API int tfim_tuning_load(const char* path);
/* "built-in" or the path of the table loaded last. */
TFIM_API const char* tfim_tuning_source(void);

TFIM_API void tfim_mine_opts_default(tfim_mine_opts* opts);

/*
 * Mine the maximal frequent itemsets.  The result set equals the reference engine's
 * output on the same database and threshold: every X that is maximal among frequent
 * itemsets over the counted items and whose largest dense id is a root, each with its
 * exact support.  Replaces the search loop of main (code/engine/src/kernel_bitmap.cu:
 * 841-894) and runWaveEngine (code/engine/src/kernel_bmma.cu:896-910).
 */
TFIM_API int tfim_mine(tfim_ctx* ctx, const tfim_mine_opts* opts, tfim_mine_stats* stats);

TFIM_API int64_t tfim_num_mfis(const tfim_ctx* ctx);
TFIM_API int64_t tfim_mfi_item_total(const tfim_ctx* ctx);
/* MFIs sorted by descending support; items in ORIGINAL ids, largest first
 * (the reference's print order). offsets has num_mfis+1 entries. */
TFIM_API int tfim_get_mfis(const tfim_ctx* ctx, int32_t* items, int64_t* offsets, int32_t* supports);

/*
 * All frequent itemsets of up to max_len items (supports >= min_count), level by level on the
 * counting contract: no counterpart in the reference's engines; it restates the reference's
 * level-wise prototype code/batch_proto/batch_proto.cu:257-409 (every frequent (k-1)-itemset
 * is a prefix counted against all items; extensions beyond its last item give the frequent
 * k-itemsets).  Counted items only (a parked id 0 is never a candidate); singleton supports
 * are bitmap popcounts.  Fails with TFIM_E_NOMEM, keeping nothing, when more than
 * max_itemsets are frequent.  stats (optional): waves, prefixes counted (nodes), supports.
 */
TFIM_API int tfim_mine_all(tfim_ctx* ctx, int32_t min_count, int32_t max_len, int64_t max_itemsets,
                           tfim_mine_stats* stats);
TFIM_API int64_t tfim_num_all(const tfim_ctx* ctx);
TFIM_API int64_t tfim_all_item_total(const tfim_ctx* ctx);
/* Itemsets by level, then in prefix order; items in ORIGINAL ids, ascending dense order. */
TFIM_API int tfim_get_all(const tfim_ctx* ctx, int32_t* items, int64_t* offsets, int32_t* supports);

/*
 * Write the reference's results file (code/engine/src/kernel_bitmap.cu:651-690):
 * header keys, "<i>th: <k> { ids }   support: <s>  frequency: <f>" lines, MFIsNumber.
 */
TFIM_API int tfim_write_results(const tfim_ctx* ctx, const char* trans_set_file, const char* result_path,
                       double preprocessing_s, double computation_s);

/*
 * Free a database (the reference frees nothing: its device bitmap is a module global,
 * code/engine/src/kernel_bitmap.cu:447-449).  The search's grown device pools (the resident
 * engine's records and the prefix-mask pool) are kept for the next database opened on the
 * same device, which adopts them instead of growing its own from their minimum; freed
 * device blocks stay cached in the library's stream-ordered pool up to half the device's
 * memory.
 */
TFIM_API void tfim_close(tfim_ctx* ctx);

/*
 * Free the device pools that closed databases left for reuse (see tfim_close), on
 * `device`, or on every device when device < 0.  No counterpart in the reference.
 */
TFIM_API int tfim_release_cached(int32_t device);

/* ------------------------------------------------------------------------------------
 * Learned lookahead proposal (no counterpart in the reference, which has no learned part).
 * A 32 -> 64 -> 64 -> 1 MLP (ReLU, ReLU, sigmoid), BF16 weights, FP32 accumulation,
 * trained and evaluated by the library's own CUDA kernels.  It scores a search node
 * (features: depth, head size, tail size, head support, tail-item supports, prefix
 * density, ...) with the probability that head + tail is frequent; the batched engine
 * issues the head-union-tail lookahead first only for nodes it scores high.  It decides
 * ordering and which exact checks run first only: results never depend on it.
 * Parameters (tfim_mlp_num_params() floats): W1[64][32], b1[64], W2[64][64], b2[64],
 * W3[64], b3.
 */
typedef struct tfim_mlp tfim_mlp;
#define TFIM_MLP_FEATURES 32
TFIM_API int tfim_mlp_create(int32_t device, uint64_t seed, tfim_mlp** out);
TFIM_API int tfim_mlp_num_params(void);
TFIM_API int tfim_mlp_set_params(tfim_mlp* mlp, const float* params);
TFIM_API int tfim_mlp_get_params(const tfim_mlp* mlp, float* params);
/* probs[i] = sigmoid(MLP(feats[i*32 .. i*32+32))) */
TFIM_API int tfim_mlp_predict(tfim_mlp* mlp, const float* feats, int64_t n, float* probs);
/* gradient of mean_i w_i * BCE(probs_i, labels_i) (w_i = pos_weight when label 1) with
 * respect to the FP32 parameters, through the BF16 forward pass; loss may be NULL */
TFIM_API int tfim_mlp_grad(tfim_mlp* mlp, const float* feats, const float* labels, int64_t n, float pos_weight,
                           float* grads, float* loss);
/* Adam over minibatches in the given order, on the GPU */
TFIM_API int tfim_mlp_train(tfim_mlp* mlp, const float* feats, const float* labels, int64_t n, int32_t epochs,
                            int32_t batch, float lr, float pos_weight, float weight_decay, float* final_loss);
TFIM_API void tfim_mlp_free(tfim_mlp* mlp);

/* Attach a proposal network to a context (not owned; NULL detaches).  With
 * tfim_mine_opts.lookahead == 2 the engine issues a lookahead only for nodes scored
 * >= threshold. */
TFIM_API int tfim_set_proposal(tfim_ctx* ctx, tfim_mlp* mlp, float threshold);
/* Lookahead outcomes logged by the last tfim_mine run with opts.log_lookahead = 1:
 * feats (n x 32) and labels (1 = head + tail was frequent).  Returns the number of
 * records (copies at most cap of them); negative on error. */
TFIM_API int64_t tfim_lookahead_log(const tfim_ctx* ctx, float* feats, float* labels, int64_t cap);

#ifdef __cplusplus
}
#endif
#endif /* TFIM_H */
