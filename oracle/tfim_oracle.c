/*
 * tfim_oracle.c -- CPU restatement of the reference MFI engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA engine in
 * tensorfim_b200/.  It may be built, linked and run only by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline leg.
 * Nothing in the shipped engine links or calls it.
 *
 * Parity pinning: tests/test_oracle.py checks this restatement against the reference's
 * own gold result files (data/gold_results) on the datasets that ship with the
 * reference, and against the reference engine itself compiled from its sources by
 * oracle/Makefile (oracle/_ref/), on seeded synthetic databases.
 *
 * Every function cites the reference code it restates (paths relative to the
 * reference project root; the engine is code/engine/src/kernel_bitmap.cu, identical
 * in the relevant parts to code/engine/src/kernel_bmma.cu).
 *
 * Semantics restated exactly:
 *   - parse: every '\n' ends a transaction, empty lines included; a final line
 *     without '\n' counts only if non-empty; "-<digits>" tokens are dropped; any other
 *     non-digit byte is a separator                         (kernel_bitmap.cu:205-267)
 *   - F1 counts item OCCURRENCES (a duplicated id in one row counts twice); the
 *     frequency-sorted order is a stable sort by descending count (kernel_bitmap.cu:269-298)
 *   - frequencyThreshold = transNum * supportThreshold, a double  (kernel_bitmap.cu:806)
 *   - reduction drops items with count < threshold, then empty rows (kernel_bitmap.cu:692-703)
 *   - dimensionReduced = #{ids 0..itemIDmax : double(freq)/transNum > thr} (strict;
 *     kernel_bitmap.cu:815-816); roots are the first dimensionReduced dense items in
 *     frequency order (kernel_bitmap.cu:841-850)
 *   - survivors are ids 1..itemIDmax with count >= threshold, given dense ids in
 *     ascending original-id order; a frequent id 0 is parked after them and is never a
 *     candidate                                          (kernel_bitmap.cu:342-380)
 *   - count: res[e] = popc(AND_{x in X} bv[x] & bv[e]) for every survivor e; the
 *     extra slot holds #{e : res[e] >= threshold}        (kernel_bitmap.cu:390-408)
 *   - search: a node X is an MFI iff that extra slot == |X|; otherwise every dense
 *     i < progress with res[i] >= threshold gives the child X+{i} with frequency res[i]
 *                                                        (kernel_bitmap.cu:853-894)
 *   - output: MFIs sorted by descending frequency, the results-file grammar
 *                                                        (kernel_bitmap.cu:651-690,899-908)
 *
 * The search is run depth-first per root subtree (roots in parallel with OpenMP).  The
 * reference drains one global LIFO from many threads; its output SET is independent of
 * that order, which is what the parity tests compare.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include <math.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TFO_API __attribute__((visibility("default")))

typedef struct {
    int32_t* items;   /* dense ids in insertion order (root first) */
    int32_t n;
    int32_t freq;
} tfo_mfi;

typedef struct {
    /* statistics printed in the results header */
    int64_t transNum, dimension, itemIDmin, itemIDmaxOrig, itemIDmaxDense;
    int64_t transLengthMin, transLengthMax;
    double transLengthMean;
    int64_t transNumReduced, transLengthReducedMin, transLengthReducedMax;
    double transLengthReducedMean;
    int64_t dimensionReduced;
    double supportThreshold, frequencyThreshold;
    /* dense item space */
    int32_t freqItemsNum;     /* survivors 0..freqItemsNum-1 */
    int32_t dCount;           /* + parked id 0 when it is frequent */
    int32_t* denseToOrig;     /* dCount */
    int32_t* freqDense;       /* dCount: occurrence counts */
    int32_t* itemsInFreqSort; /* dCount */
    /* bitmap: dCount rows x W64 words */
    int64_t W64;
    uint64_t* bitmap;
    /* results */
    tfo_mfi* mfis;
    int64_t nMfi, capMfi;
    int64_t nodesVisited;
    double prepTime, compTime;
} tfo_db;

/* ------------------------------------------------------------------ parse (kernel_bitmap.cu:205-267) */
typedef struct { int32_t* v; int64_t n, cap; } ivec;
static void iv_push(ivec* a, int32_t x) {
    if (a->n == a->cap) { a->cap = a->cap ? a->cap * 2 : 64; a->v = (int32_t*)realloc(a->v, (size_t)a->cap * 4); }
    a->v[a->n++] = x;
}
typedef struct { int64_t* v; int64_t n, cap; } lvec;
static void lv_push(lvec* a, int64_t x) {
    if (a->n == a->cap) { a->cap = a->cap ? a->cap * 2 : 64; a->v = (int64_t*)realloc(a->v, (size_t)a->cap * 8); }
    a->v[a->n++] = x;
}

/* rows are stored CSR: items[rowStart[r] .. rowStart[r+1]) */
static int parse_file(const char* path, ivec* items, lvec* rowStart) {
    FILE* fp = fopen(path, "rb");
    if (!fp) return -1;
    fseeko(fp, 0, SEEK_END); long long sz = ftello(fp); fseeko(fp, 0, SEEK_SET);
    char* buf = (char*)malloc(sz > 0 ? (size_t)sz : 1);
    if (sz > 0 && fread(buf, 1, (size_t)sz, fp) != (size_t)sz) { fclose(fp); free(buf); return -2; }
    fclose(fp);
    const char* p = buf; const char* end = buf + sz;
    lv_push(rowStart, 0);
    int64_t curLen = 0;
    while (p < end) {
        char c = *p;
        if (c == '\n') { lv_push(rowStart, items->n); curLen = 0; p++; continue; }
        if (c >= '0' && c <= '9') {
            long v = 0;
            while (p < end && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
            iv_push(items, (int32_t)v); curLen++;
            continue;
        }
        if (c == '-') { p++; while (p < end && *p >= '0' && *p <= '9') p++; continue; }
        p++;
    }
    if (curLen > 0) lv_push(rowStart, items->n);
    free(buf);
    return 0;
}

/* stable sort of ids by descending count (std::stable_sort, kernel_bitmap.cu:280-281) */
static const int32_t* g_sortKey;
static int cmp_desc_stable(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    if (g_sortKey[x] != g_sortKey[y]) return g_sortKey[x] > g_sortKey[y] ? -1 : 1;
    return x < y ? -1 : (x > y);   /* input is iota, so id order == original order */
}

static double now_s(void) { struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return ts.tv_sec + ts.tv_nsec * 1e-9; }

TFO_API void tfo_free(tfo_db* db) {
    if (!db) return;
    free(db->denseToOrig); free(db->freqDense); free(db->itemsInFreqSort); free(db->bitmap);
    for (int64_t i = 0; i < db->nMfi; i++) free(db->mfis[i].items);
    free(db->mfis); free(db);
}

/* Load, reduce and bitmap a transaction file (kernel_bitmap.cu:796-836). Returns NULL on
 * an unreadable file. */
static tfo_db* build_db(const int32_t* itemsv, const int64_t* rsv, int64_t nRows, double supportThreshold);

TFO_API tfo_db* tfo_load(const char* path, double supportThreshold) {
    ivec items = {0}; lvec rs = {0};
    if (parse_file(path, &items, &rs) != 0) { free(items.v); free(rs.v); return NULL; }
    tfo_db* db = build_db(items.v, rs.v, rs.n - 1, supportThreshold);
    free(items.v); free(rs.v);
    return db;
}

/* The same from a CSR transaction set already in memory (row r = items[off[r]..off[r+1])). */
TFO_API tfo_db* tfo_load_csr(const int64_t* off, const int32_t* items, int64_t nRows, double supportThreshold) {
    return build_db(items, off, nRows, supportThreshold);
}

static tfo_db* build_db(const int32_t* itemsv, const int64_t* rsv, int64_t nRows, double supportThreshold) {
    struct { const int32_t* v; } items = { itemsv };
    struct { const int64_t* v; } rs = { rsv };
    const int64_t nItemsTotal = nRows > 0 ? rsv[nRows] : 0;
    tfo_db* db = (tfo_db*)calloc(1, sizeof(tfo_db));
    db->supportThreshold = supportThreshold;
    db->transNum = nRows;
    int64_t idMin = INT_MAX, idMax = 0, lenMin = INT_MAX, lenMax = 0; double lenMean = 0;
    for (int64_t r = 0; r < nRows; r++) {
        int64_t len = rs.v[r + 1] - rs.v[r];
        for (int64_t j = rs.v[r]; j < rs.v[r + 1]; j++) {
            if (items.v[j] > idMax) idMax = items.v[j];
            if (items.v[j] < idMin) idMin = items.v[j];
        }
        if (len < lenMin) lenMin = len;
        if (len > lenMax) lenMax = len;
        lenMean += (double)len;
    }
    if (nRows > 0) lenMean /= (double)nRows;
    db->itemIDmin = idMin; db->itemIDmaxOrig = idMax;
    db->transLengthMin = lenMin; db->transLengthMax = lenMax; db->transLengthMean = lenMean;

    /* getItemsFrequenc (kernel_bitmap.cu:269-298): occurrence counts over ids 0..itemIDmax */
    int32_t* freq = (int32_t*)calloc((size_t)idMax + 1, 4);
    for (int64_t j = 0; j < nItemsTotal; j++) freq[items.v[j]]++;
    int64_t dim = 0;
    for (int64_t i = 0; i <= idMax; i++) if (freq[i]) dim++;
    db->dimension = dim;

    /* threshold, reduction, root count (kernel_bitmap.cu:806-826) */
    const double thr = (double)nRows * supportThreshold;
    db->frequencyThreshold = thr;
    int64_t dimRed = 0;
    for (int64_t i = 0; i <= idMax; i++) if ((double)freq[i] / (double)nRows > supportThreshold) dimRed++;
    db->dimensionReduced = dimRed;

    /* survivors and dense ids (kernel_bitmap.cu:342-373) */
    int32_t* origToDense = (int32_t*)malloc(((size_t)idMax + 1) * 4);
    for (int64_t i = 0; i <= idMax; i++) origToDense[i] = -1;
    int32_t nSurv = 0;
    for (int64_t i = 1; i <= idMax; i++) if (freq[i] >= thr) origToDense[i] = nSurv++;
    const int zeroFrequent = (freq[0] >= thr);
    const int32_t dCount = nSurv + (zeroFrequent ? 1 : 0);
    db->freqItemsNum = nSurv; db->dCount = dCount;
    db->denseToOrig = (int32_t*)malloc(((size_t)dCount + 1) * 4);
    db->freqDense = (int32_t*)malloc(((size_t)dCount + 1) * 4);
    for (int64_t i = 1; i <= idMax; i++) if (origToDense[i] >= 0) {
        db->denseToOrig[origToDense[i]] = (int32_t)i; db->freqDense[origToDense[i]] = freq[i];
    }
    if (zeroFrequent) { origToDense[0] = nSurv; db->denseToOrig[nSurv] = 0; db->freqDense[nSurv] = freq[0]; }
    db->itemIDmaxDense = dCount - 1;
    db->itemsInFreqSort = (int32_t*)malloc(((size_t)dCount + 1) * 4);
    for (int32_t i = 0; i < dCount; i++) db->itemsInFreqSort[i] = i;
    g_sortKey = db->freqDense;
    /* qsort is not stable, but the comparator breaks ties by id over an iota input,
     * which yields exactly the stable order */
    qsort(db->itemsInFreqSort, (size_t)dCount, 4, cmp_desc_stable);

    /* reduce rows: drop infrequent items, then empty rows; relabel to dense ids */
    ivec red = {0}; lvec rrs = {0}; lv_push(&rrs, 0);
    int64_t rMin = INT_MAX, rMax = 0; double rMean = 0;
    for (int64_t r = 0; r < nRows; r++) {
        int64_t before = red.n;
        for (int64_t j = rs.v[r]; j < rs.v[r + 1]; j++) {
            int32_t x = items.v[j];
            if (freq[x] < thr) continue;
            iv_push(&red, origToDense[x]);
        }
        if (red.n > before) {
            int64_t len = red.n - before;
            lv_push(&rrs, red.n);
            if (len < rMin) rMin = len;
            if (len > rMax) rMax = len;
            rMean += (double)len;
        }
    }
    const int64_t nRed = rrs.n - 1;
    rMean /= (double)nRed;   /* 0/0 -> nan, as the reference prints for an empty reduced set */
    db->transNumReduced = nRed; db->transLengthReducedMin = rMin; db->transLengthReducedMax = rMax;
    db->transLengthReducedMean = rMean;

    /* bitmap (kernel_bitmap.cu:374-379) */
    const int64_t W64 = (nRed + 63) / 64;
    db->W64 = W64;
    db->bitmap = (uint64_t*)calloc((size_t)(dCount > 0 ? dCount : 1) * (size_t)(W64 > 0 ? W64 : 1), 8);
    for (int64_t t = 0; t < nRed; t++)
        for (int64_t j = rrs.v[t]; j < rrs.v[t + 1]; j++)
            db->bitmap[(size_t)red.v[j] * W64 + (t >> 6)] |= (1ULL << (t & 63));

    free(freq); free(origToDense); free(red.v); free(rrs.v);
    return db;
}

/* ------------------------------------------------------------------ search (kernel_bitmap.cu:853-894) */
typedef struct { tfo_mfi* v; int64_t n, cap; int64_t nodes; } mfi_list;

static void push_mfi(mfi_list* L, const int32_t* items, int32_t n, int32_t freq) {
    if (L->n == L->cap) { L->cap = L->cap ? L->cap * 2 : 64; L->v = (tfo_mfi*)realloc(L->v, (size_t)L->cap * sizeof(tfo_mfi)); }
    L->v[L->n].items = (int32_t*)malloc((size_t)n * 4);
    memcpy(L->v[L->n].items, items, (size_t)n * 4);
    L->v[L->n].n = n; L->v[L->n].freq = freq; L->n++;
}

/* Depth-first walk of one root's subtree.  masks[k] holds AND of X[0..k]; res holds
 * the counts of the node at depth k.  The per-node counting is getResFrequency
 * (kernel_bitmap.cu:390-408) with the prefix AND carried from the parent, which gives
 * the same AND. */
/* A time-bounded sample (tfo_mine_sample) stops descending once this CLOCK_MONOTONIC time
 * has passed; 0 means no bound.  Set only outside parallel regions. */
static double g_deadline = 0.0;

static void dfs(const tfo_db* db, int32_t* X, int32_t k, int32_t freqX, uint64_t* masks,
                int32_t* resAll, mfi_list* L) {
    if (g_deadline > 0.0 && now_s() > g_deadline) return;
    const int64_t W = db->W64;
    const int32_t d = db->freqItemsNum;
    const double thr = db->frequencyThreshold;
    uint64_t* mask = masks + (size_t)(k - 1) * W;
    int32_t* res = resAll + (size_t)(k - 1) * (d + 1);
    L->nodes++;
    int32_t cnt = 0;
    for (int32_t e = 0; e < d; e++) {
        const uint64_t* bv = db->bitmap + (size_t)e * W;
        uint64_t s = 0;
        for (int64_t w = 0; w < W; w++) s += (uint64_t)__builtin_popcountll(mask[w] & bv[w]);
        res[e] = (int32_t)s;
        if ((double)res[e] >= thr) cnt++;
    }
    if (cnt == k) { push_mfi(L, X, k, freqX); return; }
    const int32_t progress = X[k - 1];
    for (int32_t i = 0; i <= progress - 1; i++) {
        if ((double)res[i] >= thr) {
            /* isOutside(i, X) is always true here: ids strictly decrease along a path */
            X[k] = i;
            uint64_t* child = masks + (size_t)k * W;
            const uint64_t* bv = db->bitmap + (size_t)i * W;
            for (int64_t w = 0; w < W; w++) child[w] = mask[w] & bv[w];
            dfs(db, X, k + 1, res[i], masks, resAll, L);
        }
    }
}

static int cmp_mfi_freq_desc(const void* a, const void* b) {
    const tfo_mfi* x = (const tfo_mfi*)a; const tfo_mfi* y = (const tfo_mfi*)b;
    if (x->freq != y->freq) return x->freq > y->freq ? -1 : 1;
    if (x->n != y->n) return x->n < y->n ? -1 : 1;
    for (int32_t i = 0; i < x->n; i++) if (x->items[i] != y->items[i]) return x->items[i] > y->items[i] ? -1 : 1;
    return 0;
}

/* Mine all MFIs (kernel_bitmap.cu:841-902).  nthreads <= 0 uses all OpenMP threads. */
TFO_API int64_t tfo_mine(tfo_db* db, int nthreads) {
    const double t0 = now_s();
    const int64_t nRoots = db->dimensionReduced < db->dCount ? db->dimensionReduced : db->dCount;
    const int64_t W = db->W64;
    const int32_t d = db->freqItemsNum;
    const int32_t maxDepth = d + 2;
    mfi_list* lists = (mfi_list*)calloc((size_t)(nRoots > 0 ? nRoots : 1), sizeof(mfi_list));
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    #pragma omp parallel num_threads(nthreads)
    {
        uint64_t* masks = (uint64_t*)malloc((size_t)maxDepth * (size_t)(W > 0 ? W : 1) * 8);
        int32_t* res = (int32_t*)malloc((size_t)maxDepth * (size_t)(d + 1) * 4);
        int32_t* X = (int32_t*)malloc((size_t)maxDepth * 4);
        #pragma omp for schedule(dynamic, 1)
        for (int64_t r = 0; r < nRoots; r++) {
            const int32_t item = db->itemsInFreqSort[r];
            X[0] = item;
            const uint64_t* bv = db->bitmap + (size_t)item * W;
            memcpy(masks, bv, (size_t)W * 8);
            dfs(db, X, 1, db->freqDense[item], masks, res, &lists[r]);
        }
        free(masks); free(res); free(X);
    }
    int64_t total = 0, nodes = 0;
    for (int64_t r = 0; r < nRoots; r++) { total += lists[r].n; nodes += lists[r].nodes; }
    for (int64_t i = 0; i < db->nMfi; i++) free(db->mfis[i].items);
    free(db->mfis);
    db->mfis = (tfo_mfi*)malloc((size_t)(total > 0 ? total : 1) * sizeof(tfo_mfi));
    db->nMfi = 0;
    for (int64_t r = 0; r < nRoots; r++) {
        for (int64_t i = 0; i < lists[r].n; i++) db->mfis[db->nMfi++] = lists[r].v[i];
        free(lists[r].v);
    }
    free(lists);
    qsort(db->mfis, (size_t)db->nMfi, sizeof(tfo_mfi), cmp_mfi_freq_desc);
    db->nodesVisited = nodes;
    db->compTime = now_s() - t0;
    return db->nMfi;
}

/* Bounded sample of the same search for CPU timing: root subtrees are taken in the
 * reference's pop order (LIFO over the frequency-ordered roots, so the least frequent
 * root first) by all threads until `budget_s` seconds have passed; subtrees already
 * started are finished.  Returns the nodes counted; *secs gets the elapsed time. */
TFO_API int64_t tfo_mine_sample(tfo_db* db, double budget_s, int nthreads, double* secs) {
    const double t0 = now_s();
    const int64_t nRoots = db->dimensionReduced < db->dCount ? db->dimensionReduced : db->dCount;
    const int64_t W = db->W64;
    const int32_t d = db->freqItemsNum;
    const int32_t maxDepth = d + 2;
    int64_t nodes = 0;
    g_deadline = t0 + budget_s;   /* a long root subtree stops at the budget too */
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    #pragma omp parallel num_threads(nthreads) reduction(+:nodes)
    {
        uint64_t* masks = (uint64_t*)malloc((size_t)maxDepth * (size_t)(W > 0 ? W : 1) * 8);
        int32_t* res = (int32_t*)malloc((size_t)maxDepth * (size_t)(d + 1) * 4);
        int32_t* X = (int32_t*)malloc((size_t)maxDepth * 4);
        mfi_list L = {0};
        #pragma omp for schedule(dynamic, 1)
        for (int64_t k = 0; k < nRoots; k++) {
            if (now_s() - t0 > budget_s) continue;
            const int32_t item = db->itemsInFreqSort[nRoots - 1 - k];
            X[0] = item;
            memcpy(masks, db->bitmap + (size_t)item * W, (size_t)W * 8);
            dfs(db, X, 1, db->freqDense[item], masks, res, &L);
        }
        nodes += L.nodes;
        for (int64_t i = 0; i < L.n; i++) free(L.v[i].items);
        free(L.v); free(masks); free(res); free(X);
    }
    g_deadline = 0.0;
    if (secs) *secs = now_s() - t0;
    return nodes;
}

/* ------------------------------------------------------------------ accessors */
/* The parse alone (kernel_bitmap.cu:205-233): sets *nRows and *nItems; fills off (nRows + 1)
 * and items when both are given and large enough.  Returns -1 when the file cannot be read. */
TFO_API int tfo_parse(const char* path, int64_t* nRows, int64_t* nItems, int64_t* off, int64_t offCap, int32_t* items,
                      int64_t itemsCap) {
    ivec it = {0}; lvec rs = {0};
    if (parse_file(path, &it, &rs) != 0) { free(it.v); free(rs.v); return -1; }
    *nRows = rs.n - 1;
    *nItems = it.n;
    if (off && items && offCap >= rs.n && itemsCap >= it.n) {
        memcpy(off, rs.v, (size_t)rs.n * 8);
        if (it.n) memcpy(items, it.v, (size_t)it.n * 4);
    }
    free(it.v); free(rs.v);
    return 0;
}

TFO_API int64_t tfo_num_mfis(const tfo_db* db) { return db->nMfi; }
TFO_API int64_t tfo_nodes_visited(const tfo_db* db) { return db->nodesVisited; }
TFO_API double tfo_comp_time(const tfo_db* db) { return db->compTime; }
TFO_API int32_t tfo_num_survivors(const tfo_db* db) { return db->freqItemsNum; }
TFO_API int64_t tfo_num_reduced(const tfo_db* db) { return db->transNumReduced; }
TFO_API int64_t tfo_num_trans(const tfo_db* db) { return db->transNum; }
TFO_API int64_t tfo_dimension_reduced(const tfo_db* db) { return db->dimensionReduced; }
TFO_API double tfo_frequency_threshold(const tfo_db* db) { return db->frequencyThreshold; }

/* Total item count over all MFIs (to size the flat buffer of tfo_get_mfis). */
TFO_API int64_t tfo_mfi_item_total(const tfo_db* db) {
    int64_t s = 0; for (int64_t i = 0; i < db->nMfi; i++) s += db->mfis[i].n; return s;
}

/* MFIs in ORIGINAL ids: items_out flat, offsets_out (nMfi+1), freq_out (nMfi). */
TFO_API void tfo_get_mfis(const tfo_db* db, int32_t* items_out, int64_t* offsets_out, int32_t* freq_out) {
    int64_t o = 0;
    for (int64_t i = 0; i < db->nMfi; i++) {
        offsets_out[i] = o;
        for (int32_t j = 0; j < db->mfis[i].n; j++) items_out[o++] = db->denseToOrig[db->mfis[i].items[j]];
        freq_out[i] = db->mfis[i].freq;
    }
    offsets_out[db->nMfi] = o;
}

/* Dense bitmap export as uint32 words: rows x W32 (W32 = 2*W64), for counting KATs. */
TFO_API int64_t tfo_w64(const tfo_db* db) { return db->W64; }
TFO_API int32_t tfo_dcount(const tfo_db* db) { return db->dCount; }
TFO_API const uint64_t* tfo_bitmap(const tfo_db* db) { return db->bitmap; }
TFO_API void tfo_dense_to_orig(const tfo_db* db, int32_t* out) { memcpy(out, db->denseToOrig, (size_t)db->dCount * 4); }
TFO_API void tfo_freq_dense(const tfo_db* db, int32_t* out) { memcpy(out, db->freqDense, (size_t)db->dCount * 4); }
TFO_API void tfo_items_in_freq_sort(const tfo_db* db, int32_t* out) { memcpy(out, db->itemsInFreqSort, (size_t)db->dCount * 4); }

/* ------------------------------------------------------------------ counting KAT
 * The counting contract of getResFrequency (kernel_bitmap.cu:390-408) for a whole
 * wave: rows are nrows x wpr uint32 words; node i's item list is lists[offs[i]..offs[i+1]);
 * counts_out[i*d + e] = popc(AND_t rows[list_i[t]] & rows[e]) for e < d;
 * nfreq_out[i] = #{e < d : counts >= minCount}.  An empty list means the all-ones mask. */
TFO_API void tfo_count_wave(const uint32_t* rows, int64_t wpr, const int32_t* lists, const int64_t* offs,
                            int32_t b, int32_t d, int32_t minCount, int32_t* counts_out, int32_t* nfreq_out) {
    #pragma omp parallel
    {
        uint32_t* mask = (uint32_t*)malloc((size_t)(wpr > 0 ? wpr : 1) * 4);
        #pragma omp for schedule(dynamic, 1)
        for (int32_t i = 0; i < b; i++) {
            for (int64_t w = 0; w < wpr; w++) mask[w] = 0xFFFFFFFFu;
            for (int64_t t = offs[i]; t < offs[i + 1]; t++) {
                const uint32_t* r = rows + (size_t)lists[t] * wpr;
                for (int64_t w = 0; w < wpr; w++) mask[w] &= r[w];
            }
            int32_t c = 0;
            for (int32_t e = 0; e < d; e++) {
                const uint32_t* r = rows + (size_t)e * wpr;
                uint64_t s = 0;
                for (int64_t w = 0; w < wpr; w++) s += (uint64_t)__builtin_popcount(mask[w] & r[w]);
                counts_out[(size_t)i * d + e] = (int32_t)s;
                if ((int32_t)s >= minCount) c++;
            }
            nfreq_out[i] = c;
        }
        free(mask);
    }
}

/* ------------------------------------------------------------------ results file (kernel_bitmap.cu:651-690) */
TFO_API int tfo_write_results(const tfo_db* db, const char* transSetFile, const char* resultPath) {
    FILE* f = fopen(resultPath, "w");
    if (!f) return -1;
    fprintf(f, "==================================================================\n");
    fprintf(f, "CPU: oracle restatement (tfim_oracle.c)\n\n");
    fprintf(f, "==================================================================\n");
    fprintf(f, "transSetFile: %s\n", transSetFile);
    fprintf(f, "dimension: %lld\n", (long long)db->dimension);
    fprintf(f, "transNum: %lld\n", (long long)db->transNum);
    fprintf(f, "itemIDmin: %lld\n", (long long)db->itemIDmin);
    fprintf(f, "itemIDmax: %lld\n", (long long)db->itemIDmaxDense);
    fprintf(f, "transLengthMin: %lld\n", (long long)db->transLengthMin);
    fprintf(f, "transLengthMax: %lld\n", (long long)db->transLengthMax);
    fprintf(f, "transLengthMean: %g\n", db->transLengthMean);
    fprintf(f, "\nsupportThreshold: %g\n\n", db->supportThreshold);
    fprintf(f, "dimensionReduced: %lld\n", (long long)db->dimensionReduced);
    fprintf(f, "transNumReduced: %lld\n", (long long)db->transNumReduced);
    fprintf(f, "transLengthReducedMin: %lld\n", (long long)db->transLengthReducedMin);
    fprintf(f, "transLengthReducedMax: %lld\n", (long long)db->transLengthReducedMax);
    fprintf(f, "transLengthReducedMean: %g\n", db->transLengthReducedMean);
    fprintf(f, "\nGPUtaskPercentage: 0%%\n");
    fprintf(f, "==================================================================\n");
    fprintf(f, "preprocessing_time(s): %g\n", db->prepTime);
    fprintf(f, "computation_time(s): %g\n", db->compTime);
    fprintf(f, "total_time(s): %g\n", db->prepTime + db->compTime);
    fprintf(f, "\nMFIsNumber: %lld\n", (long long)db->nMfi);
    fprintf(f, "============================List of MFIs:=============================\n");
    for (int64_t i = 0; i < db->nMfi; i++) {
        fprintf(f, "%lldth: %d { ", (long long)(i + 1), db->mfis[i].n);
        for (int32_t j = 0; j < db->mfis[i].n; j++) fprintf(f, "%d ", db->denseToOrig[db->mfis[i].items[j]]);
        fprintf(f, "}   support: %g  frequency: %d\n", (double)db->mfis[i].freq / (double)db->transNum, db->mfis[i].freq);
    }
    fprintf(f, "==================================================================\n");
    fclose(f);
    return 0;
}

#ifdef TFO_MAIN
/* oracle CLI: tfim_oracle <transaction file> <minsup fraction> [threads] */
int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s <transaction file> <minsup> [threads]\n", argv[0]); return 2; }
    const double thr = atof(argv[2]);
    const int threads = argc > 3 ? atoi(argv[3]) : 0;
    const double t0 = now_s();
    tfo_db* db = tfo_load(argv[1], thr);
    if (!db) { fprintf(stderr, "%s open failed!\n", argv[1]); return 1; }
    db->prepTime = now_s() - t0;
    tfo_mine(db, threads);
    char out[4096];
    snprintf(out, sizeof out, "%s-%f=Results.txt", argv[1], thr);
    tfo_write_results(db, argv[1], out);
    printf("MFIsNumber: %lld nodes: %lld computation_time(s): %g\n", (long long)db->nMfi,
           (long long)db->nodesVisited, db->compTime);
    tfo_free(db);
    return 0;
}
#endif
