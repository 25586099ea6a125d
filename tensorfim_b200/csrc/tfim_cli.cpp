// tfim -- command-line drop-in for the reference engines (CoParaCG_baseline / CoParaCG_bmma).
//
//   tfim <transaction file> <minsup fraction> [--engine resident|batched|plain]
//        [--counter auto|lop3|tensor|i8|proj] [--lookahead 0|1|2|3] [--proposal <file>] [--graphs 0|1]
//        [--superset 0|1]
//
// Same invocation as the reference (code/engine/src/kernel_bitmap.cu:796-798), same
// result file "<file>-<minsup %f>=Results.txt" next to the input (:906-908), same header
// keys and MFI line grammar (:651-690).  Exit code 0 on success, 1 on failure.
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "tfim.h"

namespace {

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

// The proposal network's weights file (written by tensorfim_b200.learn): "TFIMMLP1", int32
// parameter count, float32 threshold, float32 parameters.  Default: proposal_weights.bin in
// the parent directory of this executable.
std::string default_proposal_path() {
    char buf[4096];
    const ssize_t n = readlink("/proc/self/exe", buf, sizeof buf - 1);
    if (n <= 0) return "proposal_weights.bin";
    buf[n] = 0;
    std::string exe = buf;
    const size_t slash = exe.rfind('/');
    return (slash == std::string::npos ? std::string(".") : exe.substr(0, slash)) + "/../proposal_weights.bin";
}

bool load_proposal(const std::string& path, tfim_ctx* ctx, tfim_mlp** out) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    char magic[8];
    int32_t n = 0;
    float thr = 0.5f;
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "TFIMMLP1", 8) == 0 && fread(&n, 4, 1, f) == 1 &&
              fread(&thr, 4, 1, f) == 1 && n == tfim_mlp_num_params();
    std::vector<float> params(ok ? (size_t)n : 0);
    if (ok) ok = fread(params.data(), 4, (size_t)n, f) == (size_t)n;
    fclose(f);
    if (!ok) return false;
    if (tfim_mlp_create(0, 0, out) != TFIM_OK) return false;
    if (tfim_mlp_set_params(*out, params.data()) != TFIM_OK || tfim_set_proposal(ctx, *out, thr) != TFIM_OK) {
        tfim_mlp_free(*out);
        *out = nullptr;
        return false;
    }
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <transaction file> <minsup fraction> [--engine resident|batched|plain] "
                        "[--counter auto|lop3|tensor|i8|proj] [--lookahead 0|1|2|3] [--proposal <weights file>] "
                        "[--graphs 0|1] [--superset 0|1]\n", argv[0]);
        return 1;
    }
    const char* path = argv[1];
    const double thr = atof(argv[2]);
    tfim_mine_opts opts;
    tfim_mine_opts_default(&opts);
    std::string proposal_path;
    for (int i = 3; i + 1 < argc; i += 2) {
        const std::string k = argv[i], v = argv[i + 1];
        if (k == "--engine") {
            if (v == "plain") opts.engine = TFIM_ENGINE_PLAIN;
            else if (v == "batched") opts.engine = TFIM_ENGINE_BATCHED;
            else if (v == "resident") opts.engine = TFIM_ENGINE_RESIDENT;
            else { fprintf(stderr, "unknown engine %s\n", v.c_str()); return 1; }
        } else if (k == "--counter") {
            if (v == "auto") opts.counter = TFIM_COUNTER_AUTO;
            else if (v == "lop3") opts.counter = TFIM_COUNTER_LOP3;
            else if (v == "tensor") opts.counter = TFIM_COUNTER_TENSOR;
            else if (v == "i8") opts.counter = TFIM_COUNTER_I8;
            else if (v == "proj") opts.counter = TFIM_COUNTER_PROJ;
            else { fprintf(stderr, "unknown counter %s\n", v.c_str()); return 1; }
        } else if (k == "--lookahead") opts.lookahead = atoi(v.c_str());
        else if (k == "--proposal") proposal_path = v;
        else if (k == "--graphs") opts.use_graphs = atoi(v.c_str());
        else if (k == "--superset") opts.superset = atoi(v.c_str());
        else { fprintf(stderr, "unknown option %s\n", k.c_str()); return 1; }
    }
    // the file is read into pinned staging by worker threads, copied to the GPU in chunks and
    // parsed there (the reference's readTransSetFile rules), then ingested on the GPU
    const double t1 = now();
    tfim_ctx* ctx = nullptr;
    int rc = tfim_open_file(path, thr, 0, &ctx);
    if (rc == TFIM_E_IO) {
        printf("%s open failed!\n", path);
        return 1;
    }
    if (rc != TFIM_OK) {
        fprintf(stderr, "tfim_open_file failed (%d): %s\n", rc, tfim_last_error());
        return 1;
    }
    const double t2 = now();
    tfim_db_info info;
    tfim_db_info_get(ctx, &info);
    printf("======================================================================\n");
    printf("transSetFile: %s\n", path);
    printf("dimension: %lld\n", (long long)info.dimension);
    printf("transNum: %lld\n", (long long)info.trans_num);
    printf("itemIDmin: %lld\n", (long long)info.item_id_min);
    printf("itemIDmax: %lld\n", (long long)info.item_id_max_dense);
    printf("\nsupportThreshold: %g\n\n", info.support_threshold);
    printf("dimensionReduced: %lld\n", (long long)info.dimension_reduced);
    printf("transNumReduced: %lld\n", (long long)info.trans_num_reduced);
    tfim_mlp* proposal = nullptr;
    if (opts.lookahead == 2) {
        const std::string wp = proposal_path.empty() ? default_proposal_path() : proposal_path;
        if (!load_proposal(wp, ctx, &proposal)) {
            fprintf(stderr, "cannot load the proposal network from %s\n", wp.c_str());
            tfim_close(ctx);
            return 1;
        }
    }
    tfim_mine_stats st;
    rc = tfim_mine(ctx, &opts, &st);
    if (rc != TFIM_OK) {
        fprintf(stderr, "tfim_mine failed (%d): %s\n", rc, tfim_last_error());
        tfim_close(ctx);
        if (proposal) tfim_mlp_free(proposal);
        return 1;
    }
    char out[8192];
    snprintf(out, sizeof out, "%s-%f=Results.txt", path, thr);
    rc = tfim_write_results(ctx, path, out, t2 - t1, st.mine_seconds);
    if (rc != TFIM_OK) {
        fprintf(stderr, "tfim_write_results failed (%d): %s\n", rc, tfim_last_error());
        tfim_close(ctx);
        if (proposal) tfim_mlp_free(proposal);
        return 1;
    }
    printf("======================================================================\n");
    printf("preprocessing_time(s): %g\n", t2 - t1);
    printf("computation_time(s): %g\n", st.mine_seconds);
    printf("total_time(s): %g\n", t2 - t1 + st.mine_seconds);
    printf("\nMFIsNumber: %lld\n", (long long)st.n_mfi);
    printf("engine: %s  waves: %lld  nodes: %lld  supports: %lld  launches: %lld  lookaheads: %lld (hits %lld)  pep: %lld\n",
           opts.engine == TFIM_ENGINE_PLAIN ? "plain" : opts.engine == TFIM_ENGINE_BATCHED ? "batched" : "resident",
           (long long)st.waves, (long long)st.nodes,
           (long long)st.supports, (long long)st.launches, (long long)st.lookaheads, (long long)st.lookahead_hits,
           (long long)st.pruned_pep);
    // the reference's phase line (kernel_bmma.cu:985), measured: mask = prefix-mask building,
    // bmma = counting kernels, memcpy = result read-back and ordering, scatter = the per-row
    // expansion of counted rows into children and MFIs
    printf("BMMA phase ms: mask=%g bmma=%g memcpy=%g scatter=%g\n", st.mask_ms, st.kernel_ms, st.readback_ms,
           st.expand_ms);
    printf("count path ms: lop3=%g gram=%g b1=%g tc=%g pairs=%g proj=%g  pack=%g setup=%g\n", st.path_ms[TFIM_PATH_LOP3],
           st.path_ms[TFIM_PATH_GRAM], st.path_ms[TFIM_PATH_B1], st.path_ms[TFIM_PATH_TC], st.path_ms[TFIM_PATH_PAIRS],
           st.path_ms[TFIM_PATH_PROJ], st.pack_ms, st.setup_ms);
    printf("======================================================================\n");
    tfim_close(ctx);
    if (proposal) tfim_mlp_free(proposal);
    return 0;
}
