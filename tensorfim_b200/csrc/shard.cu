// Transaction sharding: the all-reduce steps of a context opened over one rank's slice of
// the transactions.
//
// Every count the search decides on is a sum over transactions (F1 counts, row supports,
// prefix-by-item supports), so a rank that counts its own transactions and sums the partial
// counts over the group holds the whole database's counts, exactly (integers).  The group's
// all-reduce is a host callback (tfim_group.allreduce): NCCL, torch.distributed, or anything
// that reduces device buffers in place in stream order.  One call per wave carries the b x d
// partial count matrix; ingest adds a handful of small ones.
#include "tfim_internal.h"

namespace tfim {

int group_reduce(tfim_ctx* c, void* d_buf, int64_t count, int32_t dtype, int32_t op, cudaStream_t s) {
    if (!c->sharded || c->group.world <= 1 || count <= 0) return TFIM_OK;
    const int r = c->group.allreduce(d_buf, count, dtype, op, (void*)s, c->group.user);
    TFIM_CHECK(r == 0, TFIM_E_COMM, "group all-reduce of %lld %s values failed (callback returned %d)",
               (long long)count, dtype == TFIM_DT_I64 ? "int64" : "int32", r);
    return TFIM_OK;
}

int group_reduce_host(tfim_ctx* c, int64_t* vals, int32_t n, int32_t op) {
    if (!c->sharded || c->group.world <= 1 || n <= 0) return TFIM_OK;
    cudaStream_t s = c->stream;
    c->d_group.stream = s;
    TFIM_TRY(c->d_group.reserve((size_t)n * 8));
    TFIM_CUDA(cudaMemcpyAsync(c->d_group.p, vals, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    TFIM_TRY(group_reduce(c, c->d_group.p, n, TFIM_DT_I64, op, s));
    TFIM_CUDA(cudaMemcpyAsync(vals, c->d_group.p, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    TFIM_CUDA(cudaStreamSynchronize(s));
    return TFIM_OK;
}

}  // namespace tfim
