// The gradient over a group of GPUs: row bands, the reduction of SrAdjointResult through the
// caller's sum, and a sum over NCCL loaded at run time (no link-time dependency on NCCL).
#include <dlfcn.h>
#include <nccl.h>

#include <mutex>

#include "sr_engine.h"

namespace {

constexpr int RESULT_WORDS = 10;  // loss, gradient[7], primal mismatches, star terms

void pack(const SrAdjointResult& r, double* v) {
    v[0] = r.loss;
    for (int k = 0; k < 7; ++k) v[1 + k] = r.grad[k];
    v[8] = r.primal_mismatch;
    v[9] = r.star_terms;
}

void unpack(const double* v, SrAdjointResult* r) {
    r->loss = v[0];
    for (int k = 0; k < 7; ++k) r->grad[k] = v[1 + k];
    r->primal_mismatch = v[8];
    r->star_terms = v[9];
}

using AllReduceFn = ncclResult_t (*)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);

// ncclAllReduce from the process's NCCL: the one already loaded if there is one, else libnccl.so.2.
AllReduceFn nccl_all_reduce() {
    static std::once_flag once;
    static AllReduceFn fn = nullptr;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW);
        if (h) fn = reinterpret_cast<AllReduceFn>(dlsym(h, "ncclAllReduce"));
    });
    return fn;
}

}  // namespace

extern "C" sr_status sr_adjoint_band(uint32_t height, uint32_t level, uint32_t rank, uint32_t world, uint32_t* row_begin,
                                     uint32_t* row_end) {
    if (!row_begin || !row_end || world == 0 || rank >= world || level > SR_BLOOM_LEVELS) return SR_ERR_INVALID_ARGUMENT;
    uint64_t rows = height;
    for (uint32_t k = 0; k < level; ++k) rows = (rows + 1) / 2;
    *row_begin = (uint32_t)(rows * rank / world);
    *row_end = (uint32_t)(rows * (rank + 1) / world);
    return SR_OK;
}

extern "C" sr_status sr_adjoint_reduce(SrAdjointResult* r, sr_sum_f64_fn sum, void* user) {
    if (!r || !sum) return SR_ERR_INVALID_ARGUMENT;
    double v[RESULT_WORDS];
    pack(*r, v);
    if (sum(v, RESULT_WORDS, user) != 0) return SR_ERR_CUDA;
    unpack(v, r);
    return SR_OK;
}

extern "C" sr_status sr_adjoint_group(sr_ctx* ctx, uint32_t idx, const SrGpuUniforms* u, const SrCameraF64* cam,
                                      const float* target_hdr, uint32_t level, uint32_t flags, uint32_t rank, uint32_t world,
                                      sr_sum_f64_fn sum, void* user, SrAdjointResult* out) {
    if (!ctx || !u || !out || !sum) return SR_ERR_INVALID_ARGUMENT;
    uint32_t r0 = 0, r1 = 0;
    sr_status st = sr_adjoint_band(u->size[1], level, rank, world, &r0, &r1);
    if (st != SR_OK) return st;
    SrAdjointResult part{};
    // A rank whose band is empty evaluates nothing but still joins the sum.
    if (r1 > r0 && (st = sr_adjoint_rows(ctx, idx, u, cam, target_hdr, level, flags, r0, r1, &part)) != SR_OK) return st;
    st = sr_adjoint_reduce(&part, sum, user);
    if (st != SR_OK) return st;
    *out = part;
    return SR_OK;
}

extern "C" int sr_nccl_sum_f64(double* values, size_t count, void* user) {
    auto* s = static_cast<SrNcclSum*>(user);
    if (!values || !s || !s->comm || !s->device_buf) return -2;
    AllReduceFn all_reduce = nccl_all_reduce();
    if (!all_reduce) return -1;
    cudaStream_t st = static_cast<cudaStream_t>(s->stream);
    if (cudaMemcpyAsync(s->device_buf, values, count * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) return -2;
    ncclResult_t r = all_reduce(s->device_buf, s->device_buf, count, ncclFloat64, ncclSum,
                                static_cast<ncclComm_t>(s->comm), st);
    if (r != ncclSuccess) return (int)r;
    if (cudaMemcpyAsync(values, s->device_buf, count * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -2;
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : -2;
}
