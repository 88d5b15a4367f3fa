// The fast path: the B200 node layout and the persistent, warp-cooperative render kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/specrel.h"
#include "sr_kernels.h"

namespace srk {

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevMem() { if (p) cudaFree(p); }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (!n) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// Wide node: both children's boxes in the parent (80 bytes, five 16-byte loads).
//   [0] left.min  [1] left.max  [2] right.min  [3] right.max
//   [4] (left ref, right ref, left count, right count): a leaf child has count > 0 and ref = its
//       first hot record; an internal child has count 0 and ref = its wide-node index.
// Wide nodes are internal nodes of the reference tree in the reference's depth-first order.
struct FastScene {
    DevMem wide;      // num_wide * 5 uint4
    DevMem scratch;   // build scratch (flags / scan)
    uint32_t num_wide = 0;
    uint32_t depth = 0;
    bool root_is_leaf = false;
    uint32_t root_first = 0, root_count = 0;
    float root_min[4] = {0, 0, 0, 0}, root_max[4] = {0, 0, 0, 0};
    size_t bytes() const { return wide.bytes; }
};

struct FastCtx {
    int num_sms = 148;
    int max_smem = 0;
    DevMem hits;      // per-pixel primary hit records (float4 lambda,u,v,w + uint slot)
    DevMem slots;
};

cudaError_t fast_init(FastCtx& c, const cudaDeviceProp& prop);
void fast_release(FastCtx& c);
cudaError_t fast_build(FastCtx& c, FastScene& s, const SrGpuNode* nodes, uint32_t num_nodes, uint32_t depth,
                       cudaStream_t st);
SrTuning fast_default_tuning(const FastCtx& c);
bool fast_tuning_valid(const FastCtx& c, const SrTuning& t);
// Renders the HDR image (and side outputs) of one frame; `ev` (optional) receives events after the
// trace and shade phases (ev[0], ev[1]).
cudaError_t fast_render(FastCtx& c, const FastScene& s, const SrTuning& t, const SceneDev& sd, const SrGpuUniforms& u,
                        const float4* cam_dev, const FrameDev& f, const BBConst& bb, cudaStream_t st, cudaEvent_t* ev,
                        bool count_work = false);

}  // namespace srk
