// The plain path: one thread per pixel in 8x8 tiles (the reference's dispatch, gpu.rs:28, 834-844),
// the reference's BVH2 traversal with a 64-entry per-thread stack (bvh4d.rs:445-578), then
// shading, shadow rays and the star term. It is the baseline the fast path is measured against,
// and it reproduces the reference traversal order exactly (ties at equal lambda included).
#include "sr_kernels.h"
#include "sr_shade.cuh"

namespace srk {

using namespace srd;

// Iteration bound per ray: a tree checked at upload never gets near it; a corrupted one sets
// ERR_TRAVERSAL_LIMIT and the ray ends instead of spinning.
constexpr uint32_t MAX_VISITS = 1u << 22;

struct NodeRef {
    float4 bmin, bmax;
    uint4 meta;  // right_or_first, count, left, pad
};
__device__ __forceinline__ NodeRef load_node(const SrGpuNode* nodes, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    NodeRef n;
    n.bmin = __ldg(p);
    n.bmax = __ldg(p + 1);
    n.meta = __ldg(reinterpret_cast<const uint4*>(p + 2));
    return n;
}
__device__ __forceinline__ float child_enter(const SrGpuNode* nodes, uint32_t i, float4 o, float4 inv, float t_min,
                                             float t_max) {
    const float4* p = reinterpret_cast<const float4*>(nodes + i);
    return slab_enter(__ldg(p), __ldg(p + 1), o, inv, t_min, t_max);
}

// Bvh4D::trace (bvh4d.rs:445-520). Returns the leaf slot of the closest hit or -1.
__device__ int trace_ref(const SceneDev& s, float4 o, float4 d, float t_min, float t_max, GeomHit* best,
                         uint32_t* err) {
    if (s.num_nodes == 0u) return -1;
    float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
    float re = child_enter(s.nodes, 0, o, inv, t_min, t_max);
    if (re < 0.0f) return -1;
    uint32_t sn[SR_STACK_SIZE];
    float stt[SR_STACK_SIZE];
    uint32_t sp = 1;
    sn[0] = 0;
    stt[0] = re;
    int slot = -1;
    uint32_t visits = 0;
    while (sp > 0) {
        if (++visits > MAX_VISITS) { atomicOr(err, ERR_TRAVERSAL_LIMIT); break; }
        --sp;
        uint32_t ni = sn[sp];
        if (stt[sp] >= t_max) continue;
        uint4 meta = __ldg(reinterpret_cast<const uint4*>(s.nodes + ni) + 2);
        if (meta.y > 0u) {
            uint32_t first = meta.x, end = meta.x + meta.y;
            for (uint32_t k = first; k < end; ++k) {
                GeomHit gh;
                if (intersect_geom(s.geoms + 5u * k, o, d, t_min, t_max, &gh)) {
                    t_max = gh.lambda;
                    *best = gh;
                    slot = (int)k;
                }
            }
        } else {
            uint32_t li = meta.z, ri = meta.x;
            float tl = child_enter(s.nodes, li, o, inv, t_min, t_max);
            float tr = child_enter(s.nodes, ri, o, inv, t_min, t_max);
            bool hl = tl >= 0.0f, hr = tr >= 0.0f;
            if (hl && hr) {
                if (sp + 2u <= SR_STACK_SIZE) {
                    if (tl <= tr) { sn[sp] = ri; stt[sp] = tr; sn[sp + 1] = li; stt[sp + 1] = tl; }
                    else { sn[sp] = li; stt[sp] = tl; sn[sp + 1] = ri; stt[sp + 1] = tr; }
                    sp += 2u;
                }
            } else if (hl) {
                if (sp < SR_STACK_SIZE) { sn[sp] = li; stt[sp] = tl; ++sp; }
            } else if (hr) {
                if (sp < SR_STACK_SIZE) { sn[sp] = ri; stt[sp] = tr; ++sp; }
            }
        }
    }
    return slot;
}

// Bvh4D::is_occluded (bvh4d.rs:523-578).
__device__ bool occluded_ref(const SceneDev& s, float4 o, float4 d, float t_min, float t_max, uint32_t* err) {
    if (s.num_nodes == 0u) return false;
    float4 inv = v4(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z), safe_inv(d.w));
    if (child_enter(s.nodes, 0, o, inv, t_min, t_max) < 0.0f) return false;
    uint32_t st[SR_STACK_SIZE];
    uint32_t sp = 1;
    st[0] = 0;
    uint32_t visits = 0;
    while (sp > 0) {
        if (++visits > MAX_VISITS) { atomicOr(err, ERR_TRAVERSAL_LIMIT); return false; }
        uint32_t ni = st[--sp];
        uint4 meta = __ldg(reinterpret_cast<const uint4*>(s.nodes + ni) + 2);
        if (meta.y > 0u) {
            for (uint32_t k = meta.x; k < meta.x + meta.y; ++k) {
                GeomHit gh;
                if (intersect_geom(s.geoms + 5u * k, o, d, t_min, t_max, &gh)) return true;
            }
        } else {
            uint32_t li = meta.z, ri = meta.x;
            bool hl = child_enter(s.nodes, li, o, inv, t_min, t_max) >= 0.0f;
            bool hr = child_enter(s.nodes, ri, o, inv, t_min, t_max) >= 0.0f;
            if (hr && sp < SR_STACK_SIZE) st[sp++] = ri;
            if (hl && sp < SR_STACK_SIZE) st[sp++] = li;
        }
    }
    return false;
}

struct RefOccluder {
    const SceneDev* s;
    uint32_t* err;
    __device__ bool operator()(float4 o, float4 d, float t0, float t1) { return occluded_ref(*s, o, d, t0, t1, err); }
};

__global__ void __launch_bounds__(64, 16) k_render_plain(SceneDev s, SrGpuUniforms U, const float4* cam_dev, FrameDev f,
                                                     BBConst bb) {
    uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= U.size[0] || py >= U.size[1]) return;
    const Cam cam = load_cam(U, cam_dev);
    float4 o, d;
    float sx, sy;
    camera_ray(U, cam, px, py, &o, &d, &sx, &sy);
    GeomHit gh;
    int slot = trace_ref(s, o, d, 1e-3f, 180.0f, &gh, f.counters + 1);
    uint32_t shadow_rays = 0;
    F3 color;
    Hit h;
    if (slot >= 0) {
        interpolate(s.attrs + 12u * (uint32_t)slot, o, d, gh, &h);
        RefOccluder occ{&s, f.counters + 1};
        color = shade_hit(s, U, cam, d, h, occ, &shadow_rays);
        if (U.num_haze > 0u) color = apply_haze(color, h.event, U);
    } else {
        color = shade_sky(d);
    }
    if (U.mode == 0u && s.num_stars > 0u)
        color = add(color, stars_brute(s, U, cam, o, d, sx, sy, slot >= 0 ? h.lambda : INFINITY, bb));
    size_t idx = (size_t)py * U.size[0] + px;
    f.hdr[idx] = make_float4(color.x, color.y, color.z, 0.0f);
    if (f.hit_id) f.hit_id[idx] = slot < 0 ? 0xFFFFFFFFu : (s.leaf_to_orig ? __ldg(s.leaf_to_orig + slot) : (uint32_t)slot);
    if (f.lambda) f.lambda[idx] = slot < 0 ? 0.0f : h.lambda;
    if (f.tau) f.tau[idx] = slot < 0 ? 0.0f : h.tau;
    if (shadow_rays) atomicAdd(f.counters, shadow_rays);
}

cudaError_t launch_render_plain(const SceneDev& s, const SrGpuUniforms& u, const float4* cam_dev, const FrameDev& f,
                                const BBConst& bb, cudaStream_t st) {
    dim3 block(8, 8);
    dim3 grid((u.size[0] + 7) / 8, (u.size[1] + 7) / 8);
    k_render_plain<<<grid, block, 0, st>>>(s, u, cam_dev, f, bb);
    return cudaGetLastError();
}

// Caller rays (sr_trace_rays): one thread per ray, the reference's traversal, then the hit
// record interpolated as the shading reads it.
__global__ void k_trace_rays(SceneDev s, double a0, double a1, double a2, double a3, const SrRay* rays, uint32_t n,
                             SrRayHit* hits, uint32_t* counters) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SrRay r = rays[i];
    const float4 o = v4((float)(r.origin[0] - a0), (float)(r.origin[1] - a1), (float)(r.origin[2] - a2),
                        (float)(r.origin[3] - a3));
    const float4 d = v4(r.dir[0], r.dir[1], r.dir[2], r.dir[3]);
    SrRayHit out;
    out.id = 0xFFFFFFFFu;
    out.slot = 0xFFFFFFFFu;
    out.lambda = out.proper_time = 0.0f;
    for (int k = 0; k < 4; ++k) { out.event[k] = 0.0; out.tet_bary[k] = 0.0f; }
    out.uv[0] = out.uv[1] = 0.0f;
    out.material = out.pad = 0u;
    GeomHit gh;
    const int slot = trace_ref(s, o, d, r.t_min, r.t_max, &gh, counters + 1);
    if (slot >= 0) {
        Hit h;
        interpolate(s.attrs + 12u * (uint32_t)slot, o, d, gh, &h);
        out.slot = (uint32_t)slot;
        out.id = s.leaf_to_orig ? __ldg(s.leaf_to_orig + slot) : (uint32_t)slot;
        out.lambda = h.lambda;
        out.proper_time = h.tau;
        out.event[0] = (double)h.event.x + a0;
        out.event[1] = (double)h.event.y + a1;
        out.event[2] = (double)h.event.z + a2;
        out.event[3] = (double)h.event.w + a3;
        out.tet_bary[0] = h.b0;
        out.tet_bary[1] = h.b1;
        out.tet_bary[2] = h.b2;
        out.tet_bary[3] = h.b3;
        out.uv[0] = h.uv_u;
        out.uv[1] = h.uv_v;
        out.material = h.material;
    }
    hits[i] = out;
}

cudaError_t launch_trace_rays(const SceneDev& s, const double anchor[4], const SrRay* rays, uint32_t n, SrRayHit* hits,
                              uint32_t* counters, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_trace_rays<<<(n + 127) / 128, 128, 0, st>>>(s, anchor[0], anchor[1], anchor[2], anchor[3], rays, n, hits, counters);
    return cudaGetLastError();
}

}  // namespace srk
