// Worldtube extrusion on the device (extend_worldtube_simplices, mesh4d.rs:721-854, and
// Simplex4D::new, mesh4d.rs:312-371): the events of every body at every sample, then the three
// tetrahedra of each triangle between consecutive samples, kept in the serial builder's order
// (body, sample, triangle, split) with degenerate ones dropped. The per-tetrahedron code is the host
// builder's own (host/tube_build.hpp), compiled here without contraction, so the hot records, cold
// records and boxes are the host's bit for bit.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "../host/tube_build.hpp"
#include "sr_build.h"

namespace srk {

using namespace srh;

namespace {

struct BodyDev {
    uint32_t vert_off, nv, tri_off, nt, samp_off, ns, mat, ev_off;
    uint64_t cand_off;
    uint32_t dec_off;  // first decided stamp, or NO_DECIDED (static geometry)
    uint32_t pad;
};
constexpr uint32_t NO_DECIDED = 0xFFFFFFFFu;

// The events of every vertex at every sample, and the Rindler horizon bound the reference asserts
// for a tube of two samples or more (1 + a_local . p > 0, mesh4d.rs:738-751): `bad` is set where it
// fails.
__global__ void k_tube_events(const BodyDev* bodies, const V3f* verts, const TubeSample* samples, V4f* ev,
                              uint32_t* bad) {
    const BodyDev b = bodies[blockIdx.y];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.ns * b.nv) return;
    const uint32_t s = i / b.nv, v = i % b.nv;
    const TubeSample& smp = samples[b.samp_off + s];
    const V3f p = verts[b.vert_off + v];
    if (b.ns >= 2 && !(1.0f + smp.accel.dot(p) > 0.0f)) atomicOr(bad, 1u);
    ev[b.ev_off + i] = smp.center + to_world(smp, p);
}

// The same bound on the host, for tubes that make no tetrahedra (no triangles).
bool rindler_ok(const SrTube* tubes, uint32_t num_tubes) {
    for (uint32_t b = 0; b < num_tubes; ++b) {
        const SrTube& t = tubes[b];
        if (t.num_samples < 2) continue;
        for (uint32_t s = 0; s < t.num_samples; ++s) {
            const float* a = t.samples[s].accel;
            for (uint32_t v = 0; v < t.num_vertices; ++v) {
                const float* p = t.vertices + 3 * v;
                if (!(1.0f + (a[0] * p[0] + a[1] * p[1] + a[2] * p[2]) > 0.0f)) return false;
            }
        }
    }
    return true;
}

__global__ void k_tube_tets(const BodyDev* bodies, const TubeTri* tris, const TubeSample* samples, const float* dec,
                            const V4f* ev, SrGpuGeom* cg, SrGpuAttr* ca, float4* cb, uint32_t* valid) {
    const BodyDev b = bodies[blockIdx.y];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (b.ns < 2 || i >= (b.ns - 1) * b.nt) return;
    const uint32_t st = i / b.nt, t = i % b.nt;
    Tet tet[3];
    bool ok[3];
    const float d0 = b.dec_off == NO_DECIDED ? DECIDED_STATIC : dec[b.dec_off + st];
    const float d1 = b.dec_off == NO_DECIDED ? DECIDED_STATIC : dec[b.dec_off + st + 1];
    tube_segment(tris[b.tri_off + t], ev + b.ev_off + (size_t)st * b.nv, ev + b.ev_off + (size_t)(st + 1) * b.nv,
                 samples[b.samp_off + st], samples[b.samp_off + st + 1], b.mat, d0, d1, tet, ok);
    const uint64_t c = b.cand_off + 3ull * i;
    for (int k = 0; k < 3; ++k) {
        valid[c + k] = ok[k] ? 1u : 0u;
        if (!ok[k]) continue;
        cg[c + k] = tet[k].g;
        ca[c + k] = tet[k].a;
        const Box& bx = tet[k].box;
        cb[2 * (c + k)] = make_float4(bx.lo.t, bx.lo.x, bx.lo.y, bx.lo.z);
        cb[2 * (c + k) + 1] = make_float4(bx.hi.t, bx.hi.x, bx.hi.y, bx.hi.z);
    }
}

__global__ void k_tube_compact(uint64_t ncand, const uint32_t* valid, const uint32_t* pos, const SrGpuGeom* cg,
                               const SrGpuAttr* ca, const float4* cb, SrGpuGeom* g, SrGpuAttr* a, float4* box) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < ncand; c += (uint64_t)gridDim.x * blockDim.x) {
        if (!valid[c]) continue;
        const uint32_t p = pos[c];
        g[p] = cg[c];
        a[p] = ca[c];
        box[2ull * p] = cb[2 * c];
        box[2ull * p + 1] = cb[2 * c + 1];
    }
}

// The first simplex of each tube after compaction, and the total.
__global__ void k_tube_first(const BodyDev* bodies, uint32_t num_tubes, uint64_t ncand, const uint32_t* pos,
                             uint32_t* first) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < num_tubes) first[b] = pos[bodies[b].cand_off];
    if (b == num_tubes) first[b] = pos[ncand];
}

// Scratch from the stream-ordered pool (see sr_build.cu).
template <class T>
struct DBuf {
    T* p = nullptr;
    cudaStream_t st = nullptr;
    ~DBuf() { if (p) cudaFreeAsync(p, st); }
    cudaError_t alloc(size_t n, cudaStream_t s) {
        st = s;
        return cudaMallocAsync(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T), s);
    }
};

}  // namespace

cudaError_t gpu_extrude(const SrTube* tubes, uint32_t num_tubes, ExtrudeOut* out, cudaStream_t st,
                        uint32_t* tube_first) {
    *out = ExtrudeOut{};
    if (tube_first) std::fill(tube_first, tube_first + num_tubes + 1, 0u);
    cudaError_t e = keep_build_pool();
    if (e != cudaSuccess) return e;
#define EK(x) do { if ((e = (x)) != cudaSuccess) return e; } while (0)
    std::vector<BodyDev> bodies(num_tubes);
    std::vector<V3f> verts;
    std::vector<TubeTri> tris;
    std::vector<TubeSample> samples;
    std::vector<float> decs;
    uint64_t ncand = 0;
    uint32_t nev = 0, max_ev = 0, max_seg = 0;
    for (uint32_t b = 0; b < num_tubes; ++b) {
        const SrTube& tb = tubes[b];
        BodyDev& d = bodies[b];
        d.vert_off = (uint32_t)verts.size();
        d.nv = tb.num_vertices;
        d.tri_off = (uint32_t)tris.size();
        d.nt = tb.num_triangles;
        d.samp_off = (uint32_t)samples.size();
        d.ns = tb.num_samples;
        d.mat = tb.material;
        d.ev_off = nev;
        d.cand_off = ncand;
        d.dec_off = tb.decided_at ? (uint32_t)decs.size() : NO_DECIDED;
        d.pad = 0;
        if (tb.decided_at) decs.insert(decs.end(), tb.decided_at, tb.decided_at + tb.num_samples);
        const size_t v0 = verts.size();
        for (uint32_t v = 0; v < tb.num_vertices; ++v)
            verts.push_back(V3f(tb.vertices[3 * v], tb.vertices[3 * v + 1], tb.vertices[3 * v + 2]));
        for (uint32_t t = 0; t < tb.num_triangles; ++t) {
            const SrTubeTriangle& tr = tb.triangles[t];
            tris.push_back(make_tube_tri(verts.data() + v0, tr.idx, tr.uv, V3f(tr.normal[0], tr.normal[1], tr.normal[2])));
        }
        for (uint32_t s = 0; s < tb.num_samples; ++s) {
            const SrTubeSample& q = tb.samples[s];
            TubeSample x;
            x.center = V4f(q.center[0], q.center[1], q.center[2], q.center[3]);
            x.tau = q.proper_time;
            x.phi = V3f(q.phi[0], q.phi[1], q.phi[2]);
            x.accel = V3f(q.accel[0], q.accel[1], q.accel[2]);
            for (int k = 0; k < 4; ++k) x.e[k] = V4f(q.tetrad[k][0], q.tetrad[k][1], q.tetrad[k][2], q.tetrad[k][3]);
            samples.push_back(x);
        }
        nev += tb.num_samples * tb.num_vertices;
        max_ev = std::max(max_ev, tb.num_samples * tb.num_vertices);
        if (tb.num_samples >= 2) {
            const uint32_t seg = (tb.num_samples - 1) * tb.num_triangles;
            max_seg = std::max(max_seg, seg);
            ncand += 3ull * seg;
        }
    }
    if (ncand == 0) {
        out->rindler_bad = rindler_ok(tubes, num_tubes) ? 0u : 1u;
        return cudaSuccess;
    }
    DBuf<BodyDev> db;
    DBuf<V3f> dv;
    DBuf<TubeTri> dt;
    DBuf<TubeSample> ds;
    DBuf<float> ddec;
    DBuf<V4f> dev;
    DBuf<SrGpuGeom> cg;
    DBuf<SrGpuAttr> ca;
    DBuf<float4> cb;
    DBuf<uint32_t> valid, pos, bad;
    EK(db.alloc(num_tubes, st));
    EK(bad.alloc(1, st));
    EK(cudaMemsetAsync(bad.p, 0, 4, st));
    EK(dv.alloc(verts.size(), st));
    EK(dt.alloc(tris.size(), st));
    EK(ds.alloc(samples.size(), st));
    EK(ddec.alloc(decs.size(), st));
    EK(dev.alloc(nev, st));
    EK(cg.alloc(ncand, st));
    EK(ca.alloc(ncand, st));
    EK(cb.alloc(2 * ncand, st));
    EK(valid.alloc(ncand + 1, st));
    EK(pos.alloc(ncand + 1, st));
    EK(cudaMemcpyAsync(db.p, bodies.data(), bodies.size() * sizeof(BodyDev), cudaMemcpyHostToDevice, st));
    EK(cudaMemcpyAsync(dv.p, verts.data(), verts.size() * sizeof(V3f), cudaMemcpyHostToDevice, st));
    EK(cudaMemcpyAsync(dt.p, tris.data(), tris.size() * sizeof(TubeTri), cudaMemcpyHostToDevice, st));
    EK(cudaMemcpyAsync(ds.p, samples.data(), samples.size() * sizeof(TubeSample), cudaMemcpyHostToDevice, st));
    if (!decs.empty())
        EK(cudaMemcpyAsync(ddec.p, decs.data(), decs.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    EK(cudaMemsetAsync(valid.p, 0, (ncand + 1) * 4, st));
    k_tube_events<<<dim3((max_ev + 255) / 256, num_tubes), 256, 0, st>>>(db.p, dv.p, ds.p, dev.p, bad.p);
    k_tube_tets<<<dim3((max_seg + 127) / 128, num_tubes), 128, 0, st>>>(db.p, dt.p, ds.p, ddec.p, dev.p, cg.p, ca.p,
                                                                        cb.p, valid.p);
    EK(cudaGetLastError());
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, valid.p, pos.p, (int)(ncand + 1), st);
    DBuf<unsigned char> tmp;
    EK(tmp.alloc(tmp_bytes, st));
    EK(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, valid.p, pos.p, (int)(ncand + 1), st));
    uint32_t n = 0;
    EK(cudaMemcpyAsync(&n, pos.p + ncand, 4, cudaMemcpyDeviceToHost, st));
    EK(cudaMemcpyAsync(&out->rindler_bad, bad.p, 4, cudaMemcpyDeviceToHost, st));
    DBuf<uint32_t> dfirst;
    if (tube_first) {
        EK(dfirst.alloc(num_tubes + 1, st));
        k_tube_first<<<(num_tubes + 256) / 256, 256, 0, st>>>(db.p, num_tubes, ncand, pos.p, dfirst.p);
        EK(cudaGetLastError());
        EK(cudaMemcpyAsync(tube_first, dfirst.p, (num_tubes + 1) * 4, cudaMemcpyDeviceToHost, st));
    }
    EK(cudaStreamSynchronize(st));
    EK(cudaMallocAsync(reinterpret_cast<void**>(&out->geoms), std::max<size_t>(n, 1) * sizeof(SrGpuGeom), st));
    EK(cudaMallocAsync(reinterpret_cast<void**>(&out->attrs), std::max<size_t>(n, 1) * sizeof(SrGpuAttr), st));
    EK(cudaMallocAsync(reinterpret_cast<void**>(&out->boxes), std::max<size_t>(n, 1) * 2 * sizeof(float4), st));
    out->num_prims = n;
    k_tube_compact<<<148 * 8, 256, 0, st>>>(ncand, valid.p, pos.p, cg.p, ca.p, cb.p, out->geoms, out->attrs, out->boxes);
    EK(cudaGetLastError());
    EK(cudaStreamSynchronize(st));
#undef EK
    return cudaSuccess;
}

}  // namespace srk
