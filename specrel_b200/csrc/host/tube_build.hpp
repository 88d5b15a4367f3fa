// The simplices of a worldtube (mesh4d.rs:312-371 Simplex4D::new, 678-717 TubeTriangle::new,
// 721-854 extend_worldtube_simplices), shared by the host scene builder (scene_synth.cpp, g++) and
// the device scene build (sr_extrude.cu, nvcc): the same float operations in the same order, with no
// contraction on either side, so both produce the same records bit for bit.
#pragma once
#include <cstdint>
#include <cstring>

#include "../../../include/specrel.h"
#include "sr_math.hpp"

namespace srh {

using V3f = V3<float>;
using V4f = V4<float>;

struct Box {
    V4f lo{INFINITY, INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY, -INFINITY};
};
SRH_HD inline void grow(Box& b, const V4f& p) {
    b.lo = b.lo.vmin(p);
    b.hi = b.hi.vmax(p);
}
SRH_HD inline Box unite(const Box& a, const Box& b) { return {a.lo.vmin(b.lo), a.hi.vmax(b.hi)}; }

struct Tet {
    SrGpuGeom g;
    SrGpuAttr a;
    Box box;
};

SRH_HD inline void put4(float* d, const V4f& v) {
    d[0] = v.t;
    d[1] = v.x;
    d[2] = v.y;
    d[3] = v.z;
}
SRH_HD inline float fbits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// Simplex4D::new (mesh4d.rs:312-371) writing the hot record, the transposed cold record and the
// padded box directly. Returns false for a degenerate tetrahedron.
SRH_HD inline bool make_tet(const V4f* v, const float (*uv)[2], const V3f* tb, const float* tau, const float (*gr)[2],
                            float uvs_u, float uvs_v, const V4f& nrm, const V4f& u, uint32_t mat, float dec0, float dec1,
                            const int* dec_sel, Tet* out) {
    V4f e1 = v[1] - v[0], e2 = v[2] - v[0], e3 = v[3] - v[0];
    V4f n = cross4(e1, e2, e3);
    float nl2 = n.edot(n);
    if (nl2 < 1e-16f) return false;
    V4f un = n * (1.0f / std::sqrt(nl2));
    V4f r1 = cross4(e2, e3, un), r2 = cross4(e3, e1, un), r3 = cross4(e1, e2, un);
    float d1 = r1.edot(e1), d2 = r2.edot(e2), d3 = r3.edot(e3);
    if (std::fabs(d1) < 1e-12f || std::fabs(d2) < 1e-12f || std::fabs(d3) < 1e-12f) return false;
    put4(out->g.v0, v[0]);
    put4(out->g.n, un);
    put4(out->g.b1, r1 * (1.0f / d1));
    put4(out->g.b2, r2 * (1.0f / d2));
    put4(out->g.b3, r3 * (1.0f / d3));
    SrGpuAttr& a = out->a;
    for (int k = 0; k < 4; ++k) {
        a.uv_u[k] = uv[k][0]; a.uv_v[k] = uv[k][1];
        a.tb_x[k] = tb[k].x; a.tb_y[k] = tb[k].y; a.tb_z[k] = tb[k].z;
        a.tau[k] = tau[k]; a.grad_u[k] = gr[k][0]; a.grad_v[k] = gr[k][1];
        a.decided_at[k] = dec_sel[k] ? dec1 : dec0;
    }
    put4(a.normal, nrm);
    put4(a.four_vel, u);
    a.misc[0] = uvs_u; a.misc[1] = uvs_v; a.misc[2] = fbits(mat); a.misc[3] = 0;
    Box b;
    for (int k = 0; k < 4; ++k) grow(b, v[k]);
    V4f eps(1e-4f, 1e-4f, 1e-4f, 1e-4f);
    b.lo -= eps;
    b.hi += eps;
    out->box = b;
    return true;
}

// A sample of the worldline with its tetrad as four vectors (WorldlineSample, mesh4d.rs:615-630).
struct TubeSample {
    V4f center;
    float tau;
    V3f phi, accel;
    V4f e[4];
};
SRH_HD inline V4f to_world(const TubeSample& s, const V3f& l) { return s.e[1] * l.x + s.e[2] * l.y + s.e[3] * l.z; }

// TubeTriangle::new (mesh4d.rs:678-717): the triangle with its vertex indices sorted ascending
// (stable), the matching uvs and barycentric corners, and the uv tangents.
struct TubeTri {
    uint32_t idx[3];
    V3f p[3];
    float uv[3][2];
    V3f bary[3];
    V3f tu, tv, normal;
};
inline TubeTri make_tube_tri(const V3f* verts, const uint32_t* tri_idx, const float (*tri_uv)[2], const V3f& normal) {
    TubeTri t;
    int perm[3] = {0, 1, 2};
    for (int i = 1; i < 3; ++i)  // stable insertion sort of three indices
        for (int j = i; j > 0 && tri_idx[perm[j]] < tri_idx[perm[j - 1]]; --j) {
            int x = perm[j];
            perm[j] = perm[j - 1];
            perm[j - 1] = x;
        }
    const V3f sb[3] = {V3f(1, 0, 0), V3f(0, 1, 0), V3f(0, 0, 1)};
    for (int k = 0; k < 3; ++k) {
        t.idx[k] = tri_idx[perm[k]];
        t.p[k] = verts[t.idx[k]];
        t.uv[k][0] = tri_uv[perm[k]][0];
        t.uv[k][1] = tri_uv[perm[k]][1];
        t.bary[k] = sb[perm[k]];
    }
    V3f dp1 = t.p[1] - t.p[0], dp2 = t.p[2] - t.p[0];
    float du1 = t.uv[1][0] - t.uv[0][0], dv1 = t.uv[1][1] - t.uv[0][1];
    float du2 = t.uv[2][0] - t.uv[0][0], dv2 = t.uv[2][1] - t.uv[0][1];
    float det = du1 * dv2 - dv1 * du2;
    if (std::fabs(det) > 1e-10f) {
        float inv = 1.0f / det;
        t.tu = (dp1 * dv2 - dp2 * dv1) * inv;
        t.tv = (dp2 * du1 - dp1 * du2) * inv;
    }
    t.normal = normal;
    return t;
}

// decided_at of static geometry (DECIDED_AT_STATIC, mesh4d.rs:3-5).
constexpr float DECIDED_STATIC = -1.0e9f;

// The three tetrahedra of triangle t between samples sc and sn (extend_worldtube_simplices,
// mesh4d.rs:776-854; the Dompierre split (A0,B0,C0,C1), (A0,B0,B1,C1), (A0,A1,B1,C1)). vc and vn
// are the worldtube's events at the two samples, dec0 and dec1 their causal decision stamps
// (DECIDED_STATIC for static geometry). ok[k] says whether tetrahedron k is kept (Simplex4D::new
// skips degenerate ones).
SRH_HD inline void tube_segment(const TubeTri& t, const V4f* vc, const V4f* vn, const TubeSample& sc,
                                const TubeSample& sn, uint32_t mat, float dec0, float dec1, Tet* out, bool* ok) {
    V4f ur = sc.e[0] + sn.e[0];
    V4f u = ur * (1.0f / std::sqrt(mx(-ur.mdot(ur), 1e-12f)));
    V4f a0 = vc[t.idx[0]], b0 = vc[t.idx[1]], c0 = vc[t.idx[2]];
    V4f a1 = vn[t.idx[0]], b1 = vn[t.idx[1]], c1 = vn[t.idx[2]];
    float ta0 = sc.tau + t.p[0].dot(sc.phi), tb0 = sc.tau + t.p[1].dot(sc.phi), tc0 = sc.tau + t.p[2].dot(sc.phi);
    float ta1 = sn.tau + t.p[0].dot(sn.phi), tb1 = sn.tau + t.p[1].dot(sn.phi), tc1 = sn.tau + t.p[2].dot(sn.phi);
    float uvs_u = t.tu.length(), uvs_v = t.tv.length();
    float g0[2] = {t.tu.dot(sc.phi), t.tv.dot(sc.phi)}, g1[2] = {t.tu.dot(sn.phi), t.tv.dot(sn.phi)};
    V4f nr = to_world(sc, t.normal) + to_world(sn, t.normal);
    V4f nrm = nr * (1.0f / std::sqrt(mx(nr.mdot(nr), 1e-12f)));
    const float* UA = t.uv[0];
    const float* UB = t.uv[1];
    const float* UC = t.uv[2];
    const V4f V[3][4] = {{a0, b0, c0, c1}, {a0, b0, b1, c1}, {a0, a1, b1, c1}};
    const float* UVp[3][4] = {{UA, UB, UC, UC}, {UA, UB, UB, UC}, {UA, UA, UB, UC}};
    const V3f TB[3][4] = {{t.bary[0], t.bary[1], t.bary[2], t.bary[2]},
                          {t.bary[0], t.bary[1], t.bary[1], t.bary[2]},
                          {t.bary[0], t.bary[0], t.bary[1], t.bary[2]}};
    const float TAU[3][4] = {{ta0, tb0, tc0, tc1}, {ta0, tb0, tb1, tc1}, {ta0, ta1, tb1, tc1}};
    const int SEL[3][4] = {{0, 0, 0, 1}, {0, 0, 1, 1}, {0, 1, 1, 1}};
    for (int k = 0; k < 3; ++k) {
        float uv[4][2], gr[4][2];
        for (int j = 0; j < 4; ++j) {
            uv[j][0] = UVp[k][j][0];
            uv[j][1] = UVp[k][j][1];
            const float* g = SEL[k][j] ? g1 : g0;
            gr[j][0] = g[0];
            gr[j][1] = g[1];
        }
        ok[k] = make_tet(V[k], uv, TB[k], TAU[k], gr, uvs_u, uvs_v, nrm, u, mat, dec0, dec1, SEL[k], &out[k]);
    }
}

}  // namespace srh
