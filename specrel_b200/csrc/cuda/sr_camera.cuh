// FP64 observer setup: the tetrad of Tetrad::rest().boost_local(rapidity) followed by
// rotate_local (minkowski.rs:424-596), evaluated in double precision, and the observer event
// rebased to the scene's FP64 anchor; both then rounded to the f32 values the traversal uses.
// Rebasing the ray origin is the same translation as rebasing every vertex to camera-relative
// coordinates, done once per frame instead of once per vertex.
#pragma once
#include "sr_device.cuh"

namespace srk {

struct D4 {
    double t, x, y, z;
};
__device__ __forceinline__ D4 dadd(D4 a, D4 b) { return D4{a.t + b.t, a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D4 dsub(D4 a, D4 b) { return D4{a.t - b.t, a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D4 dmul(D4 a, double s) { return D4{a.t * s, a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dm(D4 a, D4 b) { return -a.t * b.t + a.x * b.x + a.y * b.y + a.z * b.z; }

struct DTetrad {
    D4 e[4];
    __device__ void rest() {
        e[0] = D4{1, 0, 0, 0};
        e[1] = D4{0, 1, 0, 0};
        e[2] = D4{0, 0, 1, 0};
        e[3] = D4{0, 0, 0, 1};
    }
    __device__ void reorthonormalize() {
        double n0 = sqrt(fmax(-dm(e[0], e[0]), 1e-12));
        e[0] = dmul(e[0], (e[0].t >= 0.0 ? 1.0 : -1.0) / n0);
        for (int a = 1; a <= 3; ++a) {
            D4 v = e[a];
            v = dadd(v, dmul(e[0], dm(v, e[0])));
            for (int b = 1; b < a; ++b) v = dsub(v, dmul(e[b], dm(v, e[b])));
            e[a] = dmul(v, 1.0 / sqrt(fmax(dm(v, v), 1e-12)));
        }
    }
    __device__ void boost_to(D4 nu) {
        double ns = dm(nu, nu);
        D4 u2{1, 0, 0, 0};
        if (ns < -1e-12) u2 = dmul(nu, (nu.t >= 0.0 ? 1.0 : -1.0) * (1.0 / sqrt(-ns)));
        D4 u1 = e[0];
        e[0] = u2;
        for (int a = 1; a <= 3; ++a) {  // lorentz_boost_u1_to_u2 (minkowski.rs:385-392)
            double denom = 1.0 - dm(u1, u2);
            D4 sum = dadd(u1, u2);
            e[a] = dsub(dadd(e[a], dmul(sum, dm(sum, e[a]) / denom)), dmul(u2, 2.0 * dm(u1, e[a])));
        }
        reorthonormalize();
    }
    __device__ void boost_local(double rx, double ry, double rz) {
        double eta = sqrt(rx * rx + ry * ry + rz * rz);
        if (eta < 1e-8) return;
        double ie = 1.0 / eta;
        D4 s = dadd(dadd(dmul(e[1], rx * ie), dmul(e[2], ry * ie)), dmul(e[3], rz * ie));
        boost_to(dadd(dmul(e[0], cosh(eta)), dmul(s, sinh(eta))));
    }
    __device__ void rot(int a, int b, double ang) {
        double s = sin(ang), c = cos(ang);
        D4 ea = e[a], eb = e[b];
        e[a] = dsub(dmul(ea, c), dmul(eb, s));
        e[b] = dadd(dmul(ea, s), dmul(eb, c));
    }
};

// Writes 6 float4: the anchor-relative event, e0..e3, and the frontier origin (the camera event
// when the uniform block's frontier is the camera, FrameDynamics::frontier_or_camera; an explicit
// frontier is taken as already anchor-relative).
__device__ __forceinline__ void camera_f64(const SrCameraF64& c, const double* anchor, const SrGpuUniforms& U, float4* out) {
    DTetrad t;
    t.rest();
    t.boost_local(c.rapidity[0], c.rapidity[1], c.rapidity[2]);
    bool rotated = false;
    if (fabs(c.yaw) > 1e-8) { t.rot(1, 3, c.yaw); rotated = true; }
    if (fabs(c.pitch) > 1e-8) { t.rot(2, 3, c.pitch); rotated = true; }
    if (fabs(c.roll) > 1e-8) { t.rot(1, 2, c.roll); rotated = true; }
    if (rotated) t.reorthonormalize();
    float4 pos = make_float4((float)(c.event[0] - anchor[0]), (float)(c.event[1] - anchor[1]),
                             (float)(c.event[2] - anchor[2]), (float)(c.event[3] - anchor[3]));
    out[0] = pos;
    for (int a = 0; a < 4; ++a) out[1 + a] = make_float4((float)t.e[a].t, (float)t.e[a].x, (float)t.e[a].y, (float)t.e[a].z);
    bool is_camera = U.frontier_origin[0] == U.cam_pos[0] && U.frontier_origin[1] == U.cam_pos[1] &&
                     U.frontier_origin[2] == U.cam_pos[2] && U.frontier_origin[3] == U.cam_pos[3];
    out[5] = is_camera ? pos
                       : make_float4(U.frontier_origin[0], U.frontier_origin[1], U.frontier_origin[2], U.frontier_origin[3]);
}

}  // namespace srk
