// FP64 observer setup: the tetrad of Tetrad::rest().boost_local(rapidity) followed by
// rotate_local (minkowski.rs:424-596), evaluated in double precision, and the observer event
// rebased to the scene's FP64 anchor; both then rounded to the f32 values the traversal uses.
// Rebasing the ray origin is the same translation as rebasing every vertex to camera-relative
// coordinates, done once per frame instead of once per vertex.
#pragma once
#include "sr_device.cuh"

namespace srk {

// The algebra is templated on the scalar: double here, and a double carrying derivatives with
// respect to the rapidity for the gradient kernel (sr_adjoint.cuh), with the same operations.
template <class S> struct D4T {
    S t, x, y, z;
};
template <class S> __device__ __forceinline__ D4T<S> dadd(D4T<S> a, D4T<S> b) { return D4T<S>{a.t + b.t, a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> __device__ __forceinline__ D4T<S> dsub(D4T<S> a, D4T<S> b) { return D4T<S>{a.t - b.t, a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S, class K> __device__ __forceinline__ D4T<S> dmul(D4T<S> a, K s) { return D4T<S>{a.t * s, a.x * s, a.y * s, a.z * s}; }
template <class S> __device__ __forceinline__ S dm(D4T<S> a, D4T<S> b) { return -a.t * b.t + a.x * b.x + a.y * b.y + a.z * b.z; }
using D4 = D4T<double>;

// The derivative of boost_local at zero rapidity, where it returns early: none for plain doubles
// (an overload for the gradient's scalar adds the boost generators).
template <class S>
__device__ __forceinline__ void zero_boost_tangent(D4T<S>* e, const S& rx, const S& ry, const S& rz) {}

template <class S> struct TetradT {
    D4T<S> e[4];
    __device__ void rest() {
        e[0] = D4T<S>{S(1.0), S(0.0), S(0.0), S(0.0)};
        e[1] = D4T<S>{S(0.0), S(1.0), S(0.0), S(0.0)};
        e[2] = D4T<S>{S(0.0), S(0.0), S(1.0), S(0.0)};
        e[3] = D4T<S>{S(0.0), S(0.0), S(0.0), S(1.0)};
    }
    __device__ void reorthonormalize() {
        S n0 = sqrt(fmax(-dm(e[0], e[0]), 1e-12));
        e[0] = dmul(e[0], (e[0].t >= 0.0 ? 1.0 : -1.0) / n0);
        for (int a = 1; a <= 3; ++a) {
            D4T<S> v = e[a];
            v = dadd(v, dmul(e[0], dm(v, e[0])));
            for (int b = 1; b < a; ++b) v = dsub(v, dmul(e[b], dm(v, e[b])));
            e[a] = dmul(v, 1.0 / sqrt(fmax(dm(v, v), 1e-12)));
        }
    }
    __device__ void boost_to(D4T<S> nu) {
        S ns = dm(nu, nu);
        D4T<S> u2{S(1.0), S(0.0), S(0.0), S(0.0)};
        if (ns < -1e-12) u2 = dmul(nu, (nu.t >= 0.0 ? 1.0 : -1.0) * (1.0 / sqrt(-ns)));
        D4T<S> u1 = e[0];
        e[0] = u2;
        for (int a = 1; a <= 3; ++a) {  // lorentz_boost_u1_to_u2 (minkowski.rs:385-392)
            S denom = 1.0 - dm(u1, u2);
            D4T<S> sum = dadd(u1, u2);
            e[a] = dsub(dadd(e[a], dmul(sum, dm(sum, e[a]) / denom)), dmul(u2, 2.0 * dm(u1, e[a])));
        }
        reorthonormalize();
    }
    __device__ void boost_local(S rx, S ry, S rz) {
        S eta = sqrt(rx * rx + ry * ry + rz * rz);
        if (eta < 1e-8) {
            zero_boost_tangent(e, rx, ry, rz);
            return;
        }
        S ie = 1.0 / eta;
        D4T<S> s = dadd(dadd(dmul(e[1], rx * ie), dmul(e[2], ry * ie)), dmul(e[3], rz * ie));
        boost_to(dadd(dmul(e[0], cosh(eta)), dmul(s, sinh(eta))));
    }
    __device__ void rot(int a, int b, double ang) {
        double s = sin(ang), c = cos(ang);
        D4T<S> ea = e[a], eb = e[b];
        e[a] = dsub(dmul(ea, c), dmul(eb, s));
        e[b] = dadd(dmul(ea, s), dmul(eb, c));
    }
    // Tetrad::rest().boost_local(rapidity) then rotate_local (yaw, pitch, roll).
    __device__ void observer(S rx, S ry, S rz, double yaw, double pitch, double roll) {
        rest();
        boost_local(rx, ry, rz);
        bool rotated = false;
        if (fabs(yaw) > 1e-8) { rot(1, 3, yaw); rotated = true; }
        if (fabs(pitch) > 1e-8) { rot(2, 3, pitch); rotated = true; }
        if (fabs(roll) > 1e-8) { rot(1, 2, roll); rotated = true; }
        if (rotated) reorthonormalize();
    }
};
using DTetrad = TetradT<double>;

// Writes 6 float4: the anchor-relative event, e0..e3, and the frontier origin (the camera event
// when the uniform block's frontier is the camera, FrameDynamics::frontier_or_camera; an explicit
// frontier is taken as already anchor-relative).
__device__ __forceinline__ void camera_f64(const SrCameraF64& c, const double* anchor, const SrGpuUniforms& U, float4* out) {
    DTetrad t;
    t.observer(c.rapidity[0], c.rapidity[1], c.rapidity[2], c.yaw, c.pitch, c.roll);
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
