// Forward-mode dual numbers for the gradient kernel: a float value and its derivatives with respect
// to the observer parameters (rapidity x, y, z, event t, x, y, z). The value parts are computed with
// exactly the operations, in exactly the order, of the forward shading code they mirror, so they
// reproduce the forward frame's values bit for bit; the derivative parts follow the chain rule.
// Min/max/clamp select by value and carry the selected operand's derivatives (zero for a constant).
// The types live in their own namespace so that their overloads never hide the float ones.
#pragma once
#include "sr_device.cuh"

namespace srg {

using srd::F3;

constexpr int NT = 7;  // tangents

struct DF {
    float v;
    float d[NT];
};

__device__ __forceinline__ DF dconst(float v) {
    DF r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = 0.0f;
    return r;
}
__device__ __forceinline__ DF operator+(const DF& a, const DF& b) {
    DF r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
__device__ __forceinline__ DF operator-(const DF& a, const DF& b) {
    DF r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
__device__ __forceinline__ DF operator-(const DF& a) {
    DF r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = -a.d[i];
    return r;
}
__device__ __forceinline__ DF operator*(const DF& a, const DF& b) {
    DF r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
__device__ __forceinline__ DF operator/(const DF& a, const DF& b) {
    DF r;
    r.v = a.v / b.v;
    const float ib = 1.0f / b.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
__device__ __forceinline__ DF operator+(const DF& a, float b) {
    DF r = a;
    r.v = a.v + b;
    return r;
}
__device__ __forceinline__ DF operator+(float a, const DF& b) {
    DF r = b;
    r.v = a + b.v;
    return r;
}
__device__ __forceinline__ DF operator-(const DF& a, float b) {
    DF r = a;
    r.v = a.v - b;
    return r;
}
__device__ __forceinline__ DF operator-(float a, const DF& b) {
    DF r;
    r.v = a - b.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = -b.d[i];
    return r;
}
__device__ __forceinline__ DF operator*(const DF& a, float s) {
    DF r;
    r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] * s;
    return r;
}
__device__ __forceinline__ DF operator*(float s, const DF& a) {
    DF r;
    r.v = s * a.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = s * a.d[i];
    return r;
}
__device__ __forceinline__ DF operator/(const DF& a, float b) {
    DF r;
    r.v = a.v / b;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] / b;
    return r;
}
__device__ __forceinline__ DF operator/(float a, const DF& b) {
    DF r;
    r.v = a / b.v;
    const float ib = 1.0f / b.v;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = -r.v * b.d[i] * ib;
    return r;
}
__device__ __forceinline__ DF dsqrt(const DF& a) {
    DF r;
    r.v = sqrtf(a.v);
    const float k = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] * k;
    return r;
}
__device__ __forceinline__ DF dexp(const DF& a) {
    DF r;
    r.v = expf(a.v);
#pragma unroll
    for (int i = 0; i < NT; ++i) r.d[i] = a.d[i] * r.v;
    return r;
}
// fmaxf(a, b) / fminf(a, b) with a constant b.
__device__ __forceinline__ DF dmaxc(const DF& a, float b) { return fmaxf(a.v, b) == a.v && a.v >= b ? a : dconst(fmaxf(a.v, b)); }
__device__ __forceinline__ DF dminc(const DF& a, float b) { return fminf(a.v, b) == a.v && a.v <= b ? a : dconst(fminf(a.v, b)); }
__device__ __forceinline__ DF dclamp(const DF& x, float lo, float hi) {  // clampf_
    if (x.v < lo) return dconst(lo);
    if (x.v > hi) return dconst(hi);
    return x;
}

struct DF3 {
    DF x, y, z;
};
struct DF4 {
    DF x, y, z, w;  // (t, x, y, z)
};

__device__ __forceinline__ DF4 dconst4(float4 a) { return DF4{dconst(a.x), dconst(a.y), dconst(a.z), dconst(a.w)}; }
__device__ __forceinline__ float4 val4(const DF4& a) { return make_float4(a.x.v, a.y.v, a.z.v, a.w.v); }
__device__ __forceinline__ DF4 add4(const DF4& a, const DF4& b) { return DF4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
__device__ __forceinline__ DF4 sub4(const DF4& a, const DF4& b) { return DF4{a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
__device__ __forceinline__ DF4 sub4(float4 a, const DF4& b) { return DF4{a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
__device__ __forceinline__ DF4 mul4(const DF4& a, const DF& s) { return DF4{a.x * s, a.y * s, a.z * s, a.w * s}; }
__device__ __forceinline__ DF4 mul4(const DF4& a, float s) { return DF4{a.x * s, a.y * s, a.z * s, a.w * s}; }
__device__ __forceinline__ DF4 mul4(float4 a, const DF& s) { return DF4{a.x * s, a.y * s, a.z * s, a.w * s}; }
__device__ __forceinline__ DF4 neg4(const DF4& a) { return DF4{-a.x, -a.y, -a.z, -a.w}; }
// mdot / edot in the forward code's order.
__device__ __forceinline__ DF mdot(const DF4& a, const DF4& b) { return -a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ DF mdot(const DF4& a, float4 b) { return -a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ DF edot(float4 a, const DF4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ DF3 spatial(const DF4& a) { return DF3{a.y, a.z, a.w}; }
__device__ __forceinline__ DF dot3(const DF3& a, const DF3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DF3 add(const DF3& a, const DF3& b) { return DF3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ DF3 mul(const DF3& a, const DF& s) { return DF3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ DF3 mul(F3 a, const DF& s) { return DF3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ DF3 mulv(const DF3& a, F3 b) { return DF3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ DF3 dconst3(F3 a) { return DF3{dconst(a.x), dconst(a.y), dconst(a.z)}; }
__device__ __forceinline__ DF len3(const DF3& a) { return dsqrt(dot3(a, a)); }
__device__ __forceinline__ DF3 normalized3(const DF3& a) {
    DF l = len3(a);
    if (l.v > 1e-12f) {
        DF il = 1.0f / l;
        return DF3{a.x * il, a.y * il, a.z * il};
    }
    return DF3{dconst(0.0f), dconst(0.0f), dconst(0.0f)};
}

// A double with its derivatives with respect to the three rapidity components, for the FP64
// tetrad (TetradT<DD3> in sr_camera.cuh).
struct DD3 {
    double v, d[3];
    __device__ DD3(double x = 0.0) : v(x), d{0.0, 0.0, 0.0} {}
};
__device__ __forceinline__ DD3 operator+(const DD3& a, const DD3& b) {
    DD3 r(a.v + b.v);
    for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
__device__ __forceinline__ DD3 operator-(const DD3& a, const DD3& b) {
    DD3 r(a.v - b.v);
    for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
__device__ __forceinline__ DD3 operator-(const DD3& a) {
    DD3 r(-a.v);
    for (int i = 0; i < 3; ++i) r.d[i] = -a.d[i];
    return r;
}
__device__ __forceinline__ DD3 operator*(const DD3& a, const DD3& b) {
    DD3 r(a.v * b.v);
    for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
__device__ __forceinline__ DD3 operator/(const DD3& a, const DD3& b) {
    DD3 r(a.v / b.v);
    for (int i = 0; i < 3; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
__device__ __forceinline__ DD3 operator+(double a, const DD3& b) { return DD3(a) + b; }
__device__ __forceinline__ DD3 operator-(double a, const DD3& b) { return DD3(a) - b; }
__device__ __forceinline__ DD3 operator*(double a, const DD3& b) { return DD3(a) * b; }
__device__ __forceinline__ DD3 operator*(const DD3& a, double b) { return a * DD3(b); }
__device__ __forceinline__ DD3 operator/(double a, const DD3& b) { return DD3(a) / b; }
__device__ __forceinline__ bool operator<(const DD3& a, double b) { return a.v < b; }
__device__ __forceinline__ bool operator>=(const DD3& a, double b) { return a.v >= b; }
__device__ __forceinline__ DD3 sqrt(const DD3& a) {
    DD3 r(::sqrt(a.v));
    for (int i = 0; i < 3; ++i) r.d[i] = r.v > 0.0 ? a.d[i] * (0.5 / r.v) : 0.0;
    return r;
}
__device__ __forceinline__ DD3 fmax(const DD3& a, double b) { return ::fmax(a.v, b) == a.v && a.v >= b ? a : DD3(::fmax(a.v, b)); }
__device__ __forceinline__ DD3 cosh(const DD3& a) {
    DD3 r(::cosh(a.v));
    const double s = ::sinh(a.v);
    for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * s;
    return r;
}
__device__ __forceinline__ DD3 sinh(const DD3& a) {
    DD3 r(::sinh(a.v));
    const double c = ::cosh(a.v);
    for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * c;
    return r;
}

}  // namespace srg
