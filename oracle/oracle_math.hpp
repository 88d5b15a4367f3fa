// TEST INFRASTRUCTURE ONLY — part of the CPU oracle that the parity tests use as the checker.
// Nothing in the shipped library includes, links or calls this file.
//
// Scalar helpers and Minkowski algebra restated from the reference renderer, templated on the
// scalar type: `float` reproduces the Rust `f32` code path bit for bit (compile with
// -O2 -ffp-contract=off, no fast-math), `double` is the FP64 oracle.
//
// Reference: src/minkowski.rs (whole file).
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <limits>

namespace orc {

// ------------------------------------------------------------------------------------------
// Transcendentals. Rust `f32::{sin,cos,exp,...}` call the platform libm (glibc on Linux), so
// the float oracle calls the same functions. `perturb_ulps()` moves every transcendental result
// by that many ulps; the parity harness renders at +k and -k to find pixels whose colour
// depends on the last bits of a transcendental (the near-threshold mask).
// ------------------------------------------------------------------------------------------
inline int& perturb_ulps() {
    static int p = 0;
    return p;
}

template <class T>
inline T bump(T r) {
    int k = perturb_ulps();
    if (k == 0 || !std::isfinite(r)) return r;
    T dir = k > 0 ? std::numeric_limits<T>::infinity() : -std::numeric_limits<T>::infinity();
    for (int i = 0; i < std::abs(k); ++i) r = std::nextafter(r, dir);
    return r;
}

inline float m_sin(float x) { return bump(::sinf(x)); }
inline double m_sin(double x) { return bump(::sin(x)); }
inline float m_cos(float x) { return bump(::cosf(x)); }
inline double m_cos(double x) { return bump(::cos(x)); }
inline float m_exp(float x) { return bump(::expf(x)); }
inline double m_exp(double x) { return bump(::exp(x)); }
inline float m_atan2(float y, float x) { return bump(::atan2f(y, x)); }
inline double m_atan2(double y, double x) { return bump(::atan2(y, x)); }
inline float m_acos(float x) { return bump(::acosf(x)); }
inline double m_acos(double x) { return bump(::acos(x)); }
inline float m_tan(float x) { return ::tanf(x); }
inline double m_tan(double x) { return ::tan(x); }
inline float m_cosh(float x) { return ::coshf(x); }
inline double m_cosh(double x) { return ::cosh(x); }
inline float m_sinh(float x) { return ::sinhf(x); }
inline double m_sinh(double x) { return ::sinh(x); }
inline float m_powf(float x, float y) { return ::powf(x, y); }
inline double m_powf(double x, double y) { return ::pow(x, y); }
inline float m_sqrt(float x) { return ::sqrtf(x); }
inline double m_sqrt(double x) { return ::sqrt(x); }

// Rust `f32::min` / `f32::max` (IEEE minNum/maxNum: a NaN operand yields the other).
template <class T> inline T fmin_(T a, T b) { return std::fmin(a, b); }
template <class T> inline T fmax_(T a, T b) { return std::fmax(a, b); }
// Rust `f32::clamp`.
template <class T> inline T clamp_(T x, T lo, T hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// Rust `f32::rem_euclid`: `r = self % rhs; if r < 0 { r + rhs.abs() } else { r }`.
template <class T> inline T rem_euclid(T x, T m) {
    T r = std::fmod(x, m);
    return r < T(0) ? r + std::fabs(m) : r;
}
// Rust `f32::round` (half away from zero).
template <class T> inline T round_(T x) { return std::round(x); }
// Rust `x as i32` (saturating, NaN -> 0).
template <class T> inline int32_t as_i32(T x) {
    if (std::isnan(x)) return 0;
    if (x >= T(2147483648.0)) return INT32_MAX;
    if (x < T(-2147483648.0)) return INT32_MIN;
    return (int32_t)x;
}
// Rust `x as usize` (saturating, NaN -> 0).
template <class T> inline uint64_t as_usize(T x) {
    if (std::isnan(x) || x <= T(0)) return 0;
    if (x >= T(18446744073709551616.0)) return UINT64_MAX;
    return (uint64_t)x;
}
// Rust i32 `+` in a release build (wrapping).
inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
// Rust i32::rem_euclid.
inline int32_t rem_euclid_i32(int32_t a, int32_t m) {
    int32_t r = a % m;
    return r < 0 ? r + (m < 0 ? -m : m) : r;
}

template <class T> struct C {
    static constexpr T PI = T(3.14159265358979323846264338327950288);
    static constexpr T TAU = T(6.28318530717958647692528676655900577);
    static constexpr T FRAC_1_PI = T(0.318309886183790671537767526745028724);
};

// ------------------------------------------------------------------------------------------
// Vec3 / Vec4 (minkowski.rs:5-359). Division by a scalar multiplies by its reciprocal
// (minkowski.rs:128, :349), exactly as the reference does.
// ------------------------------------------------------------------------------------------
template <class T> struct V3 {
    T x = 0, y = 0, z = 0;
    V3() = default;
    V3(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}
    static V3 splat(T v) { return V3(v, v, v); }
    T dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3& o) const {
        return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
    }
    T length_sq() const { return dot(*this); }
    T length() const { return m_sqrt(length_sq()); }
    V3 normalized() const {
        T len = length();
        if (len > T(1e-12)) return (*this) * (T(1) / len);
        return V3(0, 0, 0);
    }
    V3 clamp(T lo, T hi) const { return V3(clamp_(x, lo, hi), clamp_(y, lo, hi), clamp_(z, lo, hi)); }
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator*(T s) const { return V3(x * s, y * s, z * s); }
    V3 operator*(const V3& o) const { return V3(x * o.x, y * o.y, z * o.z); }
    V3 operator/(T s) const { return (*this) * (T(1) / s); }
    V3 operator-() const { return V3(-x, -y, -z); }
    V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
};

template <class T> struct V4 {
    T t = 0, x = 0, y = 0, z = 0;
    V4() = default;
    V4(T t_, T x_, T y_, T z_) : t(t_), x(x_), y(y_), z(z_) {}
    static V4 from_time_space(T t, const V3<T>& s) { return V4(t, s.x, s.y, s.z); }
    static V4 splat(T v) { return V4(v, v, v, v); }
    V3<T> spatial() const { return V3<T>(x, y, z); }
    T mdot(const V4& o) const { return -t * o.t + x * o.x + y * o.y + z * o.z; }
    T mnorm_sq() const { return mdot(*this); }
    T edot(const V4& o) const { return t * o.t + x * o.x + y * o.y + z * o.z; }
    T elen_sq() const { return edot(*this); }
    T elen() const { return m_sqrt(elen_sq()); }
    V4 vmin(const V4& o) const { return V4(fmin_(t, o.t), fmin_(x, o.x), fmin_(y, o.y), fmin_(z, o.z)); }
    V4 vmax(const V4& o) const { return V4(fmax_(t, o.t), fmax_(x, o.x), fmax_(y, o.y), fmax_(z, o.z)); }
    T axis(int i) const { return i == 0 ? t : i == 1 ? x : i == 2 ? y : z; }
    V4 operator+(const V4& o) const { return V4(t + o.t, x + o.x, y + o.y, z + o.z); }
    V4 operator-(const V4& o) const { return V4(t - o.t, x - o.x, y - o.y, z - o.z); }
    V4 operator*(T s) const { return V4(t * s, x * s, y * s, z * s); }
    V4 operator/(T s) const { return (*this) * (T(1) / s); }
    V4 operator-() const { return V4(-t, -x, -y, -z); }
    V4& operator+=(const V4& o) { t += o.t; x += o.x; y += o.y; z += o.z; return *this; }
    V4& operator-=(const V4& o) { t -= o.t; x -= o.x; y -= o.y; z -= o.z; return *this; }

    // minkowski.rs:247-262 — hyperplane covector annihilating span(u, v, w).
    static V4 cross4(const V4& u, const V4& v, const V4& w) {
        T m_xy = v.x * w.y - v.y * w.x;
        T m_xz = v.x * w.z - v.z * w.x;
        T m_yz = v.y * w.z - v.z * w.y;
        T m_tx = v.t * w.x - v.x * w.t;
        T m_ty = v.t * w.y - v.y * w.t;
        T m_tz = v.t * w.z - v.z * w.t;
        T nt = u.x * m_yz - u.y * m_xz + u.z * m_xy;
        T nx = -(u.t * m_yz - u.y * m_tz + u.z * m_ty);
        T ny = u.t * m_xz - u.x * m_tz + u.z * m_tx;
        T nz = -(u.t * m_xy - u.x * m_ty + u.y * m_tx);
        return V4(nt, nx, ny, nz);
    }
    // minkowski.rs:266-270 (beta^2 clamped to 0.999999).
    static V4 four_velocity_from_beta(const V3<T>& beta) {
        T b2 = fmin_(beta.length_sq(), T(0.999999));
        T gamma = T(1) / m_sqrt(T(1) - b2);
        return from_time_space(gamma, beta * gamma);
    }
    // minkowski.rs:274-280.
    V3<T> beta_from_four_velocity() const {
        if (std::fabs(t) > T(1e-12)) return spatial() / t;
        return V3<T>();
    }
};

template <class T> inline V3<T> operator*(T s, const V3<T>& v) { return v * s; }
template <class T> inline V4<T> operator*(T s, const V4<T>& v) { return v * s; }

// minkowski.rs:364-380.
template <class T> inline V4<T> project_to_rest_space(const V4<T>& v, const V4<T>& u) {
    return v + u * v.mdot(u);
}
template <class T> inline T rest_frame_cos(const V4<T>& v, const V4<T>& n, const V4<T>& u) {
    V4<T> vp = project_to_rest_space(v, u);
    T len_sq = vp.mnorm_sq();
    if (len_sq > T(1e-12)) return clamp_(vp.mdot(n) / m_sqrt(len_sq), T(-1), T(1));
    return T(0);
}
// minkowski.rs:385-392.
template <class T> inline V4<T> lorentz_boost_u1_to_u2(const V4<T>& v, const V4<T>& u1, const V4<T>& u2) {
    T u1_dot_u2 = u1.mdot(u2);
    T denom = T(1) - u1_dot_u2;
    V4<T> sum = u1 + u2;
    T sum_dot_v = sum.mdot(v);
    T u1_dot_v = u1.mdot(v);
    return v + sum * (sum_dot_v / denom) - u2 * (T(2) * u1_dot_v);
}

// minkowski.rs:399-609.
template <class T> struct Tetrad {
    std::array<V4<T>, 4> e;
    static Tetrad rest() {
        Tetrad r;
        r.e = {V4<T>(1, 0, 0, 0), V4<T>(0, 1, 0, 0), V4<T>(0, 0, 1, 0), V4<T>(0, 0, 0, 1)};
        return r;
    }
    static Tetrad from_beta(const V3<T>& beta) {
        Tetrad t = rest();
        t.boost_to(V4<T>::four_velocity_from_beta(beta));
        return t;
    }
    void boost_to(const V4<T>& new_u0) {
        T norm_sq = new_u0.mnorm_sq();
        V4<T> u2;
        if (norm_sq < T(-1e-12)) {
            T inv = T(1) / m_sqrt(-norm_sq);
            T sign = new_u0.t >= T(0) ? T(1) : T(-1);
            u2 = new_u0 * (sign * inv);
        } else {
            u2 = V4<T>(1, 0, 0, 0);
        }
        V4<T> u1 = e[0];
        e[0] = u2;
        for (int a = 1; a <= 3; ++a) e[a] = lorentz_boost_u1_to_u2(e[a], u1, u2);
        reorthonormalize();
    }
    void fermi_walker_transport(const V4<T>& new_u0) { boost_to(new_u0); }
    void boost_local(const V3<T>& d_rapidity) {
        T eta = d_rapidity.length();
        if (eta < T(1e-8)) return;
        V3<T> dir = d_rapidity / eta;
        V4<T> s = local_spatial_to_world(dir);
        T ch = m_cosh(eta);
        T sh = m_sinh(eta);
        V4<T> new_u0 = e[0] * ch + s * sh;
        boost_to(new_u0);
    }
    void rotate_local(T yaw, T pitch, T roll) {
        if (std::fabs(yaw) > T(1e-8)) {
            T s = ::std::sin(yaw), c = ::std::cos(yaw);
            V4<T> e1 = e[1], e3 = e[3];
            e[1] = e1 * c - e3 * s;
            e[3] = e1 * s + e3 * c;
        }
        if (std::fabs(pitch) > T(1e-8)) {
            T s = ::std::sin(pitch), c = ::std::cos(pitch);
            V4<T> e2 = e[2], e3 = e[3];
            e[2] = e2 * c - e3 * s;
            e[3] = e2 * s + e3 * c;
        }
        if (std::fabs(roll) > T(1e-8)) {
            T s = ::std::sin(roll), c = ::std::cos(roll);
            V4<T> e1 = e[1], e2 = e[2];
            e[1] = e1 * c - e2 * s;
            e[2] = e1 * s + e2 * c;
        }
        reorthonormalize();
    }
    V4<T> local_spatial_to_world(const V3<T>& l) const { return e[1] * l.x + e[2] * l.y + e[3] * l.z; }
    V4<T> local_to_world(const V4<T>& l) const { return e[0] * l.t + e[1] * l.x + e[2] * l.y + e[3] * l.z; }
    V4<T> world_to_local(const V4<T>& v) const {
        return V4<T>(-v.mdot(e[0]), v.mdot(e[1]), v.mdot(e[2]), v.mdot(e[3]));
    }
    V3<T> world_to_local_spatial(const V4<T>& v) const {
        return V3<T>(v.mdot(e[1]), v.mdot(e[2]), v.mdot(e[3]));
    }
    V4<T> past_light_ray_direction(const V3<T>& dir_local) const {
        V3<T> n = dir_local.normalized();
        return -e[0] + e[1] * n.x + e[2] * n.y + e[3] * n.z;
    }
    V4<T> future_light_ray_direction(const V3<T>& dir_local) const {
        V3<T> n = dir_local.normalized();
        return e[0] + e[1] * n.x + e[2] * n.y + e[3] * n.z;
    }
    void reorthonormalize() {
        T n0 = m_sqrt(fmax_(-e[0].mnorm_sq(), T(1e-12)));
        T sign = e[0].t >= T(0) ? T(1) : T(-1);
        e[0] = e[0] * (sign / n0);
        for (int a = 1; a <= 3; ++a) {
            V4<T> v = e[a];
            v += e[0] * v.mdot(e[0]);
            for (int b = 1; b < a; ++b) v -= e[b] * v.mdot(e[b]);
            T na = m_sqrt(fmax_(v.mnorm_sq(), T(1e-12)));
            e[a] = v * (T(1) / na);
        }
    }
    T gamma() const { return e[0].t; }
    V3<T> beta() const { return e[0].beta_from_four_velocity(); }
};

}  // namespace orc
