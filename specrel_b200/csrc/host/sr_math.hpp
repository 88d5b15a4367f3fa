// Host-side Minkowski algebra for the scene builder and the frame setup (the caller's side of the
// boundary). Follows src/minkowski.rs operation for operation so that the f32 results equal the
// reference's: the library is compiled without FMA contraction (-ffp-contract=off) and division
// by a scalar multiplies by the reciprocal (minkowski.rs:128, :349).
#pragma once
#include <array>
#include <cmath>
#include <cstdint>

// Also compiled for the device (the scene build kernels): the vector algebra is marked for both.
#ifdef __CUDACC__
#define SRH_HD __host__ __device__
#else
#define SRH_HD
#endif

namespace srh {

template <class T> SRH_HD inline T mn(T a, T b) { return std::fmin(a, b); }
template <class T> SRH_HD inline T mx(T a, T b) { return std::fmax(a, b); }

template <class T> struct V3 {
    T x = 0, y = 0, z = 0;
    V3() = default;
    SRH_HD V3(T a, T b, T c) : x(a), y(b), z(c) {}
    SRH_HD T dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    SRH_HD T length() const { return std::sqrt(dot(*this)); }
    SRH_HD V3 normalized() const {
        T l = length();
        return l > T(1e-12) ? (*this) * (T(1) / l) : V3();
    }
    SRH_HD V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    SRH_HD V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    SRH_HD V3 operator*(T s) const { return V3(x * s, y * s, z * s); }
    SRH_HD V3 operator/(T s) const { return (*this) * (T(1) / s); }
    SRH_HD V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
};

template <class T> struct V4 {
    T t = 0, x = 0, y = 0, z = 0;
    V4() = default;
    SRH_HD V4(T a, T b, T c, T d) : t(a), x(b), y(c), z(d) {}
    SRH_HD V3<T> sp() const { return V3<T>(x, y, z); }
    SRH_HD T mdot(const V4& o) const { return -t * o.t + x * o.x + y * o.y + z * o.z; }
    SRH_HD T edot(const V4& o) const { return t * o.t + x * o.x + y * o.y + z * o.z; }
    SRH_HD T ax(int i) const { return i == 0 ? t : i == 1 ? x : i == 2 ? y : z; }
    SRH_HD V4 vmin(const V4& o) const { return V4(mn(t, o.t), mn(x, o.x), mn(y, o.y), mn(z, o.z)); }
    SRH_HD V4 vmax(const V4& o) const { return V4(mx(t, o.t), mx(x, o.x), mx(y, o.y), mx(z, o.z)); }
    SRH_HD V4 operator+(const V4& o) const { return V4(t + o.t, x + o.x, y + o.y, z + o.z); }
    SRH_HD V4 operator-(const V4& o) const { return V4(t - o.t, x - o.x, y - o.y, z - o.z); }
    SRH_HD V4 operator*(T s) const { return V4(t * s, x * s, y * s, z * s); }
    SRH_HD V4 operator-() const { return V4(-t, -x, -y, -z); }
    SRH_HD V4& operator+=(const V4& o) { t += o.t; x += o.x; y += o.y; z += o.z; return *this; }
    SRH_HD V4& operator-=(const V4& o) { t -= o.t; x -= o.x; y -= o.y; z -= o.z; return *this; }
};

// minkowski.rs:247-262.
template <class T> SRH_HD inline V4<T> cross4(const V4<T>& u, const V4<T>& v, const V4<T>& w) {
    T m_xy = v.x * w.y - v.y * w.x, m_xz = v.x * w.z - v.z * w.x, m_yz = v.y * w.z - v.z * w.y;
    T m_tx = v.t * w.x - v.x * w.t, m_ty = v.t * w.y - v.y * w.t, m_tz = v.t * w.z - v.z * w.t;
    return V4<T>(u.x * m_yz - u.y * m_xz + u.z * m_xy, -(u.t * m_yz - u.y * m_tz + u.z * m_ty),
                 u.t * m_xz - u.x * m_tz + u.z * m_tx, -(u.t * m_xy - u.x * m_ty + u.y * m_tx));
}

// minkowski.rs:266-270.
template <class T> inline V4<T> four_velocity(const V3<T>& b) {
    T b2 = mn(b.dot(b), T(0.999999));
    T g = T(1) / std::sqrt(T(1) - b2);
    V3<T> s = b * g;
    return V4<T>(g, s.x, s.y, s.z);
}

// minkowski.rs:385-392.
template <class T> inline V4<T> boost_u1_u2(const V4<T>& v, const V4<T>& u1, const V4<T>& u2) {
    T denom = T(1) - u1.mdot(u2);
    V4<T> sum = u1 + u2;
    return v + sum * (sum.mdot(v) / denom) - u2 * (T(2) * u1.mdot(v));
}

// Tetrad (minkowski.rs:399-609).
template <class T> struct Tetrad {
    std::array<V4<T>, 4> e{V4<T>(1, 0, 0, 0), V4<T>(0, 1, 0, 0), V4<T>(0, 0, 1, 0), V4<T>(0, 0, 0, 1)};
    static Tetrad from_beta(const V3<T>& b) {
        Tetrad t;
        t.boost_to(four_velocity(b));
        return t;
    }
    void boost_to(const V4<T>& nu) {
        T ns = nu.mdot(nu);
        V4<T> u2(1, 0, 0, 0);
        if (ns < T(-1e-12)) u2 = nu * ((nu.t >= T(0) ? T(1) : T(-1)) * (T(1) / std::sqrt(-ns)));
        V4<T> u1 = e[0];
        e[0] = u2;
        for (int a = 1; a <= 3; ++a) e[a] = boost_u1_u2(e[a], u1, u2);
        reorthonormalize();
    }
    void boost_local(const V3<T>& d) {
        T eta = d.length();
        if (eta < T(1e-8)) return;
        V4<T> s = local_spatial_to_world(d / eta);
        boost_to(e[0] * std::cosh(eta) + s * std::sinh(eta));
    }
    void rotate_local(T yaw, T pitch, T roll) {
        auto rot = [](V4<T>& a, V4<T>& b, T ang) {
            T s = std::sin(ang), c = std::cos(ang);
            V4<T> a0 = a, b0 = b;
            a = a0 * c - b0 * s;
            b = a0 * s + b0 * c;
        };
        if (std::fabs(yaw) > T(1e-8)) rot(e[1], e[3], yaw);
        if (std::fabs(pitch) > T(1e-8)) rot(e[2], e[3], pitch);
        if (std::fabs(roll) > T(1e-8)) rot(e[1], e[2], roll);
        reorthonormalize();
    }
    V4<T> local_spatial_to_world(const V3<T>& l) const { return e[1] * l.x + e[2] * l.y + e[3] * l.z; }
    V3<T> world_to_local_spatial(const V4<T>& v) const { return V3<T>(v.mdot(e[1]), v.mdot(e[2]), v.mdot(e[3])); }
    void reorthonormalize() {
        T n0 = std::sqrt(mx(-e[0].mdot(e[0]), T(1e-12)));
        e[0] = e[0] * ((e[0].t >= T(0) ? T(1) : T(-1)) / n0);
        for (int a = 1; a <= 3; ++a) {
            V4<T> v = e[a];
            v += e[0] * v.mdot(e[0]);
            for (int b = 1; b < a; ++b) v -= e[b] * v.mdot(e[b]);
            e[a] = v * (T(1) / std::sqrt(mx(v.mdot(v), T(1e-12))));
        }
    }
};

}  // namespace srh
