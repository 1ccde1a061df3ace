// oracle_math.h - scalar FP32 vector/quaternion math of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This header belongs to the oracle, a CPU restatement of the Dynamis
// WGSL rigid-body step used by tests/ and bench.py's cpu_baseline leg as the checker. Nothing in
// the dynamis_b200 package includes or links it.
//
// Every operation restates a WGSL builtin or a crates/dynamis-shader/shaders/core.wgsl helper with
// the operand order written out, so the oracle's IEEE-754 binary32 results are fully determined:
//   * built with -ffp-contract=off (no fused multiply-add), no -ffast-math;
//   * dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z, length = sqrt(dot), normalize = v / length;
//   * sin / cos / atan2 follow S. L. Moshier's Cephes single-precision method (sinf.c, atanf.c of
//     the Cephes Math Library): Cody-Waite reduction by pi/4 in three parts, then the Cephes
//     minimax polynomials. WGSL leaves these builtins' rounding to the backend (naga 30.0.1 maps
//     them to the platform's sin/cos/atan2), so the reference pins no bit pattern for them; the
//     oracle fixes one, and tests compare it with libm within a few ulp.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

struct V3 {
    float x, y, z;
};
struct V4 {
    float x, y, z, w;
};

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 splat3(float s) { return V3{s, s, s}; }
inline V4 v4(float x, float y, float z, float w) { return V4{x, y, z, w}; }
inline V3 xyz(V4 q) { return V3{q.x, q.y, q.z}; }

inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, V3 b) { return V3{a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
inline V4 operator+(V4 a, V4 b) { return V4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline V4 operator-(V4 a, V4 b) { return V4{a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline V4 operator-(V4 a) { return V4{-a.x, -a.y, -a.z, -a.w}; }
inline V4 operator*(float s, V4 a) { return V4{s * a.x, s * a.y, s * a.z, s * a.w}; }
inline V4 operator*(V4 a, float s) { return V4{a.x * s, a.y * s, a.z * s, a.w * s}; }
inline V4 operator/(V4 a, float s) { return V4{a.x / s, a.y / s, a.z / s, a.w / s}; }

inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(V4 a, V4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline float length(V4 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { return a / length(a); }
inline V4 normalize(V4 a) { return a / length(a); }
inline float fminw(float a, float b) { return a < b ? a : b; }  // WGSL min on non-NaN input
inline float fmaxw(float a, float b) { return a > b ? a : b; }  // WGSL max on non-NaN input
inline float clampw(float x, float lo, float hi) { return fminw(fmaxw(x, lo), hi); }
inline V3 vabs(V3 a) { return V3{std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline V3 vmin(V3 a, V3 b) { return V3{fminw(a.x, b.x), fminw(a.y, b.y), fminw(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return V3{fmaxw(a.x, b.x), fmaxw(a.y, b.y), fmaxw(a.z, b.z)}; }
inline V3 vclamp(V3 x, V3 lo, V3 hi) { return vmin(vmax(x, lo), hi); }
inline float comp(V3 v, uint32_t i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
inline bool veq(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// ---- Cephes single-precision sin/cos (Moshier, Cephes Math Library, sinf.c) ----
constexpr float kFourOverPi = 1.27323954473516f;
constexpr float kDP1 = 0.78515625f;
constexpr float kDP2 = 2.4187564849853515625e-4f;
constexpr float kDP3 = 3.77489497744594108e-8f;

inline float cephes_sin_poly(float x, float z) {
    return ((-1.9515295891e-4f * z + 8.3321608736e-3f) * z - 1.6666654611e-1f) * z * x + x;
}
inline float cephes_cos_poly(float z) {
    return ((2.443315711809948e-5f * z - 1.388731625493765e-3f) * z + 4.166664568298827e-2f) * z * z
        - 0.5f * z + 1.0f;
}
inline float reduce_octant(float x, int* octant) {
    if (x > 8192.0f) {
        x = std::fmod(x, 6.28318530717958647692f);
    }
    int j = (int)(kFourOverPi * x);
    float y = (float)j;
    if (j & 1) {
        j += 1;
        y += 1.0f;
    }
    *octant = j & 7;
    return ((x - y * kDP1) - y * kDP2) - y * kDP3;
}
inline float osin(float value) {
    float x = value;
    int sign = 1;
    if (x < 0.0f) {
        sign = -1;
        x = -x;
    }
    int j = 0;
    x = reduce_octant(x, &j);
    if (j > 3) {
        sign = -sign;
        j -= 4;
    }
    float z = x * x;
    float y = (j == 1 || j == 2) ? cephes_cos_poly(z) : cephes_sin_poly(x, z);
    return sign < 0 ? -y : y;
}
inline float ocos(float value) {
    float x = std::fabs(value);
    int sign = 1;
    int j = 0;
    x = reduce_octant(x, &j);
    if (j > 3) {
        j -= 4;
        sign = -sign;
    }
    if (j > 1) {
        sign = -sign;
    }
    float z = x * x;
    float y = (j == 1 || j == 2) ? cephes_sin_poly(x, z) : cephes_cos_poly(z);
    return sign < 0 ? -y : y;
}

// ---- Cephes single-precision atan / atan2 (Moshier, atanf.c) ----
constexpr float kPi = 3.14159265358979323846f;
constexpr float kPiOver2 = 1.57079632679489661923f;
constexpr float kPiOver4 = 0.78539816339744830962f;

inline float oatan(float value) {
    float x = value;
    int sign = 1;
    if (x < 0.0f) {
        sign = -1;
        x = -x;
    }
    float y;
    if (x > 2.414213562373095f) {
        y = kPiOver2;
        x = -(1.0f / x);
    } else if (x > 0.4142135623730950f) {
        y = kPiOver4;
        x = (x - 1.0f) / (x + 1.0f);
    } else {
        y = 0.0f;
    }
    float z = x * x;
    y = y + ((((8.05374449538e-2f * z - 1.38776856032e-1f) * z + 1.99777106478e-1f) * z
                 - 3.33329491539e-1f) * z * x + x);
    return sign < 0 ? -y : y;
}
inline float oatan2(float y, float x) {
    if (x == 0.0f) {
        if (y > 0.0f) return kPiOver2;
        if (y < 0.0f) return -kPiOver2;
        return 0.0f;
    }
    if (y == 0.0f) {
        return x < 0.0f ? kPi : 0.0f;
    }
    float w = 0.0f;
    if (x < 0.0f) {
        w = y < 0.0f ? -kPi : kPi;
    }
    return w + oatan(y / x);
}
// acos(x) = atan2(sqrt((1 - x)(1 + x)), x) on [-1, 1]: the WGSL acos of quat_slerp / quat_angle
// (core.wgsl:149-168), resting on the same Cephes atan as the rest of the restatement.
inline float oacos(float x) { return oatan2(std::sqrt((1.0f - x) * (1.0f + x)), x); }

// ---- quaternions: crates/dynamis-shader/shaders/core.wgsl:132-178 ----
inline V4 quat_mul(V4 a, V4 b) {
    V3 av = xyz(a), bv = xyz(b);
    V3 v = a.w * bv + b.w * av + cross(av, bv);
    return V4{v.x, v.y, v.z, a.w * b.w - dot(av, bv)};
}
inline V4 quat_conjugate(V4 q) { return V4{-q.x, -q.y, -q.z, q.w}; }
inline V3 quat_rotate(V4 q, V3 v) {
    V3 u = xyz(q);
    float s = q.w;
    return 2.0f * dot(u, v) * u + (s * s - dot(u, u)) * v + 2.0f * s * cross(u, v);
}
inline V3 rotate_about(V3 rotation, V3 v) {
    float angle = length(rotation);
    if (angle < 1e-8f) {
        return v;
    }
    V3 axis = rotation / angle;
    V3 offset = cross(axis, v);
    return v + osin(angle) * offset + (1.0f - ocos(angle)) * cross(axis, offset);
}
inline V3 sign_normalize(V3 v) {
    float n = length(v);
    if (n > 1e-8f) {
        return v / n;
    }
    return V3{0.0f, 1.0f, 0.0f};
}

}  // namespace orc
