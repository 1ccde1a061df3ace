// dmath.cuh - FP32 vector, quaternion and transcendental helpers for the sm_100a step kernels.
//
// The WGSL step (crates/dynamis-shader/shaders/core.wgsl) is deterministic only up to its
// builtins; this header fixes every operation so that one body state always maps to one bit
// pattern, on the GPU and in any CPU restatement built with the same rules:
//   * the .cu files are compiled with -fmad=false -prec-div=true -prec-sqrt=true, so + - * / sqrt
//     are single IEEE-754 binary32 operations and nothing is fused;
//   * dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z, length = sqrt(dot), normalize = v / length;
//   * sin / cos / atan2 use S. L. Moshier's Cephes single-precision method (sinf.c, atanf.c):
//     Cody-Waite reduction by pi/4 in three parts and the Cephes minimax polynomials, evaluated
//     in plain float arithmetic. They are not CUDA's sinf/cosf/atan2f, whose rounding is the
//     backend's business.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define DYN_HD __host__ __device__ __forceinline__
#else
#define DYN_HD inline
#include <cmath>
#endif

namespace dyn {

struct f3 {
    float x, y, z;
};

DYN_HD f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
DYN_HD f3 s3(float s) { return f3{s, s, s}; }
DYN_HD f3 xyz(float4 q) { return f3{q.x, q.y, q.z}; }
DYN_HD float4 mk4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

DYN_HD f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
DYN_HD f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
DYN_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
DYN_HD f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
DYN_HD f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
DYN_HD f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
DYN_HD f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
DYN_HD float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
DYN_HD float4 scale4(float s, float4 a) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }

DYN_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DYN_HD float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
DYN_HD f3 cross(f3 a, f3 b) { return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
DYN_HD float length(f3 a) { return sqrtf(dot(a, a)); }
DYN_HD f3 normalize(f3 a) { return a / length(a); }
DYN_HD float4 normalize4(float4 q) {
    float n = sqrtf(dot4(q, q));
    return make_float4(q.x / n, q.y / n, q.z / n, q.w / n);
}
// WGSL min/max/clamp on ordinary (non-NaN) values.
DYN_HD float wmin(float a, float b) { return a < b ? a : b; }
DYN_HD float wmax(float a, float b) { return a > b ? a : b; }
DYN_HD float wclamp(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
DYN_HD f3 vabs(f3 a) { return f3{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
DYN_HD f3 vmin(f3 a, f3 b) { return f3{wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z)}; }
DYN_HD f3 vmax(f3 a, f3 b) { return f3{wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z)}; }
DYN_HD f3 vclamp(f3 x, f3 lo, f3 hi) { return vmin(vmax(x, lo), hi); }
DYN_HD float comp(f3 v, uint32_t i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
DYN_HD bool veq(f3 a, f3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
DYN_HD bool is_zero3(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

DYN_HD uint32_t fbits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    return u;
#endif
}
DYN_HD float bitsf(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

// ---- Cephes single-precision sin / cos (Moshier, sinf.c) ----
DYN_HD float cephes_sin_poly(float x, float z) {
    return ((-1.9515295891e-4f * z + 8.3321608736e-3f) * z - 1.6666654611e-1f) * z * x + x;
}
DYN_HD float cephes_cos_poly(float z) {
    return ((2.443315711809948e-5f * z - 1.388731625493765e-3f) * z + 4.166664568298827e-2f) * z * z
        - 0.5f * z + 1.0f;
}
DYN_HD float cephes_reduce(float x, int* octant) {
    if (x > 8192.0f) {
        x = fmodf(x, 6.28318530717958647692f);
    }
    int j = (int)(1.27323954473516f * x);
    float y = (float)j;
    if (j & 1) {
        j += 1;
        y += 1.0f;
    }
    *octant = j & 7;
    return ((x - y * 0.78515625f) - y * 2.4187564849853515625e-4f) - y * 3.77489497744594108e-8f;
}
DYN_HD float dsin(float value) {
    float x = value;
    int sign = 1;
    if (x < 0.0f) {
        sign = -1;
        x = -x;
    }
    int j = 0;
    x = cephes_reduce(x, &j);
    if (j > 3) {
        sign = -sign;
        j -= 4;
    }
    float z = x * x;
    float y = (j == 1 || j == 2) ? cephes_cos_poly(z) : cephes_sin_poly(x, z);
    return sign < 0 ? -y : y;
}
DYN_HD float dcos(float value) {
    float x = fabsf(value);
    int sign = 1;
    int j = 0;
    x = cephes_reduce(x, &j);
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
DYN_HD float datan(float value) {
    float x = value;
    int sign = 1;
    if (x < 0.0f) {
        sign = -1;
        x = -x;
    }
    float y;
    if (x > 2.414213562373095f) {
        y = 1.57079632679489661923f;
        x = -(1.0f / x);
    } else if (x > 0.4142135623730950f) {
        y = 0.78539816339744830962f;
        x = (x - 1.0f) / (x + 1.0f);
    } else {
        y = 0.0f;
    }
    float z = x * x;
    y = y + ((((8.05374449538e-2f * z - 1.38776856032e-1f) * z + 1.99777106478e-1f) * z - 3.33329491539e-1f) * z * x + x);
    return sign < 0 ? -y : y;
}
DYN_HD float datan2(float y, float x) {
    if (x == 0.0f) {
        if (y > 0.0f) return 1.57079632679489661923f;
        if (y < 0.0f) return -1.57079632679489661923f;
        return 0.0f;
    }
    if (y == 0.0f) {
        return x < 0.0f ? 3.14159265358979323846f : 0.0f;
    }
    float w = 0.0f;
    if (x < 0.0f) {
        w = y < 0.0f ? -3.14159265358979323846f : 3.14159265358979323846f;
    }
    return w + datan(y / x);
}
// acos through the identity acos(x) = atan2(sqrt((1 - x)(1 + x)), x) on [-1, 1], so that it rests on
// the same Cephes atan as the rest of the step.
DYN_HD float dacos(float value) { return datan2(sqrtf((1.0f - value) * (1.0f + value)), value); }

// ---- quaternions (xyz = vector part, w = scalar) ----
DYN_HD float4 quat_mul(float4 a, float4 b) {
    f3 av = xyz(a), bv = xyz(b);
    f3 v = a.w * bv + b.w * av + cross(av, bv);
    return make_float4(v.x, v.y, v.z, a.w * b.w - dot(av, bv));
}
DYN_HD float4 quat_conj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
DYN_HD f3 quat_rotate(float4 q, f3 v) {
    f3 u = xyz(q);
    float s = q.w;
    return 2.0f * dot(u, v) * u + (s * s - dot(u, u)) * v + 2.0f * s * cross(u, v);
}
DYN_HD f3 rotate_about(f3 rotation, f3 v) {
    float angle = length(rotation);
    if (angle < 1e-8f) {
        return v;
    }
    f3 axis = rotation / angle;
    f3 offset = cross(axis, v);
    return v + dsin(angle) * offset + (1.0f - dcos(angle)) * cross(axis, offset);
}
DYN_HD f3 sign_normalize(f3 v) {
    float n = length(v);
    if (n > 1e-8f) {
        return v / n;
    }
    return f3{0.0f, 1.0f, 0.0f};
}
// Symmetric 3x3 tensor stored (xx, xy, xz, yy, yz, zz) applied to v.
DYN_HD f3 sym_apply(float4 t0, float2 t1, f3 v) {
    return f3{t0.x * v.x + t0.y * v.y + t0.z * v.z, t0.y * v.x + t0.w * v.y + t1.x * v.z,
              t0.z * v.x + t1.x * v.y + t1.y * v.z};
}

}  // namespace dyn
