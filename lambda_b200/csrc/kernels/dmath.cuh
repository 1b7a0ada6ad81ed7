// Device float geometry, constants and the per-pixel PCG32 stream.
//
// Every kernel that shares results with the reference's CPU build is compiled
// with --fmad=false, and the helpers below evaluate in the reference's operand
// order (src/math/vector.h, src/core/utils.h), so ray and primitive arithmetic
// rounds exactly as the reference's SSE2 code does.
#pragma once

#include <cstdint>

#include "pcg32.h"

namespace lambda_dev {

constexpr float kEps = 1e-4f;               // constants.h:5
constexpr float kEpsSq = kEps * kEps;       // constants.h:6
constexpr float kPi = 3.14159265358979323846f;
constexpr float kMax = 1e30f;               // constants.h:16
constexpr int kHero = 4;                    // constants.h:12
constexpr int kRrStartDepth = 5;            // constants.h:14
constexpr int kStackDepth = 20;             // BVH_MAX_DEPTH, constants.h:10
constexpr int kCieBins = 471;

struct f3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return a * s; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length_sq(f3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__device__ __forceinline__ float length(f3 a) { return sqrtf(length_sq(a)); }
// 1 / x rounded to nearest: the same correctly rounded value as the IEEE division
// 1.0f / x, without the division routine.
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

__device__ __forceinline__ f3 normalize(f3 a) {
    const float l = length(a);
    return mk(a.x / l, a.y / l, a.z / l);
}
__device__ __forceinline__ float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// Four hero-wavelength samples (SampledSpectrum, spectrum.h:8-156).
struct s4 {
    float v[kHero];
};

__device__ __forceinline__ s4 s4_fill(float a) { return s4{{a, a, a, a}}; }
__device__ __forceinline__ s4 operator*(s4 a, s4 b) { return s4{{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}}; }
__device__ __forceinline__ s4 operator*(s4 a, float s) { return s4{{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}}; }
__device__ __forceinline__ s4 operator/(s4 a, float s) { return s4{{a.v[0] / s, a.v[1] / s, a.v[2] / s, a.v[3] / s}}; }
__device__ __forceinline__ s4 operator+(s4 a, s4 b) { return s4{{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}}; }
__device__ __forceinline__ float s4_max(s4 a) {
    float m = a.v[0];
    for (int i = 1; i < kHero; i++)
        if (a.v[i] > m) m = a.v[i];
    return m;
}
__device__ __forceinline__ float4 to_f4(s4 a) { return make_float4(a.v[0], a.v[1], a.v[2], a.v[3]); }
__device__ __forceinline__ s4 from_f4(float4 a) { return s4{{a.x, a.y, a.z, a.w}}; }

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

// MIS power heuristic (utils.h:67-72)
__device__ __forceinline__ float power_heuristic(float a, float b) {
    a *= a;
    b *= b;
    return a / (a + b);
}

// utils.h:74-87
__device__ __forceinline__ f3 reflected(f3 v, f3 n) { return v - 2 * dot(v, n) * n; }
__device__ __forceinline__ f3 refracted(f3 v, f3 n, float ratio) {
    const float vn = dot(v, n);
    const float root = 1 - ratio * ratio * (1 - vn * vn);
    if (root < 0) return v - 2 * vn * n;
    return ratio * v - (ratio * vn + sqrtf(root)) * n;
}

// Homogeneous transform with projective divide (utils.h:89-95). m is row-major.
__device__ __forceinline__ f3 xform(const float *m, f3 v, float w) {
    float den = m[12] * v.x + m[13] * v.y + m[14] * v.z + m[15] * w;
    if (fabsf(den) < kEps) den = 1;
    const f3 r = mk(m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3] * w, m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7] * w,
                    m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11] * w);
    if (den == 1.0f) return r;  // x / 1 is x exactly: affine transforms skip the divide
    return r / den;
}

// The same with the transpose of m (normals use transpose(inverse)).
__device__ __forceinline__ f3 xform_t(const float *m, f3 v, float w) {
    float den = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * w;
    if (fabsf(den) < kEps) den = 1;
    const f3 r = mk(m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * w, m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * w,
                    m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * w);
    if (den == 1.0f) return r;
    return r / den;
}

// Per-pixel PCG32 (random.h): the stream of pixel p has increment 2p+1.
// PCG32 of one pixel. Streams are pixel indices below 2^30, so the increment
// 2 * stream + 1 fits 32 bits and is widened only in the state update.
struct Rng {
    uint64_t state;
    uint32_t inc;
    __device__ __forceinline__ float next() { return lambda_rng::pcg_next_float(state, uint64_t(inc)); }
};

__device__ __forceinline__ Rng pixel_rng(uint64_t state, int stream) {
    return Rng{state, uint32_t(lambda_rng::pcg_increment(uint64_t(stream)))};
}

// randomUnitVector (utils.h:20-24). The reference's three draws are constructor
// arguments, which its compiler (GCC, x86-64) evaluates right to left: the first
// draw becomes z and the last x.
__device__ __forceinline__ f3 random_unit_vector(Rng &r) {
    const float z = r.next() * 2 - 1;
    const float y = r.next() * 2 - 1;
    const float x = r.next() * 2 - 1;
    return normalize(mk(x, y, z));
}

// Orthonormal frame around w used by both hemisphere and cone sampling (utils.h:38-44).
__device__ __forceinline__ f3 frame_dir(f3 n, float x, float y, float z) {
    const f3 w = normalize(n);
    f3 u = fabsf(w.x) > fabsf(w.y) ? mk(0, 0, 1) : mk(1, 0, 0);
    u = normalize(cross(u, w));
    const f3 v = cross(w, u);
    return x * u + y * v + z * w;
}

// randomInHemisphere (utils.h:26-45): cosine-weighted.
__device__ __forceinline__ f3 random_in_hemisphere(f3 n, Rng &r) {
    const float r1 = r.next();
    const float r2 = r.next();
    const float phi = 2 * kPi * r1;
    const float rad = sqrtf(r2);
    const float x = rad * cosf(phi);
    const float y = rad * sinf(phi);
    const float z = sqrtf(1 - r2);
    return frame_dir(n, x, y, z);
}

// randomInCone (utils.h:47-65)
__device__ __forceinline__ f3 random_in_cone(f3 n, float cos_max, Rng &r) {
    const float r1 = r.next();
    const float r2 = r.next();
    const float cos_t = 1 + r1 * (cos_max - 1);
    const float sin_t = sqrtf(1 - cos_t * cos_t);
    const float phi = 2 * kPi * r2;
    const float x = sin_t * cosf(phi);
    const float y = sin_t * sinf(phi);
    return frame_dir(n, x, y, cos_t);
}

}  // namespace lambda_dev
