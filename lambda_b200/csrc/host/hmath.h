// Host-side float geometry for scene construction (parser, BVH build, lights).
//
// The scene the kernels see must be the one the reference builds: the BVH split
// decisions, instance matrices, light powers and bounding sphere all come out of
// float arithmetic on the host. Every helper here therefore evaluates in the same
// order as the reference's Vector/Matrix4 code (src/math/vector.h,
// src/math/matrix.h, transform() in src/core/utils.h:89-95), left to right, with
// no fused multiply-add (this file is compiled with -ffp-contract=off).
#pragma once

#include <cmath>

namespace lambda_host {

constexpr float kEpsilon = 1e-4f;            // constants.h:5
constexpr float kPi = 3.14159265358979323846f;
constexpr float kMax = 1e30f;                // constants.h:16
constexpr int kBinCount = 16;                // constants.h:9
constexpr int kMaxDepth = 20;                // constants.h:10

struct V3 {
    float c[3];
    float operator[](int i) const { return c[i]; }
    float &operator[](int i) { return c[i]; }
};

inline V3 v3(float x, float y, float z) { return V3{{x, y, z}}; }
inline V3 operator+(const V3 &a, const V3 &b) { return v3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline V3 operator-(const V3 &a, const V3 &b) { return v3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline V3 operator*(const V3 &a, float s) { return v3(a[0] * s, a[1] * s, a[2] * s); }
inline V3 operator*(float s, const V3 &a) { return a * s; }
inline V3 operator/(const V3 &a, float s) { return v3(a[0] / s, a[1] / s, a[2] / s); }
inline float dot(const V3 &a, const V3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross(const V3 &a, const V3 &b) {
    return v3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
inline float length_sq(const V3 &a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
inline float length(const V3 &a) { return std::sqrt(length_sq(a)); }
inline V3 normalize(const V3 &a) {
    float l = length(a);
    return v3(a[0] / l, a[1] / l, a[2] / l);
}
inline V3 vmin(const V3 &a, const V3 &b) { return v3(std::fmin(a[0], b[0]), std::fmin(a[1], b[1]), std::fmin(a[2], b[2])); }
inline V3 vmax(const V3 &a, const V3 &b) { return v3(std::fmax(a[0], b[0]), std::fmax(a[1], b[1]), std::fmax(a[2], b[2])); }

// Row-major 4x4.
struct M4 {
    float m[16];
};

inline M4 mat_mul(const M4 &a, const M4 &b) {
    M4 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float s = a.m[i * 4] * b.m[j];
            s += a.m[i * 4 + 1] * b.m[4 + j];
            s += a.m[i * 4 + 2] * b.m[8 + j];
            s += a.m[i * 4 + 3] * b.m[12 + j];
            r.m[i * 4 + j] = s;
        }
    return r;
}

inline M4 mat_transpose(const M4 &a) {
    M4 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) r.m[i * 4 + j] = a.m[j * 4 + i];
    return r;
}

// First-row Laplace expansion (matrix.h:232).
inline float mat_det(const M4 &a) {
    const float *d = a.m;
    return d[0] * (d[5] * (d[10] * d[15] - d[11] * d[14]) - d[6] * (d[9] * d[15] - d[11] * d[13]) + d[7] * (d[9] * d[14] - d[10] * d[13])) -
           d[1] * (d[4] * (d[10] * d[15] - d[11] * d[14]) - d[6] * (d[8] * d[15] - d[11] * d[12]) + d[7] * (d[8] * d[14] - d[10] * d[12])) +
           d[2] * (d[4] * (d[9] * d[15] - d[11] * d[13]) - d[5] * (d[8] * d[15] - d[11] * d[12]) + d[7] * (d[8] * d[13] - d[9] * d[12])) -
           d[3] * (d[4] * (d[9] * d[14] - d[10] * d[13]) - d[5] * (d[8] * d[14] - d[10] * d[12]) + d[6] * (d[8] * d[13] - d[9] * d[12]));
}

// Inverse by 2x2 sub-determinants of the top (s) and bottom (c) row pairs,
// divided by the first-row expansion determinant (matrix.h:236-255).
inline M4 mat_inverse(const M4 &a) {
    const float *d = a.m;
    const float det = mat_det(a);
    const float s0 = d[0] * d[5] - d[1] * d[4], s1 = d[0] * d[6] - d[2] * d[4], s2 = d[0] * d[7] - d[3] * d[4];
    const float s3 = d[1] * d[6] - d[2] * d[5], s4 = d[1] * d[7] - d[3] * d[5], s5 = d[2] * d[7] - d[3] * d[6];
    const float c0 = d[8] * d[13] - d[9] * d[12], c1 = d[8] * d[14] - d[10] * d[12], c2 = d[8] * d[15] - d[11] * d[12];
    const float c3 = d[9] * d[14] - d[10] * d[13], c4 = d[9] * d[15] - d[11] * d[13], c5 = d[10] * d[15] - d[11] * d[14];
    M4 r;
    r.m[0] = (d[5] * c5 - d[6] * c4 + d[7] * c3) / det;
    r.m[1] = (-d[1] * c5 + d[2] * c4 - d[3] * c3) / det;
    r.m[2] = (d[13] * s5 - d[14] * s4 + d[15] * s3) / det;
    r.m[3] = (-d[9] * s5 + d[10] * s4 - d[11] * s3) / det;
    r.m[4] = (-d[4] * c5 + d[6] * c2 - d[7] * c1) / det;
    r.m[5] = (d[0] * c5 - d[2] * c2 + d[3] * c1) / det;
    r.m[6] = (-d[12] * s5 + d[14] * s2 - d[15] * s1) / det;
    r.m[7] = (d[8] * s5 - d[10] * s2 + d[11] * s1) / det;
    r.m[8] = (d[4] * c4 - d[5] * c2 + d[7] * c0) / det;
    r.m[9] = (-d[0] * c4 + d[1] * c2 - d[3] * c0) / det;
    r.m[10] = (d[12] * s4 - d[13] * s2 + d[15] * s0) / det;
    r.m[11] = (-d[8] * s4 + d[9] * s2 - d[11] * s0) / det;
    r.m[12] = (-d[4] * c3 + d[5] * c1 - d[6] * c0) / det;
    r.m[13] = (d[0] * c3 - d[1] * c1 + d[2] * c0) / det;
    r.m[14] = (-d[12] * s3 + d[13] * s1 - d[14] * s0) / det;
    r.m[15] = (d[8] * s3 - d[9] * s1 + d[10] * s0) / det;
    return r;
}

// Homogeneous transform with projective divide; w = 1 for points, 0 for vectors
// (utils.h:89-95).
inline V3 transform(const float *m, const V3 &v, float w) {
    float den = m[12] * v[0] + m[13] * v[1] + m[14] * v[2] + m[15] * w;
    if (std::fabs(den) < kEpsilon) den = 1;
    V3 r = v3(m[0] * v[0] + m[1] * v[1] + m[2] * v[2] + m[3] * w,
              m[4] * v[0] + m[5] * v[1] + m[6] * v[2] + m[7] * w,
              m[8] * v[0] + m[9] * v[1] + m[10] * v[2] + m[11] * w);
    return r / den;
}

}  // namespace lambda_host
