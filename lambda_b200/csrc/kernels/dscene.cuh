// Device scene: layouts in HBM and the functions the render loop calls on them.
//
// Layouts (all read-only during a render; uploaded once per scene):
//   nodes      float4[2n]   (min.xyz, index)  (max.xyz, count); index/count are int bits
//   prims      float4[4m]   p0 = (corner or centre .xyz, type), p1 = (horizontal.xyz or
//                           radius, material), p2 = (vertical.xyz, 0), p3 = (normal.xyz, 0)
//   tri_attr   float4[4m]   (n0.xyz, n1.x) (n1.yz, n2.xy) (n2.z, u0, u1, u2) (v0, v1, v2, 0)
//   instances  float4[9k]   (object, count, node, material as int bits), M rows, M^-1 rows
//   spectra    float[s][471] plus a per-spectrum "all bins equal" flag
//   cspectra   double2[c][471] (complex refractive indices)
// Functions follow the reference's object.h, instance.h, scene.h, texture.h,
// background.h and material.h, in its operand order (see dmath.cuh).
#pragma once

#include <climits>

#include <cstdint>

#include "dmath.cuh"
#include "dtypes.cuh"

namespace lambda_dev {


// ---------------------------------------------------------------------------
// Spectra (DenseSpectrum::operator(), spectrum.h:176-188): linear interpolation
// on the 1 nm grid with the index held in double, result rounded to float.
// ---------------------------------------------------------------------------

__device__ __forceinline__ float spectrum_at(const DeviceScene &s, int k, float lambda) {
    const float *d = s.spectra + size_t(k) * kCieBins;
    if (s.spectrum_flat[k]) return d[0];  // all bins equal: interpolation returns the bin value exactly
    const double index = double(lambda - 360.0f);
    const int lo = int(index);
    if (lo == kCieBins - 1) return d[lo];
    const int hi = lo + 1;
    return float((double(hi) - index) * double(d[lo]) + (index - double(lo)) * double(d[hi]));
}

__device__ __forceinline__ double2 cspectrum_at(const DeviceScene &s, int k, float lambda) {
    const double2 *d = s.cspectra + size_t(k) * kCieBins;
    if (s.cspectrum_flat[k]) return d[0];
    const double index = double(lambda - 360.0f);
    const int lo = int(index);
    if (lo == kCieBins - 1) return d[lo];
    const int hi = lo + 1;
    const double a = double(hi) - index, b = index - double(lo);
    return make_double2(a * d[lo].x + b * d[hi].x, a * d[lo].y + b * d[hi].y);
}

// ---------------------------------------------------------------------------
// Noise (utils.h:97-171)
// ---------------------------------------------------------------------------

__device__ __forceinline__ int perm_at(const DeviceScene &s, int i) { return s.perm[i & 255]; }

// t^5-style fade t^3 (t (6t - 15) + 10). The reference takes t^3 from powf; the
// cube is formed exactly in double (t^2 has 48 significant bits) and rounded once.
__device__ __forceinline__ float fade(float t) {
    const double t2 = double(t) * double(t);
    const float cube = float(t2 * double(t));
    return cube * (t * (6 * t - 15) + 10);
}

__device__ __forceinline__ float grad(int hash, float x, float y, float z) {
    switch (hash % 12) {
        case 0: return x + y;
        case 1: return -x + y;
        case 2: return x - y;
        case 3: return -x - y;
        case 4: return x + z;
        case 5: return -x + z;
        case 6: return x - z;
        case 7: return -x - z;
        case 8: return y + z;
        case 9: return -y + z;
        case 10: return y - z;
        case 11: return -y - z;
        default: return 0;
    }
}

__device__ __forceinline__ float lerp(float a, float b, float x) { return a + x * (b - a); }

// Improved noise mapped to [0, 1] (utils.h:123-148).
__device__ inline float perlin_noise(const DeviceScene &s, f3 p) {
    const float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
    const int i = int(fx) & 255, j = int(fy) & 255, k = int(fz) & 255;
    const float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
    const float u = fade(tx), v = fade(ty), w = fade(tz);
    const int pi0 = perm_at(s, i), pi1 = perm_at(s, i + 1);
    const int a0 = perm_at(s, pi0 + j), a1 = perm_at(s, pi0 + j + 1);
    const int b0 = perm_at(s, pi1 + j), b1 = perm_at(s, pi1 + j + 1);
    const int aaa = perm_at(s, a0 + k), aba = perm_at(s, a1 + k), aab = perm_at(s, a0 + k + 1), abb = perm_at(s, a1 + k + 1);
    const int baa = perm_at(s, b0 + k), bba = perm_at(s, b1 + k), bab = perm_at(s, b0 + k + 1), bbb = perm_at(s, b1 + k + 1);
    float x1 = lerp(grad(aaa, tx, ty, tz), grad(baa, tx - 1, ty, tz), u);
    float x2 = lerp(grad(aba, tx, ty - 1, tz), grad(bba, tx - 1, ty - 1, tz), u);
    const float y1 = lerp(x1, x2, v);
    x1 = lerp(grad(aab, tx, ty, tz - 1), grad(bab, tx - 1, ty, tz - 1), u);
    x2 = lerp(grad(abb, tx, ty - 1, tz - 1), grad(bbb, tx - 1, ty - 1, tz - 1), u);
    const float y2 = lerp(x1, x2, v);
    return (lerp(y1, y2, w) + 1) / 2;
}

__device__ __forceinline__ float fract(float x) { return x - floorf(x); }

// Feature offset of one Worley lattice cell: fract(sin(cell . k) * 43758.5453)
// per axis (utils.h:165). Cells inside the scene's table were evaluated on the host
// with the C library's sinf at upload; others are computed here, with the sine
// taken in double and rounded to float.
__device__ __forceinline__ f3 worley_feature(const DeviceScene &s, int cx, int cy, int cz) {
    const int ix = cx - s.worley_lo.x, iy = cy - s.worley_lo.y, iz = cz - s.worley_lo.z;
    if (unsigned(ix) < unsigned(s.worley_dim.x) && unsigned(iy) < unsigned(s.worley_dim.y) &&
        unsigned(iz) < unsigned(s.worley_dim.z)) {
        const float4 h = __ldg(&s.worley_cells[(size_t(iz) * s.worley_dim.y + iy) * s.worley_dim.x + ix]);
        return mk(h.x, h.y, h.z);
    }
    const f3 c = mk(float(cx), float(cy), float(cz));
    const float a = dot(c, mk(127.1f, 311.7f, 74.7f));
    const float b = dot(c, mk(269.5f, 183.3f, 246.1f));
    const float d = dot(c, mk(113.5f, 271.9f, 124.6f));
    return mk(fract(float(sin(double(a))) * 43758.5453f), fract(float(sin(double(b))) * 43758.5453f),
              fract(float(sin(double(d))) * 43758.5453f));
}

// F1 Worley distance over the 27 neighbouring cells (utils.h:154-171). Results
// equal the reference's:
// - The minimum does not depend on visit order, so cells are visited nearest
//   first. A cell is skipped when every point of its box [c, c+1]^3 (where its
//   feature lies) is farther than the best so far, with a relative margin that
//   covers float rounding.
// - sqrtf is correctly rounded and monotone, so the minimum of the distances is
//   the square root of the minimum squared distance: one sqrtf at the end.
// - When the whole 3x3x3 neighbourhood lies inside the host-built feature table,
//   cells are read from it at offsets from one base, without per-cell range checks.
// Neighbour offsets ordered by |xo| + |yo| + |zo|, packed as (xo+1) | (yo+1) << 2 | (zo+1) << 4.
__constant__ unsigned char kWorleyOrder[27] = {0x15, 0x14, 0x16, 0x11, 0x19, 0x05, 0x25, 0x10, 0x18,
                                               0x12, 0x1a, 0x04, 0x24, 0x06, 0x26, 0x01, 0x21, 0x09,
                                               0x29, 0x00, 0x20, 0x08, 0x28, 0x02, 0x22, 0x0a, 0x2a};

__device__ inline float worley_noise(const DeviceScene &s, f3 p) {
    const int xi = int(floorf(p.x)), yi = int(floorf(p.y)), zi = int(floorf(p.z));
    const float fx = p.x - float(xi), fy = p.y - float(yi), fz = p.z - float(zi);
    const int dx = s.worley_dim.x, dxy = s.worley_dim.x * s.worley_dim.y;
    const int ix = xi - 1 - s.worley_lo.x, iy = yi - 1 - s.worley_lo.y, iz = zi - 1 - s.worley_lo.z;
    const bool inside = ix >= 0 && iy >= 0 && iz >= 0 && ix + 2 < s.worley_dim.x && iy + 2 < s.worley_dim.y &&
                        iz + 2 < s.worley_dim.z;
    float d2 = 0;
    if (inside) {
        // The walk unrolled, in rounds of independent loads instead of a chain: the
        // centre and its six face neighbours unconditionally, then the 20 edge and
        // corner cells four at a time, each group's cells tested against the minimum
        // before the group and loaded together. Each cell's offsets, and so its gaps,
        // are constants; the squared gaps per axis and side are formed once. A cell is
        // skipped only when its box is farther (with the margin) than a distance
        // already found, which never skips the nearest feature, so the minimum is the
        // one the sequential walk below finds.
        constexpr unsigned char kOrder[27] = {0x15, 0x14, 0x16, 0x11, 0x19, 0x05, 0x25, 0x10, 0x18,
                                              0x12, 0x1a, 0x04, 0x24, 0x06, 0x26, 0x01, 0x21, 0x09,
                                              0x29, 0x00, 0x20, 0x08, 0x28, 0x02, 0x22, 0x0a, 0x2a};
        const float4 *block = s.worley_cells + (size_t(iz) * dxy + size_t(iy) * dx + ix);
        const float gxx[3] = {fx * fx, 0.0f, (1 - fx) * (1 - fx)};
        const float gyy[3] = {fy * fy, 0.0f, (1 - fy) * (1 - fy)};
        const float gzz[3] = {fz * fz, 0.0f, (1 - fz) * (1 - fz)};
        auto cell_d2 = [&](int c, const float4 &h) {
            const int ox = kOrder[c] & 3, oy = (kOrder[c] >> 2) & 3, oz = (kOrder[c] >> 4) & 3;
            const f3 feature = mk(h.x, h.y, h.z) + mk(float(xi + ox - 1), float(yi + oy - 1), float(zi + oz - 1));
            return length_sq(p - feature);
        };
        auto cell_at = [&](int c) {
            const int ox = kOrder[c] & 3, oy = (kOrder[c] >> 2) & 3, oz = (kOrder[c] >> 4) & 3;
            return block + (oz * dxy + oy * dx + ox);
        };
        float4 h1[7];
#pragma unroll
        for (int c = 0; c < 7; c++) h1[c] = __ldg(cell_at(c));
        d2 = cell_d2(0, h1[0]);
#pragma unroll
        for (int c = 1; c < 7; c++) d2 = fminf(d2, cell_d2(c, h1[c]));
#pragma unroll
        for (int c0 = 7; c0 < 27; c0 += 4) {
            const float reach = d2 * 1.0001f + 1e-6f;
            float4 h[4];
            bool near[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int c = c0 + k;
                near[k] = !(gxx[kOrder[c] & 3] + gyy[(kOrder[c] >> 2) & 3] + gzz[(kOrder[c] >> 4) & 3] > reach);
                h[k] = near[k] ? __ldg(cell_at(c)) : make_float4(0, 0, 0, 0);
            }
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (near[k]) d2 = fminf(d2, cell_d2(c0 + k, h[k]));
        }
        return fminf(9999.0f, sqrtf(d2));
    }
#pragma unroll 1
    for (int c = 0; c < 27; c++) {
        const int code = kWorleyOrder[c];
        const int xo = (code & 3) - 1, yo = ((code >> 2) & 3) - 1, zo = ((code >> 4) & 3) - 1;
        if (c > 0) {
            const float gx = xo < 0 ? fx : (xo > 0 ? 1 - fx : 0);
            const float gy = yo < 0 ? fy : (yo > 0 ? 1 - fy : 0);
            const float gz = zo < 0 ? fz : (zo > 0 ? 1 - fz : 0);
            const float lb2 = gx * gx + gy * gy + gz * gz;
            if (lb2 > d2 * 1.0001f + 1e-6f) continue;
        }
        const f3 off = worley_feature(s, xi + xo, yi + yo, zi + zo);
        const f3 feature = off + mk(float(xi + xo), float(yi + yo), float(zi + zo));
        const float e2 = length_sq(p - feature);
        d2 = c == 0 ? e2 : fminf(d2, e2);
    }
    return fminf(9999.0f, sqrtf(d2));
}

// ---------------------------------------------------------------------------
// Textures (texture.h)
// ---------------------------------------------------------------------------

struct ShadePoint {
    f3 point;
    float u, v;
};

__device__ __forceinline__ float scalar_texture(const DeviceScene &s, int t, f3 p) {
    const float4 x = __ldg(&s.scalar_tex[t]);
    const int type = __float_as_int(x.x);
    if (type == 0) return x.y;                                            // constant
    if (type == 1) return x.y + (x.z - x.y) * perlin_noise(s, p * x.w);   // perlin
    return x.y + (x.z - x.y) * worley_noise(s, p * x.w);                  // worley
}

__device__ __forceinline__ float spectrum_texture(const DeviceScene &s, int t, const ShadePoint &sp, float lambda) {
    const int4 x = __ldg(&s.spectrum_tex[t]);
    if (x.x == 0) return spectrum_at(s, x.y, lambda);
    if (x.x == 1) {
        const float scale = __int_as_float(x.w);
        const int cx = int(floorf(sp.u / scale));
        const int cy = int(floorf(sp.v / scale));
        return (cx + cy) % 2 == 0 ? spectrum_at(s, x.y, lambda) : spectrum_at(s, x.z, lambda);
    }
    return scalar_texture(s, x.y, sp.point);
}

// A spectrum texture at the four hero wavelengths; a texture that does not
// depend on the wavelength (scalar) is evaluated once.
__device__ __forceinline__ s4 spectrum_texture4(const DeviceScene &s, int t, const ShadePoint &sp, const s4 &lam) {
    const int4 x = __ldg(&s.spectrum_tex[t]);
    if (x.x == 2) return s4_fill(scalar_texture(s, x.y, sp.point));
    s4 r;
    for (int k = 0; k < kHero; k++) r.v[k] = spectrum_texture(s, t, sp, lam.v[k]);
    return r;
}

// Background::evaluate (background.h:81-95): equirectangular lookup of direction d.
__device__ __forceinline__ s4 background_eval(const DeviceScene &s, f3 d, const s4 &lam) {
    ShadePoint sp;
    sp.point = d;
    sp.u = (atan2f(d.z, d.x) + kPi) / (2 * kPi);
    sp.v = acosf(d.y) / kPi;
    return spectrum_texture4(s, s.background_texture, sp, lam);
}

// ---------------------------------------------------------------------------
// Geometry: BVH node slab test and primitive intersection (bvh.h:30-52,
// object.h:301-400). Traversal only needs t; attributes of the winning
// primitive are computed once at the end with the same arithmetic.
// ---------------------------------------------------------------------------

struct Ray3 {
    f3 o, d, inv;
};

__device__ __forceinline__ Ray3 make_ray(f3 o, f3 d) { return Ray3{o, d, mk(rcp(d.x), rcp(d.y), rcp(d.z))}; }

__device__ __forceinline__ bool slab(float4 lo, float4 hi, const Ray3 &r, float &t_entry) {
    float t1 = 0, t2 = kMax;
    {
        float a = (lo.x - r.o.x) * r.inv.x, b = (hi.x - r.o.x) * r.inv.x;
        if (r.inv.x < 0) { const float t = a; a = b; b = t; }
        t1 = fmaxf(a, t1);
        t2 = fminf(b, t2);
    }
    {
        float a = (lo.y - r.o.y) * r.inv.y, b = (hi.y - r.o.y) * r.inv.y;
        if (r.inv.y < 0) { const float t = a; a = b; b = t; }
        t1 = fmaxf(a, t1);
        t2 = fminf(b, t2);
    }
    {
        float a = (lo.z - r.o.z) * r.inv.z, b = (hi.z - r.o.z) * r.inv.z;
        if (r.inv.z < 0) { const float t = a; a = b; b = t; }
        t1 = fmaxf(a, t1);
        t2 = fminf(b, t2);
    }
    t_entry = t1;
    return t1 <= t2 && t2 >= 0;
}

struct Prim {
    float4 p0, p1, p2, p3;
};

__device__ __forceinline__ Prim load_prim(const DeviceScene &s, int i) {
    const float4 *p = s.prims + 4 * size_t(i);
    return Prim{__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)};
}

__device__ __forceinline__ int prim_type(const Prim &p) { return __float_as_int(p.p0.w); }
__device__ __forceinline__ int prim_material(const Prim &p) { return __float_as_int(p.p1.w); }

// t of the first intersection beyond EPSILON that is closer than `best`, else -1.
__device__ __forceinline__ float intersect_t(const Prim &p, const Ray3 &r, float best) {
    const int type = prim_type(p);
    if (type == 0) {  // sphere
        const f3 c = mk(p.p0.x, p.p0.y, p.p0.z);
        const float rad = p.p1.x;
        const f3 oc = r.o - c;
        const float a = length_sq(r.d);
        const float b = 2 * dot(r.d, oc);
        const float cc = dot(oc, oc) - rad * rad;
        float disc = b * b - 4 * a * cc;
        if (disc < 0) return -1;
        disc = sqrtf(disc);
        const float t1 = (-b - disc) / (2 * a);
        const float t2 = (-b + disc) / (2 * a);
        if (t1 < kEps && t2 < kEps) return -1;
        const float t = (t1 < kEps) ? t2 : t1;
        return t >= best ? -1 : t;
    }
    const f3 corner = mk(p.p0.x, p.p0.y, p.p0.z);
    const f3 h = mk(p.p1.x, p.p1.y, p.p1.z);
    const f3 v = mk(p.p2.x, p.p2.y, p.p2.z);
    if (type == 1) {  // quad
        const f3 nn = mk(p.p3.x, p.p3.y, p.p3.z);
        const f3 n = normalize(nn);
        const float den = dot(n, r.d);
        if (fabsf(den) < kEps) return -1;
        const float t = dot(n, corner - r.o) / den;
        if (t < kEps || t >= best) return -1;
        const f3 point = r.o + t * r.d;
        const f3 proj = point - corner;
        const float nsq = length_sq(nn);
        const float alpha = dot(nn, cross(proj, v)) / nsq;
        const float beta = dot(nn, cross(h, proj)) / nsq;
        if (alpha < 0 || alpha > 1 || beta < 0 || beta > 1) return -1;
        return t;
    }
    // triangle
    const f3 rcv = cross(r.d, v);
    const float det = dot(h, rcv);
    if (fabsf(det) < kEpsSq) return -1;
    const float inv = rcp(det);
    const f3 oc = r.o - corner;
    const float alpha = inv * dot(oc, rcv);
    if (alpha < 0 || alpha > 1) return -1;
    const f3 och = cross(oc, h);
    const float beta = inv * dot(r.d, och);
    if (beta < 0 || alpha + beta > 1) return -1;
    const float t = inv * dot(v, och);
    if (t < kEps || t >= best) return -1;
    return t;
}

struct Hit {
    float t;
    int instance;
    int object;
    f3 point;
    f3 normal;
    float u, v;
    bool front;
};

struct InstanceRef {
    const float4 *base;
    __device__ __forceinline__ int4 header() const {
        const float4 h = __ldg(base);
        return make_int4(__float_as_int(h.x), __float_as_int(h.y), __float_as_int(h.z), __float_as_int(h.w));
    }
    __device__ __forceinline__ void load_m(float *m, int which) const {
        const float4 *p = base + 1 + 4 * which;
        for (int r = 0; r < 4; r++) {
            const float4 q = __ldg(p + r);
            m[4 * r] = q.x;
            m[4 * r + 1] = q.y;
            m[4 * r + 2] = q.z;
            m[4 * r + 3] = q.w;
        }
    }
};

__device__ __forceinline__ InstanceRef instance_ref(const DeviceScene &s, int i) { return InstanceRef{s.instances + 9 * size_t(i)}; }

// Full attributes of a hit on primitive p in instance space (object.h:301-400). A
// sphere's (u, v) takes an atan2 and an acos; without want_uv (its material reads
// no (u, v)) they are left 0.
__device__ __forceinline__ void prim_attributes(const DeviceScene &s, int obj, const Prim &p, f3 o, f3 d, float t, Hit &h,
                                                bool want_uv = true) {
    const int type = prim_type(p);
    h.t = t;
    h.point = o + t * d;
    if (type == 0) {
        const f3 c = mk(p.p0.x, p.p0.y, p.p0.z);
        h.normal = normalize(h.point - c);
        h.u = want_uv ? (atan2f(-h.normal.z, h.normal.x) + kPi) / (2 * kPi) : 0.0f;
        h.v = want_uv ? acosf(-h.normal.y) / kPi : 0.0f;
        h.front = dot(d, h.normal) < 0;
        if (!h.front) h.normal = h.normal * -1.0f;
        return;
    }
    const f3 corner = mk(p.p0.x, p.p0.y, p.p0.z);
    const f3 hz = mk(p.p1.x, p.p1.y, p.p1.z);
    const f3 v = mk(p.p2.x, p.p2.y, p.p2.z);
    const f3 nn = mk(p.p3.x, p.p3.y, p.p3.z);
    if (type == 1) {
        const f3 proj = h.point - corner;
        const float nsq = length_sq(nn);
        h.u = dot(nn, cross(proj, v)) / nsq;
        h.v = dot(nn, cross(hz, proj)) / nsq;
        h.normal = normalize(nn);
        h.front = dot(d, h.normal) < 0;
        if (!h.front) h.normal = h.normal * -1.0f;
        return;
    }
    const f3 rcv = cross(d, v);
    const float det = dot(hz, rcv);
    const float inv = rcp(det);
    const f3 oc = o - corner;
    const float alpha = inv * dot(oc, rcv);
    const f3 och = cross(oc, hz);
    const float beta = inv * dot(d, och);
    const float4 *ta = s.tri_attr + 4 * size_t(obj);
    const float4 a0 = __ldg(ta), a1 = __ldg(ta + 1), a2 = __ldg(ta + 2), a3 = __ldg(ta + 3);
    const f3 n0 = mk(a0.x, a0.y, a0.z), n1 = mk(a0.w, a1.x, a1.y), n2 = mk(a1.z, a1.w, a2.x);
    const float w0 = 1 - alpha - beta;
    h.normal = normalize(w0 * n0 + alpha * n1 + beta * n2);
    h.u = w0 * a2.y + alpha * a2.z + beta * a2.w;
    h.v = w0 * a3.x + alpha * a3.y + beta * a3.z;
    h.front = dot(d, nn) < 0;
    if (!h.front) h.normal = h.normal * -1.0f;
}

// Traversal stack of one thread in shared memory, entry-major (entry i of thread t
// at base[i * stride + t], so a warp's pushes and pops hit 32 different banks). An
// entry is a wide-BVH code and the entry distance of its box. The capacity is the
// most entries the scene's trees can need (computed when the scene is uploaded).
struct WideStack {
    int *code;
    float *te;
    int stride;
    int cap;
    __device__ __forceinline__ void put(int i, int c, float t) const {
        code[i * stride] = c;
        te[i * stride] = t;
    }
};

// World ray wr -> instance space (instance.h:50-52), given the instance's flags. An
// identity instance's transform reduces exactly to adding +0 (which only turns -0
// into +0), so it is done that way; when no direction component is zero the
// direction, and so its reciprocals, are the world ray's.
__device__ __forceinline__ Ray3 to_local(uint32_t flags, const InstanceRef &ir, const Ray3 &wr) {
    const f3 zero = mk(0.0f, 0.0f, 0.0f);
    if (flags & 1u) {
        if (wr.d.x != 0.0f && wr.d.y != 0.0f && wr.d.z != 0.0f) return Ray3{wr.o + zero, wr.d, wr.inv};
        return make_ray(wr.o + zero, wr.d + zero);
    }
    float mi[16];
    ir.load_m(mi, 1);
    return make_ray(xform(mi, wr.o, 1), xform(mi, wr.d, 0));
}

// Instance space -> world for a hit (instance.h:42, :48).
__device__ __forceinline__ void to_world(const DeviceScene &s, int inst, const InstanceRef &ir, Hit &h) {
    if (s.instance_flags[inst] & 1u) {
        h.normal = normalize(h.normal + mk(0.0f, 0.0f, 0.0f));
        h.point = h.point + mk(0.0f, 0.0f, 0.0f);
        return;
    }
    float m[16];
    ir.load_m(m, 1);
    h.normal = normalize(xform_t(m, h.normal, 0));
    ir.load_m(m, 0);
    h.point = xform(m, h.point, 1);
}

// BVH layout, the template parameter L of the traversal code: the wide width (2, 4
// or 8), plus kCompressed for the compressed node records (wide_bvh.h). With the
// exact records a stack entry is (code, entry distance); with the compressed ones a
// child's entry is (its record slot w * width + i, its quantized entry distance),
// tested on its exact record when popped, and a root's entry carries its code
// (root_entry). Both visit the same nodes in the same order (wide_bvh.h).
constexpr int kCompressed = 16;
template <int L>
constexpr int kWidthOf = L & 15;
template <int L>
constexpr bool kQuantOf = (L & kCompressed) != 0;
template <int L>
constexpr int kQuantWords = 1 + (6 * kWidthOf<L> + 15) / 16;

// The stack entry of a tree root (or a BLAS root) whose box test was done exactly.
template <int L>
__device__ __forceinline__ int root_entry(const DeviceScene &s, int code) {
    if constexpr (kQuantOf<L>) return -1 - (code + s.num_leaves);
    else return code;
}

// The code of a popped entry (v, te) under ray r, or INT_MIN when it is culled: its
// distance is beyond `best`, or (compressed layout) the child's exact box is missed
// or entered beyond `best`; te becomes the exact entry distance.
template <int L>
__device__ __forceinline__ int pop_code(const DeviceScene &s, int v, float &te, const Ray3 &r, float best) {
    if (te > best) return INT_MIN;
    if constexpr (!kQuantOf<L>) {
        return v;
    } else {
        if (v < 0) return -1 - v - s.num_leaves;
        const float4 lo = __ldg(s.wide + 2 * size_t(v)), hi = __ldg(s.wide + 2 * size_t(v) + 1);
        if (!slab(lo, hi, r, te) || te > best) return INT_MIN;
        return __float_as_int(lo.w);
    }
}

// One byte of a compressed node's child bytes (words 1.. of its record).
template <int N>
__device__ __forceinline__ float qbyte(const uint32_t (&b)[N], int i) {
    return float((b[i >> 2] >> (8 * (i & 3))) & 0xFFu);
}

// Expands wide node w: tests its children (wide_bvh.h) against ray r and pushes
// the ones whose box the ray enters no farther than `best`, last-visited first, with
// their entry distances. Returns the new stack size; sets `overflow` (and stops)
// if the stack is full, which the stack sizes computed for the scene rule out.
// Compressed layout: the children's quantized boxes decode as o + q * s in FP32
// (one multiply, one add, as the encoder checked them), and each child that passes
// is pushed as its record slot.
template <int L>
__device__ __forceinline__ int wide_expand(const DeviceScene &s, int w, const Ray3 &r, float best, const WideStack &st,
                                           int sp, bool &overflow) {
    constexpr int K = kWidthOf<L>;
    const float4 *c = s.wide + size_t(w) * (2 * K);
    if constexpr (kQuantOf<L>) {
        constexpr int QW = kQuantWords<L>;
        const uint4 *q = s.wide_q + size_t(w) * QW;
        const uint4 h = __ldg(q);
        const int m = int((h.w >> 24) & 15u);
        if (h.w & 0x80000000u) {  // not quantized: the exact records
#pragma unroll
            for (int i = K - 1; i >= 0; i--) {
                if (i >= m) continue;
                const float4 lo = __ldg(c + 2 * i), hi = __ldg(c + 2 * i + 1);
                float te;
                if (slab(lo, hi, r, te) && !(te > best)) {
                    if (sp >= st.cap) {
                        overflow = true;
                        return sp;
                    }
                    st.put(sp++, w * K + i, te);
                }
            }
            return sp;
        }
        uint32_t b[4 * (QW - 1)];
#pragma unroll
        for (int k = 1; k < QW; k++) {
            const uint4 x = __ldg(q + k);
            b[4 * (k - 1)] = x.x;
            b[4 * (k - 1) + 1] = x.y;
            b[4 * (k - 1) + 2] = x.z;
            b[4 * (k - 1) + 3] = x.w;
        }
        const float ox = __uint_as_float(h.x), oy = __uint_as_float(h.y), oz = __uint_as_float(h.z);
        const float sx = __uint_as_float((h.w & 0xFFu) << 23), sy = __uint_as_float(((h.w >> 8) & 0xFFu) << 23),
                    sz = __uint_as_float(((h.w >> 16) & 0xFFu) << 23);
#pragma unroll
        for (int i = K - 1; i >= 0; i--) {
            if (i >= m) continue;
            const float4 lo = make_float4(ox + qbyte(b, 6 * i) * sx, oy + qbyte(b, 6 * i + 1) * sy,
                                          oz + qbyte(b, 6 * i + 2) * sz, 0.0f);
            const float4 hi = make_float4(ox + qbyte(b, 6 * i + 3) * sx, oy + qbyte(b, 6 * i + 4) * sy,
                                          oz + qbyte(b, 6 * i + 5) * sz, 0.0f);
            float te;
            if (slab(lo, hi, r, te) && !(te > best)) {
                if (sp >= st.cap) {
                    overflow = true;
                    return sp;
                }
                st.put(sp++, w * K + i, te);
            }
        }
        return sp;
    } else {
#pragma unroll
        for (int i = K - 1; i >= 0; i--) {
            const float4 lo = __ldg(c + 2 * i), hi = __ldg(c + 2 * i + 1);
            float te;
            if (slab(lo, hi, r, te) && !(te > best)) {
                if (sp >= st.cap) {
                    overflow = true;
                    return sp;
                }
                st.put(sp++, __float_as_int(lo.w), te);
            }
        }
        return sp;
    }
}

// The hit record of a finished closest-hit traversal of world ray wr: the winning
// primitive's attributes in instance space, then in world space. Returns false on a
// miss (best_obj < 0).
__device__ __forceinline__ bool closest_hit_finish(const DeviceScene &s, const Ray3 &wr, float best, int best_obj,
                                                   int best_inst, Hit &h) {
    if (best_obj < 0) {
        h.t = kMax;
        h.instance = -1;
        h.object = -1;
        return false;
    }
    const InstanceRef ir = instance_ref(s, best_inst);
    const Ray3 lr = to_local(s.instance_flags[best_inst], ir, wr);
    const Prim pr = load_prim(s, best_obj);
    const int inst_material = ir.header().w;
    const int mat = inst_material >= 0 ? inst_material : prim_material(pr);
    prim_attributes(s, best_obj, pr, lr.o, lr.d, best, h, s.material_uv[mat] != 0);
    h.instance = best_inst;
    h.object = best_obj;
    to_world(s, best_inst, ir, h);
    return true;
}

// Scene::hit in closest-hit mode (scene.h:51-124) over the wide BVH: two-level
// depth-first traversal that visits the nodes the reference visits in the order it
// visits them (right child first), culls an entry when its box starts beyond the best
// hit, lets a TLAS leaf test only its first instance (scene.h:80), and accepts
// candidates when t < best. This is the traversal alone: best, best_obj and
// best_inst come back (best_obj < 0 on a miss); closest_hit_finish makes the hit
// record from them.
template <int K>
__device__ __forceinline__ void closest_hit_ids_w(const DeviceScene &s, const Ray3 &wr, float &best, int &best_obj,
                                                  int &best_inst, bool &overflow, const WideStack &st,
                                                  const WideStack &sub) {
    best = kMax;
    best_obj = -1;
    best_inst = -1;
    int sp = 0;
    float te;
    if (slab(__ldg(&s.nodes[0]), __ldg(&s.nodes[1]), wr, te)) st.put(sp++, root_entry<K>(s, __ldg(&s.wide_code[0])), te);
    while (sp > 0) {
        --sp;
        te = st.te[sp * st.stride];
        const int code = pop_code<K>(s, st.code[sp * st.stride], te, wr, best);
        if (code == INT_MIN) continue;
        if (code >= 0) {
            sp = wide_expand<K>(s, code, wr, best, st, sp, overflow);
            if (overflow) break;
            continue;
        }
        const int inst = __ldg(&s.wide_leaves[-code - 1]).x;
        const uint32_t flags = s.instance_flags[inst];
        const InstanceRef ir = instance_ref(s, inst);
        const int root = ir.header().z;
        const Ray3 lr = to_local(flags, ir, wr);
        // a root box equal to the leaf's, under the same ray, was just tested (te)
        if (!(flags & 2u) && (!slab(__ldg(&s.nodes[2 * root]), __ldg(&s.nodes[2 * root + 1]), lr, te) || te > best))
            continue;
        int ssp = 0;
        sub.put(ssp++, root_entry<K>(s, __ldg(&s.wide_code[root])), te);
        while (ssp > 0) {
            --ssp;
            float te2 = sub.te[ssp * sub.stride];
            const int c2 = pop_code<K>(s, sub.code[ssp * sub.stride], te2, lr, best);
            if (c2 == INT_MIN) continue;
            if (c2 >= 0) {
                ssp = wide_expand<K>(s, c2, lr, best, sub, ssp, overflow);
                if (overflow) break;
                continue;
            }
            const int2 lf = __ldg(&s.wide_leaves[-c2 - 1]);
            for (int k = 0; k < lf.y; k++) {
                const float t = intersect_t(load_prim(s, lf.x + k), lr, best);
                if (t >= 0) {
                    best = t;
                    best_obj = lf.x + k;
                    best_inst = inst;
                }
            }
        }
        if (overflow) break;
    }
}

// Scene::hit in closest-hit mode with the hit record. Returns false on a miss.
template <int K>
__device__ __forceinline__ bool closest_hit_w(const DeviceScene &s, f3 o, f3 d, Hit &h, bool &overflow,
                                              const WideStack &st, const WideStack &sub) {
    const Ray3 wr = make_ray(o, d);
    float best;
    int best_obj, best_inst;
    closest_hit_ids_w<K>(s, wr, best, best_obj, best_inst, overflow, st, sub);
    return closest_hit_finish(s, wr, best, best_obj, best_inst, h);
}

// Scene::hit in shadow mode (scene.h:51-124 with occludedInstance/Object) over the
// wide BVH: for a scene light, first intersect the light primitive itself (a miss
// counts as occluded), then any primitive other than the light closer than it
// occludes. For the background light (-1, -1), any hit occludes. On a visible
// light, `light` holds the light's hit record for its emission lookup.
template <int K>
__device__ __forceinline__ bool occluded_w(const DeviceScene &s, f3 o, f3 d, int light_inst, int light_obj, Hit &light,
                                           bool &overflow, const WideStack &st, const WideStack &sub) {
    const Ray3 wr = make_ray(o, d);
    float best = kMax;
    if (light_inst != -1) {
        const InstanceRef ir = instance_ref(s, light_inst);
        const Ray3 lr = to_local(s.instance_flags[light_inst], ir, wr);
        const Prim p = load_prim(s, light_obj);
        const float t = intersect_t(p, lr, kMax);
        if (t < 0) return true;
        prim_attributes(s, light_obj, p, lr.o, lr.d, t, light);
        light.instance = light_inst;
        light.object = light_obj;
        to_world(s, light_inst, ir, light);
        best = t;
    }
    int sp = 0;
    float te;
    if (slab(__ldg(&s.nodes[0]), __ldg(&s.nodes[1]), wr, te)) st.put(sp++, root_entry<K>(s, __ldg(&s.wide_code[0])), te);
    while (sp > 0) {
        --sp;
        te = st.te[sp * st.stride];
        const int code = pop_code<K>(s, st.code[sp * st.stride], te, wr, best);
        if (code == INT_MIN) continue;
        if (code >= 0) {
            sp = wide_expand<K>(s, code, wr, best, st, sp, overflow);
            if (overflow) return true;
            continue;
        }
        const int inst = __ldg(&s.wide_leaves[-code - 1]).x;
        const uint32_t flags = s.instance_flags[inst];
        const InstanceRef ir = instance_ref(s, inst);
        const int root = ir.header().z;
        const Ray3 lr = to_local(flags, ir, wr);
        if (!(flags & 2u) && (!slab(__ldg(&s.nodes[2 * root]), __ldg(&s.nodes[2 * root + 1]), lr, te) || te > best))
            continue;
        int ssp = 0;
        sub.put(ssp++, root_entry<K>(s, __ldg(&s.wide_code[root])), te);
        while (ssp > 0) {
            --ssp;
            float te2 = sub.te[ssp * sub.stride];
            const int c2 = pop_code<K>(s, sub.code[ssp * sub.stride], te2, lr, best);
            if (c2 == INT_MIN) continue;
            if (c2 >= 0) {
                ssp = wide_expand<K>(s, c2, lr, best, sub, ssp, overflow);
                if (overflow) return true;
                continue;
            }
            const int2 lf = __ldg(&s.wide_leaves[-c2 - 1]);
            for (int k = 0; k < lf.y; k++) {
                if (light_inst != -1 && inst == light_inst && lf.x + k == light_obj) continue;
                if (intersect_t(load_prim(s, lf.x + k), lr, best) >= 0) return true;
            }
        }
    }
    return false;
}

// The two traversal stacks of this thread in dynamic shared memory: TLAS codes,
// TLAS distances, BLAS codes, BLAS distances, each [cap][blockDim.x].
__device__ __forceinline__ void wide_stacks(int *smem, const DeviceScene &s, WideStack &a, WideStack &b) {
    const int B = blockDim.x, t = threadIdx.x, ca = s.stack_tlas, cb = s.stack_blas;
    a = WideStack{smem + t, reinterpret_cast<float *>(smem + ca * B) + t, B, ca};
    b = WideStack{smem + 2 * ca * B + t, reinterpret_cast<float *>(smem + 2 * ca * B + cb * B) + t, B, cb};
}

__host__ __device__ inline size_t wide_stack_bytes(int block, int stack_tlas, int stack_blas) {
    return size_t(block) * size_t(stack_tlas + stack_blas) * 8;
}

// ---------------------------------------------------------------------------
// Lights (object.h:201-299, instance.h:105-111, background.h:77-79)
// ---------------------------------------------------------------------------

__device__ __forceinline__ float prim_pdf(const Prim &p, f3 point, f3 dir) {
    const int type = prim_type(p);
    if (type == 0) {
        const f3 c = mk(p.p0.x, p.p0.y, p.p0.z);
        const float rad = p.p1.x;
        const f3 oc = c - point;
        const float dsq = length_sq(oc);
        const float rsq = rad * rad;
        if (dsq <= rsq) return 1 / (4 * kPi);
        const float cos_max = sqrtf(1 - rsq / dsq);
        const float cos_t = dot(normalize(oc), dir);
        if (cos_t < cos_max) return 0;
        return 1 / (2 * kPi * (1 - cos_max));
    }
    const f3 corner = mk(p.p0.x, p.p0.y, p.p0.z);
    const f3 h = mk(p.p1.x, p.p1.y, p.p1.z);
    const f3 v = mk(p.p2.x, p.p2.y, p.p2.z);
    const f3 nn = mk(p.p3.x, p.p3.y, p.p3.z);
    if (type == 1) {
        const float cos_t = dot(normalize(nn), dir);
        if (fabsf(cos_t) < kEps) return 0;
        const float t = dot(corner - point, normalize(nn)) / cos_t;
        if (t < kEps) return 0;
        const f3 local = (point + dir * t) - corner;
        const float u = dot(nn, cross(local, v)) / length_sq(nn);
        const float w = dot(nn, cross(h, local)) / length_sq(nn);
        if (u < 0 || u > 1 || w < 0 || w > 1) return 0;
        return t * t / (fabsf(cos_t) * length(nn));
    }
    const f3 rcv = cross(dir, v);
    const float det = dot(h, rcv);
    if (fabsf(det) < kEpsSq) return 0;
    const float inv = rcp(det);
    const f3 oc = point - corner;
    const float alpha = inv * dot(oc, rcv);
    if (alpha < 0 || alpha > 1) return 0;
    const f3 och = cross(oc, h);
    const float beta = inv * dot(dir, och);
    if (beta < 0 || alpha + beta > 1) return 0;
    const float t = inv * dot(v, och);
    if (t < kEps) return 0;
    const float area = length(nn) * 0.5f;
    const float cos_t = dot(normalize(nn), dir);
    return t * t / (fabsf(cos_t) * area);
}

__device__ __forceinline__ f3 prim_sample(const Prim &p, f3 point, Rng &rng) {
    const int type = prim_type(p);
    if (type == 0) {
        const f3 c = mk(p.p0.x, p.p0.y, p.p0.z);
        const float rad = p.p1.x;
        const f3 oc = c - point;
        const float dsq = length_sq(oc);
        const float rsq = rad * rad;
        if (dsq <= rsq) return random_unit_vector(rng);
        const float cos_max = sqrtf(1 - rsq / dsq);
        return random_in_cone(oc, cos_max, rng);
    }
    const f3 corner = mk(p.p0.x, p.p0.y, p.p0.z);
    const f3 h = mk(p.p1.x, p.p1.y, p.p1.z);
    const f3 v = mk(p.p2.x, p.p2.y, p.p2.z);
    float u = rng.next();
    float w = rng.next();
    if (type == 2 && u + w > 1) {
        u = 1 - u;
        w = 1 - w;
    }
    const f3 q = corner + h * u + v * w;
    return normalize(q - point);
}

// Instance::area (instance.h:107): primitive area times |column 0 of M|^2.
__device__ __forceinline__ float prim_area(const Prim &p) {
    const int type = prim_type(p);
    if (type == 0) return 4 * kPi * p.p1.x * p.p1.x;
    const float l = length(mk(p.p3.x, p.p3.y, p.p3.z));
    return type == 1 ? l : l / 2;
}

// ---------------------------------------------------------------------------
// Materials (material.h)
// ---------------------------------------------------------------------------

enum : int { kLambertian = 0, kMirror = 1, kDielectric = 2, kEmissive = 3, kThinFilm = 4 };

// CIE 1931 lookup with linear interpolation (utils.h:195-203) and the
// spectrum -> XYZ -> linear sRGB conversion (utils.h:212-231).
__device__ __forceinline__ float xyz31(const DeviceScene &s, float lambda, int i) {
    const int lo = int(lambda);
    if (lo == 830) return s.cie[(lo - 360) * 3 + i];
    const int hi = lo + 1;
    return (float(hi) - lambda) * s.cie[(lo - 360) * 3 + i] + (lambda - float(lo)) * s.cie[(hi - 360) * 3 + i];
}

__device__ __forceinline__ f3 spectrum_to_rgb(const DeviceScene &s, const s4 &L, const s4 &lam, float range) {
    float x = 0, y = 0, z = 0;
    const float w = range / kHero;
    for (int i = 0; i < kHero; i++) {
        const float l = lam.v[i];
        const float r = L.v[i];
        x += xyz31(s, l, 0) * r * w;
        y += xyz31(s, l, 1) * r * w;
        z += xyz31(s, l, 2) * r * w;
    }
    x /= 106.856895f;
    y /= 106.856895f;
    z /= 106.856895f;
    return mk(x * 3.2406255f - y * 1.5372080f - z * 0.4986286f, -x * 0.9689307f + y * 1.8757561f + z * 0.0415175f,
              x * 0.0557101f - y * 0.2040211f + z * 1.0569959f);
}

}  // namespace lambda_dev
