// Thin-film transfer matrix (characteristic matrices of interfaces and layers).
//
// Follows Material::thinFilmReflectance (src/scene/material.h:263-309) and the
// interface/propagation matrices of src/core/utils.h:173-193: cosines carried as
// complex numbers through Snell's law, interface matrices (1/t)[[1, r], [r, 1]]
// with the Fresnel r, t of each polarisation, layer matrices diag(e^{-i phi},
// e^{i phi}) with phi = n (2 pi / lambda) d cos(theta), and R = |M01 / M00|^2.
// The reference returns only (R_s + R_p) / 2; this also gives the transmittances
// T = Re(n_out cos_out) / Re(n_in cos_in) |1 / M00|^2 (conjugated indices for p),
// which for real indices satisfy R + T = 1.
//
// The work splits in two: film_prepare() forms everything that depends only on
// the indices and the incidence angle (Snell cosines, interface matrices), and
// film_apply() multiplies in the layer phases for one wavelength. With
// non-dispersive indices the four hero wavelengths of a hit share one prepare.
// Templated on the real type: float for the render path, double for the
// training-label generator and the error audit.
#pragma once

namespace lambda_dev {

template <typename R>
struct cx {
    R re, im;
};

template <typename R> __device__ __forceinline__ cx<R> cmk(R a, R b) { return cx<R>{a, b}; }
template <typename R> __device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return cmk(a.re + b.re, a.im + b.im); }
template <typename R> __device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return cmk(a.re - b.re, a.im - b.im); }
template <typename R> __device__ __forceinline__ cx<R> operator*(cx<R> a, cx<R> b) {
    return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R> __device__ __forceinline__ cx<R> operator*(cx<R> a, R s) { return cmk(a.re * s, a.im * s); }

template <typename R> __device__ __forceinline__ R rdiv(R a, R b) {
    if constexpr (sizeof(R) == 4) return __fdividef(a, b);  // 2 ulp: far inside the 1e-5 budget
    else return a / b;
}

template <typename R> __device__ __forceinline__ cx<R> operator/(cx<R> a, cx<R> b) {
    // Smith's method: stable when one component of b dominates.
    if (fabs(b.re) >= fabs(b.im)) {
        const R q = rdiv(b.im, b.re);
        const R den = b.re + b.im * q;
        return cmk(rdiv(a.re + a.im * q, den), rdiv(a.im - a.re * q, den));
    }
    const R q = rdiv(b.re, b.im);
    const R den = b.re * q + b.im;
    return cmk(rdiv(a.re * q + a.im, den), rdiv(a.im * q - a.re, den));
}
template <typename R> __device__ __forceinline__ R cabs2(cx<R> a) { return a.re * a.re + a.im * a.im; }

// Principal square root (branch cut on the negative real axis; the sign of a
// zero imaginary part selects the side, as C99 csqrt does).
template <typename R> __device__ __forceinline__ cx<R> csqrt_(cx<R> z) {
    const R r = hypot(z.re, z.im);
    if (r == R(0)) return cmk(R(0), z.im);
    if (z.re >= R(0)) {
        const R s = sqrt((r + z.re) * R(0.5));
        return cmk(s, rdiv(z.im, R(2) * s));
    }
    R t = sqrt((r - z.re) * R(0.5));
    t = copysign(t, z.im);
    return cmk(rdiv(z.im, R(2) * t), t);
}

template <typename R> __device__ __forceinline__ cx<R> cexp_(cx<R> z) {
    R sn, cs;
    if constexpr (sizeof(R) == 4) {
        sincosf(z.im, &sn, &cs);
        const R e = expf(z.re);
        return cmk(e * cs, e * sn);
    } else {
        sincos(z.im, &sn, &cs);
        const R e = exp(z.re);
        return cmk(e * cs, e * sn);
    }
}

template <typename R>
struct m2 {
    cx<R> a, b, c, d;  // [[a, b], [c, d]]
};

template <typename R> __device__ __forceinline__ m2<R> mmul(const m2<R> &x, const m2<R> &y) {
    return m2<R>{x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}

// diag(e_minus, e_plus) * y
template <typename R> __device__ __forceinline__ m2<R> dmul(cx<R> em, cx<R> ep, const m2<R> &y) {
    return m2<R>{em * y.a, em * y.b, ep * y.c, ep * y.d};
}

// Interface matrix (1/t) [[1, r], [r, 1]] (utils.h:173-191).
template <typename R>
__device__ __forceinline__ m2<R> interface_matrix(cx<R> n1, cx<R> n2, cx<R> c1, cx<R> c2, bool p_pol) {
    cx<R> num, den;
    if (!p_pol) {
        num = n1 * c1 - n2 * c2;
        den = n1 * c1 + n2 * c2;
    } else {
        num = n2 * c1 - n1 * c2;
        den = n2 * c1 + n1 * c2;
    }
    // 1/t = den / (2 n1 c1) and r/t = num / (2 n1 c1)
    const cx<R> two_n1c1 = cmk(R(2), R(0)) * n1 * c1;
    const cx<R> inv_t = den / two_n1c1;
    const cx<R> r_t = num / two_n1c1;
    return m2<R>{inv_t, r_t, r_t, inv_t};
}

template <typename R>
struct FilmResult {
    R rs, rp, ts, tp;
};

// Everything of a stack of up to MAXL layers that does not depend on the
// wavelength once the indices are fixed: n[0] incidence medium, n[1..L] layers,
// n[L+1] exit medium.
template <typename R, int MAXL>
struct FilmPrep {
    int L;
    m2<R> is[MAXL + 1], ip[MAXL + 1];
    cx<R> n_layer[MAXL > 0 ? MAXL : 1];
    cx<R> cos_layer[MAXL > 0 ? MAXL : 1];
    cx<R> n_in, n_out, cos_out;
    R cos0;
    // One real-index film with real cosines everywhere (no total internal
    // reflection): the Fresnel coefficients of its two interfaces (s, p) for the
    // Airy form in film_apply.
    bool airy;
    R rs01, rs12, rp01, rp12;
};

template <typename R, int MAXL>
__device__ __forceinline__ void film_prepare(int L, const cx<R> *n, R cos0, FilmPrep<R, MAXL> &f) {
    f.L = L < MAXL ? L : MAXL;
    f.cos0 = cos0;
    if constexpr (sizeof(R) == 4 && MAXL >= 1) {
        // One film with real indices: Snell's law in real arithmetic. Without total
        // internal reflection every cosine is real, and the Airy form in film_apply
        // needs only the four Fresnel coefficients, not the interface matrices.
        if (L == 1 && n[0].im == R(0) && n[1].im == R(0) && n[2].im == R(0)) {
            const R n0 = n[0].re, n1 = n[1].re, n2 = n[2].re, c0 = cos0;
            const R q01 = n0 / n1, q12 = n1 / n2;
            const R sin1 = q01 * (q01 * (R(1) - c0 * c0));  // sin^2 in the film
            const R sin2 = q12 * (q12 * sin1);              // and in the substrate
            if (sin1 <= R(1) && sin2 <= R(1)) {
                const R c1 = sqrtf(R(1) - sin1), c2 = sqrtf(R(1) - sin2);
                f.airy = true;
                f.n_layer[0] = cmk(n1, R(0));
                f.cos_layer[0] = cmk(c1, R(0));
                f.rs01 = (n0 * c0 - n1 * c1) / (n0 * c0 + n1 * c1);
                f.rs12 = (n1 * c1 - n2 * c2) / (n1 * c1 + n2 * c2);
                f.rp01 = (n1 * c0 - n0 * c1) / (n1 * c0 + n0 * c1);
                f.rp12 = (n2 * c1 - n1 * c2) / (n2 * c1 + n1 * c2);
                return;
            }
        }
    }
    cx<R> cos_cur = cmk(cos0, R(0));
    cx<R> sin_next = n[0] / n[1];
    sin_next = sin_next * (sin_next * (cmk(R(1), R(0)) - cos_cur * cos_cur));
    cx<R> cos_next = csqrt_(cmk(R(1), R(0)) - sin_next);
    f.is[0] = interface_matrix(n[0], n[1], cos_cur, cos_next, false);
    f.ip[0] = interface_matrix(n[0], n[1], cos_cur, cos_next, true);
#pragma unroll
    for (int j = 0; j < MAXL; j++) {
        if (j < f.L) {
            const cx<R> a = n[j + 1], b = n[j + 2];
            cos_cur = cos_next;
            const cx<R> sin_cur = sin_next;
            sin_next = a / b;
            sin_next = sin_next * (sin_next * sin_cur);
            cos_next = csqrt_(cmk(R(1), R(0)) - sin_next);
            f.is[j + 1] = interface_matrix(a, b, cos_cur, cos_next, false);
            f.ip[j + 1] = interface_matrix(a, b, cos_cur, cos_next, true);
            f.n_layer[j] = a;
            f.cos_layer[j] = cos_cur;
        }
    }
    f.n_in = n[0];
    f.n_out = n[f.L + 1];
    f.cos_out = cos_next;
    f.airy = false;
}

// Reflectance of one film from its two interface coefficients and the cosine of the
// round-trip phase (Airy summation, the closed form of the 2x2 product). The
// denominator is at least (1 - |r01 r12|)^2, far from zero for real indices, so FP32
// keeps it within a few 1e-7 of FP64.
// The quotient takes the fast division (2 ulp), well inside the FP32 form's 1e-5.
__device__ __forceinline__ float airy_r(float r01, float r12, float cos2phi) {
    const float ab = r01 * r12, t = 2 * ab * cos2phi;
    return __fdividef(r01 * r01 + r12 * r12 + t, 1 + ab * ab + t);
}

// cos x of a film's round-trip phase (|x| up to about 1e5), for the FP32 form only.
// Cody and Waite's reduction: x less n 2 pi, n the integer nearest x / (2 pi), with
// 2 pi split into two floats (c1, 2 pi rounded to float; c2, the float nearest
// 2 pi - c1; the remainder, 6.9e-15, times n stays below 1e-9) and fused
// multiply-adds, then the hardware cosine on [-pi, pi] (absolute error below 4e-7).
__device__ __forceinline__ float cos_phase(float x) {
    const float n = rintf(x * 0.159154937f);
    float r = fmaf(-n, 6.28318548f, x);
    r = fmaf(-n, -1.74845553e-7f, r);
    return __cosf(r);
}

// Layer phases at one wavelength; k = 2 pi / lambda, d[j] in nm.
template <typename R, int MAXL>
__device__ __forceinline__ FilmResult<R> film_apply(const FilmPrep<R, MAXL> &f, const R *d, R k, bool want_t) {
    if constexpr (sizeof(R) == 4 && MAXL >= 1) {
        if (f.airy) {
            // the same phase as below: ((n k) d) cos, real here; round trip 2 phi
            const R phi = ((f.n_layer[0].re * k) * d[0]) * f.cos_layer[0].re;
            const R c2 = cos_phase(2 * phi);
            FilmResult<R> out;
            out.rs = airy_r(f.rs01, f.rs12, c2);
            out.rp = airy_r(f.rp01, f.rp12, c2);
            out.ts = want_t ? 1 - out.rs : R(0);  // lossless, no total internal reflection
            out.tp = want_t ? 1 - out.rp : R(0);
            return out;
        }
    }
    m2<R> ms = f.is[0], mp = f.ip[0];
#pragma unroll
    for (int j = 0; j < MAXL; j++) {
        if (j < f.L) {
            const cx<R> phi = ((f.n_layer[j] * k) * d[j]) * f.cos_layer[j];
            // exp(-i phi) = e^{Im phi} (cos Re phi - i sin Re phi), exp(+i phi) = e^{-Im phi} (cos + i sin)
            R sn, cs, g;
            if constexpr (sizeof(R) == 4) {
                sincosf(phi.re, &sn, &cs);
                g = expf(phi.im);
            } else {
                sincos(phi.re, &sn, &cs);
                g = exp(phi.im);
            }
            const R ginv = R(1) / g;
            const cx<R> e_minus = cmk(g * cs, -(g * sn));
            const cx<R> e_plus = cmk(ginv * cs, ginv * sn);
            ms = mmul(ms, dmul(e_minus, e_plus, f.is[j + 1]));
            mp = mmul(mp, dmul(e_minus, e_plus, f.ip[j + 1]));
        }
    }
    FilmResult<R> out;
    out.rs = cabs2(ms.b / ms.a);
    out.rp = cabs2(mp.b / mp.a);
    out.ts = out.tp = R(0);
    if (want_t) {
        const cx<R> c_in = cmk(f.cos0, R(0));
        const R s_num = (f.n_out * f.cos_out).re, s_den = (f.n_in * c_in).re;
        const R p_num = (cmk(f.n_out.re, -f.n_out.im) * f.cos_out).re, p_den = (cmk(f.n_in.re, -f.n_in.im) * c_in).re;
        const R ts_amp = R(1) / cabs2(ms.a), tp_amp = R(1) / cabs2(mp.a);
        out.ts = s_den != R(0) ? s_num / s_den * ts_amp : R(0);
        out.tp = p_den != R(0) ? p_num / p_den * tp_amp : R(0);
    }
    return out;
}

template <typename R, int MAXL>
__device__ __forceinline__ FilmResult<R> film_stack(int L, const cx<R> *n, const R *d, R cos0, R lambda) {
    FilmPrep<R, MAXL> f;
    film_prepare<R, MAXL>(L, n, cos0, f);
    return film_apply<R, MAXL>(f, d, R(2) * R(3.14159265358979323846) / lambda, true);
}

// The same product formed one interface at a time (any number of layers, no
// per-layer arrays): index_of(j) gives n[j], d[j] the layer thicknesses.
template <typename R, class IndexOf>
__device__ __forceinline__ void film_amplitudes_stream(int L, IndexOf index_of, const R *d, R cos0, R k, R &rs2, R &rp2) {
    cx<R> n0 = index_of(0), n1 = index_of(1);
    cx<R> cos_cur = cmk(cos0, R(0));
    cx<R> sin_next = n0 / n1;
    sin_next = sin_next * (sin_next * (cmk(R(1), R(0)) - cos_cur * cos_cur));
    cx<R> cos_next = csqrt_(cmk(R(1), R(0)) - sin_next);
    m2<R> ms = interface_matrix(n0, n1, cos_cur, cos_next, false);
    m2<R> mp = interface_matrix(n0, n1, cos_cur, cos_next, true);
#pragma unroll 1
    for (int j = 0; j < L; j++) {
        const cx<R> a = n1;
        n1 = index_of(j + 2);
        cos_cur = cos_next;
        const cx<R> sin_cur = sin_next;
        sin_next = a / n1;
        sin_next = sin_next * (sin_next * sin_cur);
        cos_next = csqrt_(cmk(R(1), R(0)) - sin_next);
        const cx<R> phi = ((a * k) * d[j]) * cos_cur;
        R sn, cs;
        if constexpr (sizeof(R) == 4) sincosf(phi.re, &sn, &cs);
        else sincos(phi.re, &sn, &cs);
        const R g = sizeof(R) == 4 ? R(expf(float(phi.im))) : R(exp(double(phi.im)));
        const R ginv = R(1) / g;
        const cx<R> e_minus = cmk(g * cs, -(g * sn)), e_plus = cmk(ginv * cs, ginv * sn);
        ms = mmul(ms, dmul(e_minus, e_plus, interface_matrix(a, n1, cos_cur, cos_next, false)));
        mp = mmul(mp, dmul(e_minus, e_plus, interface_matrix(a, n1, cos_cur, cos_next, true)));
    }
    rs2 = cabs2(ms.b / ms.a);
    rp2 = cabs2(mp.b / mp.a);
}

template <typename R, class IndexOf>
__device__ __forceinline__ R film_reflectance_stream(int L, IndexOf index_of, const R *d, R cos0, R k) {
    R rs2, rp2;
    film_amplitudes_stream<R>(L, index_of, d, cos0, k, rs2, rp2);
    return (rs2 + rp2) * R(0.5);
}

}  // namespace lambda_dev
