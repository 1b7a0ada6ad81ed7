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
template <typename R> __device__ __forceinline__ cx<R> operator/(cx<R> a, cx<R> b) {
    // Smith's method: stable when one component of b dominates.
    if (fabs(b.re) >= fabs(b.im)) {
        const R q = b.im / b.re;
        const R den = b.re + b.im * q;
        return cmk((a.re + a.im * q) / den, (a.im - a.re * q) / den);
    }
    const R q = b.re / b.im;
    const R den = b.re * q + b.im;
    return cmk((a.re * q + a.im) / den, (a.im * q - a.re) / den);
}
template <typename R> __device__ __forceinline__ R cabs2(cx<R> a) { return a.re * a.re + a.im * a.im; }

// Principal square root (branch cut on the negative real axis; the sign of a
// zero imaginary part selects the side, as C99 csqrt does).
template <typename R> __device__ __forceinline__ cx<R> csqrt_(cx<R> z) {
    const R r = hypot(z.re, z.im);
    if (r == R(0)) return cmk(R(0), z.im);
    if (z.re >= R(0)) {
        const R s = sqrt((r + z.re) * R(0.5));
        return cmk(s, z.im / (R(2) * s));
    }
    R t = sqrt((r - z.re) * R(0.5));
    t = copysign(t, z.im);
    return cmk(z.im / (R(2) * t), t);
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
    const cx<R> r = num / den;
    const cx<R> t = (cmk(R(2), R(0)) * n1 * c1) / den;
    const cx<R> one = cmk(R(1), R(0));
    return m2<R>{one / t, r / t, r / t, one / t};
}

template <typename R>
struct FilmResult {
    R rs, rp, ts, tp;
};

// Multilayer stack: n[0] incidence medium, n[1..L] layers, n[L+1] exit medium;
// d[0..L-1] layer thicknesses in nm, in the order the light meets them.
template <typename R, int MAXL>
__device__ FilmResult<R> film_stack(int L, const cx<R> *n, const R *d, R cos0, R lambda) {
    cx<R> cos_cur = cmk(cos0, R(0));
    cx<R> sin_next = n[0] / n[1];
    sin_next = sin_next * (sin_next * (cmk(R(1), R(0)) - cos_cur * cos_cur));
    cx<R> cos_next = csqrt_(cmk(R(1), R(0)) - sin_next);
    m2<R> ms = interface_matrix(n[0], n[1], cos_cur, cos_next, false);
    m2<R> mp = interface_matrix(n[0], n[1], cos_cur, cos_next, true);
    const R k = R(2) * R(3.14159265358979323846) / lambda;
    for (int j = 0; j < L && j < MAXL; j++) {
        const cx<R> a = n[j + 1], b = n[j + 2];
        cos_cur = cos_next;
        const cx<R> sin_cur = sin_next;
        sin_next = a / b;
        sin_next = sin_next * (sin_next * sin_cur);
        cos_next = csqrt_(cmk(R(1), R(0)) - sin_next);
        const m2<R> is = interface_matrix(a, b, cos_cur, cos_next, false);
        const m2<R> ip = interface_matrix(a, b, cos_cur, cos_next, true);
        const cx<R> phi = ((a * k) * d[j]) * cos_cur;
        const cx<R> e_minus = cexp_(cmk(phi.im, -phi.re));   // exp(-i phi)
        const cx<R> e_plus = cexp_(cmk(-phi.im, phi.re));    // exp(+i phi)
        const cx<R> zero = cmk(R(0), R(0));
        const m2<R> prop{e_minus, zero, zero, e_plus};
        ms = mmul(ms, mmul(prop, is));
        mp = mmul(mp, mmul(prop, ip));
    }
    FilmResult<R> out;
    out.rs = cabs2(ms.b / ms.a);
    out.rp = cabs2(mp.b / mp.a);
    const cx<R> n_in = n[0], n_out = n[L + 1];
    const cx<R> c_in = cmk(cos0, R(0));
    const R s_num = (n_out * cos_next).re, s_den = (n_in * c_in).re;
    const R p_num = (cmk(n_out.re, -n_out.im) * cos_next).re, p_den = (cmk(n_in.re, -n_in.im) * c_in).re;
    const cx<R> one = cmk(R(1), R(0));
    const R ts_amp = cabs2(one / ms.a), tp_amp = cabs2(one / mp.a);
    out.ts = s_den != R(0) ? s_num / s_den * ts_amp : R(0);
    out.tp = p_den != R(0) ? p_num / p_den * tp_amp : R(0);
    return out;
}

}  // namespace lambda_dev
