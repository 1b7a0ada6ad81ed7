/*
 * lambda_oracle.c - CPU restatement of the reference render loop (test oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the product never links or calls this file. Tests,
 * the smoke check and the benchmark's CPU-baseline arm use it as the checker.
 *
 * It restates, in plain C over the flat scene arrays of include/lambda_gpu.h, the
 * reference's CPU path (dakotaerskine/lambda, src/):
 *   render/renderer.h:42-195   renderImage, renderPixel, trace
 *   scene/scene.h:51-124        Scene::hit (closest and shadow modes)
 *   scene/bvh.h:30-52           BVHNode::intersect (slab test)
 *   scene/object.h:146-400      sphere/quad/triangle intersect, pdf, sample, area
 *   scene/instance.h:40-111     instance transforms, light pdf/sample/area
 *   scene/material.h:99-309     Lambertian, mirror, dielectric, thin film (FP64 TMM)
 *   scene/texture.h, background.h, core/utils.h   textures, noise, sampling, colour
 *   math/random.h               PCG32
 * with the reference's operand order, built with -ffp-contract=off and no -march
 * (SSE2 scalar, no fused multiply-add) so that results match its CPU build. It
 * also provides an FP64 transfer matrix with transmittances and an FP64 MLP
 * forward/backward for gradient checks of the surrogate.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lambda_gpu.h"

#include "../lambda_b200/csrc/host/tables.inc"

#define EPS 1e-4f
#define EPS_SQ (EPS * EPS)
#define PI_F 3.14159265358979323846f
#define MAXF 1e30f
#define HERO 4
#define RR_START 5
#define STACK 20
#define BINS 471

typedef struct { float x, y, z; } v3;

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 scl(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 dvs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float len2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline float len(v3 a) { return sqrtf(len2(a)); }
static inline v3 nrm(v3 a) { float l = len(a); return V(a.x / l, a.y / l, a.z / l); }
static inline v3 load3(const float *p) { return V(p[0], p[1], p[2]); }
static inline float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

typedef struct { float v[HERO]; } s4;

/* ---------------- PCG32 (random.h:7-30) ---------------- */
typedef struct { uint64_t state, inc; } pcg;

static inline uint32_t pcg_step(pcg *r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}
static inline pcg pcg_new(uint64_t seed, uint64_t stream) {
    pcg r;
    r.state = 0;
    r.inc = (stream << 1) | 1;
    pcg_step(&r);
    r.state += seed;
    pcg_step(&r);
    return r;
}
static inline float rnd(pcg *r) { return (float)pcg_step(r) / 4294967296.0f; }

/* ---------------- scene view ---------------- */
typedef struct {
    const lambda_scene_desc *d;
    const lambda_render_settings *rs;
    float range;
} Scene;

typedef struct {
    int instance, object;
    float t;
    v3 point, normal;
    float u, v;
    int front;
} Isect;

static inline Isect isect_init(void) {
    Isect i;
    memset(&i, 0, sizeof(i));
    i.instance = -1;
    i.object = -1;
    i.t = MAXF;
    return i;
}

/* utils.h:89-95 */
static inline v3 xform(const float *m, v3 v, float w) {
    float den = m[12] * v.x + m[13] * v.y + m[14] * v.z + m[15] * w;
    if (fabsf(den) < EPS) den = 1;
    v3 r = V(m[0] * v.x + m[1] * v.y + m[2] * v.z + m[3] * w, m[4] * v.x + m[5] * v.y + m[6] * v.z + m[7] * w,
             m[8] * v.x + m[9] * v.y + m[10] * v.z + m[11] * w);
    return dvs(r, den);
}
static inline v3 xform_t(const float *m, v3 v, float w) {
    float t[16];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) t[4 * i + j] = m[4 * j + i];
    return xform(t, v, w);
}

/* ---------------- spectra (spectrum.h:176-188) ---------------- */
static float spec_at(const Scene *s, int k, float lambda) {
    const float *d = s->d->spectra + (size_t)k * BINS;
    double index = (double)(lambda - 360.0f);
    int lo = (int)index;
    if (lo == BINS - 1) return d[lo];
    int hi = lo + 1;
    return (float)(((double)hi - index) * (double)d[lo] + (index - (double)lo) * (double)d[hi]);
}
static double complex cspec_at(const Scene *s, int k, float lambda) {
    const double *d = s->d->complex_spectra + (size_t)k * BINS * 2;
    double index = (double)(lambda - 360.0f);
    int lo = (int)index;
    if (lo == BINS - 1) return CMPLX(d[2 * lo], d[2 * lo + 1]);
    int hi = lo + 1;
    double a = (double)hi - index, b = index - (double)lo;
    return CMPLX(a * d[2 * lo] + b * d[2 * hi], a * d[2 * lo + 1] + b * d[2 * hi + 1]);
}

/* ---------------- noise (utils.h:97-171) ---------------- */
static inline float fade(float t) { return powf(t, 3) * (t * (6 * t - 15) + 10); }
static inline int perm(int i) { return kPerlinPermutation[i & 255]; }
static inline float grad(int h, float x, float y, float z) {
    switch (h % 12) {
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
static inline float lerpf_(float a, float b, float x) { return a + x * (b - a); }

float oracle_perlin(const float *p3) {
    v3 p = load3(p3);
    int i = (int)floorf(p.x) & 255, j = (int)floorf(p.y) & 255, k = (int)floorf(p.z) & 255;
    float tx = p.x - floorf(p.x), ty = p.y - floorf(p.y), tz = p.z - floorf(p.z);
    float u = fade(tx), v = fade(ty), w = fade(tz);
    int aaa = perm(perm(perm(i) + j) + k), aba = perm(perm(perm(i) + j + 1) + k);
    int aab = perm(perm(perm(i) + j) + k + 1), abb = perm(perm(perm(i) + j + 1) + k + 1);
    int baa = perm(perm(perm(i + 1) + j) + k), bba = perm(perm(perm(i + 1) + j + 1) + k);
    int bab = perm(perm(perm(i + 1) + j) + k + 1), bbb = perm(perm(perm(i + 1) + j + 1) + k + 1);
    float x1 = lerpf_(grad(aaa, tx, ty, tz), grad(baa, tx - 1, ty, tz), u);
    float x2 = lerpf_(grad(aba, tx, ty - 1, tz), grad(bba, tx - 1, ty - 1, tz), u);
    float y1 = lerpf_(x1, x2, v);
    x1 = lerpf_(grad(aab, tx, ty, tz - 1), grad(bab, tx - 1, ty, tz - 1), u);
    x2 = lerpf_(grad(abb, tx, ty - 1, tz - 1), grad(bbb, tx - 1, ty - 1, tz - 1), u);
    float y2 = lerpf_(x1, x2, v);
    return (lerpf_(y1, y2, w) + 1) / 2;
}

static inline float fractf_(float x) { return x - floorf(x); }

float oracle_worley(const float *p3) {
    v3 p = load3(p3);
    int xi = (int)floorf(p.x), yi = (int)floorf(p.y), zi = (int)floorf(p.z);
    float dist = 9999;
    for (int xo = -1; xo <= 1; xo++)
        for (int yo = -1; yo <= 1; yo++)
            for (int zo = -1; zo <= 1; zo++) {
                v3 c = V((float)(xi + xo), (float)(yi + yo), (float)(zi + zo));
                v3 f = V(fractf_(sinf(dot3(c, V(127.1f, 311.7f, 74.7f))) * 43758.5453f),
                         fractf_(sinf(dot3(c, V(269.5f, 183.3f, 246.1f))) * 43758.5453f),
                         fractf_(sinf(dot3(c, V(113.5f, 271.9f, 124.6f))) * 43758.5453f));
                f = add(f, c);
                dist = fminf(dist, len(sub(p, f)));
            }
    return dist;
}

/* ---------------- textures (texture.h) ---------------- */
static float scalar_tex(const Scene *s, int t, v3 point) {
    const lambda_scalar_texture *x = &s->d->scalar_textures[t];
    float p[3];
    switch (x->type) {
        case LAMBDA_SCALAR_CONSTANT: return x->p[0];
        case LAMBDA_SCALAR_PERLIN: {
            v3 q = scl(point, x->p[2]);
            p[0] = q.x; p[1] = q.y; p[2] = q.z;
            return x->p[0] + (x->p[1] - x->p[0]) * oracle_perlin(p);
        }
        default: {
            v3 q = scl(point, x->p[2]);
            p[0] = q.x; p[1] = q.y; p[2] = q.z;
            return x->p[0] + (x->p[1] - x->p[0]) * oracle_worley(p);
        }
    }
}
static float spec_tex(const Scene *s, int t, const Isect *i, float lambda) {
    const lambda_spectrum_texture *x = &s->d->spectrum_textures[t];
    switch (x->type) {
        case LAMBDA_SPECTRUM_CONSTANT: return spec_at(s, x->value1, lambda);
        case LAMBDA_SPECTRUM_CHECKER: {
            int cx = (int)floorf(i->u / x->scale), cy = (int)floorf(i->v / x->scale);
            return (cx + cy) % 2 == 0 ? spec_at(s, x->value1, lambda) : spec_at(s, x->value2, lambda);
        }
        default: return scalar_tex(s, x->value1, i->point);
    }
}
static float spec_avg(const Scene *s, int k) {
    const float *d = s->d->spectra + (size_t)k * BINS;
    float sum = 0;
    for (int i = 0; i < BINS; i++) sum += d[i];
    return sum / BINS;
}
static float spec_tex_avg(const Scene *s, int t) {
    const lambda_spectrum_texture *x = &s->d->spectrum_textures[t];
    if (x->type == LAMBDA_SPECTRUM_CONSTANT) return spec_avg(s, x->value1);
    if (x->type == LAMBDA_SPECTRUM_CHECKER) return 0.5f * (spec_avg(s, x->value1) + spec_avg(s, x->value2));
    const lambda_scalar_texture *y = &s->d->scalar_textures[x->value1];
    return y->type == LAMBDA_SCALAR_CONSTANT ? y->p[0] : (y->p[0] + y->p[1]) / 2;
}
/* background.h:81-95 */
static s4 bg_eval(const Scene *s, v3 d, const s4 *lam) {
    Isect i = isect_init();
    i.point = d;
    i.u = (atan2f(d.z, d.x) + PI_F) / (2 * PI_F);
    i.v = acosf(d.y) / PI_F;
    s4 r;
    for (int k = 0; k < HERO; k++) r.v[k] = spec_tex(s, s->d->background_texture, &i, lam->v[k]);
    return r;
}

/* ---------------- geometry (object.h, bvh.h) ---------------- */
static int slab(const lambda_bvh_node *n, v3 o, v3 d, float *te) {
    float t1 = 0, t2 = MAXF;
    for (int i = 0; i < 3; i++) {
        float inv = 1 / comp(d, i);
        float a = (n->min[i] - comp(o, i)) * inv, b = (n->max[i] - comp(o, i)) * inv;
        if (inv < 0) { float t = a; a = b; b = t; }
        t1 = fmaxf(a, t1);
        t2 = fminf(b, t2);
    }
    *te = t1;
    return t1 <= t2 && t2 >= 0;
}

/* Object::intersect: writes the full record when t < it->t (object.h:301-400). */
static int obj_intersect(const lambda_object *ob, int idx, v3 o, v3 d, Isect *it) {
    const float *g = ob->g;
    if (ob->type == LAMBDA_OBJECT_SPHERE) {
        v3 c = load3(g);
        float r = g[3];
        v3 oc = sub(o, c);
        float a = len2(d), b = 2 * dot3(d, oc), cc = dot3(oc, oc) - r * r;
        float disc = b * b - 4 * a * cc;
        if (disc < 0) return 0;
        disc = sqrtf(disc);
        float t1 = (-b - disc) / (2 * a), t2 = (-b + disc) / (2 * a);
        if (t1 < EPS && t2 < EPS) return 0;
        float t = t1 < EPS ? t2 : t1;
        if (t >= it->t) return 0;
        it->object = idx;
        it->t = t;
        it->point = add(o, scl(d, t));
        it->normal = nrm(sub(it->point, c));
        it->u = (atan2f(-it->normal.z, it->normal.x) + PI_F) / (2 * PI_F);
        it->v = acosf(-it->normal.y) / PI_F;
        it->front = dot3(d, it->normal) < 0;
        if (!it->front) it->normal = scl(it->normal, -1);
        return 1;
    }
    v3 corner = load3(g), h = load3(g + 3), v = load3(g + 6), nn = load3(g + 9);
    if (ob->type == LAMBDA_OBJECT_QUAD) {
        v3 n = nrm(nn);
        float den = dot3(n, d);
        if (fabsf(den) < EPS) return 0;
        float t = dot3(n, sub(corner, o)) / den;
        if (t < EPS || t >= it->t) return 0;
        v3 p = add(o, scl(d, t));
        v3 pr = sub(p, corner);
        float al = dot3(nn, cross3(pr, v)) / len2(nn);
        float be = dot3(nn, cross3(h, pr)) / len2(nn);
        if (al < 0 || al > 1 || be < 0 || be > 1) return 0;
        it->object = idx;
        it->t = t;
        it->point = p;
        it->normal = nrm(nn);
        it->u = al;
        it->v = be;
        it->front = dot3(d, it->normal) < 0;
        if (!it->front) it->normal = scl(it->normal, -1);
        return 1;
    }
    v3 rcv = cross3(d, v);
    float det = dot3(h, rcv);
    if (fabsf(det) < EPS_SQ) return 0;
    float inv = 1 / det;
    v3 oc = sub(o, corner);
    float al = inv * dot3(oc, rcv);
    if (al < 0 || al > 1) return 0;
    v3 och = cross3(oc, h);
    float be = inv * dot3(d, och);
    if (be < 0 || al + be > 1) return 0;
    float t = inv * dot3(v, och);
    if (t < EPS || t >= it->t) return 0;
    float w0 = 1 - al - be;
    it->object = idx;
    it->t = t;
    it->point = add(o, scl(d, t));
    it->normal = nrm(add(add(scl(load3(g + 12), w0), scl(load3(g + 15), al)), scl(load3(g + 18), be)));
    it->u = w0 * g[21] + al * g[22] + be * g[23];
    it->v = w0 * g[24] + al * g[25] + be * g[26];
    it->front = dot3(d, nn) < 0;
    if (!it->front) it->normal = scl(it->normal, -1);
    return 1;
}

static float obj_pdf(const lambda_object *ob, v3 p, v3 dir) {
    const float *g = ob->g;
    if (ob->type == LAMBDA_OBJECT_SPHERE) {
        v3 oc = sub(load3(g), p);
        float dsq = len2(oc), rsq = g[3] * g[3];
        if (dsq <= rsq) return 1 / (4 * PI_F);
        float cmax = sqrtf(1 - rsq / dsq);
        float ct = dot3(nrm(oc), dir);
        if (ct < cmax) return 0;
        return 1 / (2 * PI_F * (1 - cmax));
    }
    v3 corner = load3(g), h = load3(g + 3), v = load3(g + 6), nn = load3(g + 9);
    if (ob->type == LAMBDA_OBJECT_QUAD) {
        float ct = dot3(nrm(nn), dir);
        if (fabsf(ct) < EPS) return 0;
        float t = dot3(sub(corner, p), nrm(nn)) / ct;
        if (t < EPS) return 0;
        v3 local = sub(add(p, scl(dir, t)), corner);
        float u = dot3(nn, cross3(local, v)) / len2(nn);
        float w = dot3(nn, cross3(h, local)) / len2(nn);
        if (u < 0 || u > 1 || w < 0 || w > 1) return 0;
        return t * t / (fabsf(ct) * len(nn));
    }
    v3 rcv = cross3(dir, v);
    float det = dot3(h, rcv);
    if (fabsf(det) < EPS_SQ) return 0;
    float inv = 1 / det;
    v3 oc = sub(p, corner);
    float al = inv * dot3(oc, rcv);
    if (al < 0 || al > 1) return 0;
    v3 och = cross3(oc, h);
    float be = inv * dot3(dir, och);
    if (be < 0 || al + be > 1) return 0;
    float t = inv * dot3(v, och);
    if (t < EPS) return 0;
    float area = len(nn) * 0.5f;
    float ct = dot3(nrm(nn), dir);
    return t * t / (fabsf(ct) * area);
}

/* randomUnitVector: GCC evaluates the three constructor arguments right to
 * left, so the first draw is z (utils.h:20-24). */
static v3 rand_unit(pcg *r) {
    float z = rnd(r) * 2 - 1;
    float y = rnd(r) * 2 - 1;
    float x = rnd(r) * 2 - 1;
    return nrm(V(x, y, z));
}
static v3 frame(v3 n, float x, float y, float z) {
    v3 w = nrm(n);
    v3 u = fabsf(w.x) > fabsf(w.y) ? V(0, 0, 1) : V(1, 0, 0);
    u = nrm(cross3(u, w));
    v3 v = cross3(w, u);
    return add(add(scl(u, x), scl(v, y)), scl(w, z));
}
static v3 rand_hemi(v3 n, pcg *r) {
    float r1 = rnd(r), r2 = rnd(r);
    float phi = 2 * PI_F * r1;
    float rad = sqrtf(r2);
    return frame(n, rad * cosf(phi), rad * sinf(phi), sqrtf(1 - r2));
}
static v3 rand_cone(v3 n, float cmax, pcg *r) {
    float r1 = rnd(r), r2 = rnd(r);
    float ct = 1 + r1 * (cmax - 1);
    float st = sqrtf(1 - ct * ct);
    float phi = 2 * PI_F * r2;
    return frame(n, st * cosf(phi), st * sinf(phi), ct);
}
static v3 obj_sample(const lambda_object *ob, v3 p, pcg *r) {
    const float *g = ob->g;
    if (ob->type == LAMBDA_OBJECT_SPHERE) {
        v3 oc = sub(load3(g), p);
        float dsq = len2(oc), rsq = g[3] * g[3];
        if (dsq <= rsq) return rand_unit(r);
        return rand_cone(oc, sqrtf(1 - rsq / dsq), r);
    }
    float u = rnd(r), v = rnd(r);
    if (ob->type == LAMBDA_OBJECT_TRI && u + v > 1) {
        u = 1 - u;
        v = 1 - v;
    }
    v3 q = add(add(load3(g), scl(load3(g + 3), u)), scl(load3(g + 6), v));
    return nrm(sub(q, p));
}
static float obj_area(const lambda_object *ob) {
    if (ob->type == LAMBDA_OBJECT_SPHERE) return 4 * PI_F * ob->g[3] * ob->g[3];
    float l = len(load3(ob->g + 9));
    return ob->type == LAMBDA_OBJECT_QUAD ? l : l / 2;
}

/* Scene::hit (scene.h:51-124) */
static int scene_hit(const Scene *s, v3 o, v3 d, Isect *it, int occ_inst, int occ_obj) {
    const lambda_scene_desc *D = s->d;
    int stack[STACK], sp = 0, sub_[STACK], ssp = 0, hit = 0;
    stack[sp++] = 0;
    if (occ_inst != -1) {
        const lambda_instance *in = &D->instances[occ_inst];
        v3 lo = xform(in->inverse_transform, o, 1), ld = xform(in->inverse_transform, d, 0);
        if (!obj_intersect(&D->objects[occ_obj], occ_obj, lo, ld, it)) return 1;
        it->instance = occ_inst;
        it->point = xform(in->transform, it->point, 1);
        it->normal = nrm(xform_t(in->inverse_transform, it->normal, 0));
    }
    while (sp > 0) {
        int cur = stack[--sp];
        float te;
        const lambda_bvh_node *n = &D->nodes[cur];
        if (!slab(n, o, d, &te) || te > it->t) continue;
        if (n->count > 0) {
            int ii = n->index;
            const lambda_instance *in = &D->instances[ii];
            sub_[ssp++] = in->node;
            v3 lo = xform(in->inverse_transform, o, 1), ld = xform(in->inverse_transform, d, 0);
            while (ssp > 0) {
                int sc = sub_[--ssp];
                const lambda_bvh_node *m = &D->nodes[sc];
                if (!slab(m, lo, ld, &te) || te > it->t) continue;
                if (m->count > 0) {
                    for (int k = 0; k < m->count; k++) {
                        int oi = m->index + k;
                        if (occ_inst != -1 && ii == occ_inst && oi == occ_obj) continue;
                        if (obj_intersect(&D->objects[oi], oi, lo, ld, it)) {
                            it->instance = ii;
                            it->point = xform(in->transform, it->point, 1);
                            it->normal = nrm(xform_t(in->inverse_transform, it->normal, 0));
                            if (occ_obj != -2) return 1;
                            hit = 1;
                        }
                    }
                } else {
                    if (ssp + 2 > STACK) return hit;
                    sub_[ssp++] = sc + 1;
                    sub_[ssp++] = m->index;
                }
            }
        } else {
            if (sp + 2 > STACK) return hit;
            stack[sp++] = cur + 1;
            stack[sp++] = n->index;
        }
    }
    return hit;
}

/* ---------------- thin film (material.h:228-309, utils.h:173-193) ---------------- */
typedef struct { double complex a, b, c, d; } m2c;

static m2c m2mul(m2c x, m2c y) {
    m2c r;
    r.a = x.a * y.a + x.b * y.c;
    r.b = x.a * y.b + x.b * y.d;
    r.c = x.c * y.a + x.d * y.c;
    r.d = x.c * y.b + x.d * y.d;
    return r;
}
static m2c iface(double complex n1, double complex n2, double complex c1, double complex c2, int p) {
    double complex r = p ? (n2 * c1 - n1 * c2) / (n2 * c1 + n1 * c2) : (n1 * c1 - n2 * c2) / (n1 * c1 + n2 * c2);
    double complex t = p ? (CMPLX(2, 0) * n1 * c1) / (n2 * c1 + n1 * c2) : (CMPLX(2, 0) * n1 * c1) / (n1 * c1 + n2 * c2);
    m2c m;
    m.a = CMPLX(1, 0) / t;
    m.b = r / t;
    m.c = r / t;
    m.d = CMPLX(1, 0) / t;
    return m;
}

/* Characteristic-matrix stack: n[0] incidence, n[1..L] layers, n[L+1] exit.
 * out = (R_s, R_p, T_s, T_p). lambda_k is 2*pi/lambda as the caller forms it. */
static void film_stack(int L, const double complex *n, const double *dd, double cos0, double k, double *out) {
    double complex cc = CMPLX(cos0, 0);
    double complex sn = n[0] / n[1];
    sn *= sn * (CMPLX(1, 0) - cc * cc);
    double complex cn = csqrt(CMPLX(1, 0) - sn);
    m2c ms = iface(n[0], n[1], cc, cn, 0), mp = iface(n[0], n[1], cc, cn, 1);
    for (int j = 0; j < L; j++) {
        double complex a = n[j + 1], b = n[j + 2];
        cc = cn;
        double complex sc = sn;
        sn = a / b;
        sn *= sn * sc;
        cn = csqrt(CMPLX(1, 0) - sn);
        m2c is = iface(a, b, cc, cn, 0), ip = iface(a, b, cc, cn, 1);
        double complex phi = a * CMPLX(k, 0);
        phi = CMPLX(creal(phi) * dd[j], cimag(phi) * dd[j]);
        phi = phi * cc;
        m2c pr;
        pr.a = cexp(CMPLX(0, -1) * phi);
        pr.b = 0;
        pr.c = 0;
        pr.d = cexp(CMPLX(0, 1) * phi);
        ms = m2mul(ms, m2mul(pr, is));
        mp = m2mul(mp, m2mul(pr, ip));
    }
    double rs = cabs(ms.b / ms.a), rp = cabs(mp.b / mp.a);
    out[0] = rs * rs;
    out[1] = rp * rp;
    double complex ci = CMPLX(cos0, 0);
    double sden = creal(n[0] * ci), pden = creal(conj(n[0]) * ci);
    double snum = creal(n[L + 1] * cn), pnum = creal(conj(n[L + 1]) * cn);
    double ts = cabs(CMPLX(1, 0) / ms.a), tp = cabs(CMPLX(1, 0) / mp.a);
    out[2] = sden != 0 ? snum / sden * ts * ts : 0;
    out[3] = pden != 0 ? pnum / pden * tp * tp : 0;
}

/* FP64 single film on a substrate, outer index 1: out[4n] = (Rs, Rp, Ts, Tp). */
void oracle_film(const lambda_film_query *q, int n, double *out) {
    for (int i = 0; i < n; i++) {
        double complex idx[3] = {CMPLX(1, 0), CMPLX(q[i].n_film, 0), CMPLX(q[i].n_sub, 0)};
        double d = q[i].thickness_nm;
        film_stack(1, idx, &d, q[i].cos_theta, 2 * 3.14159265358979323846 / (double)q[i].lambda_nm, out + 4 * (size_t)i);
    }
}

/* thinFilmReflectance (material.h:263-309): R = (Rs + Rp) / 2 rounded as the
 * reference rounds it (|r| to float, squared in float). */
static float thin_film_r(const Scene *s, const lambda_material *m, const Isect *it, v3 dir, float lambda) {
    int L = m->p[0];
    const int *mp = s->d->material_properties;
    int off = it->front ? 0 : L + 1, sg = it->front ? 1 : -1;
    double complex n0 = cspec_at(s, mp[m->p[1] + off], lambda), n1 = cspec_at(s, mp[m->p[1] + off + sg], lambda);
    double complex cc = CMPLX((double)dot3(it->normal, scl(dir, -1)), 0);
    double complex sn = n0 / n1;
    sn *= sn * (CMPLX(1, 0) - cc * cc);
    double complex cn = csqrt(CMPLX(1, 0) - sn);
    m2c ms = iface(n0, n1, cc, cn, 0), mq = iface(n0, n1, cc, cn, 1);
    for (int j = 0; j < L; j++) {
        int di = it->front ? j : L - 1 - j;
        n0 = cspec_at(s, mp[m->p[1] + off + sg * (j + 1)], lambda);
        n1 = cspec_at(s, mp[m->p[1] + off + sg * (j + 2)], lambda);
        cc = cn;
        double complex sc = sn;
        sn = n0 / n1;
        sn *= sn * sc;
        cn = csqrt(CMPLX(1, 0) - sn);
        m2c is = iface(n0, n1, cc, cn, 0), ip = iface(n0, n1, cc, cn, 1);
        double thick = (double)scalar_tex(s, mp[m->p[2] + di], it->point);
        double complex phi = n0 * CMPLX((double)(2 * PI_F / lambda), 0);
        phi = CMPLX(creal(phi) * thick, cimag(phi) * thick);
        phi = phi * cc;
        m2c pr;
        pr.a = cexp(CMPLX(0, -1) * phi);
        pr.b = 0;
        pr.c = 0;
        pr.d = cexp(CMPLX(0, 1) * phi);
        ms = m2mul(ms, m2mul(pr, is));
        mq = m2mul(mq, m2mul(pr, ip));
    }
    float rs = (float)cabs(ms.b / ms.a), rp = (float)cabs(mq.b / mq.a);
    rs *= rs;
    rp *= rp;
    return (rs + rp) * 0.5f;
}

/* ---------------- materials and the bounce loop (renderer.h:94-195) ---------------- */
static inline v3 reflect_(v3 v, v3 n) { return sub(v, scl(n, 2 * dot3(v, n))); }
static inline v3 refract_(v3 v, v3 n, float ratio) {
    float vn = dot3(v, n);
    float root = 1 - ratio * ratio * (1 - vn * vn);
    if (root < 0) return sub(v, scl(n, 2 * vn));
    return sub(scl(v, ratio), scl(n, ratio * vn + sqrtf(root)));
}
static inline float ph(float a, float b) {
    a *= a;
    b *= b;
    return a / (a + b);
}
static inline int material_of(const Scene *s, const lambda_instance *in, int obj) {
    return in->material >= 0 ? in->material : s->d->objects[obj].material;
}
static inline float clampf_(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

static s4 trace(const Scene *s, v3 o, v3 d, const s4 *lam, pcg *rng) {
    const lambda_scene_desc *D = s->d;
    s4 L = {{0, 0, 0, 0}}, T = {{1, 1, 1, 1}};
    float prev = 1;
    int specular = 1;
    for (int i = 0; i <= s->rs->depth; i++) {
        Isect it = isect_init();
        if (!scene_hit(s, o, d, &it, -1, -2)) {
            float w = 1;
            if (!specular && D->total_light_power > 0)
                w = ph(prev, 1 / (4 * PI_F) * D->light_powers[D->num_lights - 1] / D->total_light_power);
            s4 e = bg_eval(s, d, lam);
            for (int k = 0; k < HERO; k++) L.v[k] += T.v[k] * e.v[k] * w;
            break;
        }
        const lambda_instance *in = &D->instances[it.instance];
        int mi = material_of(s, in, it.object);
        const lambda_material *m = &D->materials[mi];
        if (m->type == LAMBDA_MATERIAL_EMISSIVE) {
            float w = 1;
            if (!specular && D->total_light_power > 0) {
                v3 c0 = V(in->transform[0], in->transform[4], in->transform[8]);
                float lp = obj_area(&D->objects[it.object]) * len2(c0) * spec_tex_avg(s, m->p[0]);
                float pdf = obj_pdf(&D->objects[it.object], xform(in->inverse_transform, o, 1),
                                    nrm(xform(in->inverse_transform, d, 0)));
                w = ph(prev, pdf * lp / D->total_light_power);
            }
            for (int k = 0; k < HERO; k++) L.v[k] += T.v[k] * spec_tex(s, m->p[0], &it, lam->v[k]) * w;
            break;
        }
        if (m->type == LAMBDA_MATERIAL_LAMBERTIAN && D->total_light_power > 0) {
            float target = D->total_light_power * rnd(rng);
            float cum = 0;
            int li = D->light_instances[0], lo = D->light_objects[0];
            float lp = D->light_powers[0];
            for (int j = 0; j < D->num_lights; j++) {
                cum += D->light_powers[j];
                if (cum >= target) {
                    li = D->light_instances[j];
                    lo = D->light_objects[j];
                    lp = D->light_powers[j];
                    break;
                }
            }
            v3 ld;
            float lpdf;
            if (li != -1) {
                const lambda_instance *lin = &D->instances[li];
                v3 pl = xform(lin->inverse_transform, it.point, 1);
                ld = nrm(xform(lin->transform, obj_sample(&D->objects[lo], pl, rng), 0));
                lpdf = obj_pdf(&D->objects[lo], xform(lin->inverse_transform, it.point, 1),
                               nrm(xform(lin->inverse_transform, ld, 0)));
            } else {
                ld = rand_unit(rng);
                lpdf = 1 / (4 * PI_F);
            }
            float ct = dot3(it.normal, ld);
            if (lpdf > 0 && ct > 0) {
                lpdf *= lp / D->total_light_power;
                Isect sh = isect_init();
                if (!scene_hit(s, it.point, ld, &sh, li, lo)) {
                    s4 e, att;
                    if (li != -1) {
                        const lambda_material *lm = &D->materials[material_of(s, &D->instances[li], lo)];
                        for (int k = 0; k < HERO; k++)
                            e.v[k] = lm->type == LAMBDA_MATERIAL_EMISSIVE ? spec_tex(s, lm->p[0], &sh, lam->v[k]) : 0;
                    } else {
                        e = bg_eval(s, ld, lam);
                    }
                    int pos = dot3(it.normal, ld) > 0;
                    for (int k = 0; k < HERO; k++) att.v[k] = pos ? spec_tex(s, m->p[0], &it, lam->v[k]) / PI_F : 0;
                    float cl = dot3(it.normal, ld);
                    float spdf = cl > 0 ? cl / PI_F : 0;
                    float w = ph(lpdf, spdf);
                    for (int k = 0; k < HERO; k++) L.v[k] += T.v[k] * att.v[k] * ct * e.v[k] * w / lpdf;
                }
            }
        }
        s4 att;
        v3 nd;
        float pdf = 0;
        int spec = 1;
        if (m->type == LAMBDA_MATERIAL_LAMBERTIAN) {
            nd = rand_hemi(it.normal, rng);
            int pos = dot3(it.normal, nd) > 0;
            for (int k = 0; k < HERO; k++) att.v[k] = pos ? spec_tex(s, m->p[0], &it, lam->v[k]) / PI_F : 0;
            float cl = dot3(it.normal, nd);
            pdf = cl > 0 ? cl / PI_F : 0;
            spec = 0;
        } else if (m->type == LAMBDA_MATERIAL_MIRROR) {
            nd = reflect_(d, it.normal);
            for (int k = 0; k < HERO; k++) att.v[k] = spec_tex(s, m->p[0], &it, lam->v[k]);
        } else if (m->type == LAMBDA_MATERIAL_DIELECTRIC) {
            float factor = powf(1 + dot3(d, it.normal), 5);
            float n0h = spec_at(s, m->p[0], lam->v[0]), n1h = spec_at(s, m->p[1], lam->v[0]);
            float ratio = it.front ? n0h / n1h : n1h / n0h;
            float r0 = (n0h - n1h) / (n0h + n1h);
            r0 *= r0;
            float rh = r0 + (1 - r0) * factor;
            int refl = rnd(rng) < rh;
            nd = refl ? reflect_(d, it.normal) : refract_(d, it.normal, ratio);
            att.v[0] = 1;
            for (int k = 1; k < HERO; k++) {
                float a0 = spec_at(s, m->p[0], lam->v[k]), a1 = spec_at(s, m->p[1], lam->v[k]);
                float rr = (a0 - a1) / (a0 + a1);
                rr *= rr;
                float r = rr + (1 - rr) * factor;
                att.v[k] = refl ? r / rh : (fabsf(a0 - n0h) < EPS && fabsf(a1 - n1h) < EPS) ? (1 - r) / (1 - rh) : 0;
            }
        } else {
            const int *mp = D->material_properties;
            int outer = mp[m->p[1]], subst = mp[m->p[1] + m->p[0] + 1];
            float n0h = (float)creal(cspec_at(s, outer, lam->v[0]));
            float n1h = (float)creal(cspec_at(s, subst, lam->v[0]));
            float ratio = it.front ? n0h / n1h : n1h / n0h;
            float rh = thin_film_r(s, m, &it, d, lam->v[0]);
            int refl = rnd(rng) < rh;
            nd = refl ? reflect_(d, it.normal) : refract_(d, it.normal, ratio);
            att.v[0] = 1;
            for (int k = 1; k < HERO; k++) {
                float a0 = (float)creal(cspec_at(s, outer, lam->v[k]));
                float a1 = (float)creal(cspec_at(s, subst, lam->v[k]));
                float r = thin_film_r(s, m, &it, d, lam->v[k]);
                att.v[k] = refl ? r / rh : (fabsf(a0 - n0h) < EPS && fabsf(a1 - n1h) < EPS) ? (1 - r) / (1 - rh) : 0;
            }
        }
        o = it.point;
        d = nd;
        prev = pdf;
        specular = spec;
        if (spec) {
            for (int k = 0; k < HERO; k++) T.v[k] *= att.v[k];
        } else {
            float c = dot3(it.normal, d);
            for (int k = 0; k < HERO; k++) T.v[k] *= att.v[k] * c / prev;
        }
        if (i >= RR_START) {
            float mx = T.v[0];
            for (int k = 1; k < HERO; k++)
                if (T.v[k] > mx) mx = T.v[k];
            float q = 1 - clampf_(mx, 0.05f, 0.95f);
            if (rnd(rng) < q) break;
            for (int k = 0; k < HERO; k++) T.v[k] /= 1 - q;
        }
    }
    return L;
}

/* utils.h:195-231 */
static float xyz31(float lambda, int i) {
    int lo = (int)lambda;
    if (lo == 830) return (float)kCieXyz1931[lo - 360][i];
    int hi = lo + 1;
    return ((float)hi - lambda) * (float)kCieXyz1931[lo - 360][i] + (lambda - (float)lo) * (float)kCieXyz1931[hi - 360][i];
}
static v3 spectrum_to_rgb(const s4 *L, const s4 *lam, float range) {
    float x = 0, y = 0, z = 0, w = range / HERO;
    for (int i = 0; i < HERO; i++) {
        x += xyz31(lam->v[i], 0) * L->v[i] * w;
        y += xyz31(lam->v[i], 1) * L->v[i] * w;
        z += xyz31(lam->v[i], 2) * L->v[i] * w;
    }
    x /= 106.856895f;
    y /= 106.856895f;
    z /= 106.856895f;
    return V(x * 3.2406255f - y * 1.5372080f - z * 0.4986286f, -x * 0.9689307f + y * 1.8757561f + z * 0.0415175f,
             x * 0.0557101f - y * 0.2040211f + z * 1.0569959f);
}

/* renderPixel (renderer.h:64-92) */
static void render_pixel(const Scene *s, uint64_t seed, int px, int py, float *out) {
    const lambda_render_settings *rs = s->rs;
    pcg rng = pcg_new(seed, (uint64_t)py * (uint64_t)rs->width + (uint64_t)px);
    v3 color = V(0, 0, 0);
    v3 pos = load3(rs->camera.position), cor = load3(rs->camera.corner);
    v3 hor = load3(rs->camera.horizontal), ver = load3(rs->camera.vertical);
    for (int i = 0; i < rs->sqrt_samples; i++)
        for (int j = 0; j < rs->sqrt_samples; j++) {
            float u = ((float)px + ((float)i + rnd(&rng)) / (float)rs->sqrt_samples) / (float)rs->width;
            float v = ((float)py + ((float)j + rnd(&rng)) / (float)rs->sqrt_samples) / (float)rs->height;
            float l0 = rs->lambda_min + rnd(&rng) * (rs->lambda_max - rs->lambda_min);
            s4 lam;
            for (int k = 0; k < HERO; k++)
                lam.v[k] = rs->lambda_min + fmodf(l0 - rs->lambda_min + (float)k * s->range / HERO, s->range);
            v3 dir = nrm(sub(add(add(cor, scl(hor, u)), scl(ver, v)), pos));
            s4 L = trace(s, pos, dir, &lam, &rng);
            color = add(color, spectrum_to_rgb(&L, &lam, s->range));
        }
    color = dvs(color, (float)rs->samples);
    out[0] = color.x;
    out[1] = color.y;
    out[2] = color.z;
}

/* Renders rows [row0, row1) of the image into out (full image layout). */
void oracle_render_rows(const lambda_scene_desc *d, const lambda_render_settings *rs, uint64_t seed, int row0,
                        int row1, float *out) {
    Scene s = {d, rs, rs->lambda_max - rs->lambda_min};
#pragma omp parallel for schedule(guided)
    for (int py = row0; py < row1; py++)
        for (int px = 0; px < rs->width; px++) render_pixel(&s, seed, px, py, out + 3 * ((size_t)py * rs->width + px));
}

void oracle_render(const lambda_scene_desc *d, const lambda_render_settings *rs, uint64_t seed, float *out) {
    oracle_render_rows(d, rs, seed, 0, rs->height, out);
}

void oracle_hit(const lambda_scene_desc *d, const float *rays, int n, int32_t *inst, int32_t *obj, float *t) {
    lambda_render_settings rs;
    memset(&rs, 0, sizeof(rs));
    Scene s = {d, &rs, 1};
    for (int k = 0; k < n; k++) {
        Isect it = isect_init();
        int h = scene_hit(&s, load3(rays + 6 * k), load3(rays + 6 * k + 3), &it, -1, -2);
        inst[k] = h ? it.instance : -1;
        obj[k] = h ? it.object : -1;
        t[k] = it.t;
    }
}

void oracle_shadow(const lambda_scene_desc *d, const float *rays, const int32_t *li, const int32_t *lo, int n,
                   int32_t *occ) {
    lambda_render_settings rs;
    memset(&rs, 0, sizeof(rs));
    Scene s = {d, &rs, 1};
    for (int k = 0; k < n; k++) {
        Isect it = isect_init();
        occ[k] = scene_hit(&s, load3(rays + 6 * k), load3(rays + 6 * k + 3), &it, li[k], lo[k]);
    }
}

void oracle_pcg(uint64_t seed, uint64_t stream, int n, float *out) {
    pcg r = pcg_new(seed, stream);
    for (int i = 0; i < n; i++) out[i] = rnd(&r);
}

/* ---------------- surrogate MLP in FP64 (gradient checks) ----------------
 * 5 -> 64 -> 64 -> 64 -> 4, ReLU on hidden layers, linear output. Inputs are
 * normalised to [-1, 1] over the training range by the caller. Parameters in
 * the order W1[64][5] b1 W2[64][64] b2 W3[64][64] b3 W4[4][64] b4. */
#define H 64
static const int kIn = 5, kOut = 4;

/* Round to the nearest BF16 value (ties to even), as the tensor-core path stores
 * weights, inputs and hidden activations. */
static double bf16(double v) {
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return f;
}

static int g_round_bf16 = 0;

void oracle_mlp_set_bf16(int on) { g_round_bf16 = on; }

static void layer(const double *W, const double *b, const double *x, int nin, int nout, double *y, int relu) {
    for (int o = 0; o < nout; o++) {
        double a = b[o];
        for (int i = 0; i < nin; i++) a += (g_round_bf16 ? bf16(W[o * nin + i]) : W[o * nin + i]) * x[i];
        a = relu && a < 0 ? 0 : a;
        y[o] = relu && g_round_bf16 ? bf16(a) : a;
    }
}

void oracle_mlp_forward(const double *p, const double *x, int n, double *y) {
    const double *W1 = p, *b1 = W1 + H * kIn, *W2 = b1 + H, *b2 = W2 + H * H, *W3 = b2 + H, *b3 = W3 + H * H;
    const double *W4 = b3 + H, *b4 = W4 + kOut * H;
    for (int r = 0; r < n; r++) {
        double h1[H], h2[H], h3[H], xr[5];
        for (int i = 0; i < kIn; i++) xr[i] = g_round_bf16 ? bf16(x[kIn * r + i]) : x[kIn * r + i];
        layer(W1, b1, xr, kIn, H, h1, 1);
        layer(W2, b2, h1, H, H, h2, 1);
        layer(W3, b3, h2, H, H, h3, 1);
        layer(W4, b4, h3, H, kOut, y + kOut * r, 0);
    }
}

/* Mean squared error over n rows and 4 outputs, and its gradient w.r.t. p. */
double oracle_mlp_grad(const double *p, const double *x, const double *t, int n, double *g) {
    const int np = H * kIn + H + 2 * (H * H + H) + kOut * H + kOut;
    memset(g, 0, sizeof(double) * np);
    const double *W1 = p, *b1 = W1 + H * kIn, *W2 = b1 + H, *b2 = W2 + H * H, *W3 = b2 + H, *b3 = W3 + H * H;
    const double *W4 = b3 + H, *b4 = W4 + kOut * H;
    double *gW1 = g, *gb1 = gW1 + H * kIn, *gW2 = gb1 + H, *gb2 = gW2 + H * H, *gW3 = gb2 + H, *gb3 = gW3 + H * H;
    double *gW4 = gb3 + H, *gb4 = gW4 + kOut * H;
    double loss = 0;
    const double scale = 1.0 / ((double)n * kOut);
    for (int r = 0; r < n; r++) {
        double in[5];
        for (int i = 0; i < kIn; i++) in[i] = g_round_bf16 ? bf16(x[kIn * r + i]) : x[kIn * r + i];
        double h1[H], h2[H], h3[H], y[4], dy[4], d3[H], d2[H], d1[H];
        layer(W1, b1, in, kIn, H, h1, 1);
        layer(W2, b2, h1, H, H, h2, 1);
        layer(W3, b3, h2, H, H, h3, 1);
        layer(W4, b4, h3, H, kOut, y, 0);
        for (int o = 0; o < kOut; o++) {
            double e = y[o] - t[kOut * r + o];
            loss += e * e * scale;
            dy[o] = 2 * e * scale;
        }
        for (int o = 0; o < kOut; o++) {
            gb4[o] += dy[o];
            for (int i = 0; i < H; i++) gW4[o * H + i] += dy[o] * h3[i];
        }
        for (int i = 0; i < H; i++) {
            double a = 0;
            for (int o = 0; o < kOut; o++) a += (g_round_bf16 ? bf16(W4[o * H + i]) : W4[o * H + i]) * dy[o];
            d3[i] = h3[i] > 0 ? a : 0;
        }
        for (int o = 0; o < H; o++) {
            gb3[o] += d3[o];
            for (int i = 0; i < H; i++) gW3[o * H + i] += d3[o] * h2[i];
        }
        for (int i = 0; i < H; i++) {
            double a = 0;
            for (int o = 0; o < H; o++) a += (g_round_bf16 ? bf16(W3[o * H + i]) : W3[o * H + i]) * d3[o];
            d2[i] = h2[i] > 0 ? a : 0;
        }
        for (int o = 0; o < H; o++) {
            gb2[o] += d2[o];
            for (int i = 0; i < H; i++) gW2[o * H + i] += d2[o] * h1[i];
        }
        for (int i = 0; i < H; i++) {
            double a = 0;
            for (int o = 0; o < H; o++) a += (g_round_bf16 ? bf16(W2[o * H + i]) : W2[o * H + i]) * d2[o];
            d1[i] = h1[i] > 0 ? a : 0;
        }
        for (int o = 0; o < H; o++) {
            gb1[o] += d1[o];
            for (int i = 0; i < kIn; i++) gW1[o * kIn + i] += d1[o] * in[i];
        }
    }
    return loss;
}
