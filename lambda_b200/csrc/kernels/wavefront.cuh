// Wavefront path state and the per-stage kernels of one sample wave.
//
// A sample wave advances sample s of every pixel: pixel p's PCG32 stream is
// consumed in the reference's order (renderer.h:64-92, :94-195), so each pixel
// must finish sample s before it starts s+1, and the wave is the unit of
// parallelism (W*H paths in flight). Per bounce i the stages are
//   intersect  closest hit of every active path            (scene.h:51)
//   shade      miss/emitter terms, NEE light sampling, BSDF scatter, Russian
//              roulette; survivors and shadow rays are pushed to queues with one
//              atomic per warp (ballot + popc)                (renderer.h:101-191)
//   shadow     occlusion of the NEE rays and their radiance  (renderer.h:166-173)
// All path state is structure-of-arrays indexed by pixel; queues hold pixel ids.
#pragma once

#include <cstdint>

#include "dscene.cuh"
#include "tmm.cuh"

namespace lambda_dev {

// Queue push with one atomic per warp. Must be reached by all 32 lanes.
__device__ __forceinline__ int warp_push(int *counter, bool want) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return want ? base + __popc(mask & ((1u << lane) - 1u)) : -1;
}

__device__ __forceinline__ s4 hero_wavelengths(const RenderParams &rp, float lambda0) {
    s4 l;
    for (int k = 0; k < kHero; k++)
        l.v[k] = rp.lambda_min + fmodf(lambda0 - rp.lambda_min + float(k) * rp.lambda_range / kHero, rp.lambda_range);
    return l;
}

// Every pixel: seed its stream, zero film and radiance.
__global__ void k_init(RenderParams rp, PathState ps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= rp.num_pixels) return;
    ps.rng[p] = lambda_rng::pcg_seed(rp.seed, uint64_t(p));
    ps.film[p] = make_float4(0, 0, 0, 0);
    ps.radiance[p] = make_float4(0, 0, 0, 0);
    ps.lam[p] = make_float4(rp.lambda_min, rp.lambda_min, rp.lambda_min, rp.lambda_min);
    if (p == 0) {
        ps.wave[0] = 0;
        ps.wave[1] = 0;
    }
}

// Wave prologue (one block): fold the last wave's queue sizes into the
// statistics, clear the counters, advance the wave index.
__global__ void k_wave_prologue(int depth, PathState ps) {
    const int n = 2 * (depth + 2);
    __shared__ unsigned long long seg, sh;
    if (threadIdx.x == 0) {
        seg = 0;
        sh = 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int c = ps.counts[i];
        if (i < depth + 2) atomicAdd(&seg, (unsigned long long)c);
        else atomicAdd(&sh, (unsigned long long)c);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) ps.counts[i] = 0;
    if (threadIdx.x == 0) {
        ps.stats[0] += seg;
        ps.stats[1] += sh;
        ps.wave[1] = ps.wave[0];
        ps.wave[0] += 1;
    }
}

// Film += linear sRGB of the finished sample (renderer.h:84), then start the
// next sample: stratified jitter, hero wavelength, camera ray (renderer.h:69-81).
__global__ void k_raygen(RenderParams rp, DeviceScene sc, PathState ps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= rp.num_pixels) return;
    const int s = ps.wave[1];
    const int i = s / rp.sqrt_samples, j = s % rp.sqrt_samples;
    const int px = p % rp.width, py = p / rp.width;

    const f3 rgb = spectrum_to_rgb(sc, from_f4(ps.radiance[p]), from_f4(ps.lam[p]), rp.lambda_range);
    float4 film = ps.film[p];
    film.x += rgb.x;
    film.y += rgb.y;
    film.z += rgb.z;
    ps.film[p] = film;

    Rng rng{ps.rng[p], lambda_rng::pcg_increment(uint64_t(p))};
    const float u = (float(px) + (float(i) + rng.next()) / float(rp.sqrt_samples)) / float(rp.width);
    const float v = (float(py) + (float(j) + rng.next()) / float(rp.sqrt_samples)) / float(rp.height);
    const float lambda0 = rp.lambda_min + rng.next() * (rp.lambda_max - rp.lambda_min);
    const s4 lam = hero_wavelengths(rp, lambda0);
    const f3 dir = normalize(rp.cam_corner + rp.cam_h * u + rp.cam_v * v - rp.cam_pos);

    ps.rng[p] = rng.state;
    ps.lam[p] = to_f4(lam);
    ps.ray_o[p] = make_float4(rp.cam_pos.x, rp.cam_pos.y, rp.cam_pos.z, 1.0f);
    ps.ray_d[p] = make_float4(dir.x, dir.y, dir.z, 1.0f);
    ps.throughput[p] = make_float4(1, 1, 1, 1);
    ps.radiance[p] = make_float4(0, 0, 0, 0);
    ps.queue[0][p] = p;
    if (p == 0) ps.counts[0] = rp.num_pixels;
}

__global__ void __launch_bounds__(256) k_intersect(int bounce, DeviceScene sc, PathState ps) {
    const int n = ps.counts[bounce];
    const int *q = ps.queue[bounce & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const int p = q[idx];
        const float4 o = ps.ray_o[p], d = ps.ray_d[p];
        Hit h;
        bool overflow = false;
        if (closest_hit(sc, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), h, overflow)) {
            ps.hit_p[p] = make_float4(h.point.x, h.point.y, h.point.z, h.u);
            ps.hit_n[p] = make_float4(h.normal.x, h.normal.y, h.normal.z, h.v);
            ps.hit_id[p] = make_int4(h.instance, h.object, h.front ? 1 : 0, 0);
        } else {
            ps.hit_id[p] = make_int4(-1, -1, 0, 0);
        }
        if (overflow) atomicOr(ps.error, 1);
    }
}

// Material index of object `obj` in instance `inst` (instance.h:38).
__device__ __forceinline__ int material_of(const DeviceScene &sc, int inst_material, int obj) {
    return inst_material >= 0 ? inst_material : prim_material(load_prim(sc, obj));
}

// Thin-film reflectance (R_s + R_p) / 2 at one wavelength (material.h:263-309),
// FP32 transfer matrix. Layer order and thicknesses reverse on back-face hits.
__device__ inline float thin_film_r(const DeviceScene &sc, const int4 &m, bool front, float cos0, float lambda,
                             const float *thickness) {
    const int L = m.y < kMaxFilmLayers ? m.y : kMaxFilmLayers;
    cx<float> n[kMaxFilmLayers + 2];
    float d[kMaxFilmLayers];
    for (int k = 0; k < L + 2; k++) {
        const int src = front ? k : L + 1 - k;
        const double2 c = cspectrum_at(sc, sc.material_props[m.z + src], lambda);
        n[k] = cx<float>{float(c.x), float(c.y)};
    }
    for (int k = 0; k < L; k++) d[k] = thickness[front ? k : L - 1 - k];
    const FilmResult<float> r = film_stack<float, kMaxFilmLayers>(L, n, d, cos0, lambda);
    return (r.rs + r.rp) * 0.5f;
}

// powf(x, 5) of the dielectric's Schlick factor (material.h:186), formed in double
// and rounded once.
__device__ __forceinline__ float pow5(float x) {
    const double x2 = double(x) * double(x);
    return float(x2 * x2 * double(x));
}

__global__ void __launch_bounds__(256) k_shade(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    const int n = ps.counts[bounce];
    const int *q = ps.queue[bounce & 1];
    int *q_next = ps.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    // uniform trip count per warp so that the queue pushes below see all lanes
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        bool alive = false, nee = false;
        int p = 0;
        if (idx < n) {
            p = q[idx];
            const int4 id = ps.hit_id[p];
            float4 o4 = ps.ray_o[p], d4 = ps.ray_d[p];
            const f3 d = mk(d4.x, d4.y, d4.z);
            const float prev_pdf = o4.w;
            const bool specular = d4.w != 0.0f;
            s4 T = from_f4(ps.throughput[p]);
            s4 L = from_f4(ps.radiance[p]);
            const s4 lam = from_f4(ps.lam[p]);
            const bool lights = sc.total_light_power > 0;
            if (id.x < 0) {
                // miss: background with MIS against its NEE pdf (renderer.h:105-113)
                float w = 1;
                if (!specular && lights)
                    w = power_heuristic(prev_pdf, (1 / (4 * kPi)) * sc.light_power[sc.num_lights - 1] / sc.total_light_power);
                L = L + T * background_eval(sc, d, lam) * w;
                ps.radiance[p] = to_f4(L);
            } else {
                const float4 hp = ps.hit_p[p], hn = ps.hit_n[p];
                ShadePoint sp;
                sp.point = mk(hp.x, hp.y, hp.z);
                sp.u = hp.w;
                sp.v = hn.w;
                const f3 nrm = mk(hn.x, hn.y, hn.z);
                const bool front = id.z != 0;
                const InstanceRef ir = instance_ref(sc, id.x);
                const int4 ih = ir.header();
                const int mat = material_of(sc, ih.w, id.y);
                const int4 m = __ldg(&sc.materials[mat]);
                if (m.x == kEmissive) {
                    // emitter hit (renderer.h:119-131)
                    float w = 1;
                    if (!specular && lights) {
                        float M[16], Mi[16];
                        ir.load_m(M, 0);
                        ir.load_m(Mi, 1);
                        const Prim pr = load_prim(sc, id.y);
                        const f3 c0 = mk(M[0], M[4], M[8]);
                        const float light_power = prim_area(pr) * length_sq(c0) * sc.material_emission[mat];
                        const f3 o = mk(o4.x, o4.y, o4.z);
                        const float pdf = prim_pdf(pr, xform(Mi, o, 1), normalize(xform(Mi, d, 0)));
                        w = power_heuristic(prev_pdf, pdf * light_power / sc.total_light_power);
                    }
                    L = L + T * spectrum_texture4(sc, m.y, sp, lam) * w;
                    ps.radiance[p] = to_f4(L);
                } else {
                    Rng rng{ps.rng[p], lambda_rng::pcg_increment(uint64_t(p))};
                    s4 albedo = s4_fill(0);
                    if (m.x == kLambertian || m.x == kMirror) albedo = spectrum_texture4(sc, m.y, sp, lam);
                    // next-event estimation (renderer.h:133-175)
                    if (m.x == kLambertian && lights) {
                        const float target = sc.total_light_power * rng.next();
                        int li = sc.light_inst[0], lo = sc.light_obj[0];
                        float lp = sc.light_power[0];
                        for (int j = 0; j < sc.num_lights; j++) {
                            if (sc.light_cdf[j] >= target) {
                                li = sc.light_inst[j];
                                lo = sc.light_obj[j];
                                lp = sc.light_power[j];
                                break;
                            }
                        }
                        f3 ldir;
                        float lpdf;
                        if (li != -1) {
                            const InstanceRef lr = instance_ref(sc, li);
                            float M[16], Mi[16];
                            lr.load_m(M, 0);
                            lr.load_m(Mi, 1);
                            const Prim pr = load_prim(sc, lo);
                            const f3 lp_local = xform(Mi, sp.point, 1);
                            ldir = normalize(xform(M, prim_sample(pr, lp_local, rng), 0));
                            lpdf = prim_pdf(pr, lp_local, normalize(xform(Mi, ldir, 0)));
                        } else {
                            ldir = random_unit_vector(rng);
                            lpdf = 1 / (4 * kPi);
                        }
                        const float cos_t = dot(nrm, ldir);
                        if (lpdf > 0 && cos_t > 0) {
                            lpdf *= lp / sc.total_light_power;
                            // Lambertian evaluate/pdf toward the light (material.h:151-166)
                            const float cl = dot(nrm, ldir);
                            const s4 att = cl <= 0 ? s4_fill(0) : albedo / kPi;
                            const float spdf = cl > 0 ? cl / kPi : 0;
                            const float w = power_heuristic(lpdf, spdf);
                            const s4 a = (T * att) * cos_t;
                            ps.sh_o[p] = make_float4(sp.point.x, sp.point.y, sp.point.z, w);
                            ps.sh_d[p] = make_float4(ldir.x, ldir.y, ldir.z, lpdf);
                            ps.sh_a[p] = to_f4(a);
                            ps.sh_light[p] = make_int2(li, lo);
                            nee = true;
                        }
                    }
                    // BSDF sampling (material.h:117-261)
                    s4 att;
                    f3 nd;
                    float pdf = 0;
                    bool spec = true;
                    if (m.x == kLambertian) {
                        nd = random_in_hemisphere(nrm, rng);
                        const float cl = dot(nrm, nd);
                        att = cl <= 0 ? s4_fill(0) : albedo / kPi;
                        pdf = cl > 0 ? cl / kPi : 0;
                        spec = false;
                    } else if (m.x == kMirror) {
                        nd = reflected(d, nrm);
                        att = albedo;
                    } else if (m.x == kDielectric) {
                        const float factor = pow5(1 + dot(d, nrm));
                        const float n0h = spectrum_at(sc, m.y, lam.v[0]);
                        const float n1h = spectrum_at(sc, m.z, lam.v[0]);
                        const float ratio = front ? n0h / n1h : n1h / n0h;
                        float r0 = (n0h - n1h) / (n0h + n1h);
                        r0 *= r0;
                        const float rh = r0 + (1 - r0) * factor;
                        const bool refl = rng.next() < rh;
                        nd = refl ? reflected(d, nrm) : refracted(d, nrm, ratio);
                        att.v[0] = 1;
                        for (int k = 1; k < kHero; k++) {
                            const float a0 = spectrum_at(sc, m.y, lam.v[k]);
                            const float a1 = spectrum_at(sc, m.z, lam.v[k]);
                            float rr = (a0 - a1) / (a0 + a1);
                            rr *= rr;
                            const float r = rr + (1 - rr) * factor;
                            att.v[k] = refl ? r / rh
                                            : (fabsf(a0 - n0h) < kEps && fabsf(a1 - n1h) < kEps) ? (1 - r) / (1 - rh) : 0;
                        }
                    } else {  // thin film (material.h:228-261)
                        const int Lc = m.y < kMaxFilmLayers ? m.y : kMaxFilmLayers;
                        float thick[kMaxFilmLayers];
                        for (int k = 0; k < Lc; k++) thick[k] = scalar_texture(sc, sc.material_props[m.w + k], sp.point);
                        const float cos0 = dot(nrm, -d);
                        const int outer = sc.material_props[m.z], sub = sc.material_props[m.z + m.y + 1];
                        const float n0h = float(cspectrum_at(sc, outer, lam.v[0]).x);
                        const float n1h = float(cspectrum_at(sc, sub, lam.v[0]).x);
                        const float ratio = front ? n0h / n1h : n1h / n0h;
                        const float rh = thin_film_r(sc, m, front, cos0, lam.v[0], thick);
                        const bool refl = rng.next() < rh;
                        nd = refl ? reflected(d, nrm) : refracted(d, nrm, ratio);
                        att.v[0] = 1;
                        for (int k = 1; k < kHero; k++) {
                            const float a0 = float(cspectrum_at(sc, outer, lam.v[k]).x);
                            const float a1 = float(cspectrum_at(sc, sub, lam.v[k]).x);
                            const float r = thin_film_r(sc, m, front, cos0, lam.v[k], thick);
                            att.v[k] = refl ? r / rh
                                            : (fabsf(a0 - n0h) < kEps && fabsf(a1 - n1h) < kEps) ? (1 - r) / (1 - rh) : 0;
                        }
                    }
                    if (spec) T = T * att;
                    else T = T * ((att * dot(nrm, nd)) / pdf);
                    alive = true;
                    if (bounce >= kRrStartDepth) {
                        const float qq = 1 - clampf(s4_max(T), 0.05f, 0.95f);
                        if (rng.next() < qq) alive = false;
                        else T = T / (1 - qq);
                    }
                    if (bounce >= rp.depth) alive = false;
                    ps.rng[p] = rng.state;
                    ps.throughput[p] = to_f4(T);
                    ps.ray_o[p] = make_float4(sp.point.x, sp.point.y, sp.point.z, pdf);
                    ps.ray_d[p] = make_float4(nd.x, nd.y, nd.z, spec ? 1.0f : 0.0f);
                }
            }
        }
        const int slot = warp_push(&ps.counts[bounce + 1], alive);
        if (alive) q_next[slot] = p;
        const int sslot = warp_push(&ps.counts[rp.depth + 2 + bounce], nee);
        if (nee) ps.shadow_queue[sslot] = p;
    }
}

__global__ void __launch_bounds__(256) k_shadow(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    const int n = ps.counts[rp.depth + 2 + bounce];
    const int stride = gridDim.x * blockDim.x;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const int p = ps.shadow_queue[idx];
        const float4 o = ps.sh_o[p], dd = ps.sh_d[p];
        const int2 light = ps.sh_light[p];
        const f3 d = mk(dd.x, dd.y, dd.z);
        Hit lh;
        bool overflow = false;
        if (!occluded(sc, mk(o.x, o.y, o.z), d, light.x, light.y, lh, overflow)) {
            const s4 lam = from_f4(ps.lam[p]);
            s4 e;
            if (light.x != -1) {
                const int4 ih = instance_ref(sc, light.x).header();
                const int mat = material_of(sc, ih.w, light.y);
                const int4 m = __ldg(&sc.materials[mat]);
                ShadePoint sp;
                sp.point = lh.point;
                sp.u = lh.u;
                sp.v = lh.v;
                e = m.x == kEmissive ? spectrum_texture4(sc, m.y, sp, lam) : s4_fill(0);
            } else {
                e = background_eval(sc, d, lam);
            }
            const s4 a = from_f4(ps.sh_a[p]);
            const s4 contrib = ((a * e) * o.w) / dd.w;
            ps.radiance[p] = to_f4(from_f4(ps.radiance[p]) + contrib);
        }
        if (overflow) atomicOr(ps.error, 1);
    }
}

// Last sample into the film, then the average (renderer.h:84-91).
__global__ void k_finish(RenderParams rp, DeviceScene sc, PathState ps, float *out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= rp.num_pixels) return;
    const f3 rgb = spectrum_to_rgb(sc, from_f4(ps.radiance[p]), from_f4(ps.lam[p]), rp.lambda_range);
    float4 film = ps.film[p];
    film.x += rgb.x;
    film.y += rgb.y;
    film.z += rgb.z;
    const float inv = float(rp.samples);
    out[3 * size_t(p)] = film.x / inv;
    out[3 * size_t(p) + 1] = film.y / inv;
    out[3 * size_t(p) + 2] = film.z / inv;
}

}  // namespace lambda_dev
