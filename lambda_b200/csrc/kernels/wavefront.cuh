// Wavefront path state and the per-stage kernels of one sample wave.
//
// A sample wave advances sample s of every pixel: pixel p's PCG32 stream is
// consumed in the reference's order (renderer.h:64-92, :94-195), so each pixel
// must finish sample s before it starts s+1, and the wave is the unit of
// parallelism (W*H paths in flight). Per bounce i the stages are
//   intersect   closest hit of every active path (scene.h:51); misses and emitter
//               hits are finished on the spot (renderer.h:105-131), the rest are
//               pushed to one queue per material family
//   lambert     NEE light sampling + cosine scatter + Russian roulette (renderer.h:133-191)
//   specular    mirror and dielectric scatter + Russian roulette
//   thin film   transfer-matrix reflectance of the four hero wavelengths, scatter
//   shadow      occlusion of the NEE rays and their radiance (renderer.h:166-173)
// so every kernel runs one material's code over a coherent batch. A sample's last
// term, the emission of the miss or emitter that ends it, is kept apart (emit) and
// added to the NEE terms (radiance) when the sample is banked: that is the
// reference's order of additions (renderer.h:105-131 comes after the previous
// bounce's NEE), and it lets bounce i's shadow rays run beside bounce i+1's
// intersect. Queue pushes
// cost one atomic per warp (ballot + popc). All path state is structure-of-arrays
// indexed by pixel; queues hold pixel ids.
#pragma once

#include <cstdint>

#include "dscene.cuh"
#include "tmm.cuh"

namespace lambda_dev {

// Translation units that only need the device helpers define
// LAMBDA_WAVEFRONT_HELPERS_ONLY; the kernels then get internal linkage there.
#ifdef LAMBDA_WAVEFRONT_HELPERS_ONLY
#define LAMBDA_KERNEL static __global__
#else
#define LAMBDA_KERNEL __global__
#endif

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

__device__ __forceinline__ s4 hero_wavelengths(const Job &job, float lambda0) {
    s4 l;
    for (int k = 0; k < kHero; k++)
        l.v[k] = job.lambda_min + fmodf(lambda0 - job.lambda_min + float(k) * job.lambda_range / kHero, job.lambda_range);
    return l;
}

// Index of the job that owns virtual pixel p (jobs ordered by base).
__device__ __forceinline__ int job_of(const RenderParams &rp, int p) {
    int lo = 0, hi = rp.num_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rp.jobs[mid].base <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The job-local pixel taken l-th when warps are to cover 8x4 tiles: the image is cut
// into bands of 4 rows and each band into blocks of 8 columns (the last ones
// narrower), row-major inside a block. A bijection of [0, width * height), so it
// changes which thread or queue slot takes a pixel, never the pixel's arithmetic.
__device__ __forceinline__ int tile_order(const Job &job, int l) {
    const int w = job.width;
    const int band = l / (4 * w);
    const int hb = min(4, job.height - 4 * band);
    const int r = l - band * 4 * w;
    const int cx = r / (8 * hb);
    const int rr = r - cx * 8 * hb;
    const int bw = min(8, w - 8 * cx);
    return (4 * band + rr / bw) * w + 8 * cx + rr % bw;
}

// Pixel p of `job`: seed its stream (job seed, job-local pixel index, as a render
// of that job alone), record its depth limit, zero film and radiance.
__device__ __forceinline__ void init_pixel(const PathState &ps, int p, const Job &job) {
    const int local = p - job.base;
    ps.rng[p] = lambda_rng::pcg_seed(job.seed, uint64_t(local));
    ps.path_info[p] = make_int2(local, job.depth);
    ps.film[p] = make_float4(0, 0, 0, 0);
    ps.radiance[p] = make_float4(0, 0, 0, 0);
    ps.emit[p] = make_float4(0, 0, 0, 0);
    ps.lam[p] = make_float4(job.lambda_min, job.lambda_min, job.lambda_min, job.lambda_min);
}

// Every pixel of the pass: init_pixel, and the wave counters.
LAMBDA_KERNEL void k_init(RenderParams rp, PathState ps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= rp.num_pixels) return;
    init_pixel(ps, p, rp.jobs[job_of(rp, p)]);
    if (p == 0) {
        ps.wave[0] = 0;
        ps.wave[1] = 0;
    }
}

// Wave prologue (one block): fold the last wave's queue sizes into the
// statistics, clear the counters, advance the wave index. Inside a graph's
// sample-wave loop (waves > 0) it also sets the loop condition, true while waves
// remain after the one starting now, so the loop runs exactly `waves` times, and
// publishes the number of waves started to `progress` (mapped host memory).
LAMBDA_KERNEL void k_wave_prologue(int depth, PathState ps, cudaGraphConditionalHandle loop, int waves, int *progress) {
    const int n = kQueues * (depth + 2);
    __shared__ unsigned long long tot[kQueues];
    if (threadIdx.x < kQueues) tot[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&tot[i % kQueues], (unsigned long long)ps.counts[i]);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) ps.counts[i] = 0;
    if (threadIdx.x == 0) {
        // stats: segments, NEE rays, thin-film hits, (fallback), Lambertian hits, specular hits
        ps.stats[0] += tot[kQActive];
        ps.stats[1] += tot[kQShadow];
        ps.stats[2] += tot[kQFilm];
        ps.stats[3] += tot[kQFilmFallback];
        ps.stats[4] += tot[kQLambert];
        ps.stats[5] += tot[kQSpecular];
        ps.wave[1] = ps.wave[0];
        const int started = ps.wave[0] + 1;
        ps.wave[0] = started;
        if (waves > 0) {
            cudaGraphSetConditional(loop, started < waves ? 1u : 0u);
            if (progress) *reinterpret_cast<volatile int *>(progress) = started;
        }
    }
}

// Radiance of a finished sample: its NEE terms, then the emission that ended it.
__device__ __forceinline__ s4 sample_radiance(const PathState &ps, int p) {
    return from_f4(ps.radiance[p]) + from_f4(ps.emit[p]);
}

// Film += linear sRGB of pixel p's finished sample (renderer.h:84).
__device__ __forceinline__ void bank_sample(const DeviceScene &sc, const PathState &ps, int p, const Job &job) {
    const f3 rgb = spectrum_to_rgb(sc, sample_radiance(ps, p), from_f4(ps.lam[p]), job.lambda_range);
    float4 film = ps.film[p];
    film.x += rgb.x;
    film.y += rgb.y;
    film.z += rgb.z;
    ps.film[p] = film;
}

// Sample s of pixel p: stratified jitter, hero wavelength and camera ray
// (renderer.h:69-81), unit throughput, no radiance yet.
__device__ __forceinline__ void start_sample(const PathState &ps, int p, const Job &job, int s) {
    const int local = p - job.base;
    const int i = s / job.sqrt_samples, j = s % job.sqrt_samples;
    const int px = local % job.width, py = local / job.width;
    Rng rng = pixel_rng(ps.rng[p], local);
    const float u = (float(px) + (float(i) + rng.next()) / float(job.sqrt_samples)) / float(job.width);
    const float v = (float(py) + (float(j) + rng.next()) / float(job.sqrt_samples)) / float(job.height);
    const float lambda0 = job.lambda_min + rng.next() * (job.lambda_max - job.lambda_min);
    const s4 lam = hero_wavelengths(job, lambda0);
    const f3 dir = normalize(job.cam_corner + job.cam_h * u + job.cam_v * v - job.cam_pos);

    ps.rng[p] = rng.state;
    ps.lam[p] = to_f4(lam);
    ps.ray_o[p] = make_float4(job.cam_pos.x, job.cam_pos.y, job.cam_pos.z, 1.0f);
    ps.ray_d[p] = make_float4(dir.x, dir.y, dir.z, 1.0f);
    ps.throughput[p] = make_float4(1, 1, 1, 1);
    ps.radiance[p] = make_float4(0, 0, 0, 0);
    ps.emit[p] = make_float4(0, 0, 0, 0);
}

// Banks the finished sample of every pixel, then starts the next one.
// Pixels of jobs whose last sample was the previous wave only bank that sample.
LAMBDA_KERNEL void k_raygen(RenderParams rp, DeviceScene sc, PathState ps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = ps.wave[1];
    const int n_now = rp.active[s];
    const int n_prev = s > 0 ? rp.active[s - 1] : n_now;
    if (p == 0) ps.counts[queue_slot(0, kQActive)] = n_now;
    if (p >= n_prev) return;
    const Job &job = rp.jobs[job_of(rp, p)];
    bank_sample(sc, ps, p, job);
    if (p >= n_now) {
        ps.radiance[p] = make_float4(0, 0, 0, 0);
        ps.emit[p] = make_float4(0, 0, 0, 0);
        return;
    }
    start_sample(ps, p, job, s);
    // the first intersect takes the wave's paths tile by tile
    ps.queue[0][p] = job.base + tile_order(job, p - job.base);
}

// Material index of object `obj` in instance `inst` (instance.h:38).
__device__ __forceinline__ int material_of(const DeviceScene &sc, int inst_material, int obj) {
    return inst_material >= 0 ? inst_material : prim_material(load_prim(sc, obj));
}

// Closest hit of path p (renderer.h:94-131). A miss or an emitter hit records the
// path's emission term and returns -1: the path ends. Any other hit is stored for the
// shade kernels and its material family returned: 0 Lambertian, 1 mirror or
// dielectric, 2 thin film. The stored hit is (material, object, distance, instance)
// alone: load_shade rebuilds the hit point, normal, (u, v) and facing from it with
// the same functions, so the traversal kernels leave that work, and its bytes, to
// the hits' shading kernels.
__device__ __forceinline__ int trace_finish(const DeviceScene &sc, const PathState &ps, int p, const float4 &o4,
                                            const float4 &d4, const Ray3 &wr, float best, int obj, int inst);

template <int K>
__device__ __forceinline__ int trace_path(const DeviceScene &sc, const PathState &ps, int p, const WideStack &st_a,
                                          const WideStack &st_b) {
    const float4 o4 = ps.ray_o[p], d4 = ps.ray_d[p];
    const Ray3 wr = make_ray(mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z));
    float best;
    int obj, inst;
    bool overflow = false;
    closest_hit_ids_w<K>(sc, wr, best, obj, inst, overflow, st_a, st_b);
    if (overflow) atomicOr(ps.error, 1);
    return trace_finish(sc, ps, p, o4, d4, wr, best, obj, inst);
}

// What trace_path does with path p's closest hit (ray o4, d4 = wr; best, obj, inst
// from the traversal, obj < 0 on a miss): a miss or an emitter hit records the
// emission term and returns -1; any other hit is stored and its material family
// returned.
__device__ __forceinline__ int trace_finish(const DeviceScene &sc, const PathState &ps, int p, const float4 &o4,
                                            const float4 &d4, const Ray3 &wr, float best, int obj, int inst) {
    const f3 o = mk(o4.x, o4.y, o4.z), d = mk(d4.x, d4.y, d4.z);
    const bool specular = d4.w != 0.0f;
    const float prev_pdf = o4.w;
    const bool lights = sc.total_light_power > 0;
    if (obj < 0) {
        const s4 lam = from_f4(ps.lam[p]);
        float w = 1;
        if (!specular && lights)
            w = power_heuristic(prev_pdf, (1 / (4 * kPi)) * sc.light_power[sc.num_lights - 1] / sc.total_light_power);
        const s4 T = from_f4(ps.throughput[p]);
        ps.emit[p] = to_f4(T * background_eval(sc, d, lam) * w);
        return -1;
    }
    const InstanceRef ir = instance_ref(sc, inst);
    const int4 ih = ir.header();
    const int mat = material_of(sc, ih.w, obj);
    const int4 m = __ldg(&sc.materials[mat]);
    if (m.x == kEmissive) {
        Hit h;
        closest_hit_finish(sc, wr, best, obj, inst, h);
        float w = 1;
        if (!specular && lights) {
            float M[16], Mi[16];
            ir.load_m(M, 0);
            ir.load_m(Mi, 1);
            const Prim pr = load_prim(sc, obj);
            const f3 c0 = mk(M[0], M[4], M[8]);
            const float light_power = prim_area(pr) * length_sq(c0) * sc.material_emission[mat];
            const float pdf = prim_pdf(pr, xform(Mi, o, 1), normalize(xform(Mi, d, 0)));
            w = power_heuristic(prev_pdf, pdf * light_power / sc.total_light_power);
        }
        ShadePoint sp;
        sp.point = h.point;
        sp.u = h.u;
        sp.v = h.v;
        const s4 lam = from_f4(ps.lam[p]);
        const s4 T = from_f4(ps.throughput[p]);
        ps.emit[p] = to_f4(T * spectrum_texture4(sc, m.y, sp, lam) * w);
        return -1;
    }
    ps.hit_id[p] = make_int4(mat, obj, __float_as_int(best), inst);
    return m.x == kLambertian ? 0 : (m.x == kThinFilm ? 2 : 1);
}

// Closest hit; misses and emitter hits record their emission term and end the
// path (renderer.h:105-131); other hits go to their material's queue.
template <int K>
LAMBDA_KERNEL void __launch_bounds__(256, 4) k_intersect(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    extern __shared__ int stack_smem[];
    WideStack st_a, st_b;
    wide_stacks(stack_smem, sc, st_a, st_b);
    const int n = ps.counts[queue_slot(bounce, kQActive)];
    const int *q = ps.queue[bounce & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        int p = 0, family = -1;
        if (idx < n) {
            p = q[idx];
            family = trace_path<K>(sc, ps, p, st_a, st_b);
        }
        for (int f = 0; f < 3; f++) {
            const int slot = warp_push(&ps.counts[queue_slot(bounce, kQLambert + f)], family == f);
            if (family == f) ps.mat_queue[f][slot] = p;
        }
    }
}

// Closest hits of the bounce's queue with rays taken lane by lane. Each lane keeps its
// traversal (stacks, instance-space ray, best hit) across iterations of one loop and
// advances it by one stack entry per iteration, in the order closest_hit_w visits
// them, so its hits are closest_hit_w's bit for bit. A lane whose ray is done
// finishes it as trace_path does, pushes it to its material queue with the lanes that
// finish at the same step, and takes the next ray from the queue's fetch counter at
// once. Lanes on different rays then step together instead of waiting for a warp's
// longest ray. The loop ends when the queue is drained: every iteration pops an
// entry, finishes a ray or takes one.
template <int K>
LAMBDA_KERNEL void __launch_bounds__(256, 2) k_intersect_fetch(int bounce, RenderParams rp, DeviceScene sc,
                                                               PathState ps) {
    extern __shared__ int stack_smem[];
    WideStack st, sub;
    wide_stacks(stack_smem, sc, st, sub);
    const int n = ps.counts[queue_slot(bounce, kQActive)];
    const int *q = ps.queue[bounce & 1];
    int *next = &ps.counts[queue_slot(bounce, kQFetch)];
    const int lane = threadIdx.x & 31;
    int p = -1;
    Ray3 wr, lr;
    float best = kMax;
    int best_obj = -1, best_inst = -1, inst = -1, sp = 0, ssp = 0;
    bool overflow = false;
    for (;;) {
        if (p < 0) {
            // the lanes that need a ray take consecutive entries, one atomic per group
            const unsigned need = __activemask();
            const int leader = __ffs(need) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(next, __popc(need));
            base = __shfl_sync(need, base, leader);
            const int idx = base + __popc(need & ((1u << lane) - 1u));
            if (idx >= n) break;
            p = q[idx];
            const float4 o4 = ps.ray_o[p], d4 = ps.ray_d[p];
            wr = make_ray(mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z));
            best = kMax;
            best_obj = best_inst = -1;
            sp = ssp = 0;
            overflow = false;
            float te;
            if (slab(__ldg(&sc.nodes[0]), __ldg(&sc.nodes[1]), wr, te))
                st.put(sp++, root_entry<K>(sc, __ldg(&sc.wide_code[0])), te);
        } else if (ssp > 0 && !overflow) {
            // one BLAS entry
            --ssp;
            float te2 = sub.te[ssp * sub.stride];
            const int c2 = pop_code<K>(sc, sub.code[ssp * sub.stride], te2, lr, best);
            if (c2 != INT_MIN) {
                if (c2 >= 0) {
                    ssp = wide_expand<K>(sc, c2, lr, best, sub, ssp, overflow);
                } else {
                    const int2 lf = __ldg(&sc.wide_leaves[-c2 - 1]);
                    for (int k = 0; k < lf.y; k++) {
                        const float t = intersect_t(load_prim(sc, lf.x + k), lr, best);
                        if (t >= 0) {
                            best = t;
                            best_obj = lf.x + k;
                            best_inst = inst;
                        }
                    }
                }
            }
        } else if (sp > 0 && !overflow) {
            // one TLAS entry; a leaf starts its instance's BLAS (the first instance only)
            --sp;
            float te = st.te[sp * st.stride];
            const int code = pop_code<K>(sc, st.code[sp * st.stride], te, wr, best);
            if (code != INT_MIN) {
                if (code >= 0) {
                    sp = wide_expand<K>(sc, code, wr, best, st, sp, overflow);
                } else {
                    inst = __ldg(&sc.wide_leaves[-code - 1]).x;
                    const uint32_t flags = sc.instance_flags[inst];
                    const InstanceRef ir = instance_ref(sc, inst);
                    const int root = ir.header().z;
                    lr = to_local(flags, ir, wr);
                    if ((flags & 2u) ||
                        (slab(__ldg(&sc.nodes[2 * root]), __ldg(&sc.nodes[2 * root + 1]), lr, te) && !(te > best)))
                        sub.put(ssp++, root_entry<K>(sc, __ldg(&sc.wide_code[root])), te);
                }
            }
        } else {
            // the ray is done (or a stack overflowed): finish it and push it
            if (overflow) atomicOr(ps.error, 1);
            const int family = trace_finish(sc, ps, p, ps.ray_o[p], ps.ray_d[p], wr, best, best_obj, best_inst);
            if (family >= 0) {
                const unsigned grp = __match_any_sync(__activemask(), family);
                const int leader = __ffs(grp) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(&ps.counts[queue_slot(bounce, kQLambert + family)], __popc(grp));
                base = __shfl_sync(grp, base, leader);
                ps.mat_queue[family][base + __popc(grp & ((1u << lane) - 1u))] = p;
            }
            p = -1;
        }
    }
}

// Per-path state a shade kernel works on.
struct ShadeIn {
    int p;
    f3 d;
    ShadePoint sp;
    f3 nrm;
    bool front;
    int4 m;
    int mat;  // the material's index
    s4 T, lam;
};

// The path's PCG32: its state and its stream, the job-local pixel index.
__device__ __forceinline__ Rng path_rng(const PathState &ps, int p) { return pixel_rng(ps.rng[p], ps.path_info[p].x); }

__device__ __forceinline__ ShadeIn load_shade(const PathState &ps, const DeviceScene &sc, int p) {
    ShadeIn s;
    s.p = p;
    const float4 o4 = ps.ray_o[p], d4 = ps.ray_d[p];
    s.d = mk(d4.x, d4.y, d4.z);
    // the hit record from (object, distance, instance), as closest_hit_w makes it
    const int4 id = ps.hit_id[p];
    Hit h;
    closest_hit_finish(sc, make_ray(mk(o4.x, o4.y, o4.z), s.d), __int_as_float(id.z), id.y, id.w, h);
    s.sp.point = h.point;
    s.sp.u = h.u;
    s.sp.v = h.v;
    s.nrm = h.normal;
    s.front = h.front;
    s.m = __ldg(&sc.materials[id.x]);
    s.mat = id.x;
    s.T = from_f4(ps.throughput[p]);
    s.lam = from_f4(ps.lam[p]);
    return s;
}

// Throughput update, Russian roulette and the depth limit (renderer.h:177-191);
// writes the scattered ray and returns whether the path continues.
__device__ __forceinline__ bool finish_scatter(const PathState &ps, const ShadeIn &s, Rng &rng, int bounce, s4 att, f3 nd,
                                               float pdf, bool spec) {
    s4 T = s.T;
    if (spec) T = T * att;
    else T = T * ((att * dot(s.nrm, nd)) / pdf);
    bool alive = true;
    if (bounce >= kRrStartDepth) {
        const float qq = 1 - clampf(s4_max(T), 0.05f, 0.95f);
        if (rng.next() < qq) alive = false;
        else T = T / (1 - qq);
    }
    if (bounce >= ps.path_info[s.p].y) alive = false;  // the depth limit of the path's job
    ps.rng[s.p] = rng.state;
    ps.throughput[s.p] = to_f4(T);
    ps.ray_o[s.p] = make_float4(s.sp.point.x, s.sp.point.y, s.sp.point.z, pdf);
    ps.ray_d[s.p] = make_float4(nd.x, nd.y, nd.z, spec ? 1.0f : 0.0f);
    return alive;
}

// Lambertian hit of path p: next-event estimation (renderer.h:133-175), leaving the
// NEE ray in the path state and setting `nee`, then cosine-weighted scatter
// (material.h:151-172). Returns whether the path continues.
__device__ __forceinline__ bool lambert_path(const DeviceScene &sc, const PathState &ps, int p, int bounce, bool &nee) {
    const ShadeIn s = load_shade(ps, sc, p);
    Rng rng = path_rng(ps, p);
    const s4 albedo = spectrum_texture4(sc, s.m.y, s.sp, s.lam);
    if (sc.total_light_power > 0) {
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
            const Prim pr = load_prim(sc, lo);
            if (sc.instance_flags[li] & 1u) {
                const f3 zero = mk(0.0f, 0.0f, 0.0f);
                const f3 local = s.sp.point + zero;
                ldir = normalize(prim_sample(pr, local, rng) + zero);
                lpdf = prim_pdf(pr, local, normalize(ldir + zero));
            } else {
                const InstanceRef lr = instance_ref(sc, li);
                float M[16], Mi[16];
                lr.load_m(M, 0);
                lr.load_m(Mi, 1);
                const f3 local = xform(Mi, s.sp.point, 1);
                ldir = normalize(xform(M, prim_sample(pr, local, rng), 0));
                lpdf = prim_pdf(pr, local, normalize(xform(Mi, ldir, 0)));
            }
        } else {
            ldir = random_unit_vector(rng);
            lpdf = 1 / (4 * kPi);
        }
        const float cos_t = dot(s.nrm, ldir);
        if (lpdf > 0 && cos_t > 0) {
            lpdf *= lp / sc.total_light_power;
            const s4 att = cos_t <= 0 ? s4_fill(0) : albedo / kPi;
            const float spdf = cos_t > 0 ? cos_t / kPi : 0;
            const float w = power_heuristic(lpdf, spdf);
            ps.sh_o[p] = make_float4(s.sp.point.x, s.sp.point.y, s.sp.point.z, w);
            ps.sh_d[p] = make_float4(ldir.x, ldir.y, ldir.z, lpdf);
            ps.sh_a[p] = to_f4((s.T * att) * cos_t);
            ps.sh_light[p] = make_int2(li, lo);
            nee = true;
        }
    }
    const f3 nd = random_in_hemisphere(s.nrm, rng);
    const float cl = dot(s.nrm, nd);
    const s4 att = cl <= 0 ? s4_fill(0) : albedo / kPi;
    const float pdf = cl > 0 ? cl / kPi : 0;
    return finish_scatter(ps, s, rng, bounce, att, nd, pdf, false);
}

// Lambertian: next-event estimation (renderer.h:133-175), then cosine-weighted
// scatter (material.h:151-172).
LAMBDA_KERNEL void __launch_bounds__(256, 3) k_shade_lambert(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    const int n = ps.counts[queue_slot(bounce, kQLambert)];
    const int *q = ps.mat_queue[0];
    int *q_next = ps.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        bool alive = false, nee = false;
        int p = 0;
        if (idx < n) {
            p = q[idx];
            alive = lambert_path(sc, ps, p, bounce, nee);
        }
        const int slot = warp_push(&ps.counts[queue_slot(bounce + 1, kQActive)], alive);
        if (alive) q_next[slot] = p;
        const int sslot = warp_push(&ps.counts[queue_slot(bounce, kQShadow)], nee);
        if (nee) ps.shadow_queue[sslot] = p;
    }
}

// powf(x, 5) of the dielectric's Schlick factor (material.h:186), formed in double
// and rounded once.
__device__ __forceinline__ float pow5(float x) {
    const double x2 = double(x) * double(x);
    return float(x2 * x2 * double(x));
}

// Mirror or dielectric hit of path p (material.h:174-226). Returns whether the path
// continues.
__device__ __forceinline__ bool specular_path(const DeviceScene &sc, const PathState &ps, int p, int bounce) {
    const ShadeIn s = load_shade(ps, sc, p);
    Rng rng = path_rng(ps, p);
    s4 att;
    f3 nd;
    if (s.m.x == kMirror) {
        nd = reflected(s.d, s.nrm);
        att = spectrum_texture4(sc, s.m.y, s.sp, s.lam);
    } else {
        const float factor = pow5(1 + dot(s.d, s.nrm));
        const float n0h = spectrum_at(sc, s.m.y, s.lam.v[0]);
        const float n1h = spectrum_at(sc, s.m.z, s.lam.v[0]);
        const float ratio = s.front ? n0h / n1h : n1h / n0h;
        float r0 = (n0h - n1h) / (n0h + n1h);
        r0 *= r0;
        const float rh = r0 + (1 - r0) * factor;
        const bool refl = rng.next() < rh;
        nd = refl ? reflected(s.d, s.nrm) : refracted(s.d, s.nrm, ratio);
        att.v[0] = 1;
        for (int k = 1; k < kHero; k++) {
            const float a0 = spectrum_at(sc, s.m.y, s.lam.v[k]);
            const float a1 = spectrum_at(sc, s.m.z, s.lam.v[k]);
            float rr = (a0 - a1) / (a0 + a1);
            rr *= rr;
            const float r = rr + (1 - rr) * factor;
            att.v[k] = refl ? r / rh : (fabsf(a0 - n0h) < kEps && fabsf(a1 - n1h) < kEps) ? (1 - r) / (1 - rh) : 0;
        }
    }
    return finish_scatter(ps, s, rng, bounce, att, nd, 0, true);
}

// Mirror and dielectric (material.h:174-226).
LAMBDA_KERNEL void __launch_bounds__(256) k_shade_specular(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    const int n = ps.counts[queue_slot(bounce, kQSpecular)];
    const int *q = ps.mat_queue[1];
    int *q_next = ps.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        bool alive = false;
        int p = 0;
        if (idx < n) {
            p = q[idx];
            alive = specular_path(sc, ps, p, bounce);
        }
        const int slot = warp_push(&ps.counts[queue_slot(bounce + 1, kQActive)], alive);
        if (alive) q_next[slot] = p;
    }
}

// Thin-film reflectance (R_s + R_p) / 2 at the four hero wavelengths
// (material.h:263-309), FP32 transfer matrix. Layer order and thicknesses
// reverse on back-face hits. With non-dispersive indices the interfaces are
// formed once for all four wavelengths.
__device__ inline s4 thin_film_r4(const DeviceScene &sc, const int4 &m, bool front, float cos0, const s4 &lam,
                                  const float *thickness, float4 ff = make_float4(0, 0, 0, 0)) {
    const int L = m.y < kMaxFilmLayers ? m.y : kMaxFilmLayers;
    if (ff.w != 0.0f) {
        // one film with real, non-dispersive indices (film_flat): the values every
        // spectrum lookup below would return
        cx<float> n[3] = {{front ? ff.x : ff.z, 0.0f}, {ff.y, 0.0f}, {front ? ff.z : ff.x, 0.0f}};
        FilmPrep<float, 1> f;
        film_prepare<float, 1>(1, n, cos0, f);
        s4 R;
#pragma unroll 1
        for (int w = 0; w < kHero; w++) {
            const FilmResult<float> r = film_apply<float, 1>(f, thickness, (2 * kPi) / lam.v[w], false);
            R.v[w] = (r.rs + r.rp) * 0.5f;
        }
        return R;
    }
    bool flat = true;
    for (int k = 0; k < L + 2; k++) flat = flat && sc.cspectrum_flat[sc.material_props[m.z + k]];
    s4 R;
    if (flat && L <= 1) {
        cx<float> n[3];
        for (int k = 0; k < L + 2; k++) {
            const int src = front ? k : L + 1 - k;
            const double2 c = cspectrum_at(sc, sc.material_props[m.z + src], lam.v[0]);
            n[k] = cx<float>{float(c.x), float(c.y)};
        }
        FilmPrep<float, 1> f;
        film_prepare<float, 1>(L, n, cos0, f);
#pragma unroll 1
        for (int w = 0; w < kHero; w++) {
            const FilmResult<float> r = film_apply<float, 1>(f, thickness, (2 * kPi) / lam.v[w], false);
            R.v[w] = (r.rs + r.rp) * 0.5f;
        }
        return R;
    }
    float d[kMaxFilmLayers];
    for (int k = 0; k < L; k++) d[k] = thickness[front ? k : L - 1 - k];
#pragma unroll 1
    for (int w = 0; w < kHero; w++) {
        const float lambda = lam.v[w];
        auto index_of = [&](int k) {
            const int src = front ? k : L + 1 - k;
            const double2 c = cspectrum_at(sc, sc.material_props[m.z + src], lambda);
            return cx<float>{float(c.x), float(c.y)};
        };
        R.v[w] = film_reflectance_stream<float>(L, index_of, d, cos0, (2 * kPi) / lambda);
    }
    return R;
}

// Thin-film reflectance as the reference evaluates it (material.h:263-309): complex
// double characteristic matrices from the complex spectra, k = 2 pi / lambda formed
// in float, |r| rounded to float and squared in float.
__device__ inline s4 thin_film_r4_fp64(const DeviceScene &sc, const int4 &m, bool front, float cos0, const s4 &lam,
                                       const float *thickness) {
    const int L = m.y < kMaxFilmLayers ? m.y : kMaxFilmLayers;
    double d[kMaxFilmLayers];
    for (int k = 0; k < L; k++) d[k] = double(thickness[front ? k : L - 1 - k]);
    s4 R;
#pragma unroll 1
    for (int w = 0; w < kHero; w++) {
        const float lambda = lam.v[w];
        auto index_of = [&](int k) {
            const int src = front ? k : L + 1 - k;
            const double2 c = cspectrum_at(sc, sc.material_props[m.z + src], lambda);
            return cx<double>{c.x, c.y};
        };
        double rs2, rp2;
        film_amplitudes_stream<double>(L, index_of, d, double(cos0), double((2 * kPi) / lambda), rs2, rp2);
        float rs = float(sqrt(rs2)), rp = float(sqrt(rp2));
        rs *= rs;
        rp *= rp;
        R.v[w] = (rs + rp) * 0.5f;
    }
    return R;
}

// Hero-wavelength reflect/refract choice and secondary-wavelength weights of the
// thin film (material.h:228-261), given the four reflectances.
__device__ __forceinline__ void thin_film_scatter(const DeviceScene &sc, const ShadeIn &s, const s4 &R, Rng &rng,
                                                  s4 &att, f3 &nd, float4 ff = make_float4(0, 0, 0, 0)) {
    if (ff.w != 0.0f) {
        // non-dispersive real indices (film_flat): no secondary wavelength terminates
        const float ratio = s.front ? ff.x / ff.z : ff.z / ff.x;
        const float rh = R.v[0];
        const bool refl = rng.next() < rh;
        nd = refl ? reflected(s.d, s.nrm) : refracted(s.d, s.nrm, ratio);
        att.v[0] = 1;
        for (int k = 1; k < kHero; k++) att.v[k] = refl ? R.v[k] / rh : (1 - R.v[k]) / (1 - rh);
        return;
    }
    const int outer = sc.material_props[s.m.z], sub = sc.material_props[s.m.z + s.m.y + 1];
    const float n0h = float(cspectrum_at(sc, outer, s.lam.v[0]).x);
    const float n1h = float(cspectrum_at(sc, sub, s.lam.v[0]).x);
    const float ratio = s.front ? n0h / n1h : n1h / n0h;
    const float rh = R.v[0];
    const bool refl = rng.next() < rh;
    nd = refl ? reflected(s.d, s.nrm) : refracted(s.d, s.nrm, ratio);
    att.v[0] = 1;
    for (int k = 1; k < kHero; k++) {
        const float a0 = float(cspectrum_at(sc, outer, s.lam.v[k]).x);
        const float a1 = float(cspectrum_at(sc, sub, s.lam.v[k]).x);
        const float r = R.v[k];
        att.v[k] = refl ? r / rh : (fabsf(a0 - n0h) < kEps && fabsf(a1 - n1h) < kEps) ? (1 - r) / (1 - rh) : 0;
    }
}

// Layer thicknesses of a thin-film hit: the thickness textures are evaluated once
// per hit (the reference evaluates them once per wavelength at the same point).
__device__ __forceinline__ void thin_film_thickness(const DeviceScene &sc, const ShadeIn &s, float *thick) {
    const int L = s.m.y < kMaxFilmLayers ? s.m.y : kMaxFilmLayers;
    for (int k = 0; k < L; k++) thick[k] = scalar_texture(sc, sc.material_props[s.m.w + k], s.sp.point);
}

// Thin-film hit of path p, evaluated exactly: in FP32 (within 1e-5 of FP64), or with
// kFp64 in the reference's complex double arithmetic. Returns whether the path
// continues.
template <bool kFp64>
__device__ __forceinline__ bool film_path(const DeviceScene &sc, const PathState &ps, int p, int bounce) {
    const ShadeIn s = load_shade(ps, sc, p);
    float thick[kMaxFilmLayers];
    thin_film_thickness(sc, s, thick);
    const float4 ff = __ldg(&sc.film_flat[s.mat]);
    const s4 R = kFp64 ? thin_film_r4_fp64(sc, s.m, s.front, dot(s.nrm, -s.d), s.lam, thick)
                       : thin_film_r4(sc, s.m, s.front, dot(s.nrm, -s.d), s.lam, thick, ff);
    Rng rng = path_rng(ps, p);
    s4 att;
    f3 nd;
    thin_film_scatter(sc, s, R, rng, att, nd, ff);
    return finish_scatter(ps, s, rng, bounce, att, nd, 0, true);
}

// Thin film evaluated exactly over the bounce's thin-film queue: in FP32 (within 1e-5
// of FP64), or with kFp64 in the reference's complex double arithmetic.
template <bool kFp64>
LAMBDA_KERNEL void __launch_bounds__(256, 3) k_shade_film_exact(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    const int n = ps.counts[queue_slot(bounce, kQFilm)];
    const int *q = ps.mat_queue[2];
    int *q_next = ps.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        bool alive = false;
        int p = 0;
        if (idx < n) {
            p = q[idx];
            alive = film_path<kFp64>(sc, ps, p, bounce);
        }
        const int slot = warp_push(&ps.counts[queue_slot(bounce + 1, kQActive)], alive);
        if (alive) q_next[slot] = p;
    }
}

// The end of path p's NEE shadow ray (renderer.h:166-173): if nothing occluded the
// light, its emission (lh: the light's hit record) times the stored weights is added
// to the path's NEE radiance.
__device__ __forceinline__ void shadow_finish(const DeviceScene &sc, const PathState &ps, int p, bool occluded,
                                              const Hit &lh, bool overflow) {
    const float4 o = ps.sh_o[p], dd = ps.sh_d[p];
    const int2 light = ps.sh_light[p];
    const f3 d = mk(dd.x, dd.y, dd.z);
    if (!occluded) {
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

// The NEE shadow ray of path p: occlusion, then shadow_finish.
template <int K>
__device__ __forceinline__ void shadow_path(const DeviceScene &sc, const PathState &ps, int p, const WideStack &st_a,
                                            const WideStack &st_b) {
    const float4 o = ps.sh_o[p], dd = ps.sh_d[p];
    const int2 light = ps.sh_light[p];
    Hit lh;
    bool overflow = false;
    const bool occ = occluded_w<K>(sc, mk(o.x, o.y, o.z), mk(dd.x, dd.y, dd.z), light.x, light.y, lh, overflow, st_a, st_b);
    shadow_finish(sc, ps, p, occ, lh, overflow);
}

template <int K>
LAMBDA_KERNEL void __launch_bounds__(256, 4) k_shadow(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    extern __shared__ int stack_smem[];
    WideStack st_a, st_b;
    wide_stacks(stack_smem, sc, st_a, st_b);
    const int n = ps.counts[queue_slot(bounce, kQShadow)];
    const int stride = gridDim.x * blockDim.x;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const int p = ps.shadow_queue[idx];
        shadow_path<K>(sc, ps, p, st_a, st_b);
    }
}

// The bounce's shadow rays taken lane by lane (with lane_fetch), as k_intersect_fetch
// takes closest hits: each lane keeps its occlusion query (stacks, instance-space ray,
// light distance) across iterations of one loop and advances it by one stack entry
// per iteration, in the order occluded_w visits them, so the answer is occluded_w's;
// a lane whose query is done finishes it (shadow_finish) and takes the next ray from
// the shadow queue's fetch counter at once.
template <int K>
LAMBDA_KERNEL void __launch_bounds__(256, 2) k_shadow_fetch(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    extern __shared__ int stack_smem[];
    WideStack st, sub;
    wide_stacks(stack_smem, sc, st, sub);
    const int n = ps.counts[queue_slot(bounce, kQShadow)];
    int *next = &ps.counts[queue_slot(bounce, kQShadowFetch)];
    const int lane = threadIdx.x & 31;
    int p = -1;
    Ray3 wr, lr;
    Hit lh;
    int2 light = make_int2(-1, -1);
    float best = kMax;
    int inst = -1, sp = 0, ssp = 0;
    bool overflow = false, occ = false;
    for (;;) {
        if (p < 0) {
            const unsigned need = __activemask();
            const int leader = __ffs(need) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(next, __popc(need));
            base = __shfl_sync(need, base, leader);
            const int idx = base + __popc(need & ((1u << lane) - 1u));
            if (idx >= n) break;
            p = ps.shadow_queue[idx];
            const float4 o4 = ps.sh_o[p], d4 = ps.sh_d[p];
            light = ps.sh_light[p];
            wr = make_ray(mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z));
            best = kMax;
            sp = ssp = 0;
            overflow = occ = false;
            // a scene light is first intersected itself; missing it counts as occluded
            if (light.x != -1) {
                const InstanceRef ir = instance_ref(sc, light.x);
                const Ray3 l0 = to_local(sc.instance_flags[light.x], ir, wr);
                const Prim pr = load_prim(sc, light.y);
                const float t = intersect_t(pr, l0, kMax);
                if (t < 0) {
                    occ = true;
                } else {
                    prim_attributes(sc, light.y, pr, l0.o, l0.d, t, lh);
                    lh.instance = light.x;
                    lh.object = light.y;
                    to_world(sc, light.x, ir, lh);
                    best = t;
                }
            }
            float te;
            if (!occ && slab(__ldg(&sc.nodes[0]), __ldg(&sc.nodes[1]), wr, te))
                st.put(sp++, root_entry<K>(sc, __ldg(&sc.wide_code[0])), te);
        } else if (!occ && ssp > 0) {
            // one BLAS entry; any primitive other than the light closer than it occludes
            --ssp;
            float te2 = sub.te[ssp * sub.stride];
            const int c2 = pop_code<K>(sc, sub.code[ssp * sub.stride], te2, lr, best);
            if (c2 != INT_MIN) {
                if (c2 >= 0) {
                    ssp = wide_expand<K>(sc, c2, lr, best, sub, ssp, overflow);
                    occ = overflow;
                } else {
                    const int2 lf = __ldg(&sc.wide_leaves[-c2 - 1]);
                    for (int k = 0; k < lf.y && !occ; k++) {
                        if (light.x != -1 && inst == light.x && lf.x + k == light.y) continue;
                        occ = intersect_t(load_prim(sc, lf.x + k), lr, best) >= 0;
                    }
                }
            }
        } else if (!occ && sp > 0) {
            // one TLAS entry; a leaf starts its instance's BLAS (the first instance only)
            --sp;
            float te = st.te[sp * st.stride];
            const int code = pop_code<K>(sc, st.code[sp * st.stride], te, wr, best);
            if (code != INT_MIN) {
                if (code >= 0) {
                    sp = wide_expand<K>(sc, code, wr, best, st, sp, overflow);
                    occ = overflow;
                } else {
                    inst = __ldg(&sc.wide_leaves[-code - 1]).x;
                    const uint32_t flags = sc.instance_flags[inst];
                    const InstanceRef ir = instance_ref(sc, inst);
                    const int root = ir.header().z;
                    lr = to_local(flags, ir, wr);
                    if ((flags & 2u) ||
                        (slab(__ldg(&sc.nodes[2 * root]), __ldg(&sc.nodes[2 * root + 1]), lr, te) && !(te > best)))
                        sub.put(ssp++, root_entry<K>(sc, __ldg(&sc.wide_code[root])), te);
                }
            }
        } else {
            // the query is done: occluded, or both stacks are empty
            shadow_finish(sc, ps, p, occ, lh, overflow);
            p = -1;
        }
    }
}

// One bounce of every active path in one kernel (tuning.fused_bounce): its closest
// hit, its material's shade and, for a Lambertian hit, its NEE shadow ray, through
// the same per-path steps as the path kernel and in the same order, so the image is
// the wavefront's. A wave is then raygen and one launch per bounce instead of four
// or more, which pays where a bounce's kernels are short and their chain of
// launches is the cost (small frames). The material and shadow counters are raised
// as the separate kernels' pushes raise them, for the statistics; those queues
// themselves stay empty.
template <int K, bool kFp64>
LAMBDA_KERNEL void __launch_bounds__(256, 3) k_bounce(int bounce, RenderParams rp, DeviceScene sc, PathState ps) {
    extern __shared__ int stack_smem[];
    WideStack st_a, st_b;
    wide_stacks(stack_smem, sc, st_a, st_b);
    const int n = ps.counts[queue_slot(bounce, kQActive)];
    const int *q = ps.queue[bounce & 1];
    int *q_next = ps.queue[(bounce + 1) & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int idx = base + threadIdx.x;
        int p = 0, family = -1;
        bool alive = false, nee = false;
        if (idx < n) {
            p = q[idx];
            family = trace_path<K>(sc, ps, p, st_a, st_b);
            if (family == 0) {
                alive = lambert_path(sc, ps, p, bounce, nee);
                if (nee) shadow_path<K>(sc, ps, p, st_a, st_b);
            } else if (family == 1) {
                alive = specular_path(sc, ps, p, bounce);
            } else if (family == 2) {
                alive = film_path<kFp64>(sc, ps, p, bounce);
            }
        }
        const int slot = warp_push(&ps.counts[queue_slot(bounce + 1, kQActive)], alive);
        if (alive) q_next[slot] = p;
        for (int f = 0; f < 3; f++) warp_push(&ps.counts[queue_slot(bounce, kQLambert + f)], family == f);
        warp_push(&ps.counts[queue_slot(bounce, kQShadow)], nee);
    }
}

// Last sample of pixel p into the film, then the average (renderer.h:84-91), into
// the job's own image.
__device__ __forceinline__ void finish_pixel(const DeviceScene &sc, const PathState &ps, int p, const Job &job) {
    const f3 rgb = spectrum_to_rgb(sc, sample_radiance(ps, p), from_f4(ps.lam[p]), job.lambda_range);
    float4 film = ps.film[p];
    film.x += rgb.x;
    film.y += rgb.y;
    film.z += rgb.z;
    const float inv = float(job.samples);
    const size_t local = size_t(p - job.base);
    job.out[3 * local] = film.x / inv;
    job.out[3 * local + 1] = film.y / inv;
    job.out[3 * local + 2] = film.z / inv;
}

// A whole pass, every job of a batch included, in one persistent launch: each warp
// takes the next 32 work indices from the work counter `work` (zeroed with the
// pass's counters) until none are left. Work indices run through the jobs in the
// order of rp.work, by decreasing samples x (depth + 1), so the costliest pixels are
// handed out first and the cheap ones fill in behind them. Lane l runs work index
// base + l (a warp covers an 8x4 tile of its job): it seeds the pixel (as k_init), runs every sample to the end, bounce by
// bounce, through the same per-path steps as the wavefront kernels and in the same
// order (bank and start a sample, closest hit, the material's shade, the NEE shadow
// ray), then banks the last sample and writes the job's image (as k_finish). The
// image therefore equals the wavefront's bit for bit, with no launch per bounce or
// per wave. After each tile the warp adds its pixels to `done` and publishes the
// total to `progress` (mapped host memory; the host keeps the largest value it has
// seen, since warps publish out of order). Thin films are evaluated exactly (FP32,
// or complex double with kFp64); surrogate renders of thin films need the
// wavefront, which batches a bounce's thin-film hits for the tensor cores. The
// statistics are the ones the wave prologue keeps from the queue sizes.
template <int K, bool kFp64>
LAMBDA_KERNEL void __launch_bounds__(256, 3) k_path(RenderParams rp, DeviceScene sc, PathState ps, int *work, int *done,
                                                 int *progress) {
    extern __shared__ int stack_smem[];
    WideStack st_a, st_b;
    wide_stacks(stack_smem, sc, st_a, st_b);
    const int lane = threadIdx.x & 31;
    unsigned n_seg = 0, n_nee = 0, n_film = 0, n_lam = 0, n_spec = 0;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(work, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= rp.num_pixels) break;
        const int v = base + lane;
        if (v < rp.num_pixels) {
            int lo = 0, hi = rp.num_jobs - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (rp.work[mid].y <= v) lo = mid;
                else hi = mid - 1;
            }
            const Job &job = rp.jobs[rp.work[lo].x];
            const int p = job.base + tile_order(job, v - rp.work[lo].y);
            init_pixel(ps, p, job);
            for (int s = 0; s < job.samples; s++) {
                bank_sample(sc, ps, p, job);
                start_sample(ps, p, job, s);
                for (int b = 0; b <= rp.depth_max; b++) {
                    n_seg++;
                    const int family = trace_path<K>(sc, ps, p, st_a, st_b);
                    if (family < 0) break;
                    bool alive, nee = false;
                    if (family == 0) {
                        n_lam++;
                        alive = lambert_path(sc, ps, p, b, nee);
                        if (nee) {
                            n_nee++;
                            shadow_path<K>(sc, ps, p, st_a, st_b);
                        }
                    } else if (family == 1) {
                        n_spec++;
                        alive = specular_path(sc, ps, p, b);
                    } else {
                        n_film++;
                        alive = film_path<kFp64>(sc, ps, p, b);
                    }
                    if (!alive) break;
                }
            }
            finish_pixel(sc, ps, p, job);
        }
        __syncwarp();
        if (lane == 0) {
            const int n = min(32, rp.num_pixels - base);
            const int total = atomicAdd(done, n) + n;
            if (progress) *reinterpret_cast<volatile int *>(progress) = total;
        }
    }
    // segments, NEE rays, thin-film hits, (fallback), Lambertian hits, specular hits
    const unsigned c[6] = {n_seg, n_nee, n_film, 0u, n_lam, n_spec};
    for (int i = 0; i < 6; i++) {
        const unsigned sum = __reduce_add_sync(0xffffffffu, c[i]);
        if (lane == 0 && sum) atomicAdd(&ps.stats[i], (unsigned long long)sum);
    }
}

// Last sample into the film, then the average, for every pixel of a wavefront pass.
// Jobs that finished before the last wave banked their last sample in k_raygen and
// hold zero radiance here.
LAMBDA_KERNEL void k_finish(RenderParams rp, DeviceScene sc, PathState ps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= rp.num_pixels) return;
    finish_pixel(sc, ps, p, rp.jobs[job_of(rp, p)]);
}

}  // namespace lambda_dev
