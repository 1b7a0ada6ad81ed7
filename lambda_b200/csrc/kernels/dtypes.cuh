// Plain structs shared by the kernels and the host-side engine: the device
// scene view, per-render parameters and the wavefront path state.
#pragma once

#include <cstdint>

#include "dmath.cuh"

namespace lambda_dev {

constexpr int kMaxFilmLayers = 8;  // thin-film layers handled by the FP32 transfer matrix

struct DeviceScene {
    const float4 *nodes;         // binary BVH (min, index) (max, count): root boxes
    const float4 *wide;          // wide BVH child records, `width` per node (wide_bvh.h)
    const int2 *wide_leaves;     // (index, count) of every binary leaf
    const int *wide_code;        // per binary node: wide code of the tree roots
    const uint4 *wide_q;         // compressed node records (wide_bvh.h), kQuantWords per node
    int num_leaves;              // binary leaves (the compressed layout's root entries encode codes with it)
    int bvh_width;               // children per wide node (2, 4 or 8)
    int stack_tlas, stack_blas;  // traversal stack entries a ray can need
    const float4 *prims;
    const float4 *tri_attr;
    const float4 *instances;
    const float *spectra;
    const uint8_t *spectrum_flat;
    const double2 *cspectra;
    const uint8_t *cspectrum_flat;
    const int4 *materials;
    const int *material_props;
    const float4 *scalar_tex;
    const int4 *spectrum_tex;
    const int *light_inst;
    const int *light_obj;
    const float *light_power;
    const float *light_cdf;      // running sums of light_power in list order
    const float *material_emission;  // per material: average emission (0 if not emissive)
    const uint8_t *material_uv;      // per material: 1 if a texture it evaluates reads the hit's (u, v)
    const float4 *film_flat;         // per material: (n_outer, n_film, n_sub, 1) of a one-layer thin film whose
                                     // indices are real and non-dispersive, else zeros
    const uint32_t *instance_flags;  // bit 0: transform and inverse are exactly the identity; bit 1: also
                                     // alone in its TLAS leaf, whose box is its BLAS root's box
    const float *cie;            // [471][3] as float
    const int *perm;             // [256]
    const float4 *worley_cells;  // feature offsets of lattice cells (xyz), cell-major
    int3 worley_lo;              // first cell of the table
    int3 worley_dim;             // cells per axis (0 when there is no table)
    int num_nodes;
    int num_objects;
    int num_instances;
    int num_lights;
    float total_light_power;
    int background_texture;
    uint32_t families;           // bit f set when some material of family f exists (0 Lambertian, 1 specular, 2 thin film)
};

// One image of a render: a single render is one job, a batch is many. The jobs'
// pixels are laid end to end in one virtual pixel range (job j owns
// [base, base + width * height)), ordered by decreasing sample count, so the pixels
// that still take a sample in wave s are a prefix of that range.
struct Job {
    int width, height, depth, samples, sqrt_samples;
    float lambda_min, lambda_max, lambda_range;
    f3 cam_pos, cam_corner, cam_h, cam_v;
    uint64_t seed;
    int base;    // first virtual pixel
    float *out;  // width * height * 3 floats of linear sRGB (device)
};

struct RenderParams {
    const Job *jobs;    // [num_jobs]
    int num_jobs;
    int num_pixels;     // all jobs' pixels
    int depth_max;      // deepest job: bounces per wave are 0..depth_max
    const int *active;  // [samples_max + 1]: pixels with a sample in wave s (a prefix)
    // the path kernel's hand-out order: (job, first work index) per job, jobs by
    // decreasing samples x (depth + 1), so the costliest pixels are taken first
    const int2 *work;   // [num_jobs]
};

struct PathState {
    uint64_t *rng;        // PCG32 state per pixel
    float4 *film;         // accumulated linear sRGB (xyz)
    float4 *lam;          // four hero wavelengths
    float4 *ray_o;        // origin xyz, w = pdf of the last scatter
    float4 *ray_d;        // direction xyz, w = 1 if the last scatter was specular
    float4 *throughput;
    float4 *radiance;     // NEE terms of the running sample
    float4 *emit;         // emission term of a sample that ended at a miss or an emitter
    int4 *hit_id;         // material, object, distance (float bits), instance of a stored hit
    float4 *sh_o;         // NEE ray origin xyz, w = MIS weight
    float4 *sh_d;         // NEE ray direction xyz, w = light pdf
    float4 *sh_a;         // throughput * BSDF * cos
    int2 *sh_light;       // light (instance, object)
    int *queue[2];        // active pixel ids, ping-pong by bounce parity
    int *mat_queue[3];    // this bounce's Lambertian, mirror/dielectric and thin-film hits
    int *shadow_queue;    // pixel ids with a pending NEE ray
    int *counts;          // [kQueues * (depth + 2)], see queue_slot()
    int *wave;            // [2]: wave to run next, wave being run
    unsigned long long *stats;  // segments, shadow rays, thin-film hits
    int *error;           // bit 0: traversal stack overflow
    int2 *path_info;      // job-local pixel index (the PCG stream), depth limit of the job
};

// Counters per bounce: paths to trace, then the three material queues, then NEE rays,
// then the thin-film hits the surrogate left to the exact transfer matrix (a count).
// kQFetch / kQShadowFetch: the next unclaimed entry of the bounce's active / shadow
// queue, for the lane-by-lane intersect and shadow kernels (lanes take rays one by one).
enum : int { kQActive = 0, kQLambert = 1, kQSpecular = 2, kQFilm = 3, kQShadow = 4, kQFilmFallback = 5, kQFetch = 6,
             kQShadowFetch = 7, kQueues = 8 };
__host__ __device__ inline int queue_slot(int bounce, int q) { return bounce * kQueues + q; }

}  // namespace lambda_dev
