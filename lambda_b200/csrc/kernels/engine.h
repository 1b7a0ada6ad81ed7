// The context object behind the C ABI and its device buffers.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "lambda_gpu.h"
#include "dtypes.cuh"

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n);
    cudaError_t upload(const void *src, size_t n, cudaStream_t s);
    void release();
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

bool is_device_pointer(const void *p);

// Index of the tuned BVH layout: widths 2, 4, 8 (0-2), then the same widths with
// compressed node records (3-5); the order of the kernel tables that dispatch on it.
int layout_index(const lambda_tuning &t);

// CTAs of `block` threads with `dyn_smem` bytes of dynamic shared memory that one SM
// holds at once, from the kernel's registers and static shared memory and the SM's
// limits (at least 1).
int resident_ctas(const void *fn, int device, int block, size_t dyn_smem);

// Brackets kernel launches with CUDA events and totals their device time per
// stage (LAMBDA_RENDER_PROFILE_STAGES).
struct StageProfiler {
    cudaStream_t stream;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
    std::vector<int> stages;
    size_t used = 0;
    double totals[LAMBDA_NUM_STAGES] = {0};
    int64_t counts[LAMBDA_NUM_STAGES] = {0};
    explicit StageProfiler(cudaStream_t s);
    ~StageProfiler();
    void begin(int stage);
    void end();
    cudaError_t collect();
};

struct SceneBuffers {
    DeviceBuffer nodes, prims, tri, instances, spectra, spectrum_flat, cspectra, cspectrum_flat, materials,
        material_props, scalar_tex, spectrum_tex, light_inst, light_obj, light_power, light_cdf, material_emission,
        material_uv, film_flat,
        cie, perm, worley, instance_flags;
    DeviceBuffer wide[3], wide_leaves[3], wide_code[3];  // wide BVH of width 2, 4, 8
    DeviceBuffer wide_q[3];                               // its compressed node records
};

struct RenderBuffers {
    DeviceBuffer rng, film, lam, ray_o, ray_d, throughput, radiance, emit, hit_id, sh_o, sh_d, sh_a, sh_light,
        q0, q1, qs, qm0, qm1, qm2, counts, wave, stats, error, out, path_info, jobs, active, work, film_rows, film_out,
        film_in_domain;
};

struct SurrogateBuffers {
    DeviceBuffer weights_bf16;  // packed tensor-core operand tiles
    DeviceBuffer weights_f32;   // master copy, LAMBDA_MLP_PARAMS floats
};

struct lambda_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    // Branches of a bounce that run beside the main stream's inside the pass graph:
    // specular and thin-film shading, and the shadow rays (fork and join events, no
    // timing).
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr}, ev_lambert = nullptr, ev_shadow = nullptr;
    std::string last_error;

    bool has_scene = false;
    int film_layers_max = 0;
    SceneBuffers scene;
    lambda_dev::DeviceScene dscene{};
    int wide_stack[3][2] = {};  // traversal stack entries (TLAS, BLAS) of the width 2, 4, 8 trees
    int wide_leaves_n[3] = {};  // binary leaves of each (codes of the compressed layout's root entries)

    RenderBuffers rbuf;
    lambda_dev::PathState pstate{};
    cudaGraphExec_t graph_exec = nullptr;
    lambda_render_stats stats{};
    lambda_stage_time stage_times[LAMBDA_NUM_STAGES]{};
    lambda_tuning tuning{256, 256, 1, 0, 4, LAMBDA_PATH_KERNEL_PIXELS, 0, 0, 0};  // launch shapes (max_pixels 0: no limit)
    lambda_limits limits{LAMBDA_DEFAULT_MMA_POLLS, 0};  // device guard limits (lambda_set_limits)
    int *progress_host = nullptr;           // waves started by the running pass graph (mapped host memory)
    int *progress_dev = nullptr;            // its device address

    // surrogate
    bool has_surrogate = false;
    int mlp_ctas_per_sm = 0;  // resident CTAs of the tensor-core MLP kernel per SM
    int film_encode_ctas = 0, film_scatter_ctas = 0;  // resident CTAs per SM of the surrogate's shade kernels
    lambda_film_range surrogate_range{};
    SurrogateBuffers sbuf;

    ~lambda_ctx();

    // The scene as the kernels see it with the wide BVH of the given width (2, 4 or 8).
    lambda_dev::DeviceScene scene_view(int width) const;
    lambda_status fail(lambda_status s, const std::string &msg);
    lambda_status cuda_fail(cudaError_t e, const char *what);
    lambda_status ensure_state(int pixels, int depth);
    lambda_status surrogate_ready();
    lambda_status ensure_surrogate_state(int pixels);
    int launch_shade_surrogate(int bounce, const lambda_dev::RenderParams &rp, const lambda_dev::DeviceScene &sc,
                               const lambda_dev::PathState &ps, StageProfiler *prof, cudaStream_t s);

    std::vector<DeviceBuffer *> all_buffers() {
        SceneBuffers &s = scene;
        RenderBuffers &r = rbuf;
        return {&s.nodes, &s.prims, &s.tri, &s.instances, &s.spectra, &s.spectrum_flat, &s.cspectra,
                &s.cspectrum_flat, &s.materials, &s.material_props, &s.scalar_tex, &s.spectrum_tex, &s.light_inst,
                &s.light_obj, &s.light_power, &s.light_cdf, &s.material_emission, &s.material_uv, &s.film_flat, &s.cie, &s.perm, &s.worley, &s.instance_flags,
                &s.wide[0], &s.wide[1], &s.wide[2], &s.wide_leaves[0], &s.wide_leaves[1], &s.wide_leaves[2],
                &s.wide_code[0], &s.wide_code[1], &s.wide_code[2], &s.wide_q[0], &s.wide_q[1], &s.wide_q[2],
                &r.rng, &r.film, &r.lam, &r.ray_o, &r.ray_d, &r.throughput, &r.radiance, &r.emit, &r.hit_id,
                &r.sh_o, &r.sh_d, &r.sh_a, &r.sh_light, &r.q0, &r.q1, &r.qs, &r.qm0, &r.qm1, &r.qm2, &r.counts, &r.wave,
                &r.stats, &r.error, &r.out, &r.path_info, &r.jobs, &r.active, &r.work, &r.film_rows, &r.film_out,
                &r.film_in_domain, &sbuf.weights_bf16, &sbuf.weights_f32};
    }
};

// Stages caller arrays (host or device) in and out of device memory.
struct Staging {
    lambda_ctx *ctx;
    std::vector<void *> owned;
    ~Staging() {
        for (void *p : owned) cudaFree(p);
    }
    template <typename T>
    cudaError_t in(const T *src, size_t n, const T **dst) {
        if (is_device_pointer(src)) {
            *dst = src;
            return cudaSuccess;
        }
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n * sizeof(T), 16));
        if (e != cudaSuccess) return e;
        owned.push_back(p);
        *dst = static_cast<const T *>(p);
        return cudaMemcpyAsync(p, src, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    }
    template <typename T>
    cudaError_t out(T *user, size_t n, T **dst, std::vector<std::pair<void *, std::pair<void *, size_t>>> &back) {
        if (is_device_pointer(user)) {
            *dst = user;
            return cudaSuccess;
        }
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n * sizeof(T), 16));
        if (e != cudaSuccess) return e;
        owned.push_back(p);
        *dst = static_cast<T *>(p);
        back.push_back({user, {p, n * sizeof(T)}});
        return cudaSuccess;
    }
};

using CopyBack = std::vector<std::pair<void *, std::pair<void *, size_t>>>;

// Copies staged results back to the caller's host arrays and waits for the stream.
lambda_status finish_staging(lambda_ctx *ctx, CopyBack &back);

