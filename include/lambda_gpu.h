/*
 * lambda_gpu.h - C ABI of the B200 spectral path-tracing render loop.
 *
 * The reference renderer's boundary is a C++ class plus one kernel:
 *   Parser::parseLRD      src/core/parser.h:29   (scene file -> 15 host containers)
 *   Renderer::setScene    src/render/renderer.h:38
 *   Renderer::setCamera   src/render/renderer.h:36
 *   Renderer::setBuffer   src/render/renderer.h:40
 *   Renderer::renderImage src/render/renderer.h:42  (CPU) / renderKernel :200 (GPU)
 *   Writer::write         src/core/writer.h:11
 * This header replaces that boundary with plain C: POD scene arrays that keep the
 * reference containers' indices and byte layouts, opaque handles, and status codes.
 * No entry point throws; every failure is a lambda_status plus a message that
 * lambda_last_error() returns.
 *
 * Pointers: unless an entry point says otherwise, array arguments may be host or
 * device memory. The library asks the CUDA runtime which one it was given and
 * stages host memory through its own device buffers.
 */
#ifndef LAMBDA_GPU_H
#define LAMBDA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LAMBDA_ABI_VERSION 1

/* Wavelength grid of every dense spectrum: 1 nm bins over [360, 830] nm
 * (src/core/constants.h:20-22, src/math/spectrum.h:158-188). */
#define LAMBDA_CIE_LAMBDA_MIN 360
#define LAMBDA_CIE_LAMBDA_MAX 830
#define LAMBDA_CIE_BINS 471
/* Wavelengths carried by one path (hero wavelength + 3 rotations), constants.h:12. */
#define LAMBDA_HERO_COUNT 4

typedef enum lambda_status {
    LAMBDA_OK = 0,
    LAMBDA_ERR_INVALID_ARGUMENT = 1,
    LAMBDA_ERR_PARSE = 2,          /* scene file error: message is "file:line: text" */
    LAMBDA_ERR_IO = 3,             /* file could not be opened or written */
    LAMBDA_ERR_CUDA = 4,           /* CUDA runtime error */
    LAMBDA_ERR_OUT_OF_MEMORY = 5,
    LAMBDA_ERR_NO_SCENE = 6,       /* render or trace before lambda_scene_upload */
    LAMBDA_ERR_UNSUPPORTED = 7,    /* input outside what this build implements */
    LAMBDA_ERR_QUEUE_OVERFLOW = 8, /* a device work queue or traversal stack overflowed */
    LAMBDA_ERR_TIMEOUT = 9,        /* a bounded device wait gave up */
    LAMBDA_ERR_ABORTED = 10,       /* the caller's abort flag was raised */
    LAMBDA_ERR_INTERNAL = 11
} lambda_status;

/* ---------------------------------------------------------------------------
 * Flat scene: the 15 containers Parser::parseLRD fills (parser.h:29), in the
 * reference's order after BVH::makeBVH reordered objects and instances
 * (bvh.h:61-108). Each struct has the byte layout of the reference class it
 * mirrors, so indices and bytes can be compared one to one.
 * ------------------------------------------------------------------------- */

/* ObjectType, src/scene/object.h:13 */
enum { LAMBDA_OBJECT_SPHERE = 0, LAMBDA_OBJECT_QUAD = 1, LAMBDA_OBJECT_TRI = 2 };

/* class Object, object.h:15-164 (116 bytes).
 * sphere: g[0..2] center, g[3] radius
 * quad:   g[0..2] corner, g[3..5] horizontal, g[6..8] vertical, g[9..11] normal = horizontal x vertical
 * tri:    as quad, then g[12..20] vertex normals n0 n1 n2, g[21..23] u0 u1 u2, g[24..26] v0 v1 v2 */
typedef struct lambda_object {
    int32_t type;
    int32_t material;
    float g[27];
} lambda_object;

/* class Instance, src/scene/instance.h:11-116 (144 bytes). transform = T*Rz*Ry*Rx*S,
 * row-major; inverse_transform is its cofactor inverse. material < 0 means "use the
 * object's own material" (instance.h:38). node is the root of the object's BLAS. */
typedef struct lambda_instance {
    int32_t object;
    int32_t count;
    int32_t node;
    int32_t material;
    float transform[16];
    float inverse_transform[16];
} lambda_instance;

/* class BVHNode, src/scene/bvh.h:14-57 (32 bytes). Leaf iff count > 0; a leaf's
 * index is its first instance (TLAS) or object (BLAS); an inner node's left
 * child is the next node and index is its right child. */
typedef struct lambda_bvh_node {
    float min[3];
    float max[3];
    int32_t index;
    int32_t count;
} lambda_bvh_node;

/* MaterialType, src/scene/material.h:15 */
enum {
    LAMBDA_MATERIAL_LAMBERTIAN = 0,
    LAMBDA_MATERIAL_MIRROR = 1,
    LAMBDA_MATERIAL_DIELECTRIC = 2,
    LAMBDA_MATERIAL_EMISSIVE = 3,
    LAMBDA_MATERIAL_THINFILM = 4
};

/* class Material, material.h:17-138 (16 bytes).
 * lambertian/mirror: p[0] albedo spectrum texture; dielectric: p[0] n0, p[1] n1 spectra;
 * emissive: p[0] emission spectrum texture;
 * thinfilm: p[0] layer count L, p[1] offset of L+2 complex-spectrum indices in
 * material_properties (outer medium, layers, substrate), p[2] offset of L scalar
 * texture indices (layer thickness in nm). */
typedef struct lambda_material {
    int32_t type;
    int32_t p[3];
} lambda_material;

/* ScalarTextureType, src/scene/texture.h:8 */
enum { LAMBDA_SCALAR_CONSTANT = 0, LAMBDA_SCALAR_PERLIN = 1, LAMBDA_SCALAR_WORLEY = 2 };

/* class ScalarTexture, texture.h:10-96 (16 bytes). constant: p[0] value;
 * perlin/worley: p[0] min, p[1] max, p[2] frequency. */
typedef struct lambda_scalar_texture {
    int32_t type;
    float p[3];
} lambda_scalar_texture;

/* SpectrumTextureType, texture.h:9 */
enum { LAMBDA_SPECTRUM_CONSTANT = 0, LAMBDA_SPECTRUM_CHECKER = 1, LAMBDA_SPECTRUM_SCALAR = 2 };

/* class SpectrumTexture, texture.h:98-210 (16 bytes). constant: value1 = spectrum;
 * checker: value1, value2 spectra, scale; scalar: value1 = scalar texture. */
typedef struct lambda_spectrum_texture {
    int32_t type;
    int32_t value1;
    int32_t value2;
    float scale;
} lambda_spectrum_texture;

/* class Camera, src/render/camera.h:7-19 */
typedef struct lambda_camera {
    float position[3];
    float corner[3];
    float horizontal[3];
    float vertical[3];
} lambda_camera;

/* The Renderer constructor arguments (renderer.h:28) plus its camera. */
typedef struct lambda_render_settings {
    int32_t width;
    int32_t height;
    int32_t depth;        /* maximum bounce index; a path has at most depth+1 segments */
    int32_t samples;      /* perfect square */
    int32_t sqrt_samples;
    float lambda_min;
    float lambda_max;
    lambda_camera camera;
} lambda_render_settings;

/* Renderer::setScene arguments (renderer.h:38). Background::makeEquirectangular
 * holds only a spectrum texture index (background.h:9-17). */
typedef struct lambda_scene_desc {
    const float *spectra;              /* [num_spectra][471] */
    int32_t num_spectra;
    const double *complex_spectra;     /* [num_complex_spectra][471][2] (re, im) */
    int32_t num_complex_spectra;
    int32_t background_texture;
    const lambda_object *objects;
    int32_t num_objects;
    const lambda_instance *instances;
    int32_t num_instances;
    const lambda_bvh_node *nodes;
    int32_t num_nodes;
    const int32_t *light_instances;    /* [num_lights]; the last light is the background (-1) */
    const int32_t *light_objects;
    const float *light_powers;
    int32_t num_lights;
    float total_light_power;
    const lambda_material *materials;
    int32_t num_materials;
    const int32_t *material_properties;
    int32_t num_material_properties;
    const lambda_scalar_texture *scalar_textures;
    int32_t num_scalar_textures;
    const lambda_spectrum_texture *spectrum_textures;
    int32_t num_spectrum_textures;
} lambda_scene_desc;

/* ---------------------------------------------------------------------------
 * Host side: scene parsing and image output (no GPU needed).
 * ------------------------------------------------------------------------- */

typedef struct lambda_host_scene lambda_host_scene;

/* Parser::parseLRD (src/core/parser.h:29-379) + Parser::parseOBJ (:639-786) +
 * BVH::makeBVH (src/scene/bvh.h:61-108). Reads a .lrd file (and the .obj files it
 * names), builds the two-level SAH BVH and the light list. On failure returns
 * LAMBDA_ERR_PARSE or LAMBDA_ERR_IO and writes the reference's message text
 * ("file:line: message" or "file: failed to open file (...)") into err. */
lambda_status lambda_parse_lrd(const char *path, lambda_host_scene **out, char *err, size_t err_len);

/* lambda_parse_lrd with the scene build's heavy steps on the context's GPU, for the
 * same scene byte for byte: every instance's world bounds and centroid
 * (Instance::min/max/center, src/scene/instance.h:54-101, which visit every object
 * of every instance) and the binned-SAH build (src/scene/bvh.h:111-246) of every
 * object group or instance set of at least gpu_min_items items (0: 65536; smaller
 * ones build faster on the host). Errors as lambda_parse_lrd's, plus
 * LAMBDA_ERR_CUDA. The build takes temporary device memory of about 260 bytes per
 * item of the largest range it builds plus about 175 MB (the per-node bins of up
 * to 65,536 nodes at a time), and frees it before returning. Declared with the host functions because it returns a host
 * scene; it needs a GPU. No reference counterpart: the reference builds on the
 * host only. */
typedef struct lambda_ctx lambda_ctx;
lambda_status lambda_parse_lrd_gpu(lambda_ctx *ctx, const char *path, int32_t gpu_min_items, lambda_host_scene **out,
                                   char *err, size_t err_len);

/* Views of a parsed scene; pointers stay valid until lambda_host_scene_destroy. */
lambda_status lambda_host_scene_get(const lambda_host_scene *scene, lambda_scene_desc *desc,
                                    lambda_render_settings *settings);

void lambda_host_scene_destroy(lambda_host_scene *scene);

/* Writer::hasValidExtension + Writer::write (src/core/writer.h:9-28): tonemap,
 * sRGB OETF, dither from PCG32(0, 0) and write ASCII P3. rgb is host memory,
 * [height][width][3] linear sRGB. Errors as in the reference (": invalid file
 * extension", ": failed to open file (...)"). */
lambda_status lambda_write_ppm(const char *path, int32_t width, int32_t height, const float *rgb,
                               char *err, size_t err_len);

/* Binary float output beside the reference's 8-bit text PPM (no counterpart in the
 * reference): a little-endian PFM ("PF", scale -1.0, rows bottom to top) of the
 * unclamped linear sRGB image, or with xyz != 0 of linear CIE XYZ (the inverse of
 * the XYZ -> sRGB matrix of utils.h:230, in double), the space image error is
 * measured in. The path must end in ".pfm". */
lambda_status lambda_write_pfm(const char *path, int32_t width, int32_t height, const float *rgb, int32_t xyz,
                               char *err, size_t err_len);

/* ---------------------------------------------------------------------------
 * GPU context (lambda_ctx, declared above with lambda_parse_lrd_gpu).
 * ------------------------------------------------------------------------- */

/* Creates a context on one CUDA device (one stream, its own device arena). No
 * reference counterpart: the reference uses the current device and managed memory
 * (src/core/buffer.h:9-44). */
lambda_status lambda_ctx_create(int32_t device, lambda_ctx **out);

void lambda_ctx_destroy(lambda_ctx *ctx);

/* Message of the last failed call on this context ("" if none). A NULL ctx
 * returns the message of the last failed lambda_ctx_create on this thread. */
const char *lambda_last_error(const lambda_ctx *ctx);

/* Renderer::setScene (renderer.h:38) with the Buffer<T> uploads of main.cpp:84-103:
 * copies the scene into device memory and derives the device layouts (SoA object
 * records, light CDF, noise lattices). Replaces any previous scene. */
lambda_status lambda_scene_upload(lambda_ctx *ctx, const lambda_scene_desc *scene);

/* Render flags */
#define LAMBDA_RENDER_THINFILM_EXACT 0u       /* FP32 transfer-matrix thin-film reflectance */
#define LAMBDA_RENDER_THINFILM_SURROGATE 1u   /* BF16 MLP on tensor cores, FP32 fallback per hit */
#define LAMBDA_RENDER_OUTPUT_DEVICE 2u        /* out_rgb is device memory: no copy back */
#define LAMBDA_RENDER_PROFILE_STAGES 4u       /* time every kernel launch with CUDA events (no graph replay) */
#define LAMBDA_RENDER_THINFILM_FP64 8u        /* the reference's complex double transfer matrix per hit */

typedef struct lambda_render_desc {
    lambda_render_settings settings;
    uint64_t seed;                            /* main.cpp:122 uses 42 */
    uint32_t flags;
    int32_t reserved;
} lambda_render_desc;

/* Renderer::renderImage(completed, seed) (renderer.h:42-55) / renderKernel
 * (renderer.h:200-213): renders the uploaded scene and writes [height][width][3]
 * linear sRGB floats (renderer.h:87-91) to out_rgb. Pixel (px, py) draws from PCG32
 * stream py*width+px seeded with desc->seed, in the reference's order, so results
 * follow the reference sample for sample. completed (may be NULL) is raised
 * monotonically towards width*height while the call runs (pixels x finished
 * sample waves / samples; a pass run by the path kernel reports its pixels when it
 * ends). Blocks until the image is written. */
lambda_status lambda_render(lambda_ctx *ctx, const lambda_render_desc *desc, float *out_rgb,
                            volatile int32_t *completed);

/* One image of a batch. */
typedef struct lambda_job {
    lambda_render_desc desc;  /* size, depth, samples, wavelength range, camera, seed, flags */
    float *out_rgb;           /* [height][width][3]; device memory if desc.flags has LAMBDA_RENDER_OUTPUT_DEVICE */
} lambda_job;

/* Renders n images of the uploaded scene (their own cameras, sizes, sample counts,
 * depths, wavelength ranges and seeds) as one wavefront: every job's pixels share
 * one path state, sample waves run until the job with the most samples is done
 * (jobs with fewer samples drop out of later waves), and the bounces of a wave run
 * to the deepest job. Each image is, bit for bit, what lambda_render gives for that
 * job alone. All jobs must use the same thin-film mode and profiling flag; the
 * output flag is per job. completed (may be NULL) rises towards the jobs' total
 * pixels. Statistics cover the whole batch. No counterpart in the reference, whose
 * renderKernel (renderer.h:200-213) renders one image per launch. */
lambda_status lambda_render_batch(lambda_ctx *ctx, const lambda_job *jobs, int32_t n, volatile int32_t *completed);

/* Launch shapes of the wavefront kernels and the choice of the path kernel for small
 * passes. lambda_autotune times a probe render under every candidate (the path kernel
 * among them, unless the probe renders thin films with the surrogate) and keeps the
 * fastest on the context. A winning path kernel covers passes up to the probe's pixels
 * (at least LAMBDA_PATH_KERNEL_PIXELS); a winning wavefront leaves the path kernel to
 * passes smaller than both the probe and LAMBDA_PATH_KERNEL_PIXELS. lambda_set_tuning
 * installs given values. No counterpart in the reference. */
typedef struct lambda_tuning {
    int32_t trace_block; /* threads per CTA of the traversal kernels (intersect, shadow): 64, 128 or 256 */
    int32_t shade_block; /* threads per CTA of the shading kernels: 64, 128 or 256 */
    int32_t grid_scale;  /* persistent grids hold grid_scale x the CTAs that fit on all SMs at once: 1 or 2 */
    int32_t max_pixels;  /* path-state capacity: a batch above it runs as several passes of whole jobs */
    int32_t bvh_width;   /* children per node of the traversed BVH: 2, 4 or 8 (every width finds the same hits) */
    int32_t path_kernel_pixels; /* a pass of at most this many pixels runs as one kernel in which each thread traces
                                   every sample of its pixel (same image, no launch per bounce), unless it renders
                                   thin films with the surrogate; 0: always the wavefront. Default
                                   LAMBDA_PATH_KERNEL_PIXELS */
    int32_t lane_fetch;  /* 1: the wavefront's intersect and shadow kernels take rays lane by lane (a lane whose ray
                            is done takes the next at once; same hits), for scenes whose rays differ widely in
                            traversal length; 0: each warp traces 32 rays to the end before taking more */
    int32_t compressed_nodes; /* 1: traverse the compressed node records (8-bit child boxes against a per-node origin
                                 and power-of-two scales, checked to contain the exact boxes; a child is tested on
                                 its exact box when popped, so the hits are the same); 0: the exact 32-byte child
                                 records */
    int32_t fused_bounce; /* 1: a wavefront bounce runs as one kernel (closest hit, the material's shade and the NEE
                             shadow ray of each path; same image), for frames whose bounces are too short to repay
                             a chain of launches; not for surrogate renders of thin films. 0: separate kernels */
} lambda_tuning;

/* Default path_kernel_pixels. Below it a sample wave holds too few paths to hide a
 * launch per bounce on any scene measured; above it the winner depends on the scene
 * (the wavefront's per-material kernels win where materials mix, the path kernel
 * where one material and deep traversal dominate), which lambda_autotune decides. */
#define LAMBDA_PATH_KERNEL_PIXELS 32768

lambda_status lambda_autotune(lambda_ctx *ctx, const lambda_render_desc *probe, lambda_tuning *out);
/* The same search over a batch: each candidate times lambda_render_batch of the n
 * probe views (same thin-film mode; images in device memory allocated here), so the
 * shapes suit many small and uneven jobs rendered together. */
lambda_status lambda_autotune_batch(lambda_ctx *ctx, const lambda_render_desc *probes, int32_t n, lambda_tuning *out);
lambda_status lambda_set_tuning(lambda_ctx *ctx, const lambda_tuning *tuning);
lambda_status lambda_get_tuning(const lambda_ctx *ctx, lambda_tuning *tuning);

/* Limits of the device-side guards. Every wait in the kernels is bounded and every
 * traversal stack push is checked; these settings let a test make a guard fire and
 * check that the call returns its error and that the next call on the same context
 * is correct. No reference counterpart (the reference's traversal stack is unchecked,
 * scene/scene.h:60-118, and its host polls the render forever, main.cpp:129-146).
 *   mma_polls      polls of each tensor-core MMA-completion wait before it gives up
 *                  (LAMBDA_DEFAULT_MMA_POLLS); 0 gives up at once. A wait that gives
 *                  up lets the MMAs already issued finish (bounded by the default)
 *                  before TMEM is read or freed, and the call returns
 *                  LAMBDA_ERR_TIMEOUT.
 *   stack_entries  cap on traversal stack entries per ray and BVH level, 0 for none:
 *                  the stacks then hold the most entries the uploaded BVH can need.
 *                  Below that, a ray that would overflow stops, and the call returns
 *                  LAMBDA_ERR_QUEUE_OVERFLOW.
 * lambda_set_limits(ctx, NULL) restores the defaults. */
#define LAMBDA_DEFAULT_MMA_POLLS 4194304u
typedef struct lambda_limits {
    uint32_t mma_polls;
    int32_t stack_entries;
} lambda_limits;

lambda_status lambda_set_limits(lambda_ctx *ctx, const lambda_limits *limits);
lambda_status lambda_get_limits(const lambda_ctx *ctx, lambda_limits *limits);

/* Statistics of the last lambda_render or lambda_render_batch on this context. */
typedef struct lambda_render_stats {
    double render_ms;          /* device time from first raygen to film write */
    int64_t paths;             /* width*height*samples, summed over a batch's jobs */
    int64_t segments;          /* ray segments traced (closest-hit queries) */
    int64_t shadow_rays;       /* NEE occlusion queries */
    int64_t thinfilm_hits;     /* thin-film scatter events */
    int64_t thinfilm_fallback; /* of those, evaluated exactly because the surrogate's range did not cover them */
    int32_t kernel_launches;   /* kernels launched by the render */
    int32_t waves;
    int32_t surrogate_ctas_per_sm; /* resident CTAs per SM of the surrogate kernel (0: exact render) */
    int32_t reserved;
} lambda_render_stats;

lambda_status lambda_get_render_stats(const lambda_ctx *ctx, lambda_render_stats *stats);

/* Per-stage device time of the last render made with LAMBDA_RENDER_PROFILE_STAGES.
 * Stages: 0 init, 1 wave prologue, 2 raygen, 3 intersect, 4 Lambertian shade,
 * 5 mirror/dielectric shade, 6 thin-film shade (exact), 7 shadow rays, 8 finish,
 * 9-11 thin-film shade with the surrogate: 9 the hits' queries encoded as MLP rows,
 * 10 the tensor-core MLP, 11 the scatter (with the exact transfer matrix for hits
 * outside the surrogate's domain), 12 the path kernel of small passes (every sample
 * and bounce of a pixel in one thread; items = segments), 13 the fused bounce kernel
 * (tuning.fused_bounce: a bounce's intersect, shade and shadow rays in one launch;
 * items = segments). items = paths, rays or hits the stage processed over the whole
 * render. No reference counterpart (the reference's single kernel has no stages). */
#define LAMBDA_NUM_STAGES 14
typedef struct lambda_stage_time {
    double ms;
    int64_t launches;
    int64_t items;
} lambda_stage_time;

lambda_status lambda_get_stage_times(const lambda_ctx *ctx, lambda_stage_time *out /* [LAMBDA_NUM_STAGES] */);

/* ---------------------------------------------------------------------------
 * Ray queries on the uploaded scene: Scene::hit (src/scene/scene.h:51-124).
 * ------------------------------------------------------------------------- */

/* Closest hit of n rays; rays is [n][6] (origin xyz, direction xyz). Writes the
 * hit instance and object index (-1 on a miss) and t (1e30 on a miss). Same
 * arithmetic and visit order as the reference, so ids and t match bit for bit. */
lambda_status lambda_trace_closest(lambda_ctx *ctx, const float *rays, int32_t n,
                                   int32_t *out_instance, int32_t *out_object, float *out_t);

/* Shadow queries Scene::hit(r, i, occludedInstance, occludedObject) (scene.h:51,
 * renderer.h:166): occluded[k] = 1 when ray k does not reach light (instance,
 * object) = (light_instance[k], light_object[k]); (-1, -1) is the background. */
lambda_status lambda_trace_shadow(lambda_ctx *ctx, const float *rays, const int32_t *light_instance,
                                  const int32_t *light_object, int32_t n, int32_t *out_occluded);

/* ---------------------------------------------------------------------------
 * Thin-film transfer matrix (material.h:263-309) and its learned surrogate.
 * ------------------------------------------------------------------------- */

/* One single-layer film query: outer medium index 1, film index n_film, substrate
 * n_sub, all real; thickness in nm; cos_theta of incidence in the outer medium. */
typedef struct lambda_film_query {
    float lambda_nm;
    float cos_theta;
    float thickness_nm;
    float n_film;
    float n_sub;
} lambda_film_query;

/* Exact FP32 transfer matrix: out is [n][4] = (R_s, R_p, T_s, T_p). */
lambda_status lambda_thinfilm_exact(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, float *out);

/* FP64 transfer matrix (the training labeller and error audit): out [n][4] doubles. */
lambda_status lambda_thinfilm_fp64(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, double *out);

/* Surrogate MLP 5->64->64->64->4 (ReLU hidden layers), BF16 weights. A query
 * (lambda, cos theta, d, n_film, n_sub) enters encoded as (cos 2delta, sin 2delta,
 * cos theta, n_film, n_sub), with 2delta = 4 pi n_film d cos(theta_film) / lambda
 * the film's round-trip phase and the last three normalised to [-1, 1] over the
 * trained range. */
#define LAMBDA_MLP_IN 5
#define LAMBDA_MLP_HIDDEN 64
#define LAMBDA_MLP_OUT 4
#define LAMBDA_MLP_PARAMS (5 * 64 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 * 4 + 4) /* 8964 */

/* Where a render trusts the surrogate inside its trained range. The network's
 * error concentrates at grazing incidence: over 2^18 uniform queries of the
 * trained box its largest |R error| is 0.19 at cos theta < 0.05, and the next
 * largest sit at a substrate index near 1 (a film in air) below cos theta 0.2.
 * A thin-film hit with cos theta < LAMBDA_SURROGATE_GRAZING_COS, or with
 * n_sub < LAMBDA_SURROGATE_LOW_SUB_INDEX and cos theta < LAMBDA_SURROGATE_LOW_SUB_COS,
 * therefore takes the exact FP32 transfer matrix, like a hit outside the range
 * (the render statistics count both as fallbacks). The query entry points
 * (lambda_surrogate_eval*) evaluate the network everywhere in the range. */
#define LAMBDA_SURROGATE_GRAZING_COS 0.05f
#define LAMBDA_SURROGATE_LOW_SUB_INDEX 1.05f
#define LAMBDA_SURROGATE_LOW_SUB_COS 0.2f

/* Trained range of the surrogate (queries outside it use the exact path). */
typedef struct lambda_film_range {
    float lambda_nm[2];
    float cos_theta[2];
    float thickness_nm[2];
    float n_film[2];
    float n_sub[2];
} lambda_film_range;

typedef struct lambda_train_desc {
    int64_t samples;        /* training set size, labelled by the FP64 transfer matrix (2^24) */
    int32_t epochs;
    int32_t batch;          /* minibatch rows */
    float learning_rate;    /* Adam step size */
    uint64_t seed;
    lambda_film_range range;
} lambda_train_desc;

typedef struct lambda_train_report {
    double train_ms;
    double label_ms;
    float final_loss;       /* mean squared error over the last epoch */
    float max_abs_error;    /* max |surrogate - fp64| over a held-out audit set */
    float mean_abs_error;
    int32_t audit_samples;
} lambda_train_report;

/* Trains the surrogate on the GPU with the library's forward/backward kernels and
 * installs it on the context. */
lambda_status lambda_surrogate_train(lambda_ctx *ctx, const lambda_train_desc *desc,
                                     lambda_train_report *report);

/* Installs surrogate weights: params is LAMBDA_MLP_PARAMS floats in the order
 * W1[64][5] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[4][64] b4[4] (row-major,
 * out x in), with the input normalisation range. */
lambda_status lambda_surrogate_set(lambda_ctx *ctx, const float *params, const lambda_film_range *range);

/* Reads back the installed weights (LAMBDA_MLP_PARAMS floats) and range. */
lambda_status lambda_surrogate_get(const lambda_ctx *ctx, float *params, lambda_film_range *range);

/* Surrogate inference on the tensor cores: out [n][4] = (R_s, R_p, T_s, T_p). */
lambda_status lambda_surrogate_eval(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, float *out);

/* Allocation-free surrogate evaluation, for callers that must not allocate device
 * memory where they evaluate films (a host renderer whose device memory belongs to
 * its own pool allocator, such as a game engine or plug-in host, and whose render
 * thread may not call cudaMalloc, which can synchronise the device and fail under
 * the host's memory budget). It has no counterpart in the reference.
 * queries [n] and out [n][4] = (R_s, R_p, T_s, T_p) are caller-owned DEVICE
 * memory of the context's own GPU, or managed memory (out 16-byte aligned); a
 * host pointer or another GPU's memory returns LAMBDA_ERR_INVALID_ARGUMENT.
 * Results equal lambda_surrogate_eval's bit for bit. The only scratch is a fixed
 * array of LAMBDA_SURROGATE_STATIC_MAX_QUERIES encoded queries (4 MiB) compiled
 * into the library, held by every GPU that loads it until the process exits; n
 * above the limit returns LAMBDA_ERR_INVALID_ARGUMENT. The first call on a device,
 * and the first after a device reset, looks up the array's device address
 * (cudaGetSymbolAddress), which can load the library's GPU module and so
 * allocate: make that first call as a warm-up, outside the code that must not
 * allocate and before any stream capture. Every call shares the array: calls that
 * overlap on the GPU race. The call blocks until `out` is written. */
#define LAMBDA_SURROGATE_STATIC_MAX_QUERIES 131072
lambda_status lambda_surrogate_eval_static(lambda_ctx *ctx, const lambda_film_query *queries, int32_t n, float *out);

/* One forward/backward of the training kernel on caller data, for gradient
 * checks: params [LAMBDA_MLP_PARAMS], x [n][5] already-encoded inputs,
 * y [n][4] targets (host memory, n <= 65536). Writes the mean squared
 * error over the 4 outputs and its gradient with respect to params. The forward
 * pass rounds weights, inputs and hidden activations to BF16 as inference does. */
lambda_status lambda_surrogate_grad(lambda_ctx *ctx, const float *params, const float *x, const float *y, int32_t n,
                                    float *grad_out, float *loss_out);

#ifdef __cplusplus
}
#endif

#endif /* LAMBDA_GPU_H */
