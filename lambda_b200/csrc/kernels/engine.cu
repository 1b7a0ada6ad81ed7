// GPU half of the C ABI (include/lambda_gpu.h): context, scene upload, the
// wavefront render loop, ray queries and thin-film queries.
//
// A render pass is one CUDA graph launch (render_pass): clear + init, a conditional
// while node whose body is one sample wave (wavefront.cuh: prologue, raygen, then
// per bounce intersect followed by the material branches, run in parallel), then the
// film average. Kernels read queue sizes from device counters and exit early when
// their queue is empty.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "lambda_gpu.h"
#include "engine.h"
#include "wavefront.cuh"
#include "wide_bvh.h"

#include "../host/tables.inc"

using namespace lambda_dev;

namespace {

thread_local std::string g_create_error;

}  // namespace

// ---------------------------------------------------------------------------
// Context plumbing
// ---------------------------------------------------------------------------

lambda_status lambda_ctx::fail(lambda_status s, const std::string &msg) {
    last_error = msg;
    return s;
}

lambda_status lambda_ctx::cuda_fail(cudaError_t e, const char *what) {
    last_error = std::string(what) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? LAMBDA_ERR_OUT_OF_MEMORY : LAMBDA_ERR_CUDA;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

cudaError_t DeviceBuffer::reserve(size_t n) {
    if (n <= bytes) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return e;
    }
    bytes = n;
    return cudaSuccess;
}

cudaError_t DeviceBuffer::upload(const void *src, size_t n, cudaStream_t st) {
    cudaError_t e = reserve(n ? n : 16);
    if (e != cudaSuccess || n == 0) return e;
    return cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, st);
}

bool is_device_pointer(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

#define CK(call, what)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return ctx->cuda_fail(e_, what); \
    } while (0)

extern "C" lambda_status lambda_ctx_create(int32_t device, lambda_ctx **out) {
    if (!out) return LAMBDA_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        g_create_error = std::string("no CUDA device (") + cudaGetErrorString(e) + ")";
        cudaGetLastError();
        return LAMBDA_ERR_CUDA;
    }
    if (device < 0 || device >= n) {
        g_create_error = "device index out of range";
        return LAMBDA_ERR_INVALID_ARGUMENT;
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaSetDevice failed (") + cudaGetErrorString(e) + ")";
        return LAMBDA_ERR_CUDA;
    }
    auto ctx = std::make_unique<lambda_ctx>();
    ctx->device = device;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    ctx->sm_count = prop.multiProcessorCount;
    if (prop.major < 10) {
        g_create_error = "this library is built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                         std::to_string(prop.minor);
        return LAMBDA_ERR_UNSUPPORTED;
    }
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaStreamCreate failed (") + cudaGetErrorString(e) + ")";
        return LAMBDA_ERR_CUDA;
    }
    cudaEventCreate(&ctx->ev_start);
    cudaEventCreate(&ctx->ev_stop);
    for (int i = 0; i < 3; i++) {
        e = cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking);
        if (e == cudaSuccess && i < 2) e = cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            g_create_error = std::string("cudaStreamCreate failed (") + cudaGetErrorString(e) + ")";
            return LAMBDA_ERR_CUDA;
        }
    }
    e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_lambert, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_shadow, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaEventCreate failed (") + cudaGetErrorString(e) + ")";
        return LAMBDA_ERR_CUDA;
    }
    *out = ctx.release();
    return LAMBDA_OK;
}

lambda_ctx::~lambda_ctx() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (progress_host) cudaFreeHost(progress_host);
    for (DeviceBuffer *b : all_buffers()) b->release();
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_lambert) cudaEventDestroy(ev_lambert);
    if (ev_shadow) cudaEventDestroy(ev_shadow);
    for (int i = 0; i < 2; i++)
        if (ev_join[i]) cudaEventDestroy(ev_join[i]);
    for (int i = 0; i < 3; i++)
        if (side[i]) cudaStreamDestroy(side[i]);
    if (stream) cudaStreamDestroy(stream);
}

extern "C" void lambda_ctx_destroy(lambda_ctx *ctx) { delete ctx; }

extern "C" const char *lambda_last_error(const lambda_ctx *ctx) {
    if (!ctx) return g_create_error.c_str();
    return ctx->last_error.c_str();
}

// ---------------------------------------------------------------------------
// Scene upload
// ---------------------------------------------------------------------------

namespace {

float host_fract(float x) { return x - std::floor(x); }

// Feature offsets of Worley cells as the reference computes them (utils.h:165)
// with the C library's sinf, for every cell the scene's Worley textures can
// reach: the world bounds (TLAS root) and the unit sphere (background lookups),
// each times the texture frequency, plus a margin of two cells.
void build_worley_table(const lambda_scene_desc &d, std::vector<float4> &cells, int3 &lo, int3 &dim) {
    dim = make_int3(0, 0, 0);
    lo = make_int3(0, 0, 0);
    if (d.num_nodes == 0) return;
    double bmin[3], bmax[3];
    bool any = false;
    for (int t = 0; t < d.num_scalar_textures; t++) {
        const lambda_scalar_texture &x = d.scalar_textures[t];
        if (x.type != LAMBDA_SCALAR_WORLEY) continue;
        const double f = std::fabs(double(x.p[2]));
        for (int k = 0; k < 3; k++) {
            const double a = std::min({double(d.nodes[0].min[k]) * f, double(d.nodes[0].max[k]) * f, -f});
            const double b = std::max({double(d.nodes[0].min[k]) * f, double(d.nodes[0].max[k]) * f, f});
            bmin[k] = any ? std::min(bmin[k], a) : a;
            bmax[k] = any ? std::max(bmax[k], b) : b;
        }
        any = true;
    }
    if (!any) return;
    long long n = 1;
    int l[3], e[3];
    for (int k = 0; k < 3; k++) {
        if (!(std::fabs(bmin[k]) < 1e6 && std::fabs(bmax[k]) < 1e6)) return;
        l[k] = int(std::floor(bmin[k])) - 2;
        e[k] = int(std::floor(bmax[k])) + 2 - l[k] + 1;
        n *= e[k];
    }
    constexpr long long kMaxCells = 8ll << 20;  // 128 MB of float4
    if (n > kMaxCells) return;
    cells.resize(size_t(n));
    for (int z = 0; z < e[2]; z++)
        for (int y = 0; y < e[1]; y++)
            for (int x = 0; x < e[0]; x++) {
                const float cx = float(l[0] + x), cy = float(l[1] + y), cz = float(l[2] + z);
                const float a = cx * 127.1f + cy * 311.7f + cz * 74.7f;
                const float b = cx * 269.5f + cy * 183.3f + cz * 246.1f;
                const float c = cx * 113.5f + cy * 271.9f + cz * 124.6f;
                cells[(size_t(z) * e[1] + y) * e[0] + x] = make_float4(host_fract(std::sin(a) * 43758.5453f),
                                                                       host_fract(std::sin(b) * 43758.5453f),
                                                                       host_fract(std::sin(c) * 43758.5453f), 0.0f);
            }
    lo = make_int3(l[0], l[1], l[2]);
    dim = make_int3(e[0], e[1], e[2]);
}

float spectrum_average_host(const float *d) {
    float s = 0;
    for (int k = 0; k < LAMBDA_CIE_BINS; k++) s += d[k];
    return s / LAMBDA_CIE_BINS;
}

float spectrum_texture_average_host(const lambda_scene_desc &d, int t) {
    const lambda_spectrum_texture &x = d.spectrum_textures[t];
    if (x.type == LAMBDA_SPECTRUM_CONSTANT) return spectrum_average_host(d.spectra + size_t(x.value1) * LAMBDA_CIE_BINS);
    if (x.type == LAMBDA_SPECTRUM_CHECKER)
        return 0.5f * (spectrum_average_host(d.spectra + size_t(x.value1) * LAMBDA_CIE_BINS) +
                       spectrum_average_host(d.spectra + size_t(x.value2) * LAMBDA_CIE_BINS));
    const lambda_scalar_texture &s = d.scalar_textures[x.value1];
    return s.type == LAMBDA_SCALAR_CONSTANT ? s.p[0] : (s.p[0] + s.p[1]) / 2;
}

lambda_status validate_scene(lambda_ctx *ctx, const lambda_scene_desc &d) {
    if (d.num_nodes < 1 || d.num_objects < 1 || d.num_instances < 1 || d.num_lights < 1 || d.num_spectra < 1 ||
        d.num_materials < 1 || d.num_spectrum_textures < 1 || d.num_scalar_textures < 1)
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "scene has an empty required container");
    if (!d.nodes || !d.objects || !d.instances || !d.spectra || !d.materials || !d.spectrum_textures ||
        !d.scalar_textures || !d.light_instances || !d.light_objects || !d.light_powers)
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "scene has a null container pointer");
    if (d.background_texture < 0 || d.background_texture >= d.num_spectrum_textures)
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "background texture index out of range");
    auto bad = [&](const char *m) { return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, m); };
    for (int i = 0; i < d.num_nodes; i++) {
        const lambda_bvh_node &n = d.nodes[i];
        if (n.count > 0 ? n.index < 0 : (n.index <= i || n.index >= d.num_nodes || i + 1 >= d.num_nodes))
            return bad("BVH node index out of range");
    }
    for (int i = 0; i < d.num_instances; i++) {
        const lambda_instance &in = d.instances[i];
        if (in.object < 0 || in.count < 1 || in.object + in.count > d.num_objects || in.node < 0 ||
            in.node >= d.num_nodes || in.material >= d.num_materials)
            return bad("instance fields out of range");
    }
    for (int i = 0; i < d.num_objects; i++)
        if (d.objects[i].material < 0 || d.objects[i].material >= d.num_materials || d.objects[i].type < 0 ||
            d.objects[i].type > 2)
            return bad("object fields out of range");
    auto spec_tex_ok = [&](int t) { return t >= 0 && t < d.num_spectrum_textures; };
    for (int i = 0; i < d.num_materials; i++) {
        const lambda_material &m = d.materials[i];
        if (m.type == LAMBDA_MATERIAL_THINFILM) {
            if (m.p[0] < 0 || m.p[0] > kMaxFilmLayers) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "thin film with more than 8 layers");
            if (!d.complex_spectra || !d.material_properties || m.p[1] < 0 ||
                m.p[1] + m.p[0] + 2 > d.num_material_properties || m.p[2] < 0 ||
                m.p[2] + m.p[0] > d.num_material_properties)
                return bad("thin-film properties out of range");
            for (int k = 0; k < m.p[0] + 2; k++) {
                const int c = d.material_properties[m.p[1] + k];
                if (c < 0 || c >= d.num_complex_spectra) return bad("thin-film index spectrum out of range");
            }
            for (int k = 0; k < m.p[0]; k++) {
                const int t = d.material_properties[m.p[2] + k];
                if (t < 0 || t >= d.num_scalar_textures) return bad("thin-film thickness texture out of range");
            }
        } else if (m.type == LAMBDA_MATERIAL_DIELECTRIC) {
            if (m.p[0] < 0 || m.p[0] >= d.num_spectra || m.p[1] < 0 || m.p[1] >= d.num_spectra)
                return bad("dielectric spectrum out of range");
        } else if (m.type == LAMBDA_MATERIAL_LAMBERTIAN || m.type == LAMBDA_MATERIAL_MIRROR ||
                   m.type == LAMBDA_MATERIAL_EMISSIVE) {
            if (!spec_tex_ok(m.p[0])) return bad("material texture out of range");
        } else {
            return bad("material type out of range");
        }
    }
    for (int i = 0; i < d.num_spectrum_textures; i++) {
        const lambda_spectrum_texture &t = d.spectrum_textures[i];
        const bool ok = t.type == LAMBDA_SPECTRUM_CONSTANT ? (t.value1 >= 0 && t.value1 < d.num_spectra)
                      : t.type == LAMBDA_SPECTRUM_CHECKER
                          ? (t.value1 >= 0 && t.value1 < d.num_spectra && t.value2 >= 0 && t.value2 < d.num_spectra)
                      : t.type == LAMBDA_SPECTRUM_SCALAR ? (t.value1 >= 0 && t.value1 < d.num_scalar_textures) : false;
        if (!ok) return bad("spectrum texture fields out of range");
    }
    for (int i = 0; i < d.num_scalar_textures; i++)
        if (d.scalar_textures[i].type < 0 || d.scalar_textures[i].type > 2) return bad("scalar texture type out of range");
    for (int i = 0; i < d.num_lights; i++) {
        const int li = d.light_instances[i], lo = d.light_objects[i];
        const bool bg = li == -1 && lo == -1;
        if (!bg && (li < 0 || li >= d.num_instances || lo < 0 || lo >= d.num_objects)) return bad("light id out of range");
    }
    if (d.light_instances[d.num_lights - 1] != -1) return bad("the last light must be the background (-1, -1)");
    return LAMBDA_OK;
}

}  // namespace

int layout_index(const lambda_tuning &t) {
    return (t.bvh_width == 2 ? 0 : (t.bvh_width == 4 ? 1 : 2)) + (t.compressed_nodes ? 3 : 0);
}

DeviceScene lambda_ctx::scene_view(int width) const {
    const int k = width == 2 ? 0 : (width == 4 ? 1 : 2);
    DeviceScene v = dscene;
    v.wide = scene.wide[k].as<float4>();
    v.wide_leaves = scene.wide_leaves[k].as<int2>();
    v.wide_code = scene.wide_code[k].as<int>();
    v.wide_q = scene.wide_q[k].as<uint4>();
    v.num_leaves = wide_leaves_n[k];
    v.bvh_width = 2 << k;
    v.stack_tlas = wide_stack[k][0];
    v.stack_blas = wide_stack[k][1];
    if (limits.stack_entries > 0) {  // a test cap (lambda_set_limits): kernels then size and check stacks by it
        v.stack_tlas = std::min(v.stack_tlas, limits.stack_entries);
        v.stack_blas = std::min(v.stack_blas, limits.stack_entries);
    }
    return v;
}

extern "C" lambda_status lambda_scene_upload(lambda_ctx *ctx, const lambda_scene_desc *desc) {
    if (!ctx || !desc) return LAMBDA_ERR_INVALID_ARGUMENT;
    const lambda_scene_desc &d = *desc;
    lambda_status st = validate_scene(ctx, d);
    if (st != LAMBDA_OK) return st;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = ctx->stream;
    SceneBuffers &b = ctx->scene;

    // nodes: (min, index) (max, count)
    std::vector<float4> nodes(2 * size_t(d.num_nodes));
    for (int i = 0; i < d.num_nodes; i++) {
        const lambda_bvh_node &n = d.nodes[i];
        float idx, cnt;
        std::memcpy(&idx, &n.index, 4);
        std::memcpy(&cnt, &n.count, 4);
        nodes[2 * i] = make_float4(n.min[0], n.min[1], n.min[2], idx);
        nodes[2 * i + 1] = make_float4(n.max[0], n.max[1], n.max[2], cnt);
    }
    std::vector<float4> prims(4 * size_t(d.num_objects)), tri(4 * size_t(d.num_objects));
    for (int i = 0; i < d.num_objects; i++) {
        const lambda_object &o = d.objects[i];
        float ty, ma;
        std::memcpy(&ty, &o.type, 4);
        std::memcpy(&ma, &o.material, 4);
        const float *g = o.g;
        if (o.type == LAMBDA_OBJECT_SPHERE) {
            prims[4 * i] = make_float4(g[0], g[1], g[2], ty);
            prims[4 * i + 1] = make_float4(g[3], 0, 0, ma);
            prims[4 * i + 2] = make_float4(0, 0, 0, 0);
            prims[4 * i + 3] = make_float4(0, 0, 0, 0);
        } else {
            prims[4 * i] = make_float4(g[0], g[1], g[2], ty);
            prims[4 * i + 1] = make_float4(g[3], g[4], g[5], ma);
            prims[4 * i + 2] = make_float4(g[6], g[7], g[8], 0);
            prims[4 * i + 3] = make_float4(g[9], g[10], g[11], 0);
        }
        if (o.type == LAMBDA_OBJECT_TRI) {
            tri[4 * i] = make_float4(g[12], g[13], g[14], g[15]);
            tri[4 * i + 1] = make_float4(g[16], g[17], g[18], g[19]);
            tri[4 * i + 2] = make_float4(g[20], g[21], g[22], g[23]);
            tri[4 * i + 3] = make_float4(g[24], g[25], g[26], 0);
        } else {
            for (int k = 0; k < 4; k++) tri[4 * i + k] = make_float4(0, 0, 0, 0);
        }
    }
    std::vector<float4> inst(9 * size_t(d.num_instances));
    for (int i = 0; i < d.num_instances; i++) {
        const lambda_instance &in = d.instances[i];
        float h[4];
        std::memcpy(h, &in.object, 16);
        inst[9 * i] = make_float4(h[0], h[1], h[2], h[3]);
        for (int r = 0; r < 4; r++) {
            inst[9 * i + 1 + r] = make_float4(in.transform[4 * r], in.transform[4 * r + 1], in.transform[4 * r + 2], in.transform[4 * r + 3]);
            inst[9 * i + 5 + r] = make_float4(in.inverse_transform[4 * r], in.inverse_transform[4 * r + 1],
                                              in.inverse_transform[4 * r + 2], in.inverse_transform[4 * r + 3]);
        }
    }
    std::vector<uint8_t> flat(d.num_spectra), cflat(std::max(d.num_complex_spectra, 1), 0);
    for (int i = 0; i < d.num_spectra; i++) {
        const float *x = d.spectra + size_t(i) * LAMBDA_CIE_BINS;
        flat[i] = std::all_of(x, x + LAMBDA_CIE_BINS, [&](float v) { return v == x[0]; }) ? 1 : 0;
    }
    for (int i = 0; i < d.num_complex_spectra; i++) {
        const double *x = d.complex_spectra + size_t(i) * LAMBDA_CIE_BINS * 2;
        bool same = true;
        for (int k = 1; k < LAMBDA_CIE_BINS && same; k++) same = x[2 * k] == x[0] && x[2 * k + 1] == x[1];
        cflat[i] = same ? 1 : 0;
    }
    std::vector<int4> mats(d.num_materials);
    std::vector<float> emission(d.num_materials, 0.0f);
    for (int i = 0; i < d.num_materials; i++) {
        const lambda_material &m = d.materials[i];
        mats[i] = make_int4(m.type, m.p[0], m.p[1], m.p[2]);
        if (m.type == LAMBDA_MATERIAL_EMISSIVE) emission[i] = spectrum_texture_average_host(d, m.p[0]);
    }
    std::vector<float4> stex(d.num_scalar_textures);
    for (int i = 0; i < d.num_scalar_textures; i++) {
        const lambda_scalar_texture &t = d.scalar_textures[i];
        float ty;
        std::memcpy(&ty, &t.type, 4);
        stex[i] = make_float4(ty, t.p[0], t.p[1], t.p[2]);
    }
    std::vector<int4> sptex(d.num_spectrum_textures);
    for (int i = 0; i < d.num_spectrum_textures; i++) {
        const lambda_spectrum_texture &t = d.spectrum_textures[i];
        int sc;
        std::memcpy(&sc, &t.scale, 4);
        sptex[i] = make_int4(t.type, t.value1, t.value2, sc);
    }
    // materials whose spectrum texture (albedo or emission) is a checker read the hit's
    // (u, v); no other texture does (scalar textures read the point)
    std::vector<uint8_t> muv(std::max(d.num_materials, 1), 0);
    for (int i = 0; i < d.num_materials; i++) {
        const lambda_material &m = d.materials[i];
        if (m.type != LAMBDA_MATERIAL_LAMBERTIAN && m.type != LAMBDA_MATERIAL_MIRROR && m.type != LAMBDA_MATERIAL_EMISSIVE)
            continue;
        const int t = m.p[0];
        muv[i] = (t < 0 || t >= d.num_spectrum_textures || d.spectrum_textures[t].type == LAMBDA_SPECTRUM_CHECKER) ? 1 : 0;
    }
    std::vector<float> cdf(d.num_lights);
    float run = 0;
    for (int i = 0; i < d.num_lights; i++) {
        run += d.light_powers[i];
        cdf[i] = run;
    }
    std::vector<float> cie(LAMBDA_CIE_BINS * 3);
    for (int i = 0; i < LAMBDA_CIE_BINS; i++)
        for (int k = 0; k < 3; k++) cie[3 * i + k] = float(kCieXyz1931[i][k]);
    std::vector<float4> worley;
    int3 wlo, wdim;
    build_worley_table(d, worley, wlo, wdim);
    const std::vector<int> props(d.material_properties, d.material_properties + d.num_material_properties);
    // Per material: the three indices (outer medium, film, substrate) of a one-layer
    // thin film whose complex spectra are all non-dispersive (every bin equal) and
    // real, with w = 1; else zeros. Those are exactly the values a spectrum lookup
    // returns at any wavelength, so the film kernels take them from here instead.
    std::vector<float4> film_flat(size_t(std::max(d.num_materials, 1)), make_float4(0, 0, 0, 0));
    for (int i = 0; i < d.num_materials; i++) {
        const lambda_material &m = d.materials[i];
        if (m.type != LAMBDA_MATERIAL_THINFILM || m.p[0] != 1) continue;
        float v[3];
        bool ok = true;
        for (int k = 0; k < 3 && ok; k++) {
            const int cs = d.material_properties[m.p[1] + k];
            const double im = d.complex_spectra[size_t(cs) * LAMBDA_CIE_BINS * 2 + 1];
            ok = cflat[size_t(cs)] != 0 && im == 0.0 && !std::signbit(im);  // +0: the fast path uses +0 imaginary parts
            if (ok) v[k] = float(d.complex_spectra[size_t(cs) * LAMBDA_CIE_BINS * 2]);
        }
        if (ok) film_flat[size_t(i)] = make_float4(v[0], v[1], v[2], 1.0f);
    }

    CK(b.nodes.upload(nodes.data(), nodes.size() * sizeof(float4), s), "upload nodes");
    CK(b.prims.upload(prims.data(), prims.size() * sizeof(float4), s), "upload objects");
    CK(b.tri.upload(tri.data(), tri.size() * sizeof(float4), s), "upload triangles");
    CK(b.instances.upload(inst.data(), inst.size() * sizeof(float4), s), "upload instances");
    CK(b.spectra.upload(d.spectra, size_t(d.num_spectra) * LAMBDA_CIE_BINS * sizeof(float), s), "upload spectra");
    CK(b.spectrum_flat.upload(flat.data(), flat.size(), s), "upload spectra");
    CK(b.cspectra.upload(d.complex_spectra, size_t(d.num_complex_spectra) * LAMBDA_CIE_BINS * 2 * sizeof(double), s),
       "upload complex spectra");
    CK(b.cspectrum_flat.upload(cflat.data(), cflat.size(), s), "upload complex spectra");
    CK(b.materials.upload(mats.data(), mats.size() * sizeof(int4), s), "upload materials");
    CK(b.material_props.upload(props.data(), props.size() * sizeof(int), s), "upload material properties");
    CK(b.scalar_tex.upload(stex.data(), stex.size() * sizeof(float4), s), "upload textures");
    CK(b.spectrum_tex.upload(sptex.data(), sptex.size() * sizeof(int4), s), "upload textures");
    CK(b.light_inst.upload(d.light_instances, size_t(d.num_lights) * sizeof(int), s), "upload lights");
    CK(b.light_obj.upload(d.light_objects, size_t(d.num_lights) * sizeof(int), s), "upload lights");
    CK(b.light_power.upload(d.light_powers, size_t(d.num_lights) * sizeof(float), s), "upload lights");
    CK(b.light_cdf.upload(cdf.data(), cdf.size() * sizeof(float), s), "upload lights");
    CK(b.material_emission.upload(emission.data(), emission.size() * sizeof(float), s), "upload materials");
    CK(b.material_uv.upload(muv.data(), muv.size(), s), "upload materials");
    CK(b.film_flat.upload(film_flat.data(), film_flat.size() * sizeof(float4), s), "upload materials");
    CK(b.cie.upload(cie.data(), cie.size() * sizeof(float), s), "upload CIE table");
    CK(b.perm.upload(kPerlinPermutation, sizeof(kPerlinPermutation), s), "upload permutation");
    CK(b.worley.upload(worley.data(), worley.size() * sizeof(float4), s), "upload Worley lattice");
    for (int k = 0; k < 3; k++) {
        lambda_host::WideBvh w = lambda_host::build_wide_bvh(d.nodes, d.num_nodes, d.instances, d.num_instances, 2 << k);
        w.records.resize(std::max<size_t>(w.records.size(), 8));
        w.leaves.resize(std::max<size_t>(w.leaves.size(), 2));
        CK(b.wide[k].upload(w.records.data(), w.records.size() * sizeof(float), s), "upload wide BVH");
        CK(b.wide_leaves[k].upload(w.leaves.data(), w.leaves.size() * sizeof(int32_t), s), "upload wide BVH");
        CK(b.wide_code[k].upload(w.code.data(), w.code.size() * sizeof(int32_t), s), "upload wide BVH");
        CK(b.wide_q[k].upload(w.quant.data(), w.quant.size() * sizeof(uint32_t), s), "upload wide BVH");
        ctx->wide_leaves_n[k] = int(w.leaves.size() / 2);
        CK(cudaStreamSynchronize(s), "upload wide BVH");  // the host vectors go out of scope
        ctx->wide_stack[k][0] = w.stack_tlas;
        ctx->wide_stack[k][1] = w.stack_blas;
    }
    std::vector<uint32_t> iflags(d.num_instances, 0);
    for (int i = 0; i < d.num_instances; i++) {
        bool ident = true;
        for (int k = 0; k < 16; k++) {
            const float e = (k % 5 == 0) ? 1.0f : 0.0f;
            ident = ident && d.instances[i].transform[k] == e && d.instances[i].inverse_transform[k] == e;
        }
        iflags[i] = ident ? 1u : 0u;
    }
    // bit 1: the instance is the only one of its TLAS leaf and that leaf's box is its
    // BLAS root's box, so (with an identity transform) the root's box test repeats
    // the leaf's and is skipped
    if (d.num_nodes > 0) {
        std::vector<int> todo = {0};
        while (!todo.empty()) {
            const int n = todo.back();
            todo.pop_back();
            const lambda_bvh_node &nd = d.nodes[n];
            if (nd.count <= 0) {
                todo.push_back(nd.index);
                todo.push_back(n + 1);
                continue;
            }
            if (nd.count != 1 || nd.index < 0 || nd.index >= d.num_instances || !(iflags[nd.index] & 1u)) continue;
            const int root = d.instances[nd.index].node;
            if (root < 0 || root >= d.num_nodes) continue;
            const lambda_bvh_node &r = d.nodes[root];
            bool same = true;
            for (int k = 0; k < 3; k++) same = same && nd.min[k] == r.min[k] && nd.max[k] == r.max[k];
            if (same) iflags[nd.index] |= 2u;
        }
    }
    CK(b.instance_flags.upload(iflags.data(), iflags.size() * sizeof(uint32_t), s), "upload instances");
    uint32_t families = 0;
    for (int i = 0; i < d.num_materials; i++) {
        const int t = d.materials[i].type;
        families |= t == LAMBDA_MATERIAL_LAMBERTIAN ? 1u : (t == LAMBDA_MATERIAL_THINFILM ? 4u : (t == LAMBDA_MATERIAL_EMISSIVE ? 0u : 2u));
    }
    CK(cudaStreamSynchronize(s), "scene upload");

    DeviceScene &ds = ctx->dscene;
    ds.nodes = b.nodes.as<float4>();
    ds.prims = b.prims.as<float4>();
    ds.tri_attr = b.tri.as<float4>();
    ds.instances = b.instances.as<float4>();
    ds.spectra = b.spectra.as<float>();
    ds.spectrum_flat = b.spectrum_flat.as<uint8_t>();
    ds.cspectra = b.cspectra.as<double2>();
    ds.cspectrum_flat = b.cspectrum_flat.as<uint8_t>();
    ds.materials = b.materials.as<int4>();
    ds.material_props = b.material_props.as<int>();
    ds.scalar_tex = b.scalar_tex.as<float4>();
    ds.spectrum_tex = b.spectrum_tex.as<int4>();
    ds.light_inst = b.light_inst.as<int>();
    ds.light_obj = b.light_obj.as<int>();
    ds.light_power = b.light_power.as<float>();
    ds.light_cdf = b.light_cdf.as<float>();
    ds.material_emission = b.material_emission.as<float>();
    ds.material_uv = b.material_uv.as<uint8_t>();
    ds.film_flat = b.film_flat.as<float4>();
    ds.instance_flags = b.instance_flags.as<uint32_t>();
    ds.families = families;
    ds.cie = b.cie.as<float>();
    ds.perm = b.perm.as<int>();
    ds.worley_cells = b.worley.as<float4>();
    ds.worley_lo = wlo;
    ds.worley_dim = wdim;
    ds.num_nodes = d.num_nodes;
    ds.num_objects = d.num_objects;
    ds.num_instances = d.num_instances;
    ds.num_lights = d.num_lights;
    ds.total_light_power = d.total_light_power;
    ds.background_texture = d.background_texture;
    ctx->dscene = ctx->scene_view(4);
    ctx->has_scene = true;
    ctx->film_layers_max = 0;
    for (int i = 0; i < d.num_materials; i++)
        if (d.materials[i].type == LAMBDA_MATERIAL_THINFILM) ctx->film_layers_max = std::max(ctx->film_layers_max, d.materials[i].p[0]);
    return LAMBDA_OK;
}

// ---------------------------------------------------------------------------
// Render
// ---------------------------------------------------------------------------

namespace {

struct Progress {
    volatile int32_t *completed;
    int32_t value;
};

void CUDART_CB progress_cb(void *p) {
    auto *pr = static_cast<Progress *>(p);
    *pr->completed = pr->value;
}

}  // namespace

StageProfiler::StageProfiler(cudaStream_t s) : stream(s) {}

StageProfiler::~StageProfiler() {
    for (auto &e : pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
}

void StageProfiler::begin(int stage) {
    if (used == pool.size()) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        pool.push_back({a, b});
        stages.push_back(0);
    }
    stages[used] = stage;
    cudaEventRecord(pool[used].first, stream);
}

void StageProfiler::end() {
    cudaEventRecord(pool[used].second, stream);
    used++;
}

cudaError_t StageProfiler::collect() {
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    for (size_t i = 0; i < used; i++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, pool[i].first, pool[i].second);
        totals[stages[i]] += ms;
        counts[stages[i]]++;
    }
    used = 0;
    return cudaSuccess;
}

lambda_status lambda_ctx::ensure_state(int pixels, int depth) {
    lambda_ctx *ctx = this;
    const size_t P = size_t(pixels);
    RenderBuffers &r = rbuf;
    CK(r.rng.reserve(P * 8), "allocate path state");
    CK(r.film.reserve(P * 16), "allocate path state");
    CK(r.lam.reserve(P * 16), "allocate path state");
    CK(r.ray_o.reserve(P * 16), "allocate path state");
    CK(r.ray_d.reserve(P * 16), "allocate path state");
    CK(r.throughput.reserve(P * 16), "allocate path state");
    CK(r.radiance.reserve(P * 16), "allocate path state");
    CK(r.emit.reserve(P * 16), "allocate path state");
    CK(r.hit_id.reserve(P * 16), "allocate path state");
    CK(r.sh_o.reserve(P * 16), "allocate path state");
    CK(r.sh_d.reserve(P * 16), "allocate path state");
    CK(r.sh_a.reserve(P * 16), "allocate path state");
    CK(r.sh_light.reserve(P * 8), "allocate path state");
    CK(r.path_info.reserve(P * 8), "allocate path state");
    CK(r.q0.reserve(P * 4), "allocate queues");
    CK(r.q1.reserve(P * 4), "allocate queues");
    CK(r.qs.reserve(P * 4), "allocate queues");
    CK(r.qm0.reserve(P * 4), "allocate queues");
    CK(r.qm1.reserve(P * 4), "allocate queues");
    CK(r.qm2.reserve(P * 4), "allocate queues");
    CK(r.counts.reserve(size_t(kQueues * (depth + 2)) * 4), "allocate queues");
    CK(r.wave.reserve(16), "allocate queues");
    CK(r.stats.reserve(8 * 8), "allocate statistics");
    CK(r.error.reserve(16), "allocate flags");
    PathState &ps = pstate;
    ps.rng = r.rng.as<uint64_t>();
    ps.film = r.film.as<float4>();
    ps.lam = r.lam.as<float4>();
    ps.ray_o = r.ray_o.as<float4>();
    ps.ray_d = r.ray_d.as<float4>();
    ps.throughput = r.throughput.as<float4>();
    ps.radiance = r.radiance.as<float4>();
    ps.emit = r.emit.as<float4>();
    ps.hit_id = r.hit_id.as<int4>();
    ps.sh_o = r.sh_o.as<float4>();
    ps.sh_d = r.sh_d.as<float4>();
    ps.sh_a = r.sh_a.as<float4>();
    ps.sh_light = r.sh_light.as<int2>();
    ps.path_info = r.path_info.as<int2>();
    ps.queue[0] = r.q0.as<int>();
    ps.queue[1] = r.q1.as<int>();
    ps.shadow_queue = r.qs.as<int>();
    ps.mat_queue[0] = r.qm0.as<int>();
    ps.mat_queue[1] = r.qm1.as<int>();
    ps.mat_queue[2] = r.qm2.as<int>();
    ps.counts = r.counts.as<int>();
    ps.wave = r.wave.as<int>();
    ps.stats = r.stats.as<unsigned long long>();
    ps.error = r.error.as<int>();
    return LAMBDA_OK;
}

int resident_ctas(const void *fn, int device, int block, size_t dyn_smem) {
    cudaFuncAttributes fa{};
    int smem_sm = 0, regs_sm = 0, threads_sm = 0, reserved = 0, blocks_sm = 0;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&blocks_sm, cudaDevAttrMaxBlocksPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const int regs = (std::max(fa.numRegs, 1) + 7) / 8 * 8;
    const int by_regs = regs_sm / (block * regs);
    const int by_smem = smem_sm / int(dyn_smem + fa.sharedSizeBytes + reserved);
    const int by_threads = threads_sm / block;
    return std::max(1, std::min({by_regs, by_smem, by_threads, blocks_sm}));
}

namespace {

lambda_status check_settings(lambda_ctx *ctx, const lambda_render_settings &st) {
    if (st.width <= 0 || st.height <= 0 || st.depth < 0 || st.samples < 1 || st.sqrt_samples * st.sqrt_samples != st.samples)
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "invalid render settings");
    if (!(st.lambda_min >= LAMBDA_CIE_LAMBDA_MIN && st.lambda_max <= LAMBDA_CIE_LAMBDA_MAX && st.lambda_min < st.lambda_max))
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "wavelength range outside [360, 830] nm");
    if (int64_t(st.width) * st.height > (int64_t(1) << 30)) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "image too large");
    if (st.depth > 1024) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "depth above 1024");
    return LAMBDA_OK;
}

Job device_job(const lambda_job &j) {
    const lambda_render_settings &st = j.desc.settings;
    Job d{};
    d.width = st.width;
    d.height = st.height;
    d.depth = st.depth;
    d.samples = st.samples;
    d.sqrt_samples = st.sqrt_samples;
    d.lambda_min = st.lambda_min;
    d.lambda_max = st.lambda_max;
    d.lambda_range = st.lambda_max - st.lambda_min;
    const lambda_camera &c = st.camera;
    d.cam_pos = mk(c.position[0], c.position[1], c.position[2]);
    d.cam_corner = mk(c.corner[0], c.corner[1], c.corner[2]);
    d.cam_h = mk(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    d.cam_v = mk(c.vertical[0], c.vertical[1], c.vertical[2]);
    d.seed = j.desc.seed;
    return d;
}

// Totals over the passes of one render call.
struct RenderTotals {
    double ms = 0;
    int64_t paths = 0, pixels = 0;
    unsigned long long stats[8] = {0};
    int launches = 0, waves = 0;
    int err = 0;
};

// Renders jobs[order[first..last)] as one wavefront pass (see lambda_render_batch).
lambda_status render_pass(lambda_ctx *ctx, const lambda_job *jobs, const std::vector<int> &order, size_t first,
                          size_t last, bool surrogate, bool fp64, StageProfiler *prof, volatile int32_t *completed,
                          int32_t completed_base, int32_t completed_total, RenderTotals &tot) {
    const size_t nj = last - first;
    std::vector<Job> dj(nj);
    int64_t P64 = 0, host_pixels = 0;
    int s_max = 0, d_max = 0;
    for (size_t k = 0; k < nj; k++) {
        const lambda_job &j = jobs[order[first + k]];
        dj[k] = device_job(j);
        dj[k].base = int(P64);
        P64 += int64_t(dj[k].width) * dj[k].height;
        if (!(j.desc.flags & LAMBDA_RENDER_OUTPUT_DEVICE)) host_pixels += int64_t(dj[k].width) * dj[k].height;
        s_max = std::max(s_max, dj[k].samples);
        d_max = std::max(d_max, dj[k].depth);
    }
    if (P64 > (int64_t(1) << 30)) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "more than 2^30 pixels in one pass");
    const int P = int(P64);
    // pixels with a sample in wave s: jobs are ordered by decreasing samples
    std::vector<int> active(size_t(s_max) + 1, 0);
    for (int s = 0; s <= s_max; s++)
        for (size_t k = 0; k < nj; k++)
            if (dj[k].samples > s) active[s] += dj[k].width * dj[k].height;

    lambda_status st = ctx->ensure_state(P, d_max);
    if (st != LAMBDA_OK) return st;
    if (surrogate) {
        // four MLP rows per thin-film hit, counted in int
        if (P > INT32_MAX / 4) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "more than 2^29 pixels in one surrogate pass");
        st = ctx->ensure_surrogate_state(P);
        if (st != LAMBDA_OK) return st;
    }
    RenderBuffers &r = ctx->rbuf;
    CK(r.out.reserve(size_t(std::max<int64_t>(host_pixels, 1)) * 12), "allocate output");
    int64_t host_off = 0;
    for (size_t k = 0; k < nj; k++) {
        const lambda_job &j = jobs[order[first + k]];
        if (j.desc.flags & LAMBDA_RENDER_OUTPUT_DEVICE) {
            dj[k].out = j.out_rgb;
        } else {
            dj[k].out = r.out.as<float>() + host_off * 3;
            host_off += int64_t(dj[k].width) * dj[k].height;
        }
    }
    // the path kernel's work order: jobs by decreasing samples x (depth + 1)
    std::vector<int> by_cost(nj);
    for (size_t k = 0; k < nj; k++) by_cost[k] = int(k);
    std::stable_sort(by_cost.begin(), by_cost.end(), [&](int a, int b) {
        return int64_t(dj[a].samples) * (dj[a].depth + 1) > int64_t(dj[b].samples) * (dj[b].depth + 1);
    });
    std::vector<int2> work(nj);
    int64_t wbase = 0;
    for (size_t i = 0; i < nj; i++) {
        work[i] = make_int2(by_cost[i], int(wbase));
        wbase += int64_t(dj[by_cost[i]].width) * dj[by_cost[i]].height;
    }
    CK(r.jobs.reserve(nj * sizeof(Job)), "allocate job table");
    CK(r.active.reserve(active.size() * 4), "allocate job table");
    CK(r.work.reserve(nj * sizeof(int2)), "allocate job table");
    cudaStream_t stream = ctx->stream;
    CK(cudaMemcpyAsync(r.jobs.ptr, dj.data(), nj * sizeof(Job), cudaMemcpyHostToDevice, stream), "upload job table");
    CK(cudaMemcpyAsync(r.active.ptr, active.data(), active.size() * 4, cudaMemcpyHostToDevice, stream),
       "upload job table");
    CK(cudaMemcpyAsync(r.work.ptr, work.data(), nj * sizeof(int2), cudaMemcpyHostToDevice, stream), "upload job table");

    RenderParams rp{};
    rp.jobs = r.jobs.as<Job>();
    rp.num_jobs = int(nj);
    rp.num_pixels = P;
    rp.depth_max = d_max;
    rp.active = r.active.as<int>();
    rp.work = r.work.as<int2>();

    const PathState ps = ctx->pstate;
    const lambda_tuning &tu = ctx->tuning;
    const DeviceScene sc = ctx->scene_view(tu.bvh_width);
    const int dev = ctx->device, sms = ctx->sm_count;
    const int tb = tu.trace_block, sb = tu.shade_block, gs = tu.grid_scale;
    const size_t stack_smem = wide_stack_bytes(tb, sc.stack_tlas, sc.stack_blas);
    // intersect: a warp traces 32 rays to the end, or (lane_fetch) lanes take rays one
    // by one; over the tuned BVH layout (width, exact or compressed node records)
    using IntersectKernel = void (*)(int, RenderParams, DeviceScene, PathState);
    const int li = layout_index(tu);
    static const IntersectKernel isect_fetch[6] = {k_intersect_fetch<2>, k_intersect_fetch<4>, k_intersect_fetch<8>, k_intersect_fetch<2 | kCompressed>, k_intersect_fetch<4 | kCompressed>, k_intersect_fetch<8 | kCompressed>}, isect_warp[6] = {k_intersect<2>, k_intersect<4>, k_intersect<8>, k_intersect<2 | kCompressed>, k_intersect<4 | kCompressed>, k_intersect<8 | kCompressed>};
    const IntersectKernel k_isect = tu.lane_fetch ? isect_fetch[li] : isect_warp[li];
    const void *f_isect = (const void *)k_isect;
    // shadow rays: a warp's 32 queries to the end, or (lane_fetch) taken lane by lane
    static const IntersectKernel shad_fetch[6] = {k_shadow_fetch<2>, k_shadow_fetch<4>, k_shadow_fetch<8>, k_shadow_fetch<2 | kCompressed>, k_shadow_fetch<4 | kCompressed>, k_shadow_fetch<8 | kCompressed>}, shad_warp[6] = {k_shadow<2>, k_shadow<4>, k_shadow<8>, k_shadow<2 | kCompressed>, k_shadow<4 | kCompressed>, k_shadow<8 | kCompressed>};
    const IntersectKernel k_shad = tu.lane_fetch ? shad_fetch[li] : shad_warp[li];
    const void *f_shadow = (const void *)k_shad;
    // fused_bounce: one kernel per bounce (closest hit, shade, shadow ray)
    static const IntersectKernel bounce64[6] = {k_bounce<2, true>, k_bounce<4, true>, k_bounce<8, true>, k_bounce<2 | kCompressed, true>, k_bounce<4 | kCompressed, true>, k_bounce<8 | kCompressed, true>}, bounce32[6] = {k_bounce<2, false>, k_bounce<4, false>, k_bounce<8, false>, k_bounce<2 | kCompressed, false>, k_bounce<4 | kCompressed, false>, k_bounce<8 | kCompressed, false>};
    const bool fused = tu.fused_bounce != 0 && !surrogate;
    const IntersectKernel k_bnc = fp64 ? bounce64[li] : bounce32[li];
    int smem_optin = 0;
    CK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "device attribute");
    if (stack_smem > size_t(smem_optin))
        return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "the scene's traversal stacks exceed shared memory at this block size");
    CK(cudaFuncSetAttribute(f_isect, cudaFuncAttributeMaxDynamicSharedMemorySize, int(stack_smem)), "configure kernels");
    CK(cudaFuncSetAttribute(f_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize, int(stack_smem)), "configure kernels");
    if (fused)
        CK(cudaFuncSetAttribute((const void *)k_bnc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(stack_smem)),
           "configure kernels");
    auto grid = [&](const void *fn, int block, size_t smem) {
        return std::max(1, std::min((P + block - 1) / block, resident_ctas(fn, dev, block, smem) * sms * gs));
    };
    const int g_isect = grid(f_isect, tb, stack_smem);
    const int g_shadow = grid(f_shadow, tb, stack_smem);
    const int g_bounce = fused ? grid((const void *)k_bnc, tb, stack_smem) : 1;
    auto intersect = [&](int b) { k_isect<<<g_isect, tb, stack_smem, stream>>>(b, rp, sc, ps); };
    auto shadow = [&](int b, cudaStream_t s) { k_shad<<<g_shadow, tb, stack_smem, s>>>(b, rp, sc, ps); };
    const int g_lambert = grid((const void *)k_shade_lambert, sb, 0);
    const int g_spec = grid((const void *)k_shade_specular, sb, 0);
    const int g_film = grid(fp64 ? (const void *)k_shade_film_exact<true> : (const void *)k_shade_film_exact<false>, sb, 0);
    const int pix_blocks = (P + 255) / 256;

    // One wave's launches. With a profiler every launch is bracketed by events, in
    // order on the library stream. Inside the pass graph's loop the prologue sets the
    // loop condition, and a bounce's shading runs as parallel branches: Lambertian
    // shade, mirror/dielectric shade and thin-film shade touch disjoint paths (each
    // path is in one material queue), so only the queue order depends on their
    // interleaving, and the next intersect waits for all three. The Lambertian
    // shade's shadow rays run on a stream of their own beside the next intersect:
    // they add to the NEE radiance, which intersect no longer touches (it records a
    // path's final emission apart), and the next Lambertian shade, which refills the
    // NEE buffers, waits for them.
    cudaError_t fork_err = cudaSuccess;
    auto wave = [&](StageProfiler *pr, cudaGraphConditionalHandle loop, int waves) -> int {
        int n = 0;
        auto timed = [&](int stage, auto &&launch) {
            if (pr) pr->begin(stage);
            launch();
            if (pr) pr->end();
            n++;
        };
        timed(1, [&] { k_wave_prologue<<<1, 256, 0, stream>>>(d_max, ps, loop, waves, ctx->progress_dev); });
        timed(2, [&] { k_raygen<<<pix_blocks, 256, 0, stream>>>(rp, sc, ps); });
        // branch k: 1 specular, 2 thin film
        auto branch = [&](int k, int b, cudaStream_t s) {
            if (k == 1) {
                timed(5, [&] { k_shade_specular<<<g_spec, sb, 0, s>>>(b, rp, sc, ps); });
            } else if (surrogate) {
                n += ctx->launch_shade_surrogate(b, rp, sc, ps, pr, s);
            } else if (fp64) {
                timed(6, [&] { k_shade_film_exact<true><<<g_film, sb, 0, s>>>(b, rp, sc, ps); });
            } else {
                timed(6, [&] { k_shade_film_exact<false><<<g_film, sb, 0, s>>>(b, rp, sc, ps); });
            }
        };
        const bool lambert_on = (sc.families & 1u) != 0;
        int branches[2], nb = 0;
        for (int k = 1; k < 3; k++)
            if (sc.families & (1u << k)) branches[nb++] = k;
        auto keep = [&](cudaError_t e) {
            if (fork_err == cudaSuccess) fork_err = e;
        };
        if (fused) {
            for (int b = 0; b <= d_max; b++) timed(13, [&] { k_bnc<<<g_bounce, tb, stack_smem, stream>>>(b, rp, sc, ps); });
            return n;
        }
        cudaStream_t shadow_stream = ctx->side[2];
        bool shadow_pending = false;
        for (int b = 0; b <= d_max; b++) {
            timed(3, [&] { intersect(b); });
            if (pr) {
                if (lambert_on) {
                    timed(4, [&] { k_shade_lambert<<<g_lambert, sb, 0, stream>>>(b, rp, sc, ps); });
                    timed(7, [&] { shadow(b, stream); });
                }
                for (int i = 0; i < nb; i++) branch(branches[i], b, stream);
                continue;
            }
            if (nb > 0) keep(cudaEventRecord(ctx->ev_fork, stream));
            for (int i = 0; i < nb; i++) {
                keep(cudaStreamWaitEvent(ctx->side[i], ctx->ev_fork, 0));
                branch(branches[i], b, ctx->side[i]);
                keep(cudaEventRecord(ctx->ev_join[i], ctx->side[i]));
            }
            if (lambert_on) {
                if (shadow_pending) keep(cudaStreamWaitEvent(stream, ctx->ev_shadow, 0));
                timed(4, [&] { k_shade_lambert<<<g_lambert, sb, 0, stream>>>(b, rp, sc, ps); });
                keep(cudaEventRecord(ctx->ev_lambert, stream));
                keep(cudaStreamWaitEvent(shadow_stream, ctx->ev_lambert, 0));
                timed(7, [&] { shadow(b, shadow_stream); });
                keep(cudaEventRecord(ctx->ev_shadow, shadow_stream));
                shadow_pending = true;
            }
            for (int i = 0; i < nb; i++) keep(cudaStreamWaitEvent(stream, ctx->ev_join[i], 0));
        }
        // the last shadow rays finish inside the wave
        if (shadow_pending) keep(cudaStreamWaitEvent(stream, ctx->ev_shadow, 0));
        return n;
    };
    auto clear = [&]() -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(ps.stats, 0, 8 * 8, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(ps.error, 0, 16, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(ps.counts, 0, size_t(kQueues * (d_max + 2)) * 4, stream);
        return e;
    };
    // pixels of this pass whose samples are all done once `waves` waves have finished
    auto pixels_done = [&](int waves) {
        int64_t done = 0;
        for (size_t k = 0; k < nj; k++)
            done += int64_t(dj[k].width) * dj[k].height * std::min(waves, dj[k].samples) / dj[k].samples;
        return int32_t(std::min<int64_t>(completed_base + done, completed_total));
    };
    int launches = 0;
    bool path_pass = false;
    std::vector<Progress> progress(completed ? size_t(s_max) : 0);
    // the surrogate flag changes nothing on a scene without thin films
    const bool film_surrogate = surrogate && (sc.families & (1u << 2)) != 0;
    if (!film_surrogate && P <= tu.path_kernel_pixels) {
        // The pass as one persistent k_path launch (it seeds, traces and finishes
        // every pixel), captured with the counter clears into one graph.
        using PathKernel = void (*)(RenderParams, DeviceScene, PathState, int *, int *, int *);
        static const PathKernel path64[6] = {k_path<2, true>, k_path<4, true>, k_path<8, true>, k_path<2 | kCompressed, true>, k_path<4 | kCompressed, true>, k_path<8 | kCompressed, true>}, path32[6] = {k_path<2, false>, k_path<4, false>, k_path<8, false>, k_path<2 | kCompressed, false>, k_path<4 | kCompressed, false>, k_path<8 | kCompressed, false>};
        const PathKernel f_path = fp64 ? path64[li] : path32[li];
        CK(cudaFuncSetAttribute((const void *)f_path, cudaFuncAttributeMaxDynamicSharedMemorySize, int(stack_smem)),
           "configure kernels");
        const int g_path = grid((const void *)f_path, tb, stack_smem);
        // counts[0]: the work counter (virtual pixels handed out); counts[1]: pixels done
        auto launch = [&] { f_path<<<g_path, tb, stack_smem, stream>>>(rp, sc, ps, ps.counts, ps.counts + 1, ctx->progress_dev); };
        *ctx->progress_host = 0;
        if (prof) {
            CK(clear(), "clear counters");
            CK(cudaEventRecord(ctx->ev_start, stream), "event");
            prof->begin(12);
            launch();
            prof->end();
            CK(cudaGetLastError(), "launch path kernel");
            CK(cudaEventRecord(ctx->ev_stop, stream), "event");
        } else {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            cudaError_t e = clear();
            launch();
            cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (e != cudaSuccess || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return ctx->cuda_fail(e != cudaSuccess ? e : ce, "capture path-kernel pass");
            }
            if (ctx->graph_exec) {
                cudaGraphExecDestroy(ctx->graph_exec);
                ctx->graph_exec = nullptr;
            }
            e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return ctx->cuda_fail(e, "instantiate path-kernel pass");
            CK(cudaEventRecord(ctx->ev_start, stream), "event");
            CK(cudaGraphLaunch(ctx->graph_exec, stream), "launch path-kernel pass");
            CK(cudaEventRecord(ctx->ev_stop, stream), "event");
        }
        launches = 1;
        path_pass = true;
    } else if (prof) {
        CK(clear(), "clear counters");
        CK(cudaEventRecord(ctx->ev_start, stream), "event");
        prof->begin(0);
        k_init<<<pix_blocks, 256, 0, stream>>>(rp, ps);
        prof->end();
        launches++;
        for (int w = 0; w < s_max; w++) {
            launches += wave(prof, 0, 0);
            CK(cudaGetLastError(), "launch wave");
            if (completed) {
                progress[w] = Progress{completed, pixels_done(w + 1)};
                CK(cudaLaunchHostFunc(stream, progress_cb, &progress[w]), "progress callback");
            }
            CK(prof->collect(), "stage timing");
        }
        prof->begin(1);
        k_wave_prologue<<<1, 256, 0, stream>>>(d_max, ps, 0, 0, nullptr);  // folds the last wave's counts in
        prof->end();
        prof->begin(8);
        k_finish<<<pix_blocks, 256, 0, stream>>>(rp, sc, ps);
        prof->end();
        launches += 2;
        CK(cudaGetLastError(), "launch finish");
        CK(cudaEventRecord(ctx->ev_stop, stream), "event");
    } else {
        // The whole pass as one graph launch: clear + k_init, a while node whose
        // body is one sample wave (run s_max times), then the last prologue and
        // k_finish.
        cudaGraph_t g = nullptr, pre = nullptr, post = nullptr;
        cudaGraphConditionalHandle loop = 0;
        auto fail = [&](cudaError_t e, const char *what) {
            if (pre) cudaGraphDestroy(pre);
            if (post) cudaGraphDestroy(post);
            if (g) cudaGraphDestroy(g);
            return ctx->cuda_fail(e, what);
        };
        cudaError_t e = cudaGraphCreate(&g, 0);
        if (e != cudaSuccess) return fail(e, "create pass graph");
        e = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) return fail(e, "create wave loop");
        e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail(e, "begin capture");
        e = clear();
        k_init<<<pix_blocks, 256, 0, stream>>>(rp, ps);
        cudaError_t ce = cudaStreamEndCapture(stream, &pre);
        if (e != cudaSuccess || ce != cudaSuccess) return fail(e != cudaSuccess ? e : ce, "capture pass prefix");
        cudaGraphNode_t n_pre = nullptr, n_loop = nullptr, n_post = nullptr;
        e = cudaGraphAddChildGraphNode(&n_pre, g, nullptr, 0, pre);
        if (e != cudaSuccess) return fail(e, "build pass graph");
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&n_loop, g, &n_pre, 1, &cp);
        if (e != cudaSuccess) return fail(e, "build wave loop");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail(e, "begin capture of the wave");
        const int wave_launches = wave(nullptr, loop, s_max);
        ce = cudaStreamEndCapture(stream, &body);
        if (fork_err != cudaSuccess) return fail(fork_err, "capture the wave's branches");
        if (ce != cudaSuccess) return fail(ce, "capture wave");
        e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail(e, "begin capture");
        k_wave_prologue<<<1, 256, 0, stream>>>(d_max, ps, 0, 0, nullptr);  // folds the last wave's counts in
        k_finish<<<pix_blocks, 256, 0, stream>>>(rp, sc, ps);
        ce = cudaStreamEndCapture(stream, &post);
        if (ce != cudaSuccess) return fail(ce, "capture pass suffix");
        e = cudaGraphAddChildGraphNode(&n_post, g, &n_loop, 1, post);
        if (e != cudaSuccess) return fail(e, "build pass graph");
        if (ctx->graph_exec) {
            cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = nullptr;
        }
        e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
        cudaGraphDestroy(pre);
        cudaGraphDestroy(post);
        cudaGraphDestroy(g);
        pre = post = g = nullptr;
        if (e != cudaSuccess) return ctx->cuda_fail(e, "instantiate pass graph");
        *ctx->progress_host = 0;
        CK(cudaEventRecord(ctx->ev_start, stream), "event");
        CK(cudaGraphLaunch(ctx->graph_exec, stream), "launch pass graph");
        CK(cudaEventRecord(ctx->ev_stop, stream), "event");
        launches = 1 + s_max * wave_launches + 2;
    }
    if (completed && !prof) {
        // progress from the mapped host counter: the waves the graph has started, or
        // the pixels a path-kernel pass has finished (the largest value seen). This
        // runs before the copies below: a copy into pageable host memory returns only
        // once the stream has drained, which would leave nothing to poll.
        int32_t seen = 0;
        for (;;) {
            const cudaError_t q = cudaStreamQuery(stream);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return ctx->cuda_fail(q, "render");
            const int v = *reinterpret_cast<volatile int *>(ctx->progress_host);
            const int32_t now = path_pass ? int32_t(std::min<int64_t>(int64_t(completed_base) + std::min(v, P), completed_total))
                                          : pixels_done(std::max(0, v - 1));
            seen = std::max(seen, now);
            *completed = seen;
            std::this_thread::sleep_for(std::chrono::milliseconds(2));
        }
    }
    for (size_t k = 0; k < nj; k++) {
        const lambda_job &j = jobs[order[first + k]];
        if (!(j.desc.flags & LAMBDA_RENDER_OUTPUT_DEVICE))
            CK(cudaMemcpyAsync(j.out_rgb, dj[k].out, size_t(dj[k].width) * dj[k].height * 12, cudaMemcpyDeviceToHost,
                               stream),
               "copy image to host");
    }
    unsigned long long stats[8] = {0};
    int err[4] = {0};
    CK(cudaMemcpyAsync(stats, ps.stats, sizeof(stats), cudaMemcpyDeviceToHost, stream), "read statistics");
    CK(cudaMemcpyAsync(err, ps.error, sizeof(err), cudaMemcpyDeviceToHost, stream), "read flags");
    CK(cudaStreamSynchronize(stream), "render");
    if (prof) CK(prof->collect(), "stage timing");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    tot.ms += ms;
    for (size_t k = 0; k < nj; k++) tot.paths += int64_t(dj[k].width) * dj[k].height * dj[k].samples;
    tot.pixels += P;
    for (int i = 0; i < 8; i++) tot.stats[i] += stats[i];
    tot.launches += launches;
    tot.waves += s_max;
    tot.err |= err[0];
    return LAMBDA_OK;
}

// Renders n jobs in passes of whole jobs (at most tuning.max_pixels pixels a pass,
// a larger single job alone), ordered by decreasing sample count.
lambda_status render_jobs(lambda_ctx *ctx, const lambda_job *jobs, int n, volatile int32_t *completed) {
    if (!ctx->has_scene) return ctx->fail(LAMBDA_ERR_NO_SCENE, "no scene uploaded");
    constexpr uint32_t kModeBits = LAMBDA_RENDER_THINFILM_SURROGATE | LAMBDA_RENDER_THINFILM_FP64 | LAMBDA_RENDER_PROFILE_STAGES;
    const uint32_t mode = jobs[0].desc.flags & kModeBits;
    if ((mode & LAMBDA_RENDER_THINFILM_SURROGATE) && (mode & LAMBDA_RENDER_THINFILM_FP64))
        return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "the surrogate and the FP64 thin film exclude each other");
    int64_t total_pixels = 0;
    for (int i = 0; i < n; i++) {
        if (!jobs[i].out_rgb) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "job without an output image");
        lambda_status s = check_settings(ctx, jobs[i].desc.settings);
        if (s != LAMBDA_OK) return s;
        if ((jobs[i].desc.flags & kModeBits) != mode)
            return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "the jobs of a batch must share the thin-film mode and profiling flag");
        total_pixels += int64_t(jobs[i].desc.settings.width) * jobs[i].desc.settings.height;
    }
    if (total_pixels > INT32_MAX) return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "more than 2^31 pixels in one batch");
    const bool surrogate = (mode & LAMBDA_RENDER_THINFILM_SURROGATE) != 0;
    const bool fp64 = (mode & LAMBDA_RENDER_THINFILM_FP64) != 0;
    const bool profile = (mode & LAMBDA_RENDER_PROFILE_STAGES) != 0;
    if (surrogate) {
        lambda_status s = ctx->surrogate_ready();
        if (s != LAMBDA_OK) return s;
    }
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    for (int i = 0; i < n; i++)
        if ((jobs[i].desc.flags & LAMBDA_RENDER_OUTPUT_DEVICE) && !is_device_pointer(jobs[i].out_rgb))
            return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "LAMBDA_RENDER_OUTPUT_DEVICE given a host pointer");
    if (!ctx->progress_host) {
        CK(cudaHostAlloc(reinterpret_cast<void **>(&ctx->progress_host), sizeof(int), cudaHostAllocMapped),
           "allocate progress counter");
        CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&ctx->progress_dev), ctx->progress_host, 0),
           "map progress counter");
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return jobs[a].desc.settings.samples > jobs[b].desc.settings.samples;
    });
    const int64_t cap = ctx->tuning.max_pixels > 0 ? ctx->tuning.max_pixels : (int64_t(1) << 30);
    StageProfiler prof(ctx->stream);
    RenderTotals tot;
    size_t first = 0;
    while (first < size_t(n)) {
        size_t last = first + 1;
        int64_t px = int64_t(jobs[order[first]].desc.settings.width) * jobs[order[first]].desc.settings.height;
        while (last < size_t(n)) {
            const int64_t add = int64_t(jobs[order[last]].desc.settings.width) * jobs[order[last]].desc.settings.height;
            if (px + add > cap) break;
            px += add;
            last++;
        }
        lambda_status s = render_pass(ctx, jobs, order, first, last, surrogate, fp64, profile ? &prof : nullptr, completed,
                                      int32_t(tot.pixels), int32_t(total_pixels), tot);
        if (s != LAMBDA_OK) return s;
        first = last;
    }
    if (completed) *completed = int32_t(total_pixels);
    ctx->stats = lambda_render_stats{};
    ctx->stats.render_ms = tot.ms;
    ctx->stats.paths = tot.paths;
    ctx->stats.segments = int64_t(tot.stats[0]);
    ctx->stats.shadow_rays = int64_t(tot.stats[1]);
    ctx->stats.thinfilm_hits = int64_t(tot.stats[2]);
    ctx->stats.thinfilm_fallback = int64_t(tot.stats[3]);
    ctx->stats.kernel_launches = tot.launches;
    ctx->stats.waves = tot.waves;
    ctx->stats.surrogate_ctas_per_sm = surrogate ? ctx->mlp_ctas_per_sm : 0;
    if (profile) {
        for (int i = 0; i < LAMBDA_NUM_STAGES; i++) {
            ctx->stage_times[i].ms = prof.totals[i];
            ctx->stage_times[i].launches = prof.counts[i];
        }
        ctx->stage_times[0].items = tot.pixels;
        ctx->stage_times[1].items = tot.waves;
        ctx->stage_times[2].items = tot.paths;
        ctx->stage_times[3].items = prof.counts[3] ? ctx->stats.segments : 0;
        ctx->stage_times[12].items = prof.counts[12] ? ctx->stats.segments : 0;
        ctx->stage_times[13].items = prof.counts[13] ? ctx->stats.segments : 0;
        ctx->stage_times[4].items = int64_t(tot.stats[4]);
        ctx->stage_times[5].items = int64_t(tot.stats[5]);
        ctx->stage_times[6].items = surrogate ? 0 : ctx->stats.thinfilm_hits;
        ctx->stage_times[7].items = ctx->stats.shadow_rays;
        ctx->stage_times[8].items = tot.pixels;
        for (int i = 9; i <= 11; i++) ctx->stage_times[i].items = surrogate ? ctx->stats.thinfilm_hits : 0;
    }
    if (tot.err & 1) return ctx->fail(LAMBDA_ERR_QUEUE_OVERFLOW, "BVH traversal stack overflow");
    if (tot.err & 2) return ctx->fail(LAMBDA_ERR_TIMEOUT, "tensor-core MMA completion wait timed out");
    return LAMBDA_OK;
}

bool tuning_ok(const lambda_tuning &t) {
    auto block_ok = [](int b) { return b == 64 || b == 128 || b == 256; };
    return block_ok(t.trace_block) && block_ok(t.shade_block) && (t.grid_scale == 1 || t.grid_scale == 2) &&
           t.max_pixels >= 0 && (t.bvh_width == 2 || t.bvh_width == 4 || t.bvh_width == 8) && t.path_kernel_pixels >= 0 &&
           (t.lane_fetch == 0 || t.lane_fetch == 1) && (t.compressed_nodes == 0 || t.compressed_nodes == 1) &&
           (t.fused_bounce == 0 || t.fused_bounce == 1);
}

}  // namespace

extern "C" lambda_status lambda_render(lambda_ctx *ctx, const lambda_render_desc *desc, float *out_rgb,
                                       volatile int32_t *completed) {
    if (!ctx || !desc || !out_rgb) return LAMBDA_ERR_INVALID_ARGUMENT;
    const lambda_job job{*desc, out_rgb};
    return render_jobs(ctx, &job, 1, completed);
}

extern "C" lambda_status lambda_render_batch(lambda_ctx *ctx, const lambda_job *jobs, int32_t n,
                                             volatile int32_t *completed) {
    if (!ctx || !jobs || n < 1) return LAMBDA_ERR_INVALID_ARGUMENT;
    return render_jobs(ctx, jobs, n, completed);
}

extern "C" lambda_status lambda_set_tuning(lambda_ctx *ctx, const lambda_tuning *tuning) {
    if (!ctx || !tuning) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (!tuning_ok(*tuning)) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "invalid tuning values");
    ctx->tuning = *tuning;
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_get_tuning(const lambda_ctx *ctx, lambda_tuning *tuning) {
    if (!ctx || !tuning) return LAMBDA_ERR_INVALID_ARGUMENT;
    *tuning = ctx->tuning;
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_set_limits(lambda_ctx *ctx, const lambda_limits *limits) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (!limits) {
        ctx->limits = lambda_limits{LAMBDA_DEFAULT_MMA_POLLS, 0};
        return LAMBDA_OK;
    }
    if (limits->stack_entries < 0) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "stack_entries must be >= 0");
    ctx->limits = *limits;
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_get_limits(const lambda_ctx *ctx, lambda_limits *limits) {
    if (!ctx || !limits) return LAMBDA_ERR_INVALID_ARGUMENT;
    *limits = ctx->limits;
    return LAMBDA_OK;
}

namespace {

// Times renders of the probe views (their images stay in device memory) under every
// combination of BVH width, traversal block, shading block and grid scale of the
// wavefront, and of BVH width and block size of the path kernel, each as the best of
// three renders after one warm-up, and keeps the fastest. The path-state
// capacity is set from free device memory: half of it, at the bytes of path state
// and queues a pixel needs.
lambda_status autotune_views(lambda_ctx *ctx, const lambda_render_desc *probes, int n, lambda_tuning *out) {
    if (!ctx || !probes || n < 1) return LAMBDA_ERR_INVALID_ARGUMENT;
    size_t pixels = 0;
    for (int i = 0; i < n; i++) {
        lambda_status s = check_settings(ctx, probes[i].settings);
        if (s != LAMBDA_OK) return s;
        pixels += size_t(probes[i].settings.width) * probes[i].settings.height;
    }
    if (!ctx->has_scene) return ctx->fail(LAMBDA_ERR_NO_SCENE, "no scene uploaded");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    DeviceBuffer img;
    CK(img.reserve(pixels * 12), "allocate probe images");
    std::vector<lambda_job> jobs(n);
    size_t off = 0;
    for (int i = 0; i < n; i++) {
        jobs[i] = lambda_job{probes[i], img.as<float>() + off * 3};
        jobs[i].desc.flags = (probes[0].flags & (LAMBDA_RENDER_THINFILM_SURROGATE | LAMBDA_RENDER_THINFILM_FP64)) |
                             LAMBDA_RENDER_OUTPUT_DEVICE;
        off += size_t(probes[i].settings.width) * probes[i].settings.height;
    }
    const lambda_tuning keep = ctx->tuning;
    lambda_tuning best = keep;
    double best_ms = 1e300;
    // one warm-up render, then the best of three timed ones
    auto trial = [&](const lambda_tuning &t, double &ms) -> lambda_status {
        ctx->tuning = t;
        lambda_status r = render_jobs(ctx, jobs.data(), n, nullptr);
        ms = 1e300;
        for (int rep = 0; rep < 3 && r == LAMBDA_OK; rep++) {
            r = render_jobs(ctx, jobs.data(), n, nullptr);
            ms = std::min(ms, ctx->stats.render_ms);
        }
        return r;
    };
    // every BVH width with every block shape: the best width can depend on the blocks
    for (int bw : {2, 4, 8})
        for (int tb : {64, 128, 256})
            for (int sb : {64, 128, 256})
                for (int gs : {1, 2}) {
                    double ms = 0;
                    const lambda_status r = trial(lambda_tuning{tb, sb, gs, keep.max_pixels, bw, 0, 0, 0, 0}, ms);
                    if (r == LAMBDA_ERR_UNSUPPORTED) continue;  // stacks too deep for shared memory at this block size
                    if (r != LAMBDA_OK) {
                        ctx->tuning = keep;
                        return r;
                    }
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = ctx->tuning;
                    }
                }
    // the intersect kernel with rays taken lane by lane, at every width and traversal
    // block, with the best wavefront's other shapes
    {
        const lambda_tuning grid_best = best;
        for (int bw : {2, 4, 8})
            for (int tb : {64, 128, 256}) {
                lambda_tuning t = grid_best;
                t.trace_block = tb;
                t.bvh_width = bw;
                t.lane_fetch = 1;
                double ms = 0;
                const lambda_status r = trial(t, ms);
                if (r == LAMBDA_ERR_UNSUPPORTED) continue;
                if (r != LAMBDA_OK) {
                    ctx->tuning = keep;
                    return r;
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best = t;
                }
            }
    }
    // the compressed node records at every width, with the best shapes so far (warp
    // or lane-by-lane traversal)
    {
        const lambda_tuning exact_best = best;
        for (int bw : {2, 4, 8}) {
            lambda_tuning t = exact_best;
            t.bvh_width = bw;
            t.compressed_nodes = 1;
            double ms = 0;
            const lambda_status r = trial(t, ms);
            if (r == LAMBDA_ERR_UNSUPPORTED) continue;
            if (r != LAMBDA_OK) {
                ctx->tuning = keep;
                return r;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        }
    }
    // one kernel per bounce at every width and traversal block, with the best shapes so
    // far (not for surrogate renders of thin films, which keep the batched MLP stage)
    if (!(probes[0].flags & LAMBDA_RENDER_THINFILM_SURROGATE) || !(ctx->dscene.families & (1u << 2))) {
        const lambda_tuning sep_best = best;
        for (int bw : {2, 4, 8})
            for (int tb : {64, 128, 256}) {
                lambda_tuning t = sep_best;
                t.trace_block = tb;
                t.bvh_width = bw;
                t.lane_fetch = 0;
                t.fused_bounce = 1;
                double ms = 0;
                const lambda_status r = trial(t, ms);
                if (r == LAMBDA_ERR_UNSUPPORTED) continue;
                if (r != LAMBDA_OK) {
                    ctx->tuning = keep;
                    return r;
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best = t;
                }
            }
    }
    // the path kernel at every BVH width, node layout and block size (not for surrogate renders of
    // thin films, which it does not run). If one wins, passes up to the probe's pixels
    // use it; if the wavefront wins, only passes below the probe's size and the default
    // threshold do.
    best.path_kernel_pixels = keep.path_kernel_pixels;
    if (!(probes[0].flags & LAMBDA_RENDER_THINFILM_SURROGATE) || !(ctx->dscene.families & (1u << 2))) {
        const int32_t probe_pixels = int32_t(std::min<size_t>(pixels, INT32_MAX));
        best.path_kernel_pixels = std::min<int32_t>(LAMBDA_PATH_KERNEL_PIXELS, probe_pixels - 1);
        const lambda_tuning wave_best = best;
        for (int bw : {2, 4, 8})
            for (int cn : {0, 1})
            for (int tb : {64, 128, 256}) {
                lambda_tuning t = wave_best;
                t.trace_block = tb;
                t.bvh_width = bw;
                t.compressed_nodes = cn;
                t.path_kernel_pixels = INT32_MAX;
                double ms = 0;
                const lambda_status r = trial(t, ms);
                if (r == LAMBDA_ERR_UNSUPPORTED) continue;
                if (r != LAMBDA_OK) {
                    ctx->tuning = keep;
                    return r;
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best = t;
                    best.path_kernel_pixels = std::max<int32_t>(LAMBDA_PATH_KERNEL_PIXELS, probe_pixels);
                }
            }
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        // path state, queues, staged image, the surrogate's MLP rows, outputs and domain flags
        constexpr size_t kBytesPerPixel = 8 + 16 * 12 + 8 + 8 + 4 * 6 + 12 + 4 * 32 + 4 * 16 + 1;
        best.max_pixels = int32_t(std::min<size_t>((free_b / 2) / kBytesPerPixel, size_t(1) << 30));
    }
    ctx->tuning = best;
    if (out) *out = best;
    return LAMBDA_OK;
}

}  // namespace

extern "C" lambda_status lambda_autotune(lambda_ctx *ctx, const lambda_render_desc *probe, lambda_tuning *out) {
    return autotune_views(ctx, probe, 1, out);
}

extern "C" lambda_status lambda_autotune_batch(lambda_ctx *ctx, const lambda_render_desc *probes, int32_t n,
                                               lambda_tuning *out) {
    return autotune_views(ctx, probes, n, out);
}

extern "C" lambda_status lambda_get_stage_times(const lambda_ctx *ctx, lambda_stage_time *out) {
    if (!ctx || !out) return LAMBDA_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < LAMBDA_NUM_STAGES; i++) out[i] = ctx->stage_times[i];
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_get_render_stats(const lambda_ctx *ctx, lambda_render_stats *stats) {
    if (!ctx || !stats) return LAMBDA_ERR_INVALID_ARGUMENT;
    *stats = ctx->stats;
    return LAMBDA_OK;
}

// ---------------------------------------------------------------------------
// Ray queries
// ---------------------------------------------------------------------------

namespace {

template <int K>
__global__ void k_trace_closest(DeviceScene sc, const float *rays, int n, int *inst, int *obj, float *t, int *error) {
    extern __shared__ int stack_smem[];
    WideStack st_a, st_b;
    wide_stacks(stack_smem, sc, st_a, st_b);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float *r = rays + 6 * size_t(k);
    Hit h;
    bool overflow = false;
    closest_hit_w<K>(sc, mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), h, overflow, st_a, st_b);
    inst[k] = h.instance;
    obj[k] = h.object;
    t[k] = h.t;
    if (overflow) atomicOr(error, 1);
}

template <int K>
__global__ void k_trace_shadow(DeviceScene sc, const float *rays, const int *li, const int *lo, int n, int *occ,
                               int *error) {
    extern __shared__ int stack_smem[];
    WideStack st_a, st_b;
    wide_stacks(stack_smem, sc, st_a, st_b);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float *r = rays + 6 * size_t(k);
    Hit h;
    bool overflow = false;
    occ[k] = occluded_w<K>(sc, mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), li[k], lo[k], h, overflow, st_a, st_b) ? 1 : 0;
    if (overflow) atomicOr(error, 1);
}

// Launches a ray-query kernel (fns: one per BVH layout, in layout_index order) of the
// tuned layout with its stacks in shared memory.
template <class... A>
cudaError_t launch_query(lambda_ctx *ctx, void (*const *fns)(DeviceScene, A...), int n, A... args) {
    const DeviceScene sc = ctx->scene_view(ctx->tuning.bvh_width);
    const size_t smem = wide_stack_bytes(128, sc.stack_tlas, sc.stack_blas);
    void (*fn)(DeviceScene, A...) = fns[layout_index(ctx->tuning)];
    cudaError_t e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    const int blocks = (n + 127) / 128;
    fn<<<blocks, 128, smem, ctx->stream>>>(sc, args...);
    return cudaGetLastError();
}

}  // namespace

lambda_status finish_staging(lambda_ctx *ctx, CopyBack &back) {
    for (auto &b : back)
        CK(cudaMemcpyAsync(b.first, b.second.first, b.second.second, cudaMemcpyDeviceToHost, ctx->stream), "copy results");
    CK(cudaStreamSynchronize(ctx->stream), "query");
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_trace_closest(lambda_ctx *ctx, const float *rays, int32_t n, int32_t *out_instance,
                                              int32_t *out_object, float *out_t) {
    if (!ctx || n < 0 || (n > 0 && (!rays || !out_instance || !out_object || !out_t))) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return ctx->fail(LAMBDA_ERR_NO_SCENE, "no scene uploaded");
    if (n == 0) return LAMBDA_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    Staging sg{ctx, {}};
    CopyBack back;
    const float *dr;
    int *di, *dobj;
    float *dt;
    CK(sg.in(rays, size_t(n) * 6, &dr), "stage rays");
    CK(sg.out(out_instance, size_t(n), &di, back), "stage results");
    CK(sg.out(out_object, size_t(n), &dobj, back), "stage results");
    CK(sg.out(out_t, size_t(n), &dt, back), "stage results");
    CK(ctx->rbuf.error.reserve(16), "allocate flags");
    int *err = ctx->rbuf.error.as<int>();
    CK(cudaMemsetAsync(err, 0, 16, ctx->stream), "clear flags");
    static void (*const closest[6])(DeviceScene, const float *, int, int *, int *, float *, int *) = {k_trace_closest<2>, k_trace_closest<4>, k_trace_closest<8>, k_trace_closest<2 | kCompressed>, k_trace_closest<4 | kCompressed>, k_trace_closest<8 | kCompressed>};
    CK(launch_query(ctx, closest, n, static_cast<const float *>(dr), n, di, dobj, dt, err),
       "launch closest-hit queries");
    CK(cudaGetLastError(), "launch trace");
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, ctx->stream), "read flags");
    lambda_status s = finish_staging(ctx, back);
    if (s != LAMBDA_OK) return s;
    if (herr & 1) return ctx->fail(LAMBDA_ERR_QUEUE_OVERFLOW, "BVH traversal stack overflow");
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_trace_shadow(lambda_ctx *ctx, const float *rays, const int32_t *light_instance,
                                             const int32_t *light_object, int32_t n, int32_t *out_occluded) {
    if (!ctx || n < 0 || (n > 0 && (!rays || !light_instance || !light_object || !out_occluded)))
        return LAMBDA_ERR_INVALID_ARGUMENT;
    if (!ctx->has_scene) return ctx->fail(LAMBDA_ERR_NO_SCENE, "no scene uploaded");
    if (n == 0) return LAMBDA_OK;
    // light ids are checked on the host: the kernel indexes instances/objects with them
    std::vector<int32_t> hli(n), hlo(n);
    if (is_device_pointer(light_instance)) CK(cudaMemcpy(hli.data(), light_instance, 4 * size_t(n), cudaMemcpyDeviceToHost), "read lights");
    else std::memcpy(hli.data(), light_instance, 4 * size_t(n));
    if (is_device_pointer(light_object)) CK(cudaMemcpy(hlo.data(), light_object, 4 * size_t(n), cudaMemcpyDeviceToHost), "read lights");
    else std::memcpy(hlo.data(), light_object, 4 * size_t(n));
    for (int k = 0; k < n; k++) {
        const bool bg = hli[k] == -1 && hlo[k] == -1;
        const bool ok = bg || (hli[k] >= 0 && hli[k] < ctx->dscene.num_instances && hlo[k] >= 0 && hlo[k] < ctx->dscene.num_objects);
        if (!ok) return ctx->fail(LAMBDA_ERR_INVALID_ARGUMENT, "light id out of range");
    }
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    Staging sg{ctx, {}};
    CopyBack back;
    const float *dr;
    const int *dli, *dlo;
    int *docc;
    CK(sg.in(rays, size_t(n) * 6, &dr), "stage rays");
    CK(sg.in(hli.data(), size_t(n), &dli), "stage lights");
    CK(sg.in(hlo.data(), size_t(n), &dlo), "stage lights");
    CK(sg.out(out_occluded, size_t(n), &docc, back), "stage results");
    CK(ctx->rbuf.error.reserve(16), "allocate flags");
    int *err = ctx->rbuf.error.as<int>();
    CK(cudaMemsetAsync(err, 0, 16, ctx->stream), "clear flags");
    static void (*const shadow[6])(DeviceScene, const float *, const int *, const int *, int, int *, int *) =
        {k_trace_shadow<2>, k_trace_shadow<4>, k_trace_shadow<8>, k_trace_shadow<2 | kCompressed>, k_trace_shadow<4 | kCompressed>, k_trace_shadow<8 | kCompressed>};
    CK(launch_query(ctx, shadow, n, static_cast<const float *>(dr), static_cast<const int *>(dli),
                    static_cast<const int *>(dlo), n, docc, err),
       "launch shadow queries");
    CK(cudaGetLastError(), "launch trace");
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, ctx->stream), "read flags");
    lambda_status s = finish_staging(ctx, back);
    if (s != LAMBDA_OK) return s;
    if (herr & 1) return ctx->fail(LAMBDA_ERR_QUEUE_OVERFLOW, "BVH traversal stack overflow");
    return LAMBDA_OK;
}

// ---------------------------------------------------------------------------
// Thin-film queries: single film between air (n = 1) and a substrate.
// ---------------------------------------------------------------------------

namespace {

template <typename R>
__global__ void k_film_query(const lambda_film_query *q, int n, R *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const lambda_film_query x = q[k];
    cx<R> idx[3] = {cx<R>{R(1), R(0)}, cx<R>{R(x.n_film), R(0)}, cx<R>{R(x.n_sub), R(0)}};
    const R d = R(x.thickness_nm);
    const FilmResult<R> r = film_stack<R, 1>(1, idx, &d, R(x.cos_theta), R(x.lambda_nm));
    out[4 * size_t(k)] = r.rs;
    out[4 * size_t(k) + 1] = r.rp;
    out[4 * size_t(k) + 2] = r.ts;
    out[4 * size_t(k) + 3] = r.tp;
}

template <typename R>
lambda_status film_query(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, R *out) {
    if (!ctx || n < 0 || (n > 0 && (!q || !out))) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (n == 0) return LAMBDA_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    Staging sg{ctx, {}};
    CopyBack back;
    const lambda_film_query *dq;
    R *dout;
    CK(sg.in(q, size_t(n), &dq), "stage queries");
    CK(sg.out(out, size_t(n) * 4, &dout, back), "stage results");
    k_film_query<R><<<(n + 127) / 128, 128, 0, ctx->stream>>>(dq, n, dout);
    CK(cudaGetLastError(), "launch thin-film query");
    return finish_staging(ctx, back);
}

}  // namespace

extern "C" lambda_status lambda_thinfilm_exact(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, float *out) {
    return film_query<float>(ctx, q, n, out);
}

extern "C" lambda_status lambda_thinfilm_fp64(lambda_ctx *ctx, const lambda_film_query *q, int32_t n, double *out) {
    return film_query<double>(ctx, q, n, out);
}
