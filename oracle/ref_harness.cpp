// Test harness around the reference renderer's own CPU code (checker only).
//
// This file is test infrastructure. It is compiled by oracle/Makefile against the
// reference headers where they lie (REF_SRC) into oracle/_ref/libref_lambda.so,
// which is never linked into the product. It exposes, over a C ABI for ctypes:
//   - Parser::parseLRD (src/core/parser.h:29) and the containers it fills,
//   - Renderer::renderImage (src/render/renderer.h:42) with OpenMP threads,
//   - Scene::hit (src/scene/scene.h:51) on caller-given rays,
//   - Material::thinFilmReflectance (src/scene/material.h:263) and the texture
//     evaluators (src/scene/texture.h), for golden vectors,
//   - Writer::write (src/core/writer.h:11).
// Private members are opened with a preprocessor switch so that the reference's
// own member functions can be called on constructed inputs.

#include <algorithm>
#include <atomic>
#include <cassert>
#include <cctype>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include <omp.h>

#define private public
#include "core/constants.h"
#include "core/parser.h"
#include "core/platform.h"
#include "core/utils.h"
#include "core/writer.h"
#include "math/random.h"
#include "math/spectrum.h"
#include "render/renderer.h"
#include "scene/background.h"
#include "scene/bvh.h"
#include "scene/material.h"
#include "scene/object.h"
#include "scene/scene.h"
#include "scene/texture.h"
#undef private

namespace {

struct RefScene {
    Renderer renderer;
    std::vector<DenseSpectrum<Float>> spectra;
    std::vector<DenseSpectrum<Complex>> complexSpectra;
    Background background;
    std::vector<Object> objects;
    std::vector<Instance> instances;
    std::vector<BVHNode> nodes;
    std::vector<int> lightInstances;
    std::vector<int> lightObjects;
    std::vector<Float> lightPowers;
    Float totalLightPower = 0;
    std::vector<Material> materials;
    std::vector<int> materialProperties;
    std::vector<ScalarTexture> scalarTextures;
    std::vector<SpectrumTexture> spectrumTextures;
};

std::vector<int> g_permutation(h_PERMUTATION, h_PERMUTATION + PERMUTATION_SIZE);
std::vector<double> g_cie(&h_CIE_XYZ_1931[0][0], &h_CIE_XYZ_1931[CIE_LAMBDA_BINS - 1][2] + 1);

void install_tables() {
    PERMUTATION = g_permutation.data();
    CIE_XYZ_1931 = g_cie.data();
}

void wire(RefScene &s) {
    install_tables();
    s.renderer.setScene(s.spectra.data(), s.complexSpectra.data(), s.background, s.objects.data(), s.instances.data(),
                        s.nodes.data(), s.lightInstances.data(), s.lightObjects.data(), int(s.lightInstances.size()),
                        s.lightPowers.data(), s.totalLightPower, s.materials.data(), s.materialProperties.data(),
                        s.scalarTextures.data(), s.spectrumTextures.data());
}

void put_err(char *err, size_t len, const std::string &msg) {
    if (!err || len == 0) return;
    size_t n = std::min(len - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = 0;
}

}  // namespace

extern "C" {

// Layout checks: the product's flat structs mirror these byte for byte.
int ref_sizeof(int which) {
    switch (which) {
        case 0: return int(sizeof(Object));
        case 1: return int(sizeof(Instance));
        case 2: return int(sizeof(BVHNode));
        case 3: return int(sizeof(Material));
        case 4: return int(sizeof(ScalarTexture));
        case 5: return int(sizeof(SpectrumTexture));
        case 6: return int(sizeof(DenseSpectrum<Float>));
        case 7: return int(sizeof(DenseSpectrum<Complex>));
        case 8: return int(sizeof(Background));
        default: return -1;
    }
}

int ref_parse(const char *path, void **out, char *err, size_t err_len) {
    auto *s = new RefScene();
    try {
        Parser::parseLRD(path, s->renderer, s->spectra, s->complexSpectra, s->background, s->objects, s->instances,
                         s->nodes, s->lightInstances, s->lightObjects, s->lightPowers, s->totalLightPower,
                         s->materials, s->materialProperties, s->scalarTextures, s->spectrumTextures);
    } catch (const std::exception &e) {
        put_err(err, err_len, e.what());
        delete s;
        return 1;
    }
    wire(*s);
    *out = s;
    return 0;
}

void ref_free(void *p) { delete static_cast<RefScene *>(p); }

// counts: spectra, complexSpectra, objects, instances, nodes, lights, materials,
// materialProperties, scalarTextures, spectrumTextures, backgroundTexture
void ref_counts(void *p, int32_t *c) {
    auto &s = *static_cast<RefScene *>(p);
    c[0] = int32_t(s.spectra.size());
    c[1] = int32_t(s.complexSpectra.size());
    c[2] = int32_t(s.objects.size());
    c[3] = int32_t(s.instances.size());
    c[4] = int32_t(s.nodes.size());
    c[5] = int32_t(s.lightInstances.size());
    c[6] = int32_t(s.materials.size());
    c[7] = int32_t(s.materialProperties.size());
    c[8] = int32_t(s.scalarTextures.size());
    c[9] = int32_t(s.spectrumTextures.size());
    c[10] = s.background.equirectangular.texture;
}

// Raw bytes of one container (which = index in ref_counts order; 10 = light
// powers, 11 = light objects, 12 = total light power, 13 = render settings).
int ref_copy(void *p, int which, void *dst) {
    auto &s = *static_cast<RefScene *>(p);
    auto cp = [&](const void *src, size_t n) { std::memcpy(dst, src, n); return 0; };
    switch (which) {
        case 0: return cp(s.spectra.data(), s.spectra.size() * sizeof(DenseSpectrum<Float>));
        case 1: return cp(s.complexSpectra.data(), s.complexSpectra.size() * sizeof(DenseSpectrum<Complex>));
        case 2: return cp(s.objects.data(), s.objects.size() * sizeof(Object));
        case 3: return cp(s.instances.data(), s.instances.size() * sizeof(Instance));
        case 4: return cp(s.nodes.data(), s.nodes.size() * sizeof(BVHNode));
        case 5: return cp(s.lightInstances.data(), s.lightInstances.size() * sizeof(int));
        case 6: return cp(s.materials.data(), s.materials.size() * sizeof(Material));
        case 7: return cp(s.materialProperties.data(), s.materialProperties.size() * sizeof(int));
        case 8: return cp(s.scalarTextures.data(), s.scalarTextures.size() * sizeof(ScalarTexture));
        case 9: return cp(s.spectrumTextures.data(), s.spectrumTextures.size() * sizeof(SpectrumTexture));
        case 10: return cp(s.lightPowers.data(), s.lightPowers.size() * sizeof(Float));
        case 11: return cp(s.lightObjects.data(), s.lightObjects.size() * sizeof(int));
        case 12: return cp(&s.totalLightPower, sizeof(Float));
        case 13: {
            const Renderer &r = s.renderer;
            int32_t iv[5] = {r.width, r.height, r.depth, r.samples, r.sqrtSamples};
            float fv[2 + 12];
            fv[0] = r.lambdaMin;
            fv[1] = r.lambdaMax;
            const Camera &c = r.camera;
            for (int k = 0; k < 3; k++) {
                fv[2 + k] = c.position[k];
                fv[5 + k] = c.corner[k];
                fv[8 + k] = c.horizontal[k];
                fv[11 + k] = c.vertical[k];
            }
            std::memcpy(dst, iv, sizeof(iv));
            std::memcpy(static_cast<char *>(dst) + sizeof(iv), fv, sizeof(fv));
            return 0;
        }
        default: return 1;
    }
}

// Overrides the sample count (a perfect square) of the parsed Render command.
void ref_set_samples(void *p, int samples) {
    auto &s = *static_cast<RefScene *>(p);
    int sq = int(std::sqrt(double(samples)));
    s.renderer.samples = samples;
    s.renderer.sqrtSamples = sq;
}

// Renderer::renderImage with `threads` OpenMP threads; returns seconds spent in it.
double ref_render(void *p, uint64_t seed, int threads, float *out_rgb) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    std::vector<Float> buffer(size_t(s.renderer.totalPixels) * 3);
    s.renderer.setBuffer(buffer.data());
    int completed = 0;
    if (threads > 0) omp_set_num_threads(threads);
    auto t0 = std::chrono::steady_clock::now();
    s.renderer.renderImage(&completed, seed);
    auto t1 = std::chrono::steady_clock::now();
    if (out_rgb) std::memcpy(out_rgb, buffer.data(), buffer.size() * sizeof(Float));
    return std::chrono::duration<double>(t1 - t0).count();
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// Renderer::trace for one pixel sample: radiance of 4 hero wavelengths of the path
// that pixel (px, py) draws for sample index `sample` (0-based, i-outer j-inner).
void ref_trace_sample(void *p, uint64_t seed, int px, int py, int sample, float *radiance_out, float *lambdas_out) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    const Renderer &r = s.renderer;
    Random state(seed, uint64_t(py) * uint64_t(r.width) + uint64_t(px));
    int k = 0;
    for (int i = 0; i < r.sqrtSamples; i++)
        for (int j = 0; j < r.sqrtSamples; j++, k++) {
            Float u = (Float(px) + (Float(i) + randomFloat(state)) / Float(r.sqrtSamples)) / Float(r.width);
            Float v = (Float(py) + (Float(j) + randomFloat(state)) / Float(r.sqrtSamples)) / Float(r.height);
            Float lambda = r.lambdaMin + randomFloat(state) * (r.lambdaMax - r.lambdaMin);
            SampledSpectrum lambdas;
            for (int h = 0; h < HERO_COUNT; h++)
                lambdas[h] = r.lambdaMin + fmodF(lambda - r.lambdaMin + Float(h) * r.lambdaRange / HERO_COUNT, r.lambdaRange);
            Ray ray = r.camera.getRay(u, v, lambdas);
            SampledSpectrum spectrum = r.trace(ray, state);
            if (k == sample) {
                for (int h = 0; h < HERO_COUNT; h++) {
                    radiance_out[h] = spectrum[h];
                    lambdas_out[h] = lambdas[h];
                }
                return;
            }
        }
}

// Renderer::renderPixel's samples of pixel (px, py) one by one: radiance_out
// [samples][4] holds each sample's spectrum at its 4 hero wavelengths, before the
// film average.
void ref_trace_pixel(void *p, uint64_t seed, int px, int py, float *radiance_out) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    const Renderer &r = s.renderer;
    Random state(seed, uint64_t(py) * uint64_t(r.width) + uint64_t(px));
    int k = 0;
    for (int i = 0; i < r.sqrtSamples; i++)
        for (int j = 0; j < r.sqrtSamples; j++, k++) {
            Float u = (Float(px) + (Float(i) + randomFloat(state)) / Float(r.sqrtSamples)) / Float(r.width);
            Float v = (Float(py) + (Float(j) + randomFloat(state)) / Float(r.sqrtSamples)) / Float(r.height);
            Float lambda = r.lambdaMin + randomFloat(state) * (r.lambdaMax - r.lambdaMin);
            SampledSpectrum lambdas;
            for (int h = 0; h < HERO_COUNT; h++)
                lambdas[h] = r.lambdaMin + fmodF(lambda - r.lambdaMin + Float(h) * r.lambdaRange / HERO_COUNT, r.lambdaRange);
            Ray ray = r.camera.getRay(u, v, lambdas);
            SampledSpectrum spectrum = r.trace(ray, state);
            for (int h = 0; h < HERO_COUNT; h++) radiance_out[4 * k + h] = spectrum[h];
        }
}

// Scene::hit closest-hit queries. rays: [n][6].
void ref_hit(void *p, const float *rays, int n, int32_t *inst, int32_t *obj, float *t, float *pn /* [n][8]: point, normal, u, v */, int32_t *front) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    SampledSpectrum l(500);
    for (int k = 0; k < n; k++) {
        Ray r(Vector(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]), Vector(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]), l);
        Intersection it;
        bool h = s.renderer.scene.hit(r, it);
        inst[k] = h ? it.instance : -1;
        obj[k] = h ? it.object : -1;
        t[k] = it.t;
        if (pn) {
            for (int c = 0; c < 3; c++) {
                pn[8 * k + c] = it.point[c];
                pn[8 * k + 3 + c] = it.normal[c];
            }
            pn[8 * k + 6] = it.u;
            pn[8 * k + 7] = it.v;
        }
        if (front) front[k] = it.frontFacing ? 1 : 0;
    }
}

// Scene::hit shadow queries (renderer.h:166).
void ref_shadow(void *p, const float *rays, const int32_t *li, const int32_t *lo, int n, int32_t *occ) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    SampledSpectrum l(500);
    for (int k = 0; k < n; k++) {
        Ray r(Vector(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]), Vector(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]), l);
        Intersection it;
        occ[k] = s.renderer.scene.hit(r, it, li[k], lo[k]) ? 1 : 0;
    }
}

// Material::thinFilmReflectance of material m for a hit with the given shading
// normal, facing flag and world point, seen along direction d, at lambda.
float ref_thinfilm(void *p, int m, const float *normal, int front, const float *point, const float *d, float lambda) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    Intersection it;
    it.normal = Vector(normal[0], normal[1], normal[2]);
    it.point = Vector(point[0], point[1], point[2]);
    it.frontFacing = front != 0;
    SampledSpectrum l(lambda);
    Ray r(it.point, Vector(d[0], d[1], d[2]), l);
    return s.materials[m].thinFilmReflectance(s.complexSpectra.data(), s.materialProperties.data(), s.scalarTextures.data(), it, r, lambda);
}

// The reference's transfer-matrix helpers (utils.h:173-193) for one film on a
// substrate, outer index 1: returns R_s, R_p in out[0..1] (double).
void ref_tmm_single(double lambda, double cos_theta, double d, double n_film, double n_sub, double *out) {
    Complex n0(1.0), n1(n_film), n2(n_sub);
    Complex cosCurrent = cos_theta;
    Complex sinNext = n0 / n1;
    sinNext *= sinNext * (Complex(1) - cosCurrent * cosCurrent);
    Complex cosNext = sqrtC(Complex(1) - sinNext);
    Matrix2<Complex> ms = interfaceMatrixS(n0, n1, cosCurrent, cosNext);
    Matrix2<Complex> mp = interfaceMatrixP(n0, n1, cosCurrent, cosNext);
    Complex cos1 = cosNext;
    Complex sin1 = sinNext;
    Complex sin2 = n1 / n2;
    sin2 *= sin2 * sin1;
    Complex cos2 = sqrtC(Complex(1) - sin2);
    Complex phi = n1 * Complex(2 * 3.14159265358979323846 / lambda) * d * cos1;
    Matrix2<Complex> prop = propagationMatrix(phi);
    ms *= prop * interfaceMatrixS(n1, n2, cos1, cos2);
    mp *= prop * interfaceMatrixP(n1, n2, cos1, cos2);
    double rs = std::abs(ms.get(0, 1) / ms.get(0, 0));
    double rp = std::abs(mp.get(0, 1) / mp.get(0, 0));
    out[0] = rs * rs;
    out[1] = rp * rp;
}

float ref_scalar_texture(void *p, int tex, const float *point) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    Intersection it;
    it.point = Vector(point[0], point[1], point[2]);
    return s.scalarTextures[tex].evaluate(it);
}

float ref_spectrum_texture(void *p, int tex, const float *point, float u, float v, float lambda) {
    auto &s = *static_cast<RefScene *>(p);
    wire(s);
    Intersection it;
    it.point = Vector(point[0], point[1], point[2]);
    it.u = u;
    it.v = v;
    return s.spectrumTextures[tex].evaluate(s.spectra.data(), s.scalarTextures.data(), it, lambda);
}

float ref_perlin(const float *point) {
    install_tables();
    return perlinNoise(Vector(point[0], point[1], point[2]));
}

float ref_worley(const float *point) { return worleyNoise(Vector(point[0], point[1], point[2])); }

void ref_spectrum_to_rgb(const float *radiance, const float *lambdas, float range, float *rgb) {
    install_tables();
    SampledSpectrum s, l;
    for (int i = 0; i < HERO_COUNT; i++) {
        s[i] = radiance[i];
        l[i] = lambdas[i];
    }
    Vector v = spectrumToRGB(s, l, range);
    rgb[0] = v[0];
    rgb[1] = v[1];
    rgb[2] = v[2];
}

// PCG32 stream (random.h): n draws of Random(seed, stream).next().
void ref_pcg(uint64_t seed, uint64_t stream, int n, float *out) {
    Random r(seed, stream);
    for (int i = 0; i < n; i++) out[i] = r.next();
}

int ref_write_ppm(const char *path, int w, int h, const float *rgb, char *err, size_t err_len) {
    try {
        Writer::write(path, w, h, const_cast<float *>(rgb));
    } catch (const std::exception &e) {
        put_err(err, err_len, e.what());
        return 1;
    }
    return 0;
}

}  // extern "C"
