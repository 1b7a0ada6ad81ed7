// Timing harness around the reference renderer's own CUDA kernel (baseline only).
//
// This file is test and benchmark infrastructure, never part of the product. It is
// compiled by oracle/Makefile (target ref_gpu) against the reference headers where
// they lie (REF_SRC), as the reference's own CUDA build compiles them (nvcc, C++20,
// relocatable device code, -O3), for sm_100a, into oracle/_ref/libref_lambda_gpu.so.
// It drives the reference's stock GPU path exactly as its main.cpp does
// (src/main.cpp:57-124): Parser::parseLRD into the host containers, a managed-memory
// Buffer per container and for the PERMUTATION / CIE tables, Renderer::setScene and
// setBuffer, then renderKernel<<<(W/16, H/16), (16, 16)>>>(completed, renderer, seed)
// (src/render/renderer.h:200-213). Only the launch is timed, with CUDA events; the
// host waits for it with a wall-clock limit instead of main.cpp's unbounded poll
// (main.cpp:129-146), and reports a timeout as an error.

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#define private public
#include "core/buffer.h"
#include "core/constants.h"
#include "core/parser.h"
#include "core/platform.h"
#include "core/utils.h"
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

struct GpuScene {
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

    // device copies, as main.cpp makes them (managed memory)
    std::unique_ptr<Buffer<int>> d_permutation;
    std::unique_ptr<Buffer<double>> d_cie, d_d65;
    std::unique_ptr<Buffer<DenseSpectrum<Float>>> d_spectra;
    std::unique_ptr<Buffer<DenseSpectrum<Complex>>> d_complexSpectra;
    std::unique_ptr<Buffer<Object>> d_objects;
    std::unique_ptr<Buffer<Instance>> d_instances;
    std::unique_ptr<Buffer<BVHNode>> d_nodes;
    std::unique_ptr<Buffer<int>> d_lightInstances, d_lightObjects, d_materialProperties;
    std::unique_ptr<Buffer<Float>> d_lightPowers, d_output;
    std::unique_ptr<Buffer<Material>> d_materials;
    std::unique_ptr<Buffer<ScalarTexture>> d_scalarTextures;
    std::unique_ptr<Buffer<SpectrumTexture>> d_spectrumTextures;
    std::unique_ptr<Buffer<int>> d_completed;
};

void put_err(char *err, size_t len, const std::string &msg) {
    if (!err || len == 0) return;
    const size_t n = std::min(len - 1, msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = 0;
}

}  // namespace

extern "C" {

// Parses the scene with the reference's parser and makes main.cpp's device copies.
int refgpu_open(const char *path, void **out, char *err, size_t err_len) {
    auto s = std::make_unique<GpuScene>();
    try {
        Parser::parseLRD(path, s->renderer, s->spectra, s->complexSpectra, s->background, s->objects, s->instances,
                         s->nodes, s->lightInstances, s->lightObjects, s->lightPowers, s->totalLightPower,
                         s->materials, s->materialProperties, s->scalarTextures, s->spectrumTextures);
        s->d_permutation = std::make_unique<Buffer<int>>(&h_PERMUTATION[0], &h_PERMUTATION[PERMUTATION_SIZE - 1] + 1);
        s->d_cie = std::make_unique<Buffer<double>>(&h_CIE_XYZ_1931[0][0], &h_CIE_XYZ_1931[CIE_LAMBDA_BINS - 1][2] + 1);
        s->d_d65 = std::make_unique<Buffer<double>>(&h_CIE_D65[0], &h_CIE_D65[CIE_D65_LAMBDA_BINS - 1] + 1);
        PERMUTATION = s->d_permutation->data();
        CIE_XYZ_1931 = s->d_cie->data();
        CIE_D65 = s->d_d65->data();
        s->d_spectra = std::make_unique<Buffer<DenseSpectrum<Float>>>(s->spectra);
        s->d_complexSpectra = std::make_unique<Buffer<DenseSpectrum<Complex>>>(s->complexSpectra);
        s->d_objects = std::make_unique<Buffer<Object>>(s->objects);
        s->d_instances = std::make_unique<Buffer<Instance>>(s->instances);
        s->d_nodes = std::make_unique<Buffer<BVHNode>>(s->nodes);
        s->d_lightInstances = std::make_unique<Buffer<int>>(s->lightInstances);
        s->d_lightObjects = std::make_unique<Buffer<int>>(s->lightObjects);
        s->d_lightPowers = std::make_unique<Buffer<Float>>(s->lightPowers);
        s->d_materials = std::make_unique<Buffer<Material>>(s->materials);
        s->d_materialProperties = std::make_unique<Buffer<int>>(s->materialProperties);
        s->d_scalarTextures = std::make_unique<Buffer<ScalarTexture>>(s->scalarTextures);
        s->d_spectrumTextures = std::make_unique<Buffer<SpectrumTexture>>(s->spectrumTextures);
        s->renderer.setScene(s->d_spectra->data(), s->d_complexSpectra->data(), s->background, s->d_objects->data(),
                             s->d_instances->data(), s->d_nodes->data(), s->d_lightInstances->data(),
                             s->d_lightObjects->data(), int(s->lightInstances.size()), s->d_lightPowers->data(),
                             s->totalLightPower, s->d_materials->data(), s->d_materialProperties->data(),
                             s->d_scalarTextures->data(), s->d_spectrumTextures->data());
        s->d_output = std::make_unique<Buffer<Float>>(size_t(s->renderer.getTotalPixels()) * 3);
        s->renderer.setBuffer(s->d_output->data());
        s->d_completed = std::make_unique<Buffer<int>>(size_t(1));
    } catch (const std::exception &e) {
        put_err(err, err_len, e.what());
        return 1;
    }
    *out = s.release();
    return 0;
}

void refgpu_close(void *p) { delete static_cast<GpuScene *>(p); }

void refgpu_set_samples(void *p, int samples) {
    auto &s = *static_cast<GpuScene *>(p);
    s.renderer.samples = samples;
    s.renderer.sqrtSamples = int(std::sqrt(double(samples)));
}

// One launch of the stock renderKernel (main.cpp's grid and block). Returns the
// kernel's device time in milliseconds through *ms and copies the image (linear
// sRGB, W*H*3) to out_rgb when it is not null. Status: 0 ok, 1 CUDA error, 2 the
// kernel did not finish within limit_s seconds.
int refgpu_render(void *p, uint64_t seed, double limit_s, float *out_rgb, double *ms, char *err, size_t err_len) {
    auto &s = *static_cast<GpuScene *>(p);
    PERMUTATION = s.d_permutation->data();
    CIE_XYZ_1931 = s.d_cie->data();
    CIE_D65 = s.d_d65->data();
    const int bw = 16, bh = 16;
    dim3 block(bw, bh);
    dim3 grid((s.renderer.getWidth() + bw - 1) / bw, (s.renderer.getHeight() + bh - 1) / bh);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemset(s.d_completed->data(), 0, sizeof(int));
    cudaEventRecord(e0);
    renderKernel<<<grid, block>>>(s.d_completed->data(), s.renderer, seed);
    cudaEventRecord(e1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        put_err(err, err_len, std::string("launch: ") + cudaGetErrorString(e));
        return 1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        e = cudaEventQuery(e1);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) {
            put_err(err, err_len, std::string("render: ") + cudaGetErrorString(e));
            return 1;
        }
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit_s) {
            put_err(err, err_len, "renderKernel did not finish within the time limit");
            return 2;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
    }
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (out_rgb) {
        e = cudaMemcpy(out_rgb, s.d_output->data(), size_t(s.renderer.getTotalPixels()) * 3 * sizeof(Float),
                       cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            put_err(err, err_len, std::string("copy: ") + cudaGetErrorString(e));
            return 1;
        }
    }
    return 0;
}

}  // extern "C"
