// ASCII PPM output (src/core/writer.h:11-41): clamp to [0,1], sRGB OETF
// (utils.h:233-238), then round value*255 plus a dither in [-0.5, 0.5) drawn from
// PCG32(seed 0, stream 0), one draw per channel in pixel order (utils.h:240-244).
#include <cerrno>
#include <cmath>
#include <cstring>
#include <fstream>
#include <string>

#include "pcg32.h"
#include "scene.h"

namespace lambda_host {

namespace {

float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

float srgb_oetf(float r) {
    if (r <= 0.0031308) return 12.92f * r;
    return 1.055f * std::pow(r, 1 / 2.4f) - 0.055f;
}

int quantize(float value, uint64_t &state, uint64_t inc) {
    const float dither = lambda_rng::pcg_next_float(state, inc) - 0.5f;
    return int(clampf(float(int(std::round(value * 255 + dither))), 0, 255));
}

}  // namespace

void write_ppm(const std::string &path, int width, int height, const float *rgb) {
    const std::string ext = ".ppm";
    if (!(path.size() >= ext.size() && path.compare(path.size() - ext.size(), ext.size(), ext) == 0))
        throw SceneError(LAMBDA_ERR_INVALID_ARGUMENT, ": invalid file extension");
    std::ofstream out(path);
    if (!out.is_open()) {
        std::string e = std::strerror(errno);
        if (!e.empty()) e[0] = char(std::tolower(e[0]));
        throw SceneError(LAMBDA_ERR_IO, ": failed to open file (" + e + ")");
    }
    uint64_t state = lambda_rng::pcg_seed(0, 0);
    const uint64_t inc = lambda_rng::pcg_increment(0);
    std::string text = "P3\n" + std::to_string(width) + " " + std::to_string(height) + "\n255\n";
    text.reserve(text.size() + size_t(width) * height * 12);
    const size_t n = size_t(width) * size_t(height);
    for (size_t i = 0; i < n; i++) {
        for (int c = 0; c < 3; c++) {
            const int q = quantize(srgb_oetf(clampf(rgb[3 * i + c], 0, 1)), state, inc);
            text += std::to_string(q);
            text += c < 2 ? ' ' : '\n';
        }
    }
    out << text;
}

}  // namespace lambda_host
