// ASCII PPM output (src/core/writer.h:11-41): clamp to [0,1], sRGB OETF
// (utils.h:233-238), then round value*255 plus a dither in [-0.5, 0.5) drawn from
// PCG32(seed 0, stream 0), one draw per channel in pixel order (utils.h:240-244).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

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

namespace {

// XYZ -> linear sRGB as spectrumToRGB applies it (utils.h:230), and its inverse
// formed in double by cofactors.
constexpr double kXyzToRgb[3][3] = {{3.2406255, -1.5372080, -0.4986286},
                                    {-0.9689307, 1.8757561, 0.0415175},
                                    {0.0557101, -0.2040211, 1.0569959}};

struct RgbToXyz {
    double m[3][3];
    RgbToXyz() {
        const auto &a = kXyzToRgb;
        const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1], c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2],
                     c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
        const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
        m[0][0] = c00 / det;
        m[1][0] = c01 / det;
        m[2][0] = c02 / det;
        m[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
        m[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
        m[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
        m[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
        m[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
        m[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    }
};

}  // namespace

// Portable float map: "PF", size, scale -1 (little-endian), then float32 RGB rows
// from the bottom row up. With xyz, each pixel is converted from linear sRGB to
// CIE XYZ in double first.
void write_pfm(const std::string &path, int width, int height, const float *rgb, bool xyz) {
    const std::string ext = ".pfm";
    if (!(path.size() >= ext.size() && path.compare(path.size() - ext.size(), ext.size(), ext) == 0))
        throw SceneError(LAMBDA_ERR_INVALID_ARGUMENT, ": invalid file extension");
    std::ofstream out(path, std::ios::binary);
    if (!out.is_open()) {
        std::string e = std::strerror(errno);
        if (!e.empty()) e[0] = char(std::tolower(e[0]));
        throw SceneError(LAMBDA_ERR_IO, ": failed to open file (" + e + ")");
    }
    static const RgbToXyz inv;
    const std::string head = "PF\n" + std::to_string(width) + " " + std::to_string(height) + "\n-1.0\n";
    out.write(head.data(), std::streamsize(head.size()));
    std::vector<float> row(size_t(width) * 3);
    for (int y = height - 1; y >= 0; y--) {
        const float *src = rgb + size_t(y) * width * 3;
        for (int x = 0; x < width; x++)
            for (int c = 0; c < 3; c++) {
                const float *p = src + 3 * size_t(x);
                row[3 * size_t(x) + c] =
                    xyz ? float(inv.m[c][0] * p[0] + inv.m[c][1] * p[1] + inv.m[c][2] * p[2]) : p[c];
            }
        out.write(reinterpret_cast<const char *>(row.data()), std::streamsize(row.size() * sizeof(float)));
    }
    if (!out) throw SceneError(LAMBDA_ERR_IO, ": failed to write file");
}

}  // namespace lambda_host
