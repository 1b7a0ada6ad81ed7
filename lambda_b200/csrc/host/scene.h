// Host scene: what the .lrd/.obj parser and the BVH builder produce, held as the
// flat POD arrays of lambda_gpu.h (the reference's 15 containers, parser.h:29).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "lambda_gpu.h"

namespace lambda_host {

constexpr int kBins = LAMBDA_CIE_BINS;

struct HostScene {
    lambda_render_settings settings{};
    std::vector<float> spectra;           // [n][471]
    std::vector<double> complex_spectra;  // [n][471][2]
    int32_t background_texture = -1;
    std::vector<lambda_object> objects;
    std::vector<lambda_instance> instances;
    std::vector<lambda_bvh_node> nodes;
    std::vector<int32_t> light_instances;
    std::vector<int32_t> light_objects;
    std::vector<float> light_powers;
    float total_light_power = 0;
    std::vector<lambda_material> materials;
    std::vector<int32_t> material_properties;
    std::vector<lambda_scalar_texture> scalar_textures;
    std::vector<lambda_spectrum_texture> spectrum_textures;

    int num_spectra() const { return int(spectra.size() / kBins); }
    int num_complex_spectra() const { return int(complex_spectra.size() / (2 * kBins)); }
    lambda_scene_desc desc() const;
};

// A parse failure (LAMBDA_ERR_PARSE) or an unreadable file (LAMBDA_ERR_IO); what()
// is the reference's message text.
struct SceneError : std::runtime_error {
    lambda_status status;
    SceneError(lambda_status s, const std::string &msg) : std::runtime_error(msg), status(s) {}
};

// Parser::parseLRD (parser.h:29-379): throws SceneError.
void parse_lrd(const std::string &path, HostScene &scene);

// BVH::makeBVH (bvh.h:61-108): builds the TLAS over instances and one BLAS per
// object group into scene.nodes, reordering scene.instances and scene.objects.
// group_offsets holds the first object of every group plus objects.size().
void build_bvh(HostScene &scene, const std::vector<int> &group_offsets);

// Light list and background power (parser.h:333-378).
void build_lights(HostScene &scene);

// Writer::write (writer.h:11-41): throws SceneError with the reference's text.
void write_ppm(const std::string &path, int width, int height, const float *rgb);
void write_pfm(const std::string &path, int width, int height, const float *rgb, bool xyz);

// Scalar/spectrum texture and spectrum statistics used while parsing.
float spectrum_average(const HostScene &s, int spectrum);
float spectrum_min(const HostScene &s, int spectrum);
float spectrum_max(const HostScene &s, int spectrum);
float spectrum_texture_min(const HostScene &s, int texture);
float spectrum_texture_max(const HostScene &s, int texture);
float spectrum_texture_average(const HostScene &s, int texture);

}  // namespace lambda_host
