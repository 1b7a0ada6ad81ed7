// Host scene: what the .lrd/.obj parser and the BVH builder produce, held as the
// flat POD arrays of lambda_gpu.h (the reference's 15 containers, parser.h:29).
#pragma once

#include <functional>
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

// Steps of the scene build that a GPU can take over. Each one must produce the
// values of the host loop it replaces float for float and byte for byte (the tests
// compare the two), and reports failures by throwing SceneError. An empty member
// leaves its step on the host.
struct BuildAccel {
    // Instance::min/max/center (instance.h:54-101) of every instance, in the order
    // of scene.instances: 9 floats each (lo xyz, hi xyz, centroid xyz).
    std::function<void(const HostScene &, std::vector<float> &)> instance_bounds;
    // The binned-SAH build (bvh.h:111-246) of items order[start, end), given each
    // item's 9 floats (lo, hi, centroid) in `items`: reorders order[start, end)
    // and appends the subtree's nodes, root first, to `nodes` as the host recursion
    // writes them.
    std::function<void(const std::vector<float> &items, std::vector<int> &order, int start, int end,
                       std::vector<lambda_bvh_node> &nodes)>
        build;
    // Ranges with at least this many items go to `build`; smaller ones stay on the host.
    int build_min_items = 1 << 16;
};

// Parser::parseLRD (parser.h:29-379): throws SceneError. With accel, the build
// steps it names run on the GPU, with the same results.
void parse_lrd(const std::string &path, HostScene &scene, const BuildAccel *accel = nullptr);

// BVH::makeBVH (bvh.h:61-108): builds the TLAS over instances and one BLAS per
// object group into scene.nodes, reordering scene.instances and scene.objects.
// group_offsets holds the first object of every group plus objects.size(). When
// instance_boxes is given it receives each instance's world bounds (lo xyz, hi xyz)
// in the reordered instance order, for build_lights.
void build_bvh(HostScene &scene, const std::vector<int> &group_offsets, const BuildAccel *accel = nullptr,
               std::vector<float> *instance_boxes = nullptr);

// Light list and background power (parser.h:333-378). instance_boxes (from
// build_bvh) lets the scene-sphere merge pass over instances that provably change
// nothing.
void build_lights(HostScene &scene, const std::vector<float> *instance_boxes = nullptr);

// The status-returning half of lambda_parse_lrd and lambda_parse_lrd_gpu: parses
// into a new handle, turning exceptions into a status and the message into err.
lambda_status parse_into(const char *path, struct ::lambda_host_scene **out, char *err, size_t err_len,
                         const BuildAccel *accel);

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

// The handle behind lambda_host_scene.
struct lambda_host_scene {
    lambda_host::HostScene scene;
};
