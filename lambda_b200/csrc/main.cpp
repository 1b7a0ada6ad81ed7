// `lambda <scene.lrd> [out.ppm]`: the reference's command-line renderer
// (src/main.cpp:27-174) on the B200 render loop. Same arguments, messages,
// progress line, seed (42) and PPM output; rendering goes through the C ABI.
#include <chrono>
#include <cstdio>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "lambda_gpu.h"

static bool has_ext(const std::string &s, const std::string &e) {
    return s.size() >= e.size() && s.compare(s.size() - e.size(), e.size(), e) == 0;
}

int main(int argc, char *argv[]) {
    if (argc != 2 && argc != 3) {
        std::cerr << argv[0] << ": invalid number of arguments" << std::endl;
        return 1;
    }
    const std::string input(argv[1]);
    if (!has_ext(input, ".lrd")) {
        std::cerr << input << ": invalid file extension" << std::endl;
        return 1;
    }
    std::string output;
    if (argc == 3) {
        output = argv[2];
        if (!has_ext(output, ".ppm")) {
            std::cerr << output << ": invalid file extension" << std::endl;
            return 1;
        }
    } else {
        output = input.substr(0, input.size() - 4) + ".ppm";
    }

    char err[1024] = {0};
    lambda_host_scene *scene = nullptr;
    // the scene build runs on the GPU when there is one (the same scene as the host build)
    lambda_ctx *ctx = nullptr;
    const bool have_gpu = lambda_ctx_create(0, &ctx) == LAMBDA_OK;
    const lambda_status parsed = have_gpu ? lambda_parse_lrd_gpu(ctx, input.c_str(), 0, &scene, err, sizeof(err))
                                          : lambda_parse_lrd(input.c_str(), &scene, err, sizeof(err));
    if (parsed != LAMBDA_OK) {
        std::cerr << err << std::endl;
        if (ctx) lambda_ctx_destroy(ctx);
        return 1;
    }
    lambda_scene_desc desc;
    lambda_render_desc rd{};
    lambda_host_scene_get(scene, &desc, &rd.settings);
    rd.seed = 42;
    rd.flags = LAMBDA_RENDER_THINFILM_EXACT;
    const int total = rd.settings.width * rd.settings.height;
    std::vector<float> image(size_t(total) * 3);

    if (!have_gpu) {
        std::cerr << argv[0] << ": " << lambda_last_error(nullptr) << std::endl;
        lambda_host_scene_destroy(scene);
        return 1;
    }
    if (lambda_scene_upload(ctx, &desc) != LAMBDA_OK) {
        std::cerr << argv[0] << ": " << lambda_last_error(ctx) << std::endl;
        lambda_ctx_destroy(ctx);
        lambda_host_scene_destroy(scene);
        return 1;
    }
    std::cout << "\r" << argv[0] << ": 0% complete" << std::flush;
    volatile int32_t completed = 0;
    lambda_status status = LAMBDA_OK;
    std::thread worker([&] { status = lambda_render(ctx, &rd, image.data(), &completed); });
    bool done = false;
    while (!done) {
        const int c = completed;
        std::cout << "\r" << argv[0] << ": " << int(100.0 * c / total) << "% complete" << std::flush;
        if (c >= total) break;
        std::this_thread::sleep_for(std::chrono::milliseconds(100));
        done = status != LAMBDA_OK;
    }
    worker.join();
    if (status != LAMBDA_OK) {
        std::cerr << std::endl << argv[0] << ": " << lambda_last_error(ctx) << std::endl;
        lambda_ctx_destroy(ctx);
        lambda_host_scene_destroy(scene);
        return 1;
    }
    std::cout << "\r" << argv[0] << ": 100% complete" << std::flush << std::endl;
    lambda_ctx_destroy(ctx);
    lambda_host_scene_destroy(scene);
    if (lambda_write_ppm(output.c_str(), rd.settings.width, rd.settings.height, image.data(), err, sizeof(err)) != LAMBDA_OK) {
        std::cerr << output << err << std::endl;
        return 1;
    }
    return 0;
}
