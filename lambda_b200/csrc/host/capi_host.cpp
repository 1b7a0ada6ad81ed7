// Host half of the C ABI (include/lambda_gpu.h): scene parsing and PPM output.
// Exceptions never cross the boundary; they become status codes and messages.
#include <cstring>
#include <new>
#include <string>

#include "lambda_gpu.h"
#include "scene.h"

namespace {

void put_error(char *err, size_t len, const std::string &msg) {
    if (!err || len == 0) return;
    const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
    std::memcpy(err, msg.data(), n);
    err[n] = 0;
}

}  // namespace

lambda_status lambda_host::parse_into(const char *path, lambda_host_scene **out, char *err, size_t err_len,
                                      const BuildAccel *accel) {
    if (!path || !out) {
        put_error(err, err_len, "lambda_parse_lrd: null argument");
        return LAMBDA_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    auto *s = new (std::nothrow) lambda_host_scene();
    if (!s) return LAMBDA_ERR_OUT_OF_MEMORY;
    try {
        lambda_host::parse_lrd(path, s->scene, accel);
    } catch (const lambda_host::SceneError &e) {
        put_error(err, err_len, e.what());
        delete s;
        return e.status;
    } catch (const std::bad_alloc &) {
        put_error(err, err_len, "out of host memory");
        delete s;
        return LAMBDA_ERR_OUT_OF_MEMORY;
    } catch (const std::exception &e) {
        put_error(err, err_len, e.what());
        delete s;
        return LAMBDA_ERR_INTERNAL;
    }
    put_error(err, err_len, "");
    *out = s;
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_parse_lrd(const char *path, lambda_host_scene **out, char *err, size_t err_len) {
    return lambda_host::parse_into(path, out, err, err_len, nullptr);
}

extern "C" lambda_status lambda_host_scene_get(const lambda_host_scene *s, lambda_scene_desc *desc,
                                               lambda_render_settings *settings) {
    if (!s) return LAMBDA_ERR_INVALID_ARGUMENT;
    if (desc) *desc = s->scene.desc();
    if (settings) *settings = s->scene.settings;
    return LAMBDA_OK;
}

extern "C" void lambda_host_scene_destroy(lambda_host_scene *s) { delete s; }

extern "C" lambda_status lambda_write_ppm(const char *path, int32_t width, int32_t height, const float *rgb,
                                          char *err, size_t err_len) {
    if (!path || !rgb || width <= 0 || height <= 0) {
        put_error(err, err_len, "lambda_write_ppm: invalid argument");
        return LAMBDA_ERR_INVALID_ARGUMENT;
    }
    try {
        lambda_host::write_ppm(path, width, height, rgb);
    } catch (const lambda_host::SceneError &e) {
        put_error(err, err_len, e.what());
        return e.status;
    } catch (const std::exception &e) {
        put_error(err, err_len, e.what());
        return LAMBDA_ERR_INTERNAL;
    }
    put_error(err, err_len, "");
    return LAMBDA_OK;
}

extern "C" lambda_status lambda_write_pfm(const char *path, int32_t width, int32_t height, const float *rgb,
                                          int32_t xyz, char *err, size_t err_len) {
    if (!path || !rgb || width <= 0 || height <= 0) {
        put_error(err, err_len, "lambda_write_pfm: invalid argument");
        return LAMBDA_ERR_INVALID_ARGUMENT;
    }
    try {
        lambda_host::write_pfm(path, width, height, rgb, xyz != 0);
    } catch (const lambda_host::SceneError &e) {
        put_error(err, err_len, e.what());
        return e.status;
    } catch (const std::exception &e) {
        put_error(err, err_len, e.what());
        return LAMBDA_ERR_INTERNAL;
    }
    put_error(err, err_len, "");
    return LAMBDA_OK;
}
