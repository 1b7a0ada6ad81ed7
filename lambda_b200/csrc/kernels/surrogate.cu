// Thin-film surrogate MLP: training, weight install, tensor-core inference.
#include <cuda_runtime.h>

#include "engine.h"
#include "lambda_gpu.h"

lambda_status lambda_ctx::surrogate_ready() {
    if (!has_surrogate) return fail(LAMBDA_ERR_INVALID_ARGUMENT, "no surrogate installed (lambda_surrogate_train or lambda_surrogate_set)");
    return LAMBDA_OK;
}

int lambda_ctx::launch_shade_surrogate(int, const lambda_dev::RenderParams &, const lambda_dev::DeviceScene &,
                                       const lambda_dev::PathState &, int, StageProfiler *) {
    return 0;
}

extern "C" lambda_status lambda_surrogate_train(lambda_ctx *ctx, const lambda_train_desc *, lambda_train_report *) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "surrogate training not built yet");
}

extern "C" lambda_status lambda_surrogate_set(lambda_ctx *ctx, const float *, const lambda_film_range *) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "surrogate not built yet");
}

extern "C" lambda_status lambda_surrogate_get(const lambda_ctx *ctx, float *, lambda_film_range *) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    return LAMBDA_ERR_UNSUPPORTED;
}

extern "C" lambda_status lambda_surrogate_eval(lambda_ctx *ctx, const lambda_film_query *, int32_t, float *) {
    if (!ctx) return LAMBDA_ERR_INVALID_ARGUMENT;
    return ctx->fail(LAMBDA_ERR_UNSUPPORTED, "surrogate not built yet");
}
