"""The device-side guards fire, return their error, and leave the context usable.

Every wait in the kernels is bounded and every traversal stack push is checked.
lambda_set_limits lowers a limit so that a guard fires on an ordinary render:
an MMA-completion wait that may poll zero times gives up (LAMBDA_ERR_TIMEOUT), and
traversal stacks capped at one entry overflow (LAMBDA_ERR_QUEUE_OVERFLOW). Neither
faults or hangs the GPU: a wait that gives up still lets the MMAs it issued finish
before TMEM is freed, and a full stack stops the ray before any write past it. The
next call with the default limits renders the same image as before, bit for bit.
"""

import ctypes as C

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import _native as N
from lambda_b200 import scenes, surrogate

pytestmark = pytest.mark.gpu

TIMEOUT, OVERFLOW = 9, 8


def _status(excinfo) -> int:
    return excinfo.value.status


def test_mma_wait_gives_up_and_context_recovers(scene_dir, ctx):
    surrogate.install(ctx)
    sc = scenes.thinfilm_spheres(scene_dir, 64, 36, 4, depth=6, name="guard_film.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    desc = scene.render_desc(seed=sc.seed, flags=lb.RENDER_THINFILM_SURROGATE)
    want = ctx.render(desc)
    q = np.array([[550.0, 0.8, 400.0, 1.33, 1.5]] * 1000, np.float32)
    want_q = ctx.surrogate_eval(q)
    try:
        ctx.set_limits(mma_polls=0)
        assert ctx.limits().mma_polls == 0
        with pytest.raises(lb.LambdaError) as e:
            ctx.render(desc)
        assert _status(e) == TIMEOUT and "timed out" in ctx.last_error
        with pytest.raises(lb.LambdaError) as e:
            ctx.surrogate_eval(q)
        assert _status(e) == TIMEOUT
        import torch

        dq = torch.from_numpy(q).cuda()
        dout = torch.empty((len(q), 4), dtype=torch.float32, device="cuda")
        st = ctx._lib.lambda_surrogate_eval_static(ctx._h, C.c_void_p(dq.data_ptr()), len(q),
                                                   C.c_void_p(dout.data_ptr()))
        assert st == TIMEOUT
    finally:
        ctx.reset_limits()
    assert ctx.limits().mma_polls == N.DEFAULT_MMA_POLLS
    got = ctx.render(desc)
    assert np.array_equal(got, want, equal_nan=True)
    assert np.array_equal(ctx.surrogate_eval(q), want_q)


@pytest.mark.parametrize("path_kernel", [True, False])
def test_stack_overflow_is_reported_and_context_recovers(scene_dir, ctx, path_kernel):
    sc = scenes.perlin_sphere(scene_dir, 48, 48, 4, levels=5, name="guard_mesh.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    t = ctx.tuning()
    ctx.set_tuning(t.trace_block, t.shade_block, t.grid_scale, t.max_pixels, t.bvh_width,
                   N.PATH_KERNEL_PIXELS if path_kernel else 0, t.lane_fetch)
    desc = scene.render_desc(seed=sc.seed)
    rays = np.concatenate([np.tile(np.array([[0.0, 0.0, -3.0]], np.float32), (256, 1)),
                           np.random.default_rng(1).normal(0, 0.1, (256, 3)).astype(np.float32) + [0, 0, 1]], 1)
    rays[:, 3:] /= np.linalg.norm(rays[:, 3:], axis=1, keepdims=True)
    try:
        want = ctx.render(desc)
        want_hits = ctx.trace_closest(rays)
        ctx.set_limits(stack_entries=1)
        with pytest.raises(lb.LambdaError) as e:
            ctx.render(desc)
        assert _status(e) == OVERFLOW and "overflow" in ctx.last_error
        with pytest.raises(lb.LambdaError) as e:
            ctx.trace_closest(rays)
        assert _status(e) == OVERFLOW
        ctx.reset_limits()
        got = ctx.render(desc)
        assert np.array_equal(got, want, equal_nan=True)
        for a, b in zip(ctx.trace_closest(rays), want_hits):
            assert np.array_equal(a, b)
    finally:
        ctx.reset_limits()
        ctx.set_tuning(t.trace_block, t.shade_block, t.grid_scale, t.max_pixels, t.bvh_width,
                       t.path_kernel_pixels, t.lane_fetch)
