"""One kernel per bounce (tuning.fused_bounce) against the separate wavefront
kernels: the same images and statistics, bit for bit, on every scene family, in the
exact and FP64 thin-film forms, at every BVH width, and for a batch; surrogate renders
of thin films keep the separate kernels."""

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import _native as N
from lambda_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {
    "cornell": lambda d: scenes.cornell(d, 48, 48, 16, name="f_cornell.lrd"),
    "thinfilm": lambda d: scenes.thinfilm_spheres(d, 64, 36, 4, depth=12, name="f_thinfilm.lrd"),
    "mesh": lambda d: scenes.perlin_sphere(d, 48, 48, 4, levels=5, name="f_mesh.lrd"),
    "instanced": lambda d: scenes.instanced_meshes(d, 64, 40, 4, depth=8, instances=120, segments=16, rings=9,
                                                   box=14.0, name="f_instanced.lrd"),
}


def _stats(ctx):
    st = ctx.stats()
    return (st.paths, st.segments, st.shadow_rays, st.thinfilm_hits, st.thinfilm_fallback)


def _set(ctx, keep, width, fused):
    ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, width, 0, 0,
                   keep.compressed_nodes, fused)


def _restore(ctx, keep):
    ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                   keep.path_kernel_pixels, keep.lane_fetch, keep.compressed_nodes, keep.fused_bounce)


@pytest.mark.parametrize("case", sorted(CASES))
def test_fused_bounce_equals_separate_kernels(case, scene_dir, ctx):
    sc = CASES[case](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    flags = [lb.RENDER_THINFILM_EXACT] + ([lb.RENDER_THINFILM_FP64] if case == "thinfilm" else [])
    try:
        for width in (2, 4, 8):
            for f in flags:
                desc = scene.render_desc(seed=sc.seed, flags=f)
                _set(ctx, keep, width, 0)
                want, ws = ctx.render(desc), _stats(ctx)
                _set(ctx, keep, width, 1)
                got, gs = ctx.render(desc), _stats(ctx)
                assert np.array_equal(got, want, equal_nan=True), f"{case} width {width} flags {f}: images differ"
                assert gs == ws, f"{case} width {width}: statistics {gs} vs {ws}"
    finally:
        _restore(ctx, keep)


def test_fused_bounce_profiled_and_batched(scene_dir, ctx):
    """The stage profile names the fused kernel (one launch per bounce), and a batch of
    uneven jobs renders each image as its job alone."""
    sc = CASES["cornell"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    try:
        _set(ctx, keep, 4, 1)
        ctx.render(scene.render_desc(seed=1, flags=N.RENDER_PROFILE_STAGES))
        st = ctx.stage_times()
        assert st["bounce"]["launches"] > 0 and st["intersect"]["launches"] == 0
        assert st["bounce"]["items"] == ctx.stats().segments
        descs = scenes.random_pose_jobs(scene, 5, seed=4, resolutions=(16, 24, 40), spps=(1, 4, 9), depth=(2, 12))
        _set(ctx, keep, 4, 0)
        alone = [ctx.render(d) for d in descs]
        _set(ctx, keep, 4, 1)
        batch = ctx.render_batch(descs)
    finally:
        _restore(ctx, keep)
    for a, b in zip(alone, batch):
        assert np.array_equal(a, b, equal_nan=True)


def test_surrogate_keeps_separate_kernels(scene_dir, ctx):
    from lambda_b200 import surrogate

    surrogate.install(ctx)
    sc = CASES["thinfilm"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    try:
        _set(ctx, keep, 4, 1)
        ctx.render(scene.render_desc(seed=1, flags=lb.RENDER_THINFILM_SURROGATE | N.RENDER_PROFILE_STAGES))
        st = ctx.stage_times()
        assert st["bounce"]["launches"] == 0 and st["film_mlp"]["launches"] > 0
    finally:
        _restore(ctx, keep)
