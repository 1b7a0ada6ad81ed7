"""The intersect kernel that takes rays lane by lane (lambda_tuning.lane_fetch)
against the one that traces a warp's 32 rays to the end: the same images and
statistics bit for bit on every scene family, BVH width and thin-film mode, alone
and in batches."""

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {
    "cornell": lambda d: scenes.cornell(d, 48, 48, 16, name="f_cornell.lrd"),
    "thinfilm": lambda d: scenes.thinfilm_spheres(d, 96, 54, 16, name="f_thinfilm.lrd"),
    "mesh": lambda d: scenes.perlin_sphere(d, 48, 48, 4, levels=5, name="f_mesh.lrd"),
    "instanced": lambda d: scenes.instanced_meshes(d, 64, 40, 9, depth=8, instances=120, segments=16, rings=9,
                                                   box=14.0, name="f_instanced.lrd"),
}


def _stats(ctx):
    st = ctx.stats()
    return (st.paths, st.segments, st.shadow_rays, st.thinfilm_hits, st.thinfilm_fallback)


def _both(ctx, render, width=4):
    keep = ctx.tuning()
    out = []
    try:
        for fetch in (0, 1):
            # path kernel off: the wavefront's intersect kernel is the one compared
            ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, width, 0, fetch)
            out.append((render(), _stats(ctx)))
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels, keep.lane_fetch)
    return out


def _same(a, b):
    if isinstance(a, list):
        return all(np.array_equal(x, y, equal_nan=True) for x, y in zip(a, b))
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("case", sorted(CASES))
def test_lane_fetch_equals_warp_tracing(case, scene_dir, ctx):
    sc = CASES[case](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    for width in (2, 4, 8):
        (a, sa), (b, sb) = _both(ctx, lambda: ctx.render(scene.render_desc(seed=sc.seed)), width)
        assert _same(a, b), f"{case} width {width}: images differ"
        assert sa == sb, f"{case} width {width}: statistics {sa} vs {sb}"


@pytest.mark.parametrize("flags", [lb.RENDER_THINFILM_FP64, lb.RENDER_THINFILM_SURROGATE])
def test_lane_fetch_thin_film_modes(flags, scene_dir, ctx):
    from lambda_b200 import surrogate

    surrogate.install(ctx)
    sc = CASES["thinfilm"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    (a, sa), (b, sb) = _both(ctx, lambda: ctx.render(scene.render_desc(seed=2, flags=flags)))
    assert _same(a, b) and sa == sb and sa[3] > 0


def test_lane_fetch_batch(scene_dir, ctx):
    sc = CASES["instanced"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    descs = scenes.random_pose_jobs(scene, 6, seed=4, resolutions=(16, 24, 40), spps=(1, 4, 9), depth=(2, 12),
                                    target=(0.0, 0.0, 0.0), distance=(10.0, 14.0), height=(-2.0, 4.0))
    (a, sa), (b, sb) = _both(ctx, lambda: ctx.render_batch(descs))
    assert _same(a, b) and sa == sb
