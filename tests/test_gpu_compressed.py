"""The compressed BVH node records (8-bit child boxes, tested exactly when popped)
against the exact records: the same images and statistics, bit for bit, in every
traversal form (warp and lane-by-lane wavefront, path kernel) and width. The ray
queries are checked against the reference in tests/test_gpu_traversal.py."""

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {
    "thinfilm": lambda d: scenes.thinfilm_spheres(d, 64, 36, 4, depth=8, name="c_thinfilm.lrd"),
    "mesh": lambda d: scenes.perlin_sphere(d, 48, 48, 4, levels=6, name="c_mesh.lrd"),
    "instanced": lambda d: scenes.instanced_meshes(d, 64, 40, 4, depth=8, instances=200, segments=16, rings=9,
                                                   box=14.0, name="c_instanced.lrd"),
}


def _stats(ctx):
    st = ctx.stats()
    return (st.paths, st.segments, st.shadow_rays, st.thinfilm_hits)


@pytest.mark.parametrize("case", sorted(CASES))
def test_compressed_renders_equal_exact(case, scene_dir, ctx):
    sc = CASES[case](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    desc = scene.render_desc(seed=sc.seed)
    keep = ctx.tuning()
    try:
        for width in (2, 4, 8):
            for lane_fetch, path_pixels in ((0, 0), (1, 0), (0, 1 << 30)):
                imgs, stats = [], []
                for compressed in (0, 1):
                    ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, width,
                                   path_pixels, lane_fetch, compressed)
                    imgs.append(ctx.render(desc))
                    stats.append(_stats(ctx))
                form = f"{case} width {width} lane_fetch {lane_fetch} path {path_pixels > 0}"
                assert np.array_equal(imgs[0], imgs[1], equal_nan=True), f"{form}: images differ"
                assert stats[0] == stats[1], f"{form}: statistics {stats[1]} vs {stats[0]}"
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels, keep.lane_fetch, keep.compressed_nodes)
