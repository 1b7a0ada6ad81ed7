"""Batched rendering (lambda_render_batch) and the launch-shape autotuner.

A batch renders many views of one scene (own camera, size, sample count, depth,
wavelength range and seed) as one wavefront. Every image must equal, bit for bit,
the single render of the same job, since each pixel keeps its own PCG32 stream
and arithmetic: the parity of single renders with the reference then carries
over to batches."""

import numpy as np
import pytest
import torch

import lambda_b200 as lb
from lambda_b200 import scenes, surrogate

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def film(scene_dir, ctx):
    sc = scenes.thinfilm_spheres(scene_dir, 48, 32, 4, depth=8, name="b_thinfilm.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    return scene


def _jobs(scene, n=7, seed=4, flags=0):
    descs = scenes.random_pose_jobs(scene, n, seed=seed, resolutions=(16, 24, 40), spps=(1, 4, 9, 16),
                                    depth=(2, 12), flags=flags)
    if n > 1:
        descs[1].settings.lambda_min, descs[1].settings.lambda_max = 400.0, 700.0
    return descs


def _same(a, b):
    return np.array_equal(a, b, equal_nan=True)


def test_batch_equals_single_renders(film, ctx):
    ctx.upload(film)
    descs = _jobs(film)
    done = np.zeros(1, np.int32)
    imgs = ctx.render_batch(descs, completed=done.ctypes.data)
    st = ctx.stats()
    total = sum(d.settings.width * d.settings.height for d in descs)
    assert int(done[0]) == total
    assert st.paths == sum(d.settings.width * d.settings.height * d.settings.samples for d in descs)
    assert st.waves == max(d.settings.samples for d in descs)
    for d, img in zip(descs, imgs):
        single = ctx.render(d)
        assert img.shape == (d.settings.height, d.settings.width, 3)
        assert _same(img, single), f"job {d.settings.width}x{d.settings.height} spp {d.settings.samples}"


def test_batch_device_outputs_and_passes(film, ctx):
    """Mixed host/device outputs, and a path-state capacity that forces several passes."""
    ctx.upload(film)
    descs = _jobs(film, n=6, seed=9)
    want = [ctx.render(d) for d in descs]
    keep = ctx.tuning()
    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, max_pixels=1200)
        outs = []
        for i, d in enumerate(descs):
            if i % 2:
                d.flags |= lb.RENDER_OUTPUT_DEVICE
                outs.append(torch.empty((d.settings.height, d.settings.width, 3), dtype=torch.float32, device="cuda"))
            else:
                outs.append(None)
        got = ctx.render_batch(descs, outs)
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels)
    for i, (g, w) in enumerate(zip(got, want)):
        g = g.cpu().numpy() if isinstance(g, torch.Tensor) else g
        assert _same(g, w), f"job {i}"


def test_batch_surrogate_equals_single(film, ctx):
    ctx.upload(film)
    surrogate.install(ctx)
    descs = _jobs(film, n=5, seed=12, flags=lb.RENDER_THINFILM_SURROGATE)
    imgs = ctx.render_batch(descs)
    assert ctx.stats().surrogate_ctas_per_sm >= 1
    for d, img in zip(descs, imgs):
        assert _same(img, ctx.render(d))


def test_batch_rejects_mixed_modes(film, ctx):
    ctx.upload(film)
    surrogate.install(ctx)
    descs = _jobs(film, n=2)
    descs[1].flags |= lb.RENDER_THINFILM_SURROGATE
    with pytest.raises(lb.LambdaError):
        ctx.render_batch(descs)
    descs = _jobs(film, n=2)
    descs[0].settings.samples = 3  # not a perfect square
    with pytest.raises(lb.LambdaError):
        ctx.render_batch(descs)


def test_launch_shapes_do_not_change_images(film, ctx):
    ctx.upload(film)
    d = _jobs(film, n=1, seed=21)[0]
    keep = ctx.tuning()
    try:
        ctx.set_tuning(256, 256, 1)
        a = ctx.render(d)
        ctx.set_tuning(64, 128, 2)
        b = ctx.render(d)
        with pytest.raises(lb.LambdaError):
            ctx.set_tuning(96, 256, 1)
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels)
    assert _same(a, b)


def test_autotune_picks_valid_shapes(film, ctx):
    ctx.upload(film)
    probe = film.render_desc(seed=5, samples=1)
    keep = ctx.tuning()
    try:
        t = ctx.autotune(probe)
        print(f"autotune: trace {t.trace_block}, shade {t.shade_block}, grid x{t.grid_scale}, "
              f"max pixels {t.max_pixels}")
        assert t.trace_block in (64, 128, 256) and t.shade_block in (64, 128, 256) and t.grid_scale in (1, 2)
        assert t.max_pixels > 1 << 20
        cur = ctx.tuning()
        assert (cur.trace_block, cur.shade_block, cur.grid_scale) == (t.trace_block, t.shade_block, t.grid_scale)
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels)


def test_batch_of_mesh_views_equals_single_renders(scene_dir, ctx):
    """The batched workload's shape: random camera poses around the Perlin-displaced
    sphere mesh (here 20,480 triangles; the workload's mesh has 1,048,576), checker
    texture and Perlin sky, each view bit for bit its single render."""
    sc = scenes.perlin_sphere(scene_dir, 32, 32, 4, levels=5, name="b_mesh.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    descs = scenes.random_pose_jobs(scene, 6, seed=4, resolutions=(16, 24, 40), spps=(1, 4, 9), depth=(4, 24),
                                    target=(0.0, 0.0, 0.0), distance=(2.6, 4.0), height=(-1.0, 1.5), jitter=0.2)
    imgs = ctx.render_batch(descs)
    for d, img in zip(descs, imgs):
        assert img.mean() > 0
        assert _same(img, ctx.render(d)), f"job {d.settings.width}x{d.settings.height} spp {d.settings.samples}"


def test_autotune_batch(film, ctx):
    """The batch autotuner times batched renders of the probe views, installs a valid
    choice, and launch shapes change no image."""
    ctx.upload(film)
    descs = _jobs(film, n=4, seed=8)
    keep = ctx.tuning()
    want = ctx.render_batch(descs)
    try:
        t = ctx.autotune_batch(descs)
        assert t.trace_block in (64, 128, 256) and t.shade_block in (64, 128, 256)
        assert t.grid_scale in (1, 2) and t.bvh_width in (2, 4, 8) and t.max_pixels > 0
        got = ctx.tuning()
        assert (got.trace_block, got.shade_block, got.grid_scale, got.bvh_width) == \
            (t.trace_block, t.shade_block, t.grid_scale, t.bvh_width)
        for w, g in zip(want, ctx.render_batch(descs)):
            assert _same(w, g)
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width)
