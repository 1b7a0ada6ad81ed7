"""The path kernel of small passes (one thread runs every sample and bounce of its
pixel) against the wavefront: the same images bit for bit, the same statistics, on
every scene family and thin-film mode it runs, alone and in batches; surrogate
renders keep the wavefront."""

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import _native as N
from lambda_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {
    "cornell": lambda d: scenes.cornell(d, 48, 48, 16, name="p_cornell.lrd"),
    "thinfilm": lambda d: scenes.thinfilm_spheres(d, 96, 54, 16, name="p_thinfilm.lrd"),
    "thinfilm_deep": lambda d: scenes.thinfilm_spheres(d, 64, 36, 4, depth=24, name="p_thinfilm_deep.lrd"),
    "mesh": lambda d: scenes.perlin_sphere(d, 48, 48, 4, levels=5, name="p_mesh.lrd"),
    "instanced": lambda d: scenes.instanced_meshes(d, 64, 40, 9, depth=8, instances=120, segments=16, rings=9,
                                                   box=14.0, name="p_instanced.lrd"),
}


def _stats(ctx):
    st = ctx.stats()
    return (st.paths, st.segments, st.shadow_rays, st.thinfilm_hits, st.thinfilm_fallback)


def _render_both(ctx, desc, width=4):
    """(wavefront image, stats, path-kernel image, stats) of one render description."""
    keep = ctx.tuning()
    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, width, 0)
        wave = ctx.render(desc)
        wave_stats = _stats(ctx)
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, width, 1 << 30)
        path = ctx.render(desc)
        path_stats = _stats(ctx)
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)
    return wave, wave_stats, path, path_stats


@pytest.mark.parametrize("case", sorted(CASES))
def test_path_kernel_equals_wavefront(case, scene_dir, ctx):
    sc = CASES[case](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    for width in (2, 4, 8):
        wave, ws, path, ps = _render_both(ctx, scene.render_desc(seed=sc.seed), width)
        assert np.array_equal(path, wave, equal_nan=True), f"{case} width {width}: images differ"
        assert ps == ws, f"{case} width {width}: statistics {ps} vs {ws}"
    print(f"{case}: paths {ps[0]}, segments {ps[1]}, shadow rays {ps[2]}, thin-film hits {ps[3]}")


def test_path_kernel_fp64_thin_film(scene_dir, ctx):
    sc = CASES["thinfilm"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    wave, ws, path, ps = _render_both(ctx, scene.render_desc(seed=2, flags=lb.RENDER_THINFILM_FP64))
    assert np.array_equal(path, wave, equal_nan=True)
    assert ps == ws and ps[3] > 0


def test_path_kernel_runs_and_is_profiled(scene_dir, ctx):
    """Below the threshold a render is one persistent launch of the path kernel (it
    seeds, traces and finishes every pixel); the stage profile names the path kernel
    and counts its segments; above it the wavefront runs."""
    sc = CASES["cornell"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       48 * 48)
        ctx.render(scene.render_desc(seed=1))
        assert ctx.stats().kernel_launches == 1
        ctx.render(scene.render_desc(seed=1, flags=N.RENDER_PROFILE_STAGES))
        st = ctx.stage_times()
        assert st["path"]["launches"] == 1 and st["intersect"]["launches"] == 0
        assert st["path"]["items"] == ctx.stats().segments > 0
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       48 * 48 - 1)
        ctx.render(scene.render_desc(seed=1))
        assert ctx.stats().kernel_launches > 1
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)


def test_path_kernel_batch_equals_single_renders(scene_dir, ctx):
    """A batch of uneven jobs (sizes, sample counts, depths) in one persistent
    path-kernel launch: each image equals its job rendered alone by the wavefront,
    and the progress counter ends at the batch's pixel count."""
    sc = CASES["thinfilm"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    descs = scenes.random_pose_jobs(scene, 7, seed=4, resolutions=(16, 24, 40), spps=(1, 4, 9, 16), depth=(2, 24))
    descs[1].settings.lambda_min, descs[1].settings.lambda_max = 400.0, 700.0
    keep = ctx.tuning()
    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width, 0)
        alone = [ctx.render(d) for d in descs]
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       1 << 30)
        import ctypes

        done = ctypes.c_int32(0)
        batch = ctx.render_batch(descs, completed=ctypes.pointer(done))
        assert ctx.stats().kernel_launches == 1
        assert done.value == sum(d.settings.width * d.settings.height for d in descs)
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)
    for a, b in zip(alone, batch):
        assert np.array_equal(a, b, equal_nan=True)


def test_surrogate_keeps_the_wavefront(scene_dir, ctx):
    from lambda_b200 import surrogate

    surrogate.install(ctx)
    sc = CASES["thinfilm"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       1 << 30)
        ctx.render(scene.render_desc(seed=1, flags=lb.RENDER_THINFILM_SURROGATE | N.RENDER_PROFILE_STAGES))
        st = ctx.stage_times()
        assert st["path"]["launches"] == 0 and st["film_mlp"]["launches"] > 0
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)


def test_surrogate_flag_without_thin_films_takes_the_path_kernel(scene_dir, ctx):
    """On a scene without thin films the surrogate flag changes nothing, so such a
    pass may run the path kernel: the image equals the exact wavefront render."""
    from lambda_b200 import surrogate

    surrogate.install(ctx)
    sc = CASES["mesh"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width, 0)
        want = ctx.render(scene.render_desc(seed=3))
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       1 << 30)
        got = ctx.render(scene.render_desc(seed=3, flags=lb.RENDER_THINFILM_SURROGATE))
        assert ctx.stats().kernel_launches == 1
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)
    assert np.array_equal(got, want, equal_nan=True)


def test_autotune_sets_the_path_kernel_threshold(scene_dir, ctx):
    """A winning path kernel covers the probe (and at least the default threshold); a
    winning wavefront keeps the path kernel for passes below both the probe and the
    default. Either way the probe's frame renders as the tuned form."""
    sc = CASES["mesh"](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    try:
        probe = scene.render_desc(seed=sc.seed)
        pixels = sc.width * sc.height
        t = ctx.autotune(probe)
        assert t.path_kernel_pixels in (max(N.PATH_KERNEL_PIXELS, pixels), min(N.PATH_KERNEL_PIXELS, pixels - 1))
        ctx.render(probe)
        path_won = t.path_kernel_pixels >= pixels
        assert (ctx.stats().kernel_launches == 1) == path_won
        print(f"autotuned on {pixels} pixels: {'path kernel' if path_won else 'wavefront'}, "
              f"threshold {t.path_kernel_pixels}")
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)


@pytest.mark.parametrize("path_kernel", [False, True])
def test_progress_rises_while_rendering(scene_dir, ctx, path_kernel):
    """The caller's `completed` counter (main.cpp's progress poll) rises while a render
    runs and never falls, for a wavefront pass (waves the graph has started) and for
    one persistent path-kernel launch (pixels its warps have finished); it ends at
    the pixel count."""
    import ctypes
    import threading
    import time

    sc = scenes.thinfilm_spheres(scene_dir, 960, 540, 64, name="p_progress.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    keep = ctx.tuning()
    done = ctypes.c_int32(0)
    seen = []
    stop = threading.Event()

    def watch():
        while not stop.is_set():
            seen.append(done.value)
            time.sleep(0.0002)

    try:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       1 << 30 if path_kernel else 0)
        t = threading.Thread(target=watch)
        t.start()
        try:
            ctx.render(scene.render_desc(seed=sc.seed), completed=ctypes.pointer(done))
        finally:
            stop.set()
            t.join()
        assert (ctx.stats().kernel_launches == 1) == path_kernel
    finally:
        ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                       keep.path_kernel_pixels)
    seen.append(done.value)
    assert all(a <= b for a, b in zip(seen, seen[1:])), "progress fell"
    assert seen[-1] == 960 * 540
    inner = sorted(set(v for v in seen if 0 < v < 960 * 540))
    print(f"{'path kernel' if path_kernel else 'wavefront'}: {len(inner)} intermediate progress values")
    assert len(inner) >= 2
