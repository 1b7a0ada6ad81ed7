"""The scene build on the GPU (lambda_parse_lrd_gpu) against the host build: the
same objects, instances, BVH nodes and light list, byte for byte, on every scene
family, with every build range sent to the GPU; and the large scenes' build times."""

import os
import time

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "scenes")


def _same(a, b):
    for c in ("objects", "instances", "nodes", "materials"):
        ra, rb = a.raw(c), b.raw(c)
        assert ra.shape == rb.shape, c
        if c == "nodes":
            bad = np.nonzero((ra != rb).any(axis=1))[0]
            assert bad.size == 0, f"{bad.size} nodes differ, first {bad[:5]}"
        assert (ra == rb).all(), c
    assert (a.light_instances == b.light_instances).all() and (a.light_objects == b.light_objects).all()
    assert (a.light_powers.view(np.uint32) == b.light_powers.view(np.uint32)).all()
    assert np.float32(a.total_light_power) == np.float32(b.total_light_power)


@pytest.mark.parametrize("name", ["cornell", "thinfilm", "thinfilm_deep", "mesh", "instanced"])
def test_gpu_build_equals_host_build(name, ctx):
    cwd = os.getcwd()
    os.chdir(GOLDEN)  # mesh paths in the fixtures are relative to the scene directory
    try:
        host = lb.HostScene.parse(f"{name}.lrd")
        gpu = lb.HostScene.parse_gpu(ctx, f"{name}.lrd", gpu_min_items=1)
    finally:
        os.chdir(cwd)
    _same(host, gpu)


def test_gpu_build_many_instances(scene_dir, ctx):
    sc = scenes.instanced_meshes(scene_dir, 32, 18, 1, instances=300, segments=24, rings=13, box=30.0,
                                 name="b_instanced.lrd")
    _same(lb.HostScene.parse(sc.lrd), lb.HostScene.parse_gpu(ctx, sc.lrd, gpu_min_items=1))


def test_gpu_build_million_triangles(scene_dir, ctx):
    """The 1,048,576-triangle mesh: identical node bytes, and the build time of each."""
    sc = scenes.perlin_sphere(scene_dir, 64, 64, 1, levels=9, name="b_mesh_1m.lrd")
    lb.HostScene.parse_gpu(ctx, sc.lrd)  # warm-up (module load, allocations)
    t0 = time.perf_counter()
    host = lb.HostScene.parse(sc.lrd)
    t1 = time.perf_counter()
    gpu = lb.HostScene.parse_gpu(ctx, sc.lrd)
    t2 = time.perf_counter()
    print(f"1M-triangle mesh: parse + build on the host {t1 - t0:.2f} s, with the GPU build {t2 - t1:.2f} s")
    _same(host, gpu)
