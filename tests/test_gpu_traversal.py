"""Hit ids and t of a seeded ray set: GPU traversal vs the reference's Scene::hit
(src/scene/scene.h:51-124), bit for bit."""

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import scenes
from oracle import port, ref
from tests.helpers import camera_rays, random_rays, ref_scene

pytestmark = pytest.mark.gpu

SCENES = {
    "cornell": lambda d: scenes.cornell(d, 32, 32, 4),
    "thinfilm": lambda d: scenes.thinfilm_spheres(d, 64, 36, 4),
    "mesh": lambda d: scenes.perlin_sphere(d, 64, 64, 4, levels=5),
    "instanced": lambda d: scenes.instanced_meshes(d, 64, 40, 4, depth=8, instances=300, segments=24, rings=13,
                                                   box=20.0, name="t_instanced.lrd"),
    # the BVH stress configuration at full size: 1,048,576 triangles, tree depth capped at 20
    "mesh_1m": lambda d: scenes.perlin_sphere(d, 64, 64, 4, levels=9, name="t_mesh_1m.lrd"),
}


@pytest.fixture(scope="module", params=sorted(SCENES))
def loaded(request, scene_dir, ctx):
    sc = SCENES[request.param](scene_dir)
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    return request.param, sc, scene


def _ray_set(scene, n=20000):
    nodes = scene.nodes_array()
    lo, hi = nodes["min"][0], nodes["max"][0]
    center = (lo + hi) / 2
    ext = (hi - lo) / 2
    return np.concatenate([random_rays(n, center - ext, center + ext, 11), camera_rays(scene.settings, n, 12)])


def _plane_rays(scene, n=6000, seed=17):
    """Rays that start exactly on BVH node planes with some direction components
    exactly zero: the slab test then meets 0 * inf = NaN bounds, which it ignores.
    Every BVH width must make the reference's decisions on them too."""
    nodes = scene.nodes_array()
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, len(nodes), n)
    lo, hi = nodes["min"][pick].astype(np.float32), nodes["max"][pick].astype(np.float32)
    o = lo + (hi - lo) * rng.uniform(0, 1, (n, 3)).astype(np.float32)
    axis = rng.integers(0, 3, n)
    side = rng.integers(0, 2, n)
    o[np.arange(n), axis] = np.where(side == 0, lo[np.arange(n), axis], hi[np.arange(n), axis])
    d = rng.normal(size=(n, 3)).astype(np.float32)
    zero = rng.integers(0, 3, n)
    d[np.arange(n), axis] = 0.0
    d[np.arange(n) % 3 == 0, zero[np.arange(n) % 3 == 0]] = 0.0
    d[(d == 0).all(axis=1), 1] = 1.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], axis=1).astype(np.float32)


def _oracle_hit(sc, scene, rays):
    if ref.available():
        r_inst, r_obj, r_t, _, _ = ref_scene(sc.lrd).hit(rays)
        return r_inst, r_obj, r_t
    return port.hit(scene, rays)


@pytest.fixture(params=["2", "4", "8", "2c", "4c", "8c"])
def width(request, ctx):
    """BVH width, and "c" for the compressed node records."""
    keep = ctx.tuning()
    w, compressed = int(request.param[0]), int(request.param.endswith("c"))
    ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, w,
                   keep.path_kernel_pixels, keep.lane_fetch, compressed)
    yield request.param
    ctx.set_tuning(keep.trace_block, keep.shade_block, keep.grid_scale, keep.max_pixels, keep.bvh_width,
                   keep.path_kernel_pixels, keep.lane_fetch, keep.compressed_nodes)


def test_closest_hit_ids_bit_exact(loaded, width, ctx):
    name, sc, scene = loaded
    ctx.upload(scene)
    rays = np.concatenate([_ray_set(scene), _plane_rays(scene)])
    inst, obj, t = ctx.trace_closest(rays)
    r_inst, r_obj, r_t = _oracle_hit(sc, scene, rays)
    assert (inst == r_inst).all(), f"{name}/{width}: instance ids differ at {np.flatnonzero(inst != r_inst)[:10]}"
    assert (obj == r_obj).all(), f"{name}/{width}: object ids differ at {np.flatnonzero(obj != r_obj)[:10]}"
    assert (t.view(np.uint32) == r_t.view(np.uint32)).all(), f"{name}/{width}: t differs"
    assert (inst >= 0).mean() > 0.2


def test_shadow_bit_exact(loaded, width, ctx):
    name, sc, scene = loaded
    ctx.upload(scene)
    rays = np.concatenate([_ray_set(scene, 10000), _plane_rays(scene, 3000, 23)])
    li_all, lo_all = scene.light_instances, scene.light_objects
    pick = np.random.default_rng(5).integers(0, len(li_all), size=rays.shape[0])
    li, lo = li_all[pick], lo_all[pick]
    occ = ctx.trace_shadow(rays, li, lo)
    r_occ = ref_scene(sc.lrd).shadow(rays, li, lo) if ref.available() else port.shadow(scene, rays, li, lo)
    assert (occ == r_occ).all(), f"{name}/{width}: occlusion differs at {np.flatnonzero(occ != r_occ)[:10]}"


def test_empty_query(loaded, ctx):
    inst, obj, t = ctx.trace_closest(np.zeros((0, 6), np.float32))
    assert inst.shape == (0,)
