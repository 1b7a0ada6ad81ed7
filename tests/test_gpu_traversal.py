"""Hit ids and t of a seeded ray set: GPU traversal vs the reference's Scene::hit
(src/scene/scene.h:51-124), bit for bit."""

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import scenes
from oracle import port, ref
from tests.helpers import camera_rays, random_rays

pytestmark = pytest.mark.gpu

SCENES = {
    "cornell": lambda d: scenes.cornell(d, 32, 32, 4),
    "thinfilm": lambda d: scenes.thinfilm_spheres(d, 64, 36, 4),
    "mesh": lambda d: scenes.perlin_sphere(d, 64, 64, 4, levels=5),
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


def _oracle_hit(sc, scene, rays):
    if ref.available():
        r_inst, r_obj, r_t, _, _ = ref.RefScene(sc.lrd).hit(rays)
        return r_inst, r_obj, r_t
    return port.hit(scene, rays)


def test_closest_hit_ids_bit_exact(loaded, ctx):
    name, sc, scene = loaded
    ctx.upload(scene)
    rays = _ray_set(scene)
    inst, obj, t = ctx.trace_closest(rays)
    r_inst, r_obj, r_t = _oracle_hit(sc, scene, rays)
    assert (inst == r_inst).all(), f"{name}: instance ids differ at {np.flatnonzero(inst != r_inst)[:10]}"
    assert (obj == r_obj).all(), f"{name}: object ids differ at {np.flatnonzero(obj != r_obj)[:10]}"
    assert (t.view(np.uint32) == r_t.view(np.uint32)).all(), f"{name}: t differs"
    assert (inst >= 0).mean() > 0.2


def test_shadow_bit_exact(loaded, ctx):
    name, sc, scene = loaded
    ctx.upload(scene)
    rays = _ray_set(scene, 10000)
    li_all, lo_all = scene.light_instances, scene.light_objects
    pick = np.random.default_rng(5).integers(0, len(li_all), size=rays.shape[0])
    li, lo = li_all[pick], lo_all[pick]
    occ = ctx.trace_shadow(rays, li, lo)
    r_occ = ref.RefScene(sc.lrd).shadow(rays, li, lo) if ref.available() else port.shadow(scene, rays, li, lo)
    assert (occ == r_occ).all(), f"{name}: occlusion differs at {np.flatnonzero(occ != r_occ)[:10]}"


def test_empty_query(loaded, ctx):
    inst, obj, t = ctx.trace_closest(np.zeros((0, 6), np.float32))
    assert inst.shape == (0,)
