"""The CPU oracle (oracle/lambda_oracle.c) pinned against golden vectors made by
the reference renderer's own CPU code (tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

import lambda_b200 as lb
from oracle import port, ref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SCN = os.path.join(GOLDEN, "scenes")
NAMES = ["cornell", "thinfilm", "thinfilm_deep", "mesh", "instanced"]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "golden.npz"))


def _parse(name):
    cwd = os.getcwd()
    os.chdir(SCN)
    try:
        return lb.HostScene.parse(f"{name}.lrd")
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("name", NAMES)
def test_render_bit_exact(name, golden):
    s = _parse(name)
    img = port.render(s, int(golden[f"{name}/seed"]))
    want = golden[f"{name}/image"]
    assert (img.view(np.uint32) == want.view(np.uint32)).all()


@pytest.mark.parametrize("name", NAMES)
def test_hits_bit_exact(name, golden):
    s = _parse(name)
    rays = golden[f"{name}/rays"]
    inst, obj, t = port.hit(s, rays)
    assert (inst == golden[f"{name}/hit_instance"]).all()
    assert (obj == golden[f"{name}/hit_object"]).all()
    assert (t.view(np.uint32) == golden[f"{name}/hit_t"].view(np.uint32)).all()
    occ = port.shadow(s, rays, golden[f"{name}/shadow_li"], golden[f"{name}/shadow_lo"])
    assert (occ == golden[f"{name}/shadow"]).all()


def test_film_against_reference_helpers(golden):
    q = golden["film/query"]
    out = port.film(q)
    assert np.abs(out[:, :2] - golden["film/rs_rp"]).max() == 0.0
    # lossless stack: R + T = 1 per polarisation
    assert np.abs(out[:, 0] + out[:, 2] - 1).max() < 1e-12
    assert np.abs(out[:, 1] + out[:, 3] - 1).max() < 1e-12


def test_noise_bit_exact(golden):
    pts = golden["noise/points"]
    per = np.array([port.perlin(p) for p in pts], np.float32)
    wor = np.array([port.worley(p) for p in pts], np.float32)
    assert (per == golden["noise/perlin"]).all()
    assert (wor == golden["noise/worley"]).all()


def test_pcg(golden):
    got = np.stack([port.pcg(42, s, 64) for s in (0, 1, 12345, 2**40 + 7)])
    assert (got == golden["pcg/draws"]).all()


def test_film_known_answers():
    # normal incidence, film index equal to the substrate: one interface
    n = np.float32(1.5)
    q = np.array([[550, 1, 300, n, n]], np.float32)
    r = port.film(q)[0]
    want = ((1 - float(n)) / (1 + float(n))) ** 2
    assert abs(r[0] - want) < 1e-15 and abs(r[1] - want) < 1e-15
    # quarter-wave antireflection coating
    nf = np.float32(np.sqrt(1.69))
    q = np.array([[550, 1, np.float32(550 / (4 * float(nf))), nf, 1.69]], np.float32)
    assert port.film(q)[0, 0] < 1e-6


def test_oracle_matches_live_reference(tmp_path):
    """When the compiled reference is present, a fresh scene renders identically."""
    if not ref.available():
        pytest.skip("reference harness not built")
    from lambda_b200 import scenes

    sc = scenes.thinfilm_spheres(str(tmp_path), 20, 12, 4, name="live.lrd")
    s = lb.HostScene.parse(sc.lrd)
    a = port.render(s, 77)
    b, _ = ref.RefScene(sc.lrd).render(77, threads=2)
    assert (a.view(np.uint32) == b.view(np.uint32)).all()


def test_mlp_gradient_finite_difference():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, 8964)
    x = rng.uniform(-1, 1, (16, 5))
    t = rng.uniform(0, 1, (16, 4))
    loss, g = port.mlp_grad(p, x, t)
    for k in rng.integers(0, 8964, 40):
        e = np.zeros_like(p)
        e[k] = 1e-6
        lp, _ = port.mlp_grad(p + e, x, t)
        lm, _ = port.mlp_grad(p - e, x, t)
        assert abs((lp - lm) / 2e-6 - g[k]) < 1e-6 * max(1, abs(g[k]))
