"""Host side (no GPU): the .lrd/.obj parser, BVH build and light list against the
reference's own containers, parse errors, and the PPM writer."""

import hashlib
import os

import numpy as np
import pytest

import lambda_b200 as lb
from oracle import ref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SCN = os.path.join(GOLDEN, "scenes")
NAMES = ["cornell", "thinfilm", "thinfilm_deep", "mesh", "instanced"]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "golden.npz"))


def _parse(name):
    cwd = os.getcwd()
    os.chdir(SCN)  # mesh paths in the fixtures are relative to the scene directory
    try:
        return lb.HostScene.parse(f"{name}.lrd")
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("name", NAMES)
def test_containers_match_reference(name, golden):
    s = _parse(name)
    for c in ("objects", "instances", "nodes"):
        raw = s.raw(c)
        if c == "objects":
            # compare the bytes the object type uses; the reference leaves the rest of its union unset
            types = raw[:, :4].copy().view(np.int32).ravel()
            used = {0: 24, 1: 56, 2: 116}
            ref_raw = None
            if ref.available():
                cwd = os.getcwd()
                os.chdir(SCN)
                try:
                    ref_raw = ref.RefScene(f"{name}.lrd").raw("objects")
                finally:
                    os.chdir(cwd)
                for i, t in enumerate(types):
                    assert (raw[i, :used[int(t)]] == ref_raw[i, :used[int(t)]]).all(), f"object {i}"
            if (types == 2).all():
                assert hashlib.sha256(raw.tobytes()).hexdigest() == str(golden[f"{name}/sha_objects"])
        else:
            assert hashlib.sha256(raw.tobytes()).hexdigest() == str(golden[f"{name}/sha_{c}"]), c
    assert (s.light_powers.view(np.uint32) == golden[f"{name}/light_powers"].view(np.uint32)).all()
    assert np.float32(s.total_light_power) == golden[f"{name}/total_light_power"]
    assert (s.spectra == golden[f"{name}/spectra"]).all()


def test_parse_error_messages(golden, tmp_path):
    from tests.golden.make_golden import ERROR_CASES

    msgs = golden["parse_errors/messages"]
    assert len(msgs) == len(ERROR_CASES)
    for i, text in enumerate(ERROR_CASES):
        p = tmp_path / f"case{i}.lrd"
        p.write_text(text)
        try:
            lb.HostScene.parse(str(p))
            got = ""
        except lb.LambdaError as e:
            got = e.message.replace(str(p), "<file>")
            assert e.status in (2, 3)
        assert got == str(msgs[i]), f"case {i}: {text!r}"


def test_missing_file():
    with pytest.raises(lb.LambdaError) as e:
        lb.HostScene.parse("/nonexistent/scene.lrd")
    assert e.value.status == 3
    assert "failed to open file (no such file or directory)" in e.value.message


def test_ppm_writer_matches_reference(golden, tmp_path):
    img = golden["ppm/image"]
    p = tmp_path / "out.ppm"
    lb.write_ppm(str(p), img)
    assert p.read_bytes() == golden["ppm/bytes"].tobytes()


def test_ppm_writer_rejects_extension(tmp_path):
    with pytest.raises(lb.LambdaError) as e:
        lb.write_ppm(str(tmp_path / "out.png"), np.zeros((2, 2, 3), np.float32))
    assert e.value.message == ": invalid file extension"


def test_scene_generators_are_deterministic(tmp_path):
    from lambda_b200 import scenes

    a = scenes.thinfilm_spheres(str(tmp_path), 64, 36, 4, name="a.lrd")
    b = scenes.thinfilm_spheres(str(tmp_path), 64, 36, 4, name="b.lrd")
    assert open(a.lrd).read() == open(b.lrd).read()
    n = scenes.write_perlin_sphere_obj(str(tmp_path / "s.obj"), levels=3)
    assert n == 4 * 4 ** 3


OBJ_HEAD = ("Render 8 8 1 1 380 780\nMaterial m lambertian 0.5\nObject o mesh m {obj}\n"
            "Instance o default (0 0 0) (0 0 0) (1 1 1)\nBackground equirectangular 0\n"
            "Camera (0 0 -3) (-0.5 0.5 -2) (1 0 0) (0 -1 0)\n")
OBJ_CASES = [
    # lines the fast reader takes, and lines it leaves to the stream reader (face
    # index 0, which the reference reads before its first vertex, is rejected here)
    "v 1. .5 -0\nv 1e-3 2E+2 3\nv 0.25 -1.5e1 2\nf 1 2 3\n",
    "v +1 2 3\nv 0 1 0\nv 0 0 1\nvt 0.5 0.25\nvn 0 0 1\nf 1/1/1 2/1/1 3/1/1\nf -3 -2 -1\n",
    "# comment\r\nv 0 0 0\r\nv 1 0 0 \r\nv 0 1 0\r\no name\r\ng grp\r\nf 1 2 3",
    "v 1e-40 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 4 3\nf 1  2\t3\n",
    "v inf 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "v 0 0 0 1\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n",
    "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n",
    "v 1 2\n",
]


@pytest.mark.skipif(not ref.available(), reason="reference harness not built")
def test_obj_reader_matches_reference(tmp_path):
    """OBJ lines on both reading paths give the reference's triangles byte for
    byte, or its error message."""
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        for i, obj in enumerate(OBJ_CASES):
            (tmp_path / f"m{i}.obj").write_bytes(obj.encode())
            lrd = tmp_path / f"s{i}.lrd"
            lrd.write_text(OBJ_HEAD.format(obj=f"m{i}.obj"))
            try:
                want = ref.RefScene(lrd.name).raw("objects")
                want_err = ""
            except ref.RefError as e:
                want, want_err = None, str(e)
            try:
                got = lb.HostScene.parse(lrd.name).raw("objects")
                got_err = ""
            except lb.LambdaError as e:
                got, got_err = None, e.message
            assert got_err == want_err, f"case {i}"
            if want is not None:
                assert got.shape == want.shape and (got == want).all(), f"case {i}"
    finally:
        os.chdir(cwd)


@pytest.mark.skipif(not ref.available(), reason="reference harness not built")
def test_instanced_light_list_matches_reference(tmp_path):
    """A scene of many instances: the background light's power comes from the
    scene-sphere merge, which passes over instances whose world box shows they change
    nothing. The light list and its powers equal the reference's bit for bit, as do
    the reordered instances and the nodes."""
    from lambda_b200 import scenes

    sc = scenes.instanced_meshes(str(tmp_path), 32, 18, 1, instances=300, segments=24, rings=13, box=30.0)
    s = lb.HostScene.parse(sc.lrd)
    r = ref.RefScene(sc.lrd)
    assert (s.light_instances == r.light_instances).all() and (s.light_objects == r.light_objects).all()
    assert (s.light_powers.view(np.uint32) == r.light_powers.view(np.uint32)).all()
    assert np.float32(s.total_light_power) == np.float32(r.total_light_power)
    assert (s.raw("instances") == r.raw("instances")).all()
    assert (s.raw("nodes") == r.raw("nodes")).all()
