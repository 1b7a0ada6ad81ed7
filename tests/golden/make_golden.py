"""Generates the golden fixtures in this directory from the reference renderer's
own CPU code (oracle/_ref/libref_lambda.so, built from the reference sources by
oracle/Makefile). Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py

Fixtures (small, committed):
  scenes/*.lrd, scenes/*.obj       the scene files the vectors were made from
  golden.npz                       images, hit ids, shadow flags, thin-film R, noise,
                                   PCG draws, parsed containers (hashes) and PPM bytes
"""

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lambda_b200 import scenes  # noqa: E402
from oracle import ref  # noqa: E402

SCN = os.path.join(HERE, "scenes")


_OK_TAIL = "Instance box default (0 0 0) (0 0 0) (1 1 1)\nBackground equirectangular 0\nCamera (0 0 -3) (-0.5 0.5 -2) (1 0 0) (0 -1 0)\n"
_OK_HEAD = "Render 8 8 2 4 380 780\n"
_OK_OBJ = "Object box quad default (-1 -1 1) (2 0 0) (0 2 0)\n"
# Malformed inputs; each line of the scene language gets at least one.
ERROR_CASES = [
    "Texture t scalar constant 1\n",
    "Render 0 8 2 4 380 780\n",
    "Render 8 8 2 5 380 780\n",
    "Render 8 8 2 4 300 780\n",
    "Render 8 8 2 4 380 900\n",
    "Render 8 8 2 4 700 600\n",
    "Render 8 8 -1 4 380 780\n",
    "Render 8 8 2 4 380\n",
    _OK_HEAD + "Texture t scalar worley 5 1 3\n",
    _OK_HEAD + "Texture t scalar bogus 1\n",
    _OK_HEAD + "Texture t spectrum scalar default\n",
    _OK_HEAD + "Texture t spectrum constant (360 0.5 900 0.5)\n",
    _OK_HEAD + "Texture t spectrum checker 0.5\n",
    _OK_HEAD + "Texture default scalar constant 1\n",
    _OK_HEAD + "Material m lambertian 1.5\n",
    _OK_HEAD + "Material m lambertian nosuchtex\n",
    _OK_HEAD + "Material m dielectric 1.0 -1.5\n",
    _OK_HEAD + "Material m thinfilm [1 1.33 1.5] [a b]\n",
    _OK_HEAD + "Material m thinfilm [1] []\n",
    _OK_HEAD + "Material m thinfilm [1 1.33 1.5] [nosuch]\n",
    _OK_HEAD + "Material m thinfilm [1 1.33+0.1i 1.5-i] [300]\n" + _OK_OBJ + _OK_TAIL,
    _OK_HEAD + "Material m glass 1\n",
    _OK_HEAD + "Object box sphere default (0 0 0) -1\n",
    _OK_HEAD + "Object box quad default (0 0 0) (1 0 0) (2 0 0)\n",
    _OK_HEAD + "Object box quad nomat (0 0 0) (1 0 0) (0 1 0)\n",
    _OK_HEAD + "Object default quad default (0 0 0) (1 0 0) (0 1 0)\n",
    _OK_HEAD + "Object box cone default\n",
    _OK_HEAD + "Object box mesh default /nonexistent/file.obj\n",
    _OK_HEAD + _OK_OBJ + "Object b2 quad default (0 0 0) (1 0 0) (0 1 0)\n" + "Object box quad default (0 0 0) (1 0 0) (0 1 0)\n",
    _OK_HEAD + _OK_OBJ + "Instance nobox default (0 0 0) (0 0 0) (1 1 1)\n",
    _OK_HEAD + _OK_OBJ + "Instance box default (0 0 0) (0 0 0) (1 0 1)\n",
    _OK_HEAD + "Material e emissive 5\nObject l quad e (0 0 0) (1 0 0) (0 1 0)\nInstance l default (0 0 0) (0 0 0) (1 2 1)\n",
    _OK_HEAD + _OK_OBJ + "Instance box default (0 0 0) (0 0 0) (1 1 1) extra\n",
    _OK_HEAD + "Background sphere 0\n",
    _OK_HEAD + "Camera (0 0 0) (0 0 0) (0 0 0) (0 1 0)\n",
    _OK_HEAD + "Frobnicate\n",
    _OK_HEAD + _OK_OBJ + "Instance box default (0 0 0) (0 0 0) (1 1 1)\nCamera (0 0 -3) (-0.5 0.5 -2) (1 0 0) (0 -1 0)\n",
    _OK_HEAD + _OK_OBJ + "Background equirectangular 0\nCamera (0 0 -3) (-0.5 0.5 -2) (1 0 0) (0 -1 0)\n",
    _OK_HEAD + _OK_OBJ + _OK_TAIL,
    _OK_HEAD + "# comment only\n" + _OK_OBJ + "Instance box default (0,0,0) (0 0 0) (1 1 1) # trailing\n" + _OK_TAIL,
]


def scene_files():
    os.makedirs(SCN, exist_ok=True)
    cwd = os.getcwd()
    os.chdir(SCN)  # .obj paths in the .lrd are written relative to this directory
    try:
        out = {
            "cornell": scenes.cornell(".", 24, 24, 4, name="cornell.lrd"),
            "thinfilm": scenes.thinfilm_spheres(".", 32, 18, 4, name="thinfilm.lrd"),
            "thinfilm_deep": scenes.thinfilm_spheres(".", 24, 14, 9, depth=24, name="thinfilm_deep.lrd"),
            "mesh": scenes.perlin_sphere(".", 24, 24, 4, levels=4, name="mesh.lrd"),
            "instanced": scenes.instanced_meshes(".", 24, 16, 4, depth=6, instances=40, segments=12, rings=7,
                                                 box=10.0, name="instanced.lrd"),
        }
    finally:
        os.chdir(cwd)
    return out


def rays_for(r: "ref.RefScene", n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    nodes = r.raw("nodes")
    lo = nodes[0, 0:12].view(np.float32)
    hi = nodes[0, 12:24].view(np.float32)
    c, e = (lo + hi) / 2, (hi - lo) / 2
    o = rng.uniform(c - e, c + e, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    files = scene_files()
    g = {}
    cwd = os.getcwd()
    os.chdir(SCN)
    try:
        for name, sc in files.items():
            r = ref.RefScene(os.path.basename(sc.lrd))
            img, _ = r.render(sc.seed, threads=1)
            g[f"{name}/image"] = img
            g[f"{name}/seed"] = np.array(sc.seed)
            rays = rays_for(r, 3000, 17)
            inst, obj, t, _, _ = r.hit(rays)
            g[f"{name}/rays"] = rays
            g[f"{name}/hit_instance"] = inst
            g[f"{name}/hit_object"] = obj
            g[f"{name}/hit_t"] = t
            li, lo = r.light_instances, r.light_objects
            pick = np.random.default_rng(5).integers(0, len(li), size=rays.shape[0])
            g[f"{name}/shadow_li"] = li[pick]
            g[f"{name}/shadow_lo"] = lo[pick]
            g[f"{name}/shadow"] = r.shadow(rays, li[pick], lo[pick])
            for c in ("objects", "instances", "nodes"):
                g[f"{name}/sha_{c}"] = np.array(digest(r.raw(c)))
            g[f"{name}/light_powers"] = r.light_powers
            g[f"{name}/total_light_power"] = np.array(r.total_light_power, np.float32)
            g[f"{name}/spectra"] = r.spectra
    finally:
        os.chdir(cwd)
    rng = np.random.default_rng(2)
    q = rng.uniform([380, 0, 150, 1.2, 1.0], [780, 1, 850, 1.8, 2.0], (400, 5)).astype(np.float32)
    g["film/query"] = q
    g["film/rs_rp"] = np.array([ref.tmm_single(*map(float, row)) for row in q])
    pts = np.random.default_rng(3).uniform(-20, 20, (1000, 3)).astype(np.float32)
    g["noise/points"] = pts
    g["noise/perlin"] = np.array([ref.perlin(p) for p in pts], np.float32)
    g["noise/worley"] = np.array([ref.worley(p) for p in pts], np.float32)
    g["pcg/draws"] = np.stack([ref.pcg(42, s, 64) for s in (0, 1, 12345, 2**40 + 7)])
    img = np.random.default_rng(4).uniform(-0.2, 1.3, (7, 5, 3)).astype(np.float32)
    path = os.path.join(HERE, "_tmp.ppm")
    ref.write_ppm(path, img)
    with open(path, "rb") as f:
        g["ppm/bytes"] = np.frombuffer(f.read(), np.uint8)
    os.unlink(path)
    g["ppm/image"] = img
    # parser error messages for malformed scenes (file names stripped)
    msgs = []
    for i, text in enumerate(ERROR_CASES):
        path = os.path.join(HERE, f"_err{i}.lrd")
        with open(path, "w") as f:
            f.write(text)
        try:
            ref.RefScene(path)
            msgs.append("")
        except ref.RefError as e:
            msgs.append(str(e).replace(path, "<file>"))
        os.unlink(path)
    g["parse_errors/messages"] = np.array(msgs)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **g)
    print("wrote", len(g), "arrays")


if __name__ == "__main__":
    main()
