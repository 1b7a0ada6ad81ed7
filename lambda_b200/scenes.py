"""Synthetic scene files (.lrd + .obj) for the benchmark workloads.

The reference ships no scenes; these generators write the workloads the
benchmark names, in the reference's scene language (README.md:19-81), so the
same files drive the reference CPU renderer and this library.

  cornell(...)     256x256, depth 8, 16 spp, 380-780 nm: five 2x2 wall quads,
                   red/green/white Lambertian walls, 0.5x0.5 ceiling light
                   (emission 15), a dielectric (1.0/1.5) and a mirror (0.9)
                   sphere of radius 0.3, pinhole camera at z=-3.
  thinfilm_spheres 1920x1080, depth 16, 256 spp, 380-780 nm: 64 spheres of
                   radius 0.4 on a jittered 8x8 grid (seed 3), thin film
                   n=[1 1.33 1.5] with Worley thickness 200-800 nm at
                   frequency 3, Lambertian ground (0.5), one quad light (10).
  perlin_sphere    1024x1024, depth 12, 64 spp, 360-830 nm: a 9x subdivided
                   tetrahedron (4*4^9 = 1,048,576 triangles) on the unit
                   sphere, radially displaced by Perlin noise (amplitude 0.1,
                   frequency 4, domain offset from seed 2), checker 0.8/0.2 at
                   scale 10, Perlin background 0.2-1.0 at frequency 1.

Every generator takes overrides (resolution, spp, depth) so tests can render
small versions of the same scene.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

__all__ = [
    "SceneFiles",
    "cornell",
    "thinfilm_spheres",
    "perlin_sphere",
    "look_at_camera",
    "random_pose_jobs",
    "instanced_meshes",
]


@dataclass
class SceneFiles:
    lrd: str
    seed: int
    width: int
    height: int
    spp: int
    depth: int


def _v(x) -> str:
    return "(" + " ".join(_f(c) for c in x) + ")"


def _f(c: float) -> str:
    return repr(float(c))


def look_at_camera(position, target, up, vfov_deg: float, aspect: float, plane_distance: float = 1.0):
    """Camera (position, corner, horizontal, vertical) for the .lrd Camera command.

    The reference's pinhole maps u in [0,1] along `horizontal` and v in [0,1]
    along `vertical` from `corner` (camera.h:13-16); v grows downwards, row 0 is
    the top row.
    """
    p = np.asarray(position, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    upv = np.asarray(up, dtype=np.float64)
    w = t - p
    w /= np.linalg.norm(w)
    u = np.cross(w, upv)
    u /= np.linalg.norm(u)
    v = np.cross(u, w)
    half_h = math.tan(math.radians(vfov_deg) / 2) * plane_distance
    half_w = half_h * aspect
    center = p + w * plane_distance
    corner = center - u * half_w + v * half_h
    horizontal = u * (2 * half_w)
    vertical = -v * (2 * half_h)
    return p, corner, horizontal, vertical


def _write(path: str, lines: list[str]) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def cornell(directory: str, width: int = 256, height: int = 256, spp: int = 16, depth: int = 8,
            name: str = "cornell.lrd") -> SceneFiles:
    path = os.path.join(directory, name)
    lines = [
        "# Cornell-style box: five 2x2 walls, ceiling light, dielectric and mirror spheres",
        f"Render {width} {height} {depth} {spp} 380 780",
        "Texture red spectrum constant (360 0.05 599 0.05 600 0.65 830 0.65)",
        "Texture green spectrum constant (360 0.05 499 0.05 500 0.65 570 0.65 571 0.05 830 0.05)",
        "Material white lambertian 0.73",
        "Material red lambertian red",
        "Material green lambertian green",
        "Material light emissive 15",
        "Material glass dielectric 1.0 1.5",
        "Material chrome mirror 0.9",
        "Object box quad white (-1 -1 1) (2 0 0) (0 2 0)",
        "Object box quad white (-1 -1 -1) (2 0 0) (0 0 2)",
        "Object box quad white (-1 1 -1) (0 0 2) (2 0 0)",
        "Object box quad red (-1 -1 -1) (0 0 2) (0 2 0)",
        "Object box quad green (1 -1 -1) (0 2 0) (0 0 2)",
        "Object lamp quad light (-0.25 0.999 -0.25) (0.5 0 0) (0 0 0.5)",
        "Object balls sphere glass (-0.4 -0.7 0.2) 0.3",
        "Object balls sphere chrome (0.4 -0.7 -0.2) 0.3",
        "Instance box default (0 0 0) (0 0 0) (1 1 1)",
        "Instance lamp default (0 0 0) (0 0 0) (1 1 1)",
        "Instance balls default (0 0 0) (0 0 0) (1 1 1)",
        "Background equirectangular 0",
        "Camera (0 0 -3) (-0.5 0.5 -2) (1 0 0) (0 -1 0)",
    ]
    _write(path, lines)
    return SceneFiles(path, 1, width, height, spp, depth)


def thinfilm_spheres(directory: str, width: int = 1920, height: int = 1080, spp: int = 256, depth: int = 16,
                     seed: int = 3, name: str = "thinfilm.lrd", film: str = "thinfilm",
                     background: str = "0", thickness: str = "worley 200 800 3") -> SceneFiles:
    """64 thin-film spheres on a jittered grid. `film` may be "dielectric" to swap
    the film for a plain 1.0/1.5 dielectric (same geometry); `thickness` is the
    film's scalar thickness texture in nm."""
    rng = np.random.default_rng(seed)
    jitter = rng.uniform(-0.1, 0.1, size=(8, 8, 2))
    path = os.path.join(directory, name)
    pos, corner, hor, ver = look_at_camera((0.0, 4.2, -8.5), (0.0, 0.3, 0.6), (0.0, 1.0, 0.0), 40.0,
                                           width / height)
    lines = [
        "# 64 thin-film spheres (r=0.4) on a jittered 8x8 grid, Lambertian ground, one quad light",
        f"Render {width} {height} {depth} {spp} 380 780",
        f"Texture thickness scalar {thickness}",
        "Material ground lambertian 0.5",
        "Material lamp emissive 10",
    ]
    if film == "thinfilm":
        lines.append("Material film thinfilm [1 1.33 1.5] [thickness]")
    elif film == "dielectric":
        lines.append("Material film dielectric 1.0 1.5")
    else:
        raise ValueError(film)
    for i in range(8):
        for j in range(8):
            cx = (i - 3.5) * 1.0 + jitter[i, j, 0]
            cz = (j - 3.5) * 1.0 + jitter[i, j, 1]
            lines.append(f"Object spheres sphere film ({_f(cx)} 0.4 {_f(cz)}) 0.4")
    lines += [
        "Object floor quad ground (-12 0 -12) (0 0 24) (24 0 0)",
        "Object light quad lamp (-1.5 6 -1.5) (3 0 0) (0 0 3)",
        "Instance spheres default (0 0 0) (0 0 0) (1 1 1)",
        "Instance floor default (0 0 0) (0 0 0) (1 1 1)",
        "Instance light default (0 0 0) (0 0 0) (1 1 1)",
        f"Background equirectangular {background}",
        f"Camera {_v(pos)} {_v(corner)} {_v(hor)} {_v(ver)}",
    ]
    _write(path, lines)
    return SceneFiles(path, seed, width, height, spp, depth)


def random_pose_jobs(scene, n: int, seed: int = 4, resolutions=(128, 256, 512, 1024), spps=(1, 4, 16, 64, 256),
                     depth=(4, 24), flags: int = 0, target=(0.0, 0.3, 0.0), distance=(8.0, 11.0),
                     height=(2.5, 6.0), jitter: float = 0.5) -> list:
    """Render descriptors of `n` views of an uploaded scene for a batch: square
    resolutions and sample counts drawn uniformly from the given sets, depth
    uniform in [depth[0], depth[1]], and a camera at a random azimuth, at a
    horizontal distance and height uniform in the given ranges, looking at `target`
    (jittered by up to `jitter` per axis) with a 35-50 degree field of view. The
    defaults frame the thin-film sphere grid. Render seed of job i is seed * 1000 + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        res = int(rng.choice(resolutions))
        spp = int(rng.choice(spps))
        dep = int(rng.integers(depth[0], depth[1] + 1))
        az = rng.uniform(0, 2 * math.pi)
        dist = rng.uniform(*distance)
        h = rng.uniform(*height)
        tgt = np.asarray(target) + rng.uniform(-jitter, jitter, 3)
        pos = (dist * math.sin(az), h, dist * math.cos(az))
        cam = look_at_camera(pos, tgt, (0.0, 1.0, 0.0), rng.uniform(35.0, 50.0), 1.0)
        d = scene.render_desc(seed=seed * 1000 + i, flags=flags)
        st = d.settings
        st.width = st.height = res
        st.depth = dep
        root = int(round(spp ** 0.5))
        st.samples, st.sqrt_samples = spp, root
        for k in range(3):
            st.camera.position[k] = cam[0][k]
            st.camera.corner[k] = cam[1][k]
            st.camera.horizontal[k] = cam[2][k]
            st.camera.vertical[k] = cam[3][k]
        out.append(d)
    return out


# --------------------------------------------------------------------------
# Perlin-displaced sphere mesh
# --------------------------------------------------------------------------

def _subdivided_tetrahedron(levels: int):
    """Vertices on the unit sphere and triangles of a tetrahedron split `levels`
    times (each split makes 4 triangles of 1): 4 * 4**levels triangles."""
    s = 1.0 / math.sqrt(3.0)
    verts = [(s, s, s), (-s, -s, s), (-s, s, -s), (s, -s, -s)]
    tris = np.array([(0, 1, 2), (0, 3, 1), (0, 2, 3), (1, 3, 2)], dtype=np.int64)
    v = np.array(verts, dtype=np.float64)
    for _ in range(levels):
        a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]
        edges = np.concatenate([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mids])
        n = len(tris)
        ab, bc, ca = inv[:n] + base, inv[n:2 * n] + base, inv[2 * n:] + base
        tris = np.concatenate([
            np.stack([a, ab, ca], 1),
            np.stack([ab, b, bc], 1),
            np.stack([ca, bc, c], 1),
            np.stack([ab, bc, ca], 1),
        ])
    return v, tris


# Improved-noise permutation (Perlin 2002), the table the reference's Perlin
# texture uses; lambda_b200/csrc/host/tables.cpp carries the same values.
def _perlin_permutation() -> np.ndarray:
    from ._tables import PERLIN_PERMUTATION
    return np.asarray(PERLIN_PERMUTATION, dtype=np.int64)


def perlin_noise_np(p: np.ndarray) -> np.ndarray:
    """Vectorised improved noise in [0,1] (float64), for mesh displacement only."""
    perm = _perlin_permutation()

    def P(i):
        return perm[np.asarray(i) & 255]

    fl = np.floor(p)
    i, j, k = (fl[:, 0].astype(np.int64) & 255, fl[:, 1].astype(np.int64) & 255, fl[:, 2].astype(np.int64) & 255)
    t = p - fl
    f = t ** 3 * (t * (6 * t - 15) + 10)
    tx, ty, tz = t[:, 0], t[:, 1], t[:, 2]

    def grad(h, x, y, z):
        h = h % 12
        table = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                          [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]], dtype=np.float64)
        g = table[h]
        return g[:, 0] * x + g[:, 1] * y + g[:, 2] * z

    def lerp(a, b, w):
        return a + w * (b - a)

    aaa = P(P(P(i) + j) + k)
    aba = P(P(P(i) + j + 1) + k)
    aab = P(P(P(i) + j) + k + 1)
    abb = P(P(P(i) + j + 1) + k + 1)
    baa = P(P(P(i + 1) + j) + k)
    bba = P(P(P(i + 1) + j + 1) + k)
    bab = P(P(P(i + 1) + j) + k + 1)
    bbb = P(P(P(i + 1) + j + 1) + k + 1)
    x1 = lerp(grad(aaa, tx, ty, tz), grad(baa, tx - 1, ty, tz), f[:, 0])
    x2 = lerp(grad(aba, tx, ty - 1, tz), grad(bba, tx - 1, ty - 1, tz), f[:, 0])
    y1 = lerp(x1, x2, f[:, 1])
    x1 = lerp(grad(aab, tx, ty, tz - 1), grad(bab, tx - 1, ty, tz - 1), f[:, 0])
    x2 = lerp(grad(abb, tx, ty - 1, tz - 1), grad(bbb, tx - 1, ty - 1, tz - 1), f[:, 0])
    y2 = lerp(x1, x2, f[:, 1])
    return (lerp(y1, y2, f[:, 2]) + 1) / 2


def write_perlin_sphere_obj(path: str, levels: int = 9, amplitude: float = 0.1, frequency: float = 4.0,
                            seed: int = 2) -> int:
    """Writes the displaced sphere as an .obj (shared vertices, no normals or uvs);
    returns the triangle count."""
    v, tris = _subdivided_tetrahedron(levels)
    offset = np.random.default_rng(seed).uniform(0, 64, size=3)
    n = perlin_noise_np(v * frequency + offset)
    v = v * (1.0 + amplitude * (2.0 * n - 1.0))[:, None]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(f"# {len(tris)} triangles: {levels}x subdivided tetrahedron, Perlin amplitude {amplitude}\n")
        np.savetxt(f, v, fmt="v %.7g %.7g %.7g")
        np.savetxt(f, tris + 1, fmt="f %d %d %d")
    return len(tris)


def perlin_sphere(directory: str, width: int = 1024, height: int = 1024, spp: int = 64, depth: int = 12,
                  levels: int = 9, seed: int = 2, name: str = "perlin_sphere.lrd") -> SceneFiles:
    obj = os.path.join(directory, f"perlin_sphere_l{levels}.obj")
    if not os.path.exists(obj):
        write_perlin_sphere_obj(obj, levels=levels, seed=seed)
    path = os.path.join(directory, name)
    pos, corner, hor, ver = look_at_camera((0.0, 0.6, -3.2), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 40.0,
                                           width / height)
    lines = [
        "# Perlin-displaced sphere mesh under a Perlin sky",
        f"Render {width} {height} {depth} {spp} 360 830",
        "Texture sky scalar perlin 0.2 1.0 1",
        "Texture tiles spectrum checker 0.8 0.2 10",
        "Material body lambertian tiles",
        f"Object mesh mesh body {obj}",
        "Instance mesh default (0 0 0) (0 0 0) (1 1 1)",
        "Background equirectangular sky",
        f"Camera {_v(pos)} {_v(corner)} {_v(hor)} {_v(ver)}",
    ]
    _write(path, lines)
    return SceneFiles(path, seed, width, height, spp, depth)


# --------------------------------------------------------------------------
# Large instanced scene
# --------------------------------------------------------------------------

def write_latlong_sphere_obj(path: str, segments: int = 250, rings: int = 201, amplitude: float = 0.1,
                             frequency: float = 4.0, seed: int = 5) -> int:
    """A latitude-longitude sphere of 2 * segments * (rings - 1) triangles (fans at
    the poles, two triangles per quad between), radially displaced by Perlin noise
    like the mesh of perlin_sphere; 250 x 201 gives exactly 100,000 triangles.
    Returns the triangle count."""
    th = np.linspace(0.0, math.pi, rings + 1)[1:-1]                 # interior latitudes
    ph = np.linspace(0.0, 2 * math.pi, segments, endpoint=False)
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    ring = np.stack([st * np.cos(ph), np.broadcast_to(ct, (len(th), segments)), st * np.sin(ph)], -1).reshape(-1, 3)
    v = np.concatenate([[[0.0, 1.0, 0.0]], ring, [[0.0, -1.0, 0.0]]])
    top, bottom = 0, len(v) - 1
    idx = lambda r, k: 1 + r * segments + (k % segments)  # noqa: E731
    tris = []
    for k in range(segments):
        tris.append((top, idx(0, k + 1), idx(0, k)))
        tris.append((bottom, idx(rings - 2, k), idx(rings - 2, k + 1)))
    for r in range(rings - 2):
        for k in range(segments):
            a, b, c, d = idx(r, k), idx(r, k + 1), idx(r + 1, k), idx(r + 1, k + 1)
            tris.append((a, b, d))
            tris.append((a, d, c))
    tris = np.asarray(tris, dtype=np.int64)
    offset = np.random.default_rng(seed).uniform(0, 64, size=3)
    n = perlin_noise_np(v * frequency + offset)
    v = v * (1.0 + amplitude * (2.0 * n - 1.0))[:, None]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(f"# {len(tris)} triangles: lat-long sphere {segments}x{rings}, Perlin amplitude {amplitude}\n")
        np.savetxt(f, v, fmt="v %.7g %.7g %.7g")
        np.savetxt(f, tris + 1, fmt="f %d %d %d")
    return len(tris)


def instanced_meshes(directory: str, width: int = 3840, height: int = 2160, spp: int = 1024, depth: int = 32,
                     instances: int = 10000, segments: int = 250, rings: int = 201, box: float = 100.0,
                     seed: int = 5, name: str = "instanced.lrd") -> SceneFiles:
    """`instances` copies of one Perlin-displaced mesh (write_latlong_sphere_obj;
    the defaults give 100,000 triangles and 10,000 instances) with a random
    translation in a box^3 cube, random rotation and uniform scale 0.5-2 (`seed`).
    Materials are set per instance (the Instance material override): 40 % thin film
    [1 1.33 1.5] with Worley thickness 200-800 nm, 30 % dielectric 1.0/1.5, 30 %
    Lambertian checker 0.8/0.2. A Perlin equirectangular sky is the only light. The
    camera stands outside the cube looking at its centre."""
    obj = os.path.join(directory, f"latlong_{segments}x{rings}.obj")
    if not os.path.exists(obj):
        write_latlong_sphere_obj(obj, segments, rings, seed=seed)
    rng = np.random.default_rng(seed)
    path = os.path.join(directory, name)
    pos, corner, hor, ver = look_at_camera((0.0, 0.35 * box, -1.6 * box), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0,
                                           width / height)
    lines = [
        "# instanced Perlin-displaced meshes under a Perlin sky",
        f"Render {width} {height} {depth} {spp} 380 780",
        "Texture sky scalar perlin 0.2 1.0 1",
        "Texture thickness scalar worley 200 800 3",
        "Texture tiles spectrum checker 0.8 0.2 10",
        "Material film thinfilm [1 1.33 1.5] [thickness]",
        "Material glass dielectric 1.0 1.5",
        "Material tiled lambertian tiles",
        f"Object mesh mesh tiled {obj}",
    ]
    u = rng.uniform(0, 1, instances)
    mats = np.where(u < 0.4, "film", np.where(u < 0.7, "glass", "tiled"))
    t = rng.uniform(-box / 2, box / 2, (instances, 3))
    r = rng.uniform(0, 2 * math.pi, (instances, 3))
    sc = rng.uniform(0.5, 2.0, instances)
    for i in range(instances):
        lines.append(f"Instance mesh {mats[i]} {_v(t[i])} {_v(r[i])} ({_f(sc[i])} {_f(sc[i])} {_f(sc[i])})")
    lines += [
        "Background equirectangular sky",
        f"Camera {_v(pos)} {_v(corner)} {_v(hor)} {_v(ver)}",
    ]
    _write(path, lines)
    return SceneFiles(path, seed, width, height, spp, depth)
