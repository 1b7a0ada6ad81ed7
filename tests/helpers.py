"""Shared helpers for the tests: seeded ray sets and image metrics."""

import numpy as np

# linear sRGB -> XYZ: the inverse of the reference's fixed XYZ -> sRGB matrix
# (src/core/utils.h:230), formed in float64.
_M = np.array([[3.2406255, -1.5372080, -0.4986286],
               [-0.9689307, 1.8757561, 0.0415175],
               [0.0557101, -0.2040211, 1.0569959]], dtype=np.float64)
RGB_TO_XYZ = np.linalg.inv(_M)


def to_xyz(rgb: np.ndarray) -> np.ndarray:
    return rgb.reshape(-1, 3).astype(np.float64) @ RGB_TO_XYZ.T


def rel_rmse(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b||_2 / ||b||_2 over all pixels x 3 channels of linear XYZ."""
    xa, xb = to_xyz(a), to_xyz(b)
    return float(np.linalg.norm(xa - xb) / max(np.linalg.norm(xb), 1e-300))


def random_rays(n: int, lo, hi, seed: int) -> np.ndarray:
    """Origins uniform in the box [lo, hi], directions uniform on the sphere."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], axis=1).astype(np.float32)


def camera_rays(settings, n: int, seed: int) -> np.ndarray:
    """Rays through random image-plane points of a scene's camera."""
    rng = np.random.default_rng(seed)
    c = settings.camera
    pos = np.array(list(c.position), np.float32)
    corner = np.array(list(c.corner), np.float32)
    h = np.array(list(c.horizontal), np.float32)
    v = np.array(list(c.vertical), np.float32)
    uv = rng.uniform(0, 1, size=(n, 2)).astype(np.float32)
    d = corner[None] + h[None] * uv[:, :1] + v[None] * uv[:, 1:] - pos[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.repeat(pos[None], n, axis=0)
    return np.concatenate([o, d], axis=1).astype(np.float32)


_REF_SCENES = {}


def ref_scene(lrd: str):
    """The reference harness's scene for an .lrd file, built once per test session
    (the reference's BVH build takes seconds on a million triangles)."""
    from oracle import ref

    if lrd not in _REF_SCENES:
        _REF_SCENES[lrd] = ref.RefScene(lrd)
    return _REF_SCENES[lrd]
