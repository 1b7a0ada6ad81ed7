"""ctypes view of oracle/liboracle.so, the plain-C restatement of the render loop
(oracle/lambda_oracle.c). Test infrastructure only: it takes the flat scene the
product's parser produces (lambda_b200.HostScene) and renders/queries on the CPU."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(LIB)
        P = C.c_void_p
        lib.oracle_render.argtypes = [P, P, C.c_uint64, P]
        lib.oracle_render_rows.argtypes = [P, P, C.c_uint64, C.c_int, C.c_int, P]
        lib.oracle_hit.argtypes = [P, P, C.c_int, P, P, P]
        lib.oracle_shadow.argtypes = [P, P, P, P, C.c_int, P]
        lib.oracle_film.argtypes = [P, C.c_int, P]
        lib.oracle_perlin.restype = C.c_float
        lib.oracle_perlin.argtypes = [P]
        lib.oracle_worley.restype = C.c_float
        lib.oracle_worley.argtypes = [P]
        lib.oracle_pcg.argtypes = [C.c_uint64, C.c_uint64, C.c_int, P]
        lib.oracle_mlp_forward.argtypes = [P, P, C.c_int, P]
        lib.oracle_mlp_grad.restype = C.c_double
        lib.oracle_mlp_grad.argtypes = [P, P, P, C.c_int, P]
        lib.oracle_mlp_set_bf16.argtypes = [C.c_int]
        _lib = lib
    return _lib


def render(scene, seed: int, samples: int | None = None, rows=None) -> np.ndarray:
    """Renders a lambda_b200.HostScene (optionally only rows [r0, r1))."""
    from lambda_b200 import _native as N

    s = N.RenderSettings()
    C.memmove(C.byref(s), C.byref(scene.settings), C.sizeof(N.RenderSettings))
    if samples is not None:
        s.samples = samples
        s.sqrt_samples = int(round(samples ** 0.5))
    out = np.zeros((s.height, s.width, 3), np.float32)
    r0, r1 = rows if rows is not None else (0, s.height)
    load().oracle_render_rows(C.byref(scene.desc), C.byref(s), seed, r0, r1, out.ctypes.data)
    return out


def hit(scene, rays):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
    n = rays.shape[0]
    inst, obj, t = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32)
    load().oracle_hit(C.byref(scene.desc), rays.ctypes.data, n, inst.ctypes.data, obj.ctypes.data, t.ctypes.data)
    return inst, obj, t


def shadow(scene, rays, li, lo):
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
    li = np.ascontiguousarray(li, np.int32)
    lo = np.ascontiguousarray(lo, np.int32)
    occ = np.empty(rays.shape[0], np.int32)
    load().oracle_shadow(C.byref(scene.desc), rays.ctypes.data, li.ctypes.data, lo.ctypes.data, rays.shape[0],
                         occ.ctypes.data)
    return occ


def film(q) -> np.ndarray:
    q = np.ascontiguousarray(q, np.float32).reshape(-1, 5)
    out = np.empty((q.shape[0], 4), np.float64)
    load().oracle_film(q.ctypes.data, q.shape[0], out.ctypes.data)
    return out


def perlin(p) -> float:
    p = np.ascontiguousarray(p, np.float32)
    return float(load().oracle_perlin(p.ctypes.data))


def worley(p) -> float:
    p = np.ascontiguousarray(p, np.float32)
    return float(load().oracle_worley(p.ctypes.data))


def pcg(seed, stream, n) -> np.ndarray:
    out = np.empty(n, np.float32)
    load().oracle_pcg(seed, stream, n, out.ctypes.data)
    return out


def mlp_forward(params, x, bf16: bool = False) -> np.ndarray:
    """FP64 forward; bf16=True rounds weights, inputs and hidden activations to BF16
    as the tensor-core kernel does (output layer weights too; biases stay FP32)."""
    load().oracle_mlp_set_bf16(1 if bf16 else 0)
    p = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 5)
    y = np.empty((x.shape[0], 4), np.float64)
    load().oracle_mlp_forward(p.ctypes.data, x.ctypes.data, x.shape[0], y.ctypes.data)
    return y


def mlp_grad(params, x, t, bf16: bool = False):
    load().oracle_mlp_set_bf16(1 if bf16 else 0)
    p = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 5)
    t = np.ascontiguousarray(t, np.float64).reshape(-1, 4)
    g = np.empty_like(p)
    loss = load().oracle_mlp_grad(p.ctypes.data, x.ctypes.data, t.ctypes.data, x.shape[0], g.ctypes.data)
    return loss, g
