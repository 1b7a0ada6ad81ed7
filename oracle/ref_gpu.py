"""ctypes view of oracle/_ref/libref_lambda_gpu.so: the reference's own CUDA
renderKernel (src/render/renderer.h:200-213), compiled from its headers by
oracle/Makefile (target ref_gpu) and driven as its main.cpp drives it. Benchmark and
test infrastructure only: the secondary GPU baseline."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_lambda_gpu.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle ref_gpu, needs the reference sources)")
        lib = C.CDLL(LIB)
        P = C.c_void_p
        lib.refgpu_open.restype = C.c_int
        lib.refgpu_open.argtypes = [C.c_char_p, C.POINTER(P), C.c_char_p, C.c_size_t]
        lib.refgpu_close.argtypes = [P]
        lib.refgpu_set_samples.argtypes = [P, C.c_int]
        lib.refgpu_render.restype = C.c_int
        lib.refgpu_render.argtypes = [P, C.c_uint64, C.c_double, P, C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
        _lib = lib
    return _lib


class RefGpuError(RuntimeError):
    pass


class RefGpuScene:
    """A scene parsed by the reference's parser, with main.cpp's managed device copies."""

    def __init__(self, path: str, width: int, height: int):
        self.lib = load()
        self.width, self.height = width, height
        h = C.c_void_p()
        err = C.create_string_buffer(4096)
        if self.lib.refgpu_open(path.encode(), C.byref(h), err, len(err)) != 0:
            raise RefGpuError(err.value.decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.refgpu_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_samples(self, samples: int):
        self.lib.refgpu_set_samples(self.h, samples)

    def render(self, seed: int, limit_s: float = 120.0, image: bool = True):
        """One renderKernel launch: (image or None, device milliseconds)."""
        out = np.zeros((self.height, self.width, 3), np.float32) if image else None
        ms = C.c_double(0.0)
        err = C.create_string_buffer(1024)
        st = self.lib.refgpu_render(self.h, seed, limit_s, out.ctypes.data if image else None, C.byref(ms), err,
                                    len(err))
        if st != 0:
            raise RefGpuError(err.value.decode())
        return out, ms.value
