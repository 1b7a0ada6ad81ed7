"""ctypes view of oracle/_ref/libref_lambda.so (the reference's CPU renderer,
compiled from its own headers by oracle/Makefile). Test infrastructure only."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_lambda.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle ref, needs the reference sources)")
        lib = C.CDLL(LIB)
        P = C.c_void_p
        lib.ref_sizeof.restype = C.c_int
        lib.ref_sizeof.argtypes = [C.c_int]
        lib.ref_parse.restype = C.c_int
        lib.ref_parse.argtypes = [C.c_char_p, C.POINTER(P), C.c_char_p, C.c_size_t]
        lib.ref_free.argtypes = [P]
        lib.ref_counts.argtypes = [P, P]
        lib.ref_copy.restype = C.c_int
        lib.ref_copy.argtypes = [P, C.c_int, P]
        lib.ref_set_samples.argtypes = [P, C.c_int]
        lib.ref_render.restype = C.c_double
        lib.ref_render.argtypes = [P, C.c_uint64, C.c_int, P]
        lib.ref_max_threads.restype = C.c_int
        lib.ref_trace_sample.argtypes = [P, C.c_uint64, C.c_int, C.c_int, C.c_int, P, P]
        lib.ref_trace_pixel.argtypes = [P, C.c_uint64, C.c_int, C.c_int, P]
        lib.ref_hit.argtypes = [P, P, C.c_int, P, P, P, P, P]
        lib.ref_shadow.argtypes = [P, P, P, P, C.c_int, P]
        lib.ref_thinfilm.restype = C.c_float
        lib.ref_thinfilm.argtypes = [P, C.c_int, P, C.c_int, P, P, C.c_float]
        lib.ref_tmm_single.argtypes = [C.c_double] * 5 + [P]
        lib.ref_scalar_texture.restype = C.c_float
        lib.ref_scalar_texture.argtypes = [P, C.c_int, P]
        lib.ref_spectrum_texture.restype = C.c_float
        lib.ref_spectrum_texture.argtypes = [P, C.c_int, P, C.c_float, C.c_float, C.c_float]
        lib.ref_perlin.restype = C.c_float
        lib.ref_perlin.argtypes = [P]
        lib.ref_worley.restype = C.c_float
        lib.ref_worley.argtypes = [P]
        lib.ref_spectrum_to_rgb.argtypes = [P, P, C.c_float, P]
        lib.ref_pcg.argtypes = [C.c_uint64, C.c_uint64, C.c_int, P]
        lib.ref_write_ppm.restype = C.c_int
        lib.ref_write_ppm.argtypes = [C.c_char_p, C.c_int, C.c_int, P, C.c_char_p, C.c_size_t]
        _lib = lib
    return _lib


class RefError(RuntimeError):
    pass


SIZES = {"objects": 116, "instances": 144, "nodes": 32, "materials": 16, "scalar_textures": 16,
         "spectrum_textures": 16}
_WHICH = {"spectra": 0, "complex_spectra": 1, "objects": 2, "instances": 3, "nodes": 4, "light_instances": 5,
          "materials": 6, "material_properties": 7, "scalar_textures": 8, "spectrum_textures": 9,
          "light_powers": 10, "light_objects": 11}


class RefScene:
    """A scene parsed by the reference's own Parser::parseLRD."""

    def __init__(self, path: str):
        self.lib = load()
        h = C.c_void_p()
        err = C.create_string_buffer(4096)
        if self.lib.ref_parse(path.encode(), C.byref(h), err, len(err)) != 0:
            raise RefError(err.value.decode())
        self.h = h
        c = (C.c_int32 * 11)()
        self.lib.ref_counts(h, c)
        self.counts = list(c)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_free(self.h)
            self.h = None

    def _copy(self, which: int, nbytes: int) -> np.ndarray:
        buf = np.zeros(max(nbytes, 1), dtype=np.uint8)
        self.lib.ref_copy(self.h, which, buf.ctypes.data)
        return buf[:nbytes]

    def raw(self, name: str) -> np.ndarray:
        idx = {"objects": 2, "instances": 3, "nodes": 4, "materials": 6, "scalar_textures": 8,
               "spectrum_textures": 9}[name]
        n = self.counts[idx]
        sz = SIZES[name]
        return self._copy(_WHICH[name], n * sz).reshape(n, sz)

    @property
    def spectra(self):
        n = self.counts[0]
        return self._copy(0, n * 471 * 4).view(np.float32).reshape(n, 471)

    @property
    def complex_spectra(self):
        n = self.counts[1]
        return self._copy(1, n * 471 * 16).view(np.float64).reshape(n, 471, 2)

    @property
    def light_instances(self):
        return self._copy(5, self.counts[5] * 4).view(np.int32)

    @property
    def light_objects(self):
        return self._copy(11, self.counts[5] * 4).view(np.int32)

    @property
    def light_powers(self):
        return self._copy(10, self.counts[5] * 4).view(np.float32)

    @property
    def material_properties(self):
        return self._copy(7, self.counts[7] * 4).view(np.int32)

    @property
    def total_light_power(self) -> float:
        return float(self._copy(12, 4).view(np.float32)[0])

    @property
    def background_texture(self) -> int:
        return self.counts[10]

    def settings(self):
        b = self._copy(13, 5 * 4 + 14 * 4)
        iv = b[:20].view(np.int32)
        fv = b[20:].view(np.float32)
        return {"width": int(iv[0]), "height": int(iv[1]), "depth": int(iv[2]), "samples": int(iv[3]),
                "sqrt_samples": int(iv[4]), "lambda_min": float(fv[0]), "lambda_max": float(fv[1]),
                "camera": fv[2:14].copy()}

    def set_samples(self, samples: int):
        self.lib.ref_set_samples(self.h, samples)

    def render(self, seed: int, threads: int = 0):
        s = self.settings()
        out = np.zeros((s["height"], s["width"], 3), dtype=np.float32)
        secs = self.lib.ref_render(self.h, seed, threads, out.ctypes.data)
        return out, secs

    def hit(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        inst = np.empty(n, np.int32)
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        pn = np.empty((n, 8), np.float32)
        front = np.empty(n, np.int32)
        self.lib.ref_hit(self.h, rays.ctypes.data, n, inst.ctypes.data, obj.ctypes.data, t.ctypes.data,
                         pn.ctypes.data, front.ctypes.data)
        return inst, obj, t, pn, front

    def shadow(self, rays, li, lo):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        li = np.ascontiguousarray(li, np.int32)
        lo = np.ascontiguousarray(lo, np.int32)
        occ = np.empty(rays.shape[0], np.int32)
        self.lib.ref_shadow(self.h, rays.ctypes.data, li.ctypes.data, lo.ctypes.data, rays.shape[0], occ.ctypes.data)
        return occ

    def trace_sample(self, seed, px, py, sample):
        rad = np.zeros(4, np.float32)
        lam = np.zeros(4, np.float32)
        self.lib.ref_trace_sample(self.h, seed, px, py, sample, rad.ctypes.data, lam.ctypes.data)
        return rad, lam

    def trace_pixel(self, seed, px, py):
        """Every sample's radiance (4 hero wavelengths) of one pixel, in order."""
        n = self.settings()["samples"]
        rad = np.zeros((n, 4), np.float32)
        self.lib.ref_trace_pixel(self.h, seed, px, py, rad.ctypes.data)
        return rad

    def thinfilm(self, material, normal, front, point, d, lam) -> float:
        n = np.ascontiguousarray(normal, np.float32)
        p = np.ascontiguousarray(point, np.float32)
        dd = np.ascontiguousarray(d, np.float32)
        return float(self.lib.ref_thinfilm(self.h, material, n.ctypes.data, int(front), p.ctypes.data,
                                           dd.ctypes.data, lam))

    def scalar_texture(self, tex, point) -> float:
        p = np.ascontiguousarray(point, np.float32)
        return float(self.lib.ref_scalar_texture(self.h, tex, p.ctypes.data))

    def spectrum_texture(self, tex, point, u, v, lam) -> float:
        p = np.ascontiguousarray(point, np.float32)
        return float(self.lib.ref_spectrum_texture(self.h, tex, p.ctypes.data, u, v, lam))


def tmm_single(lam, cos_t, d, n_film, n_sub):
    out = np.zeros(2, np.float64)
    load().ref_tmm_single(lam, cos_t, d, n_film, n_sub, out.ctypes.data)
    return out


def perlin(p) -> float:
    p = np.ascontiguousarray(p, np.float32)
    return float(load().ref_perlin(p.ctypes.data))


def worley(p) -> float:
    p = np.ascontiguousarray(p, np.float32)
    return float(load().ref_worley(p.ctypes.data))


def pcg(seed, stream, n):
    out = np.zeros(n, np.float32)
    load().ref_pcg(seed, stream, n, out.ctypes.data)
    return out


def spectrum_to_rgb(radiance, lambdas, rng):
    r = np.ascontiguousarray(radiance, np.float32)
    l = np.ascontiguousarray(lambdas, np.float32)
    out = np.zeros(3, np.float32)
    load().ref_spectrum_to_rgb(r.ctypes.data, l.ctypes.data, rng, out.ctypes.data)
    return out


def write_ppm(path, rgb):
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    err = C.create_string_buffer(1024)
    if load().ref_write_ppm(path.encode(), w, h, rgb.ctypes.data, err, len(err)) != 0:
        raise RefError(err.value.decode())


def max_threads() -> int:
    return int(load().ref_max_threads())
