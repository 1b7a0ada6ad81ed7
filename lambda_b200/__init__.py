"""lambda_b200: B200 spectral path-tracing render loop behind a C ABI.

Python view of include/lambda_gpu.h, used by the tests and the benchmark:

  HostScene.parse(path)      Parser::parseLRD (src/core/parser.h:29) -> flat arrays
  Context(device)            a GPU context (one stream, its own device arena)
    .upload(scene)           Renderer::setScene (src/render/renderer.h:38)
    .render(settings, seed)  Renderer::renderImage / renderKernel (renderer.h:42, :200)
    .trace_closest(rays)     Scene::hit closest mode (src/scene/scene.h:51)
    .trace_shadow(...)       Scene::hit shadow mode
    .thinfilm_exact/fp64     thin-film transfer matrix (src/scene/material.h:263)
  write_ppm(path, rgb)       Writer::write (src/core/writer.h:11)

Every call goes to liblambda_b200.so; there is no Python implementation of any
of them to fall back on.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import LambdaError

__all__ = [
    "HostScene",
    "Context",
    "LambdaError",
    "write_ppm",
    "write_pfm",
    "RENDER_THINFILM_EXACT",
    "RENDER_THINFILM_SURROGATE",
    "RENDER_OUTPUT_DEVICE",
]

RENDER_THINFILM_EXACT = N.RENDER_THINFILM_EXACT
RENDER_THINFILM_SURROGATE = N.RENDER_THINFILM_SURROGATE
RENDER_OUTPUT_DEVICE = N.RENDER_OUTPUT_DEVICE
RENDER_PROFILE_STAGES = N.RENDER_PROFILE_STAGES
RENDER_THINFILM_FP64 = N.RENDER_THINFILM_FP64


def _arr(ptr, n, dtype, shape=None):
    if n == 0 or not ptr:
        return np.zeros((0,) if shape is None else (0,) + tuple(shape[1:]), dtype=dtype)
    a = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
    a = a.view(dtype) if a.dtype != dtype else a
    return a.reshape(shape) if shape is not None else a


def _struct_array(ptr, n, ctype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=np.dtype((np.void, C.sizeof(ctype))))
    raw = C.string_at(ptr, n * C.sizeof(ctype))
    return np.frombuffer(raw, dtype=np.uint8).reshape(n, C.sizeof(ctype)).copy()


class HostScene:
    """A parsed .lrd scene (the reference's 15 containers, after the BVH build)."""

    def __init__(self, handle, lib):
        self._h = handle
        self._lib = lib
        self.desc = N.SceneDesc()
        self.settings = N.RenderSettings()
        lib.lambda_host_scene_get(handle, C.byref(self.desc), C.byref(self.settings))

    @classmethod
    def parse(cls, path: str) -> "HostScene":
        lib = N.load()
        h = C.c_void_p()
        err = C.create_string_buffer(4096)
        st = lib.lambda_parse_lrd(path.encode(), C.byref(h), err, len(err))
        if st != 0:
            raise LambdaError(st, err.value.decode())
        return cls(h, lib)

    @classmethod
    def parse_gpu(cls, ctx: "Context", path: str, gpu_min_items: int = 0) -> "HostScene":
        """parse() with the scene build's heavy steps on ctx's GPU (lambda_parse_lrd_gpu):
        the same scene byte for byte. gpu_min_items: the smallest object group or
        instance set built on the GPU (0: the library's default)."""
        lib = N.load()
        h = C.c_void_p()
        err = C.create_string_buffer(4096)
        st = lib.lambda_parse_lrd_gpu(ctx._h, path.encode(), gpu_min_items, C.byref(h), err, len(err))
        if st != 0:
            raise LambdaError(st, err.value.decode() or lib.lambda_last_error(ctx._h).decode())
        return cls(h, lib)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.lambda_host_scene_destroy(h)
            self._h = None

    # Raw byte rows of each container, for comparison with the reference.
    def raw(self, name: str) -> np.ndarray:
        d = self.desc
        table = {
            "objects": (d.objects, d.num_objects, N.Object),
            "instances": (d.instances, d.num_instances, N.Instance),
            "nodes": (d.nodes, d.num_nodes, N.BVHNode),
            "materials": (d.materials, d.num_materials, N.Material),
            "scalar_textures": (d.scalar_textures, d.num_scalar_textures, N.ScalarTexture),
            "spectrum_textures": (d.spectrum_textures, d.num_spectrum_textures, N.SpectrumTexture),
        }
        ptr, n, ct = table[name]
        return _struct_array(C.cast(ptr, C.c_void_p), n, ct)

    @property
    def spectra(self) -> np.ndarray:
        d = self.desc
        return _arr(d.spectra, d.num_spectra * N.CIE_BINS, np.float32, (d.num_spectra, N.CIE_BINS))

    @property
    def complex_spectra(self) -> np.ndarray:
        d = self.desc
        return _arr(d.complex_spectra, d.num_complex_spectra * N.CIE_BINS * 2, np.float64,
                    (d.num_complex_spectra, N.CIE_BINS, 2))

    @property
    def light_instances(self) -> np.ndarray:
        return _arr(self.desc.light_instances, self.desc.num_lights, np.int32)

    @property
    def light_objects(self) -> np.ndarray:
        return _arr(self.desc.light_objects, self.desc.num_lights, np.int32)

    @property
    def light_powers(self) -> np.ndarray:
        return _arr(self.desc.light_powers, self.desc.num_lights, np.float32)

    @property
    def material_properties(self) -> np.ndarray:
        return _arr(self.desc.material_properties, self.desc.num_material_properties, np.int32)

    @property
    def total_light_power(self) -> float:
        return float(np.float32(self.desc.total_light_power))

    @property
    def background_texture(self) -> int:
        return int(self.desc.background_texture)

    def objects_array(self) -> np.ndarray:
        """Objects as a structured array (type, material, g[27])."""
        dt = np.dtype([("type", "<i4"), ("material", "<i4"), ("g", "<f4", (27,))])
        return self.raw("objects").view(dt).reshape(-1)

    def instances_array(self) -> np.ndarray:
        dt = np.dtype([("object", "<i4"), ("count", "<i4"), ("node", "<i4"), ("material", "<i4"),
                       ("transform", "<f4", (16,)), ("inverse_transform", "<f4", (16,))])
        return self.raw("instances").view(dt).reshape(-1)

    def nodes_array(self) -> np.ndarray:
        dt = np.dtype([("min", "<f4", (3,)), ("max", "<f4", (3,)), ("index", "<i4"), ("count", "<i4")])
        return self.raw("nodes").view(dt).reshape(-1)

    def render_desc(self, seed: int, flags: int = 0, samples: int | None = None) -> N.RenderDesc:
        rd = N.RenderDesc()
        C.memmove(C.byref(rd.settings), C.byref(self.settings), C.sizeof(N.RenderSettings))
        if samples is not None:
            root = int(round(samples ** 0.5))
            if root * root != samples:
                raise ValueError("samples must be a perfect square")
            rd.settings.samples = samples
            rd.settings.sqrt_samples = root
        rd.seed = seed
        rd.flags = flags
        return rd


def write_ppm(path: str, rgb: np.ndarray) -> None:
    lib = N.load()
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    h, w = rgb.shape[:2]
    err = C.create_string_buffer(1024)
    st = lib.lambda_write_ppm(path.encode(), w, h, rgb.ctypes.data, err, len(err))
    if st != 0:
        raise LambdaError(st, err.value.decode())


def write_pfm(path: str, rgb: np.ndarray, xyz: bool = False) -> None:
    """Float image to a little-endian PFM: linear sRGB, or linear CIE XYZ."""
    lib = N.load()
    rgb = np.ascontiguousarray(rgb, dtype=np.float32)
    h, w = rgb.shape[:2]
    err = C.create_string_buffer(1024)
    st = lib.lambda_write_pfm(path.encode(), w, h, rgb.ctypes.data, 1 if xyz else 0, err, len(err))
    if st != 0:
        raise LambdaError(st, err.value.decode())


@dataclass
class RenderStats:
    render_ms: float
    paths: int
    segments: int
    shadow_rays: int
    thinfilm_hits: int
    thinfilm_fallback: int
    kernel_launches: int
    waves: int
    surrogate_ctas_per_sm: int


def _ptr(a) -> int:
    """Address of a numpy array (host) or a torch tensor (device or host)."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())


class Context:
    """One GPU context (lambda_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = N.load()
        h = C.c_void_p()
        st = self._lib.lambda_ctx_create(device, C.byref(h))
        if st != 0:
            raise LambdaError(st, self._lib.lambda_last_error(None).decode())
        self._h = h
        self._scene = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lambda_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != 0:
            raise LambdaError(st, self._lib.lambda_last_error(self._h).decode())

    @property
    def last_error(self) -> str:
        return self._lib.lambda_last_error(self._h).decode()

    def upload(self, scene: HostScene) -> None:
        self._check(self._lib.lambda_scene_upload(self._h, C.byref(scene.desc)))
        self._scene = scene

    def render(self, desc: N.RenderDesc, out=None, completed=None) -> np.ndarray:
        """Renders into `out` (host numpy array, or a device tensor with
        RENDER_OUTPUT_DEVICE); returns the host image when `out` is None."""
        s = desc.settings
        if out is None:
            out = np.empty((s.height, s.width, 3), dtype=np.float32)
        cptr = C.cast(completed, C.c_void_p) if completed is not None else None
        self._check(self._lib.lambda_render(self._h, C.byref(desc), C.c_void_p(_ptr(out)), cptr))
        return out

    def render_batch(self, descs, outs=None, completed=None) -> list:
        """Renders several images of the uploaded scene in one batch
        (lambda_render_batch). `outs[i]` is a host numpy array, or a device tensor
        when descs[i] has RENDER_OUTPUT_DEVICE; host arrays are made for a None."""
        n = len(descs)
        outs = list(outs) if outs is not None else [None] * n
        jobs = (N.Job * n)()
        for i, d in enumerate(descs):
            if outs[i] is None:
                outs[i] = np.empty((d.settings.height, d.settings.width, 3), dtype=np.float32)
            C.memmove(C.byref(jobs[i].desc), C.byref(d), C.sizeof(N.RenderDesc))
            jobs[i].out_rgb = _ptr(outs[i])
        cptr = C.cast(completed, C.c_void_p) if completed is not None else None
        self._check(self._lib.lambda_render_batch(self._h, jobs, n, cptr))
        return outs

    def autotune(self, probe: N.RenderDesc) -> N.Tuning:
        """Picks the wavefront launch shapes by timing `probe` (lambda_autotune)."""
        t = N.Tuning()
        self._check(self._lib.lambda_autotune(self._h, C.byref(probe), C.byref(t)))
        return t

    def autotune_batch(self, probes) -> N.Tuning:
        """Picks the launch shapes by timing batched renders of `probes`
        (lambda_autotune_batch)."""
        arr = (N.RenderDesc * len(probes))(*probes)
        t = N.Tuning()
        self._check(self._lib.lambda_autotune_batch(self._h, arr, len(probes), C.byref(t)))
        return t

    def set_tuning(self, trace_block: int, shade_block: int, grid_scale: int = 1, max_pixels: int = 0,
                   bvh_width: int = 4, path_kernel_pixels: int = N.PATH_KERNEL_PIXELS, lane_fetch: int = 0,
                   compressed_nodes: int = 0, fused_bounce: int = 0) -> None:
        t = N.Tuning(trace_block, shade_block, grid_scale, max_pixels, bvh_width, path_kernel_pixels, lane_fetch,
                     compressed_nodes, fused_bounce)
        self._check(self._lib.lambda_set_tuning(self._h, C.byref(t)))

    def tuning(self) -> N.Tuning:
        t = N.Tuning()
        self._check(self._lib.lambda_get_tuning(self._h, C.byref(t)))
        return t

    def set_limits(self, mma_polls: int = N.DEFAULT_MMA_POLLS, stack_entries: int = 0) -> None:
        """Device guard limits (lambda_set_limits), for tests that make a guard fire."""
        lim = N.Limits(mma_polls, stack_entries)
        self._check(self._lib.lambda_set_limits(self._h, C.byref(lim)))

    def reset_limits(self) -> None:
        self._check(self._lib.lambda_set_limits(self._h, None))

    def limits(self) -> N.Limits:
        lim = N.Limits()
        self._check(self._lib.lambda_get_limits(self._h, C.byref(lim)))
        return lim

    def stats(self) -> RenderStats:
        st = N.RenderStats()
        self._check(self._lib.lambda_get_render_stats(self._h, C.byref(st)))
        return RenderStats(st.render_ms, st.paths, st.segments, st.shadow_rays, st.thinfilm_hits,
                           st.thinfilm_fallback, st.kernel_launches, st.waves, st.surrogate_ctas_per_sm)

    def stage_times(self) -> dict:
        arr = (N.StageTime * N.NUM_STAGES)()
        self._check(self._lib.lambda_get_stage_times(self._h, arr))
        return {N.STAGE_NAMES[i]: {"ms": arr[i].ms, "launches": int(arr[i].launches), "items": int(arr[i].items)}
                for i in range(N.NUM_STAGES)}

    def trace_closest(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        inst = np.empty(n, np.int32)
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        self._check(self._lib.lambda_trace_closest(self._h, rays.ctypes.data, n, inst.ctypes.data, obj.ctypes.data,
                                                   t.ctypes.data))
        return inst, obj, t

    def trace_shadow(self, rays: np.ndarray, light_instance: np.ndarray, light_object: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        li = np.ascontiguousarray(light_instance, dtype=np.int32)
        lo = np.ascontiguousarray(light_object, dtype=np.int32)
        occ = np.empty(n, np.int32)
        self._check(self._lib.lambda_trace_shadow(self._h, rays.ctypes.data, li.ctypes.data, lo.ctypes.data, n,
                                                  occ.ctypes.data))
        return occ

    @staticmethod
    def _queries(q: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, 5)
        return q

    def _film(self, fn, q, out, dtype):
        """Film queries: q [n, 5] = (lambda_nm, cos_theta, thickness_nm, n_film, n_sub).
        A numpy q returns a new numpy [n, 4]; a contiguous float32 CUDA tensor q is
        evaluated in place into `out` (a [n, 4] CUDA tensor), with no host staging."""
        if not isinstance(q, np.ndarray) and getattr(q, "is_cuda", False):
            if out is None or not q.is_contiguous() or not out.is_contiguous() or q.shape[-1] != 5:
                raise ValueError("device queries need a contiguous [n, 5] tensor and a contiguous [n, 4] out")
            n = q.numel() // 5
            if out.numel() != 4 * n:
                raise ValueError("out must hold [n, 4] results")
            self._check(fn(self._h, _ptr(q), n, _ptr(out)))
            return out
        q = self._queries(q)
        res = np.empty((q.shape[0], 4), dtype)
        self._check(fn(self._h, q.ctypes.data, q.shape[0], res.ctypes.data))
        return res

    def thinfilm_exact(self, q, out=None):
        """Exact FP32 transfer matrix: (R_s, R_p, T_s, T_p) per query."""
        return self._film(self._lib.lambda_thinfilm_exact, q, out, np.float32)

    def thinfilm_fp64(self, q, out=None):
        """FP64 transfer matrix (the training labeller)."""
        return self._film(self._lib.lambda_thinfilm_fp64, q, out, np.float64)

    def surrogate_eval(self, q, out=None):
        """Tensor-core surrogate: (R_s, R_p, T_s, T_p) per query."""
        return self._film(self._lib.lambda_surrogate_eval, q, out, np.float32)

    def surrogate_train(self, samples: int = 1 << 24, epochs: int = 8, batch: int = 8192, lr: float = 2e-3,
                        seed: int = 7, film_range=None) -> N.TrainReport:
        d = N.TrainDesc()
        d.samples = samples
        d.epochs = epochs
        d.batch = batch
        d.learning_rate = lr
        d.seed = seed
        d.range = film_range if film_range is not None else default_film_range()
        rep = N.TrainReport()
        self._check(self._lib.lambda_surrogate_train(self._h, C.byref(d), C.byref(rep)))
        return rep

    def surrogate_set(self, params: np.ndarray, film_range=None) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        if p.size != N.MLP_PARAMS:
            raise ValueError(f"expected {N.MLP_PARAMS} parameters")
        r = film_range if film_range is not None else default_film_range()
        self._check(self._lib.lambda_surrogate_set(self._h, p.ctypes.data, C.byref(r)))

    def surrogate_get(self):
        p = np.empty(N.MLP_PARAMS, np.float32)
        r = N.FilmRange()
        self._check(self._lib.lambda_surrogate_get(self._h, p.ctypes.data, C.byref(r)))
        return p, r


def default_film_range() -> N.FilmRange:
    """Training domain: lambda 380-780 nm, cos 0-1, d 150-850 nm, n_film 1.2-1.8, n_sub 1.0-2.0."""
    r = N.FilmRange()
    r.lambda_nm[:] = (380.0, 780.0)
    r.cos_theta[:] = (0.0, 1.0)
    r.thickness_nm[:] = (150.0, 850.0)
    r.n_film[:] = (1.2, 1.8)
    r.n_sub[:] = (1.0, 2.0)
    return r


# ---------------------------------------------------------------------------
# Measurement helpers (benchmark)
# ---------------------------------------------------------------------------

# Algorithmic HBM bytes per processed item of each stage: the path-state
# structure-of-arrays words the stage must read and write (queue ids included),
# not counting scene data, which is read-only and cache resident for small scenes.
STAGE_BYTES = {
    "raygen": 16 * 2 + 16 * 2 + 16 + 8 * 2 + 16 * 4 + 4,   # film rw, radiance rw, lam w, rng rw, ray/T w, queue
    "intersect": 4 + 32 + 16 + 4,                          # queue id, ray read, hit id write, material push
    # the shade kernels rebuild the hit record from the ray and the hit id
    "shade_lambert": 4 + 32 + 16 + 16 * 2 + 8 * 2 + 32 + 16 + 64 + 8,  # queue, ray, hit id, T/lam, rng rw, ray w, T w, NEE w, pushes
    "shade_specular": 4 + 32 + 16 + 16 * 2 + 8 * 2 + 32 + 16 + 4,
    "shade_film": 4 + 32 + 16 + 16 * 2 + 8 * 2 + 32 + 16 + 4,
    "shadow": 4 + 16 * 3 + 8 + 16 * 2,                     # queue, NEE ray + weights, light ids, radiance rw
    "finish": 16 * 3 + 12,
    # surrogate thin film: queue, ray, hit id, T/lam, then 4 rows of 32 B and a domain flag
    "film_encode": 4 + 32 + 16 + 16 * 2 + 4 * 32 + 1,
    # queue, ray, hit id, T/lam, 4 outputs of 16 B, domain flag, rng rw, ray w, T w, push
    "film_scatter": 4 + 32 + 16 + 16 * 2 + 4 * 16 + 1 + 8 * 2 + 32 + 16 + 4,
    # per segment: the ray and hit state of intersect plus a scatter's reads and writes
    # (the path kernel keeps a pixel's state in one thread, mostly in L1/L2)
    "path": 4 + 32 + 16 + 4 + 4 + 32 + 16 + 16 * 2 + 8 * 2 + 32 + 16 + 4,
    # the fused bounce kernel: the same per-segment reads and writes as the path kernel
    "bounce": 4 + 32 + 16 + 4 + 4 + 32 + 16 + 16 * 2 + 8 * 2 + 32 + 16 + 4,
}


def stage_profile(ctx: "Context", desc, out) -> dict:
    """Renders once more with every kernel launch bracketed by CUDA events and
    returns per-stage device time, launches and processed items."""
    d = N.RenderDesc()
    C.memmove(C.byref(d), C.byref(desc), C.sizeof(N.RenderDesc))
    d.flags = desc.flags | N.RENDER_PROFILE_STAGES
    ctx.render(d, out=out)
    st = ctx.stage_times()
    total = sum(v["ms"] for v in st.values())
    for k, v in st.items():
        v["share"] = v["ms"] / total if total > 0 else 0.0
        v["avg_launch_us"] = 1000.0 * v["ms"] / v["launches"] if v["launches"] else 0.0
    return st


def stage_rooflines(stages: dict, hbm_gbs: float, bf16_tflops: float) -> dict:
    """Every timed stage as a fraction of its roofline: algorithmic bytes (STAGE_BYTES
    per item) over its device time against the measured HBM bandwidth, and for the
    surrogate's MLP stage FLOPs against the measured BF16 tensor peak."""
    out = {}
    for name, s in stages.items():
        if s["ms"] <= 0 or not s["items"]:
            continue
        if name == "film_mlp":
            tf = 17536.0 * s["items"] * 4 / (s["ms"] / 1000.0) / 1e12
            out[name] = {"bound": "tensor", "achieved_tflops": tf, "frac": tf / bf16_tflops}
        elif name in STAGE_BYTES:
            gbs = STAGE_BYTES[name] * s["items"] / (s["ms"] / 1000.0) / 1e9
            out[name] = {"bound": "hbm", "achieved_gbs": gbs, "frac": gbs / hbm_gbs}
    return out


def roofline(stages: dict, hbm_gbs: float, bf16_tflops: float, peak_kind: str) -> dict:
    """Roofline entry for the stage with the largest device time."""
    name, s = max(((k, v) for k, v in stages.items() if v["ms"] > 0), key=lambda kv: kv[1]["ms"])
    if name == "film_mlp":
        flops = 17536.0 * s["items"] * 4  # 2*(5*64+64*64+64*64+64*4) per (hit, wavelength)
        achieved = flops / (s["ms"] / 1000.0) / 1e12
        return {"bound": "tensor", "kernel": name, "achieved": achieved, "peak": bf16_tflops, "unit": "TFLOP/s",
                "frac": achieved / bf16_tflops, "traffic": None, "peak_source": peak_kind}
    per_item = STAGE_BYTES.get(name, 0)
    bytes_ = per_item * s["items"]
    achieved = bytes_ / (s["ms"] / 1000.0) / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm_gbs, "unit": "GB/s",
            "frac": achieved / hbm_gbs, "traffic": None, "bytes_per_item": per_item, "items": s["items"],
            "avg_launch_us": s["avg_launch_us"], "peak_source": peak_kind}


def scene_bytes(scene: HostScene) -> int:
    """Bytes of the flat scene arrays a scene upload copies host -> device."""
    d = scene.desc
    return int(d.num_spectra * N.CIE_BINS * 4 + d.num_complex_spectra * N.CIE_BINS * 16 + d.num_objects * 116
               + d.num_instances * 144 + d.num_nodes * 32 + d.num_lights * 12 + d.num_materials * 16
               + d.num_material_properties * 4 + d.num_scalar_textures * 16 + d.num_spectrum_textures * 16)
