"""The C ABI library loads and exports every entry point include/lambda_gpu.h
declares; entry points fail cleanly (status codes, messages) without a GPU."""

import ctypes
import os
import re
import subprocess

import pytest

from lambda_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lambda_gpu.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lambda_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_symbols():
    assert set(declared()) == set(N.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (lambda_[a-z0-9_]+)", out))
    assert set(declared()) <= exported


def test_struct_sizes_match_reference_layout():
    assert ctypes.sizeof(N.Object) == 116
    assert ctypes.sizeof(N.Instance) == 144
    assert ctypes.sizeof(N.BVHNode) == 32
    assert ctypes.sizeof(N.Material) == 16
    assert ctypes.sizeof(N.ScalarTexture) == 16
    assert ctypes.sizeof(N.SpectrumTexture) == 16
    from oracle import ref

    if ref.available():
        lib = ref.load()
        assert [lib.ref_sizeof(i) for i in range(6)] == [116, 144, 32, 16, 16, 16]


def _header_fields(struct: str) -> list:
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct " + struct + r" \{(.*?)\} " + struct + ";", text, flags=re.S).group(1)
    return re.findall(r"(\w+)\s*(?:\[[^\]]*\])?;", body)


def test_python_mirrors_match_the_header():
    """The ctypes mirrors of the tuning and stage-time records and the constants the
    Python side copies agree with include/lambda_gpu.h."""
    assert [f[0] for f in N.Tuning._fields_] == _header_fields("lambda_tuning")
    assert [f[0] for f in N.StageTime._fields_] == _header_fields("lambda_stage_time")
    text = open(HEADER).read()
    defines = dict(re.findall(r"#define (LAMBDA_\w+) (\d+)", text))
    assert int(defines["LAMBDA_NUM_STAGES"]) == N.NUM_STAGES == len(N.STAGE_NAMES)
    assert int(defines["LAMBDA_PATH_KERNEL_PIXELS"]) == N.PATH_KERNEL_PIXELS
    fdefs = {k: float(v) for k, v in re.findall(r"#define (LAMBDA_SURROGATE_\w+) ([0-9.]+)f", text)}
    assert fdefs == {"LAMBDA_SURROGATE_GRAZING_COS": N.SURROGATE_GRAZING_COS,
                     "LAMBDA_SURROGATE_LOW_SUB_INDEX": N.SURROGATE_LOW_SUB_INDEX,
                     "LAMBDA_SURROGATE_LOW_SUB_COS": N.SURROGATE_LOW_SUB_COS}


def test_null_arguments_are_rejected():
    lib = N.load()
    assert lib.lambda_scene_upload(None, None) == 1
    assert lib.lambda_render(None, None, None, None) == 1
    assert lib.lambda_trace_closest(None, None, 0, None, None, None) == 1
    assert lib.lambda_ctx_create(0, None) == 1


def test_ctx_create_without_gpu_reports_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = N.load()
    h = ctypes.c_void_p()
    st = lib.lambda_ctx_create(0, ctypes.byref(h))
    assert st in (4, 1)
    assert lib.lambda_last_error(None)


def test_cli_argument_errors(tmp_path):
    exe = os.path.join(ROOT, "lambda_b200", "bin", "lambda")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "invalid number of arguments" in r.stderr
    r = subprocess.run([exe, "scene.txt"], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.strip() == "scene.txt: invalid file extension"
    bad = tmp_path / "bad.lrd"
    bad.write_text("Camera (0 0 0) (0 0 0) (1 0 0) (0 1 0)\n")
    r = subprocess.run([exe, str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.strip() == f'{bad}:1: expected "Render", got "Camera"'


def test_write_pfm_round_trip(tmp_path):
    """Binary float output: rows bottom-up, values bit-exact; the XYZ variant equals
    the linear-sRGB -> XYZ conversion the image metric uses."""
    import numpy as np

    import lambda_b200 as lb
    from tests.helpers import to_xyz

    rng = np.random.default_rng(3)
    img = rng.uniform(-0.5, 3.0, (7, 11, 3)).astype(np.float32)

    def read(p):
        with open(p, "rb") as f:
            assert f.readline() == b"PF\n"
            w, h = map(int, f.readline().split())
            assert float(f.readline()) == -1.0
            data = np.frombuffer(f.read(), dtype="<f4").reshape(h, w, 3)
        return data[::-1]

    lb.write_pfm(str(tmp_path / "a.pfm"), img)
    assert np.array_equal(read(tmp_path / "a.pfm").view(np.uint32), img.view(np.uint32))
    lb.write_pfm(str(tmp_path / "b.pfm"), img, xyz=True)
    want = to_xyz(img).reshape(img.shape).astype(np.float32)
    assert np.allclose(read(tmp_path / "b.pfm"), want, rtol=1e-6, atol=1e-6)
    with pytest.raises(lb.LambdaError):
        lb.write_pfm(str(tmp_path / "c.ppm"), img)


def test_static_entry_point_buffer_rule(tmp_path):
    """The rule lambda_surrogate_eval_static applies to caller buffers
    (host/buffer_policy.h), compiled and run on the CPU: device memory of the
    context's own GPU or managed memory passes; host, unregistered and another
    GPU's device memory are refused, so they return an error instead of reaching a
    kernel."""
    src = tmp_path / "policy.cpp"
    src.write_text(r'''
#include "buffer_policy.h"
#include <cstdio>
using namespace lambda_host;
int main() {
    int bad = 0;
    bad += !buffer_usable_on(kMemDevice, 0, 0);
    bad += !buffer_usable_on(kMemDevice, 3, 3);
    bad += buffer_usable_on(kMemDevice, 1, 0);   // another GPU's memory
    bad += buffer_usable_on(kMemDevice, 0, 1);
    bad += !buffer_usable_on(kMemManaged, 5, 0);  // managed memory migrates
    bad += buffer_usable_on(kMemHost, 0, 0);
    bad += buffer_usable_on(kMemUnregistered, 0, 0);
    std::printf("%d\n", bad);
    return bad;
}
''')
    exe = tmp_path / "policy"
    inc = os.path.join(ROOT, "lambda_b200", "csrc", "host")
    subprocess.run(["g++", "-std=c++20", "-I", inc, str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
