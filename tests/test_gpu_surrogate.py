"""Thin-film surrogate on the GPU: training-kernel gradients against the CPU
oracle, tensor-core inference against the FP64 forward pass with the same BF16
rounding, a short training run, and renders with the surrogate against the exact
transfer matrix."""

import ctypes as C

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import _native as N
from lambda_b200 import scenes
from oracle import port
from tests.helpers import rel_rmse

pytestmark = pytest.mark.gpu


def _params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, scale, N.MLP_PARAMS).astype(np.float32)
    return p


def test_gradient_matches_oracle(ctx):
    rng = np.random.default_rng(1)
    p = _params(1)
    n = 200
    x = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    y = rng.uniform(0, 1, (n, 4)).astype(np.float32)
    g = np.empty(N.MLP_PARAMS, np.float32)
    loss = C.c_float()
    st = ctx._lib.lambda_surrogate_grad(ctx._h, p.ctypes.data, x.ctypes.data, y.ctypes.data, n, g.ctypes.data,
                                        C.byref(loss))
    assert st == 0, ctx.last_error
    want_loss, want = port.mlp_grad(p.astype(np.float64), x, y, bf16=True)
    assert abs(loss.value - want_loss) <= 1e-3 * abs(want_loss)
    cos = float(g @ want / (np.linalg.norm(g) * np.linalg.norm(want)))
    rel = float(np.linalg.norm(g - want) / np.linalg.norm(want))
    print(f"gradient cosine {cos:.6f}, relative error {rel:.2e}")
    assert cos > 0.9999 and rel < 1e-2


def test_tensor_core_inference_matches_fp64_forward(ctx):
    p = _params(2, 0.2)
    ctx.surrogate_set(p)
    rng = np.random.default_rng(3)
    q = np.stack([rng.uniform(380, 780, 5000), rng.uniform(0, 1, 5000), rng.uniform(150, 850, 5000),
                  rng.uniform(1.2, 1.8, 5000), rng.uniform(1.0, 2.0, 5000)], 1).astype(np.float32)
    got = ctx.surrogate_eval(q)
    r = lb.default_film_range()
    lo = np.array([r.lambda_nm[0], r.cos_theta[0], r.thickness_nm[0], r.n_film[0], r.n_sub[0]], np.float32)
    hi = np.array([r.lambda_nm[1], r.cos_theta[1], r.thickness_nm[1], r.n_film[1], r.n_sub[1]], np.float32)
    x = (2.0 * (q - lo) / (hi - lo) - 1.0).astype(np.float32)
    want = port.mlp_forward(p.astype(np.float64), x, bf16=True)
    err = np.abs(got - want)
    scale = np.abs(want).max()
    print(f"max |tc - fp64| {err.max():.3e} (output scale {scale:.3f}), mean {err.mean():.3e}")
    assert err.max() <= 1e-2 * scale
    assert err.mean() <= 1e-3 * scale
    back, _ = ctx.surrogate_get()
    assert (back == p).all()


@pytest.fixture(scope="module")
def trained(ctx):
    rep = ctx.surrogate_train(samples=1 << 21, epochs=4, batch=4096, lr=3e-3, seed=11)
    print(f"train {rep.train_ms:.0f} ms, labels {rep.label_ms:.0f} ms, loss {rep.final_loss:.3e}, "
          f"audit max {rep.max_abs_error:.3e} mean {rep.mean_abs_error:.3e}")
    return rep


def test_short_training_run(trained, ctx):
    assert trained.final_loss < 1e-3
    assert trained.mean_abs_error < 0.02
    q = np.array([[550, 0.8, 400, 1.33, 1.5]], np.float32)
    out = ctx.surrogate_eval(q)
    want = ctx.thinfilm_fp64(q)
    assert np.abs(out - want).max() < 0.1


def test_surrogate_render_close_to_exact(trained, scene_dir, ctx):
    sc = scenes.thinfilm_spheres(scene_dir, 96, 54, 16, name="s_thinfilm.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    exact = ctx.render(scene.render_desc(seed=sc.seed, flags=lb.RENDER_THINFILM_EXACT))
    sur = ctx.render(scene.render_desc(seed=sc.seed, flags=lb.RENDER_THINFILM_SURROGATE))
    st = ctx.stats()
    err = rel_rmse(sur, exact)
    print(f"surrogate vs exact relRMSE {err:.3e}; thin-film hits {st.thinfilm_hits}, exact fallback {st.thinfilm_fallback}")
    assert np.isfinite(sur).all()
    assert st.thinfilm_hits > 0 and st.thinfilm_fallback < st.thinfilm_hits
    assert err < 0.05
