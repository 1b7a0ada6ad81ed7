"""Thin-film surrogate on the GPU: training-kernel gradients against the CPU
oracle, tensor-core inference against the FP64 forward pass with the same BF16
rounding, a short training run, and renders with the surrogate against the exact
transfer matrix."""

import ctypes as C

import numpy as np
import pytest

import lambda_b200 as lb
from lambda_b200 import _native as N
from lambda_b200 import scenes, surrogate
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
    x = surrogate.encode(q, lb.default_film_range())
    want = port.mlp_forward(p.astype(np.float64), x, bf16=True)
    err = np.abs(got - want)
    scale = np.abs(want).max()
    print(f"max |tc - fp64| {err.max():.3e} (output scale {scale:.3f}), mean {err.mean():.3e}")
    assert err.max() <= 1e-2 * scale
    assert err.mean() <= 1e-3 * scale
    back, _ = ctx.surrogate_get()
    assert (back == p).all()


def test_tensor_core_inference_batch_sizes(ctx):
    """Every batch size gives each query the same bits: a row's result depends only on
    its own inputs, not on its tile, its chain (warpgroup), its CTA or the tile the
    chain loads next. The sizes straddle one tile (128 rows), one CTA's five chains
    (640 rows) and one tile per chain on every SM (148 x 640 rows), and the largest
    batch is checked against the FP64 forward pass with BF16 rounding."""
    p = _params(4, 0.2)
    ctx.surrogate_set(p)
    rng = np.random.default_rng(9)
    n_max = 200_003
    q = np.stack([rng.uniform(380, 780, n_max), rng.uniform(0, 1, n_max), rng.uniform(150, 850, n_max),
                  rng.uniform(1.2, 1.8, n_max), rng.uniform(1.0, 2.0, n_max)], 1).astype(np.float32)
    full = ctx.surrogate_eval(q)
    for n in (1, 127, 128, 129, 639, 640, 641, 148 * 640, 148 * 640 + 1):
        got = ctx.surrogate_eval(q[:n])
        assert np.array_equal(got.view(np.uint32), full[:n].view(np.uint32)), f"n={n}"
    x = surrogate.encode(q, lb.default_film_range())
    want = port.mlp_forward(p.astype(np.float64), x, bf16=True)
    err = np.abs(full - want)
    scale = np.abs(want).max()
    assert err.max() <= 1e-2 * scale
    assert err.mean() <= 1e-3 * scale


@pytest.fixture(scope="module")
def trained(ctx):
    rep = ctx.surrogate_train(samples=1 << 21, epochs=4, batch=8192, lr=3e-3, seed=11)
    print(f"train {rep.train_ms:.0f} ms, labels {rep.label_ms:.0f} ms, loss {rep.final_loss:.3e}, "
          f"audit max {rep.max_abs_error:.3e} mean {rep.mean_abs_error:.3e}")
    return rep


def test_short_training_run(trained, ctx):
    """The training kernels learn: 1024 Adam steps on 2^21 samples."""
    # a short run (1024 Adam steps); the shipped weights train 24 epochs of 2^24 samples
    assert trained.final_loss < 2e-3
    assert trained.mean_abs_error < 0.02
    q = np.array([[550, 0.8, 400, 1.33, 1.5]], np.float32)
    out = ctx.surrogate_eval(q)
    want = ctx.thinfilm_fp64(q)
    assert np.abs(out - want).max() < 0.1
    assert trained.audit_samples == 1 << 18


def test_trained_weights_accuracy(ctx):
    """The shipped weights (lambda_b200/data) against the FP64 transfer matrix."""
    surrogate.install(ctx)
    rng = np.random.default_rng(5)
    n = 100000
    q = np.stack([rng.uniform(380, 780, n), rng.uniform(0, 1, n), rng.uniform(150, 850, n),
                  rng.uniform(1.2, 1.8, n), rng.uniform(1.0, 2.0, n)], 1).astype(np.float32)
    a, b = ctx.surrogate_eval(q), ctx.thinfilm_fp64(q)
    e = np.abs((a[:, 0] + a[:, 1]) / 2 - (b[:, 0] + b[:, 1]) / 2)
    print(f"R error vs FP64: mean {e.mean():.2e}, p99 {np.quantile(e, 0.99):.2e}, max {e.max():.2e}")
    assert e.mean() < 3e-3 and np.quantile(e, 0.99) < 2e-2


def _bare_substrate_r(q):
    """(R_s + R_p) / 2 of air over the bare substrate (Fresnel, no film): what a
    renderer without a thin-film model would use."""
    c0 = q[:, 1].astype(np.float64)
    ns = q[:, 4].astype(np.float64)
    ct = np.sqrt(np.maximum(1 - (1 - c0 * c0) / (ns * ns), 0))
    rs = ((c0 - ns * ct) / (c0 + ns * ct)) ** 2
    rp = ((ns * c0 - ct) / (ns * c0 + ct)) ** 2
    return (rs + rp) / 2


def test_trained_network_gain(ctx):
    """What training buys: the shipped network's error on R against the FP64
    transfer matrix, beside (a) the same network untrained (its initial weights)
    and (b) dropping the film (bare-substrate Fresnel), the model a renderer
    without the thin-film term would use."""
    rng = np.random.default_rng(8)
    n = 100000
    q = np.stack([rng.uniform(380, 780, n), rng.uniform(0.05, 1, n), rng.uniform(150, 850, n),
                  rng.uniform(1.2, 1.8, n), rng.uniform(1.0, 2.0, n)], 1).astype(np.float32)
    fp64 = ctx.thinfilm_fp64(q)
    want = (fp64[:, 0] + fp64[:, 1]) / 2

    def err(out):
        return float(np.abs((out[:, 0] + out[:, 1]) / 2 - want).mean())

    surrogate.install(ctx)
    trained = err(ctx.surrogate_eval(q))
    # untrained: the initialisation the training kernels start from (one epoch at a
    # learning rate of 1e-12 leaves it in place)
    rep = ctx.surrogate_train(samples=1 << 16, epochs=1, batch=8192, lr=1e-12, seed=11)
    untrained = err(ctx.surrogate_eval(q))
    bare = float(np.abs(_bare_substrate_r(q) - want).mean())
    surrogate.install(ctx)
    print(f"mean |R - R_fp64|: trained {trained:.2e}, untrained {untrained:.2e}, no film {bare:.2e}; "
          f"untrained audit {rep.mean_abs_error:.2e}")
    assert trained < 0.1 * bare
    assert trained < 0.05 * untrained


def test_surrogate_render_unbiased(scene_dir, ctx):
    """A noisy render differs from the exact form's by no more than a second exact
    render (another seed) does, plus 1%; the image means agree within 2%."""
    surrogate.install(ctx)
    sc = scenes.thinfilm_spheres(scene_dir, 96, 54, 256, name="s_thinfilm.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    exact_a = ctx.render(scene.render_desc(seed=3, flags=lb.RENDER_THINFILM_EXACT))
    exact_b = ctx.render(scene.render_desc(seed=4, flags=lb.RENDER_THINFILM_EXACT))
    sur_b = ctx.render(scene.render_desc(seed=4, flags=lb.RENDER_THINFILM_SURROGATE))
    st = ctx.stats()
    floor = rel_rmse(exact_b, exact_a)
    err = rel_rmse(sur_b, exact_a)
    ratio = float(sur_b.mean() / exact_b.mean())
    print(f"relRMSE vs exact(seed 3): surrogate {err:.4f}, exact(seed 4) {floor:.4f}; mean ratio {ratio:.4f}; "
          f"thin-film hits {st.thinfilm_hits}, exact fallback {st.thinfilm_fallback}")
    assert np.isfinite(sur_b).all()
    assert st.thinfilm_hits > 0 and st.thinfilm_fallback < 0.05 * st.thinfilm_hits
    assert err <= floor + 0.01
    assert abs(ratio - 1) < 0.02


def test_surrogate_render_outside_domain_is_exact(scene_dir, ctx):
    """Films thicker than the surrogate's trained box (900-1000 nm against 150-850 nm)
    are all evaluated by the exact FP32 transfer matrix inside the surrogate's scatter
    kernel, so the render equals the exact render bit for bit and every thin-film hit
    counts as a fallback. A box that straddles the limit (700-1000 nm) sends only part
    of the hits there."""
    surrogate.install(ctx)
    sc = scenes.thinfilm_spheres(scene_dir, 64, 36, 16, thickness="worley 900 1000 3", name="s_thick.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    exact = ctx.render(scene.render_desc(seed=5, flags=lb.RENDER_THINFILM_EXACT))
    sur = ctx.render(scene.render_desc(seed=5, flags=lb.RENDER_THINFILM_SURROGATE))
    st = ctx.stats()
    assert st.thinfilm_hits > 0 and st.thinfilm_fallback == st.thinfilm_hits
    assert np.array_equal(sur, exact, equal_nan=True)

    sc = scenes.thinfilm_spheres(scene_dir, 64, 36, 16, thickness="worley 700 1000 3", name="s_mixed.lrd")
    scene = lb.HostScene.parse(sc.lrd)
    ctx.upload(scene)
    ctx.render(scene.render_desc(seed=5, flags=lb.RENDER_THINFILM_SURROGATE))
    st = ctx.stats()
    print(f"straddling box: {st.thinfilm_fallback} of {st.thinfilm_hits} thin-film hits exact")
    assert 0 < st.thinfilm_fallback < st.thinfilm_hits
