"""The allocation-free surrogate entry point (lambda_surrogate_eval_static).

It exists for callers that must not allocate device memory where they evaluate
films, such as a renderer inside a host application that owns all device memory
through its own pool and forbids cudaMalloc on its render thread. This file is
named to run last, so a failure here never hides the other tests. It passes
alone in a fresh process as well as after the rest of the suite.
"""

import ctypes as C

import numpy as np
import pytest

from lambda_b200 import _native as N
from lambda_b200 import surrogate

pytestmark = pytest.mark.gpu

LIMIT = 131072  # LAMBDA_SURROGATE_STATIC_MAX_QUERIES


def _queries(n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(380, 780, n), rng.uniform(0, 1, n), rng.uniform(150, 850, n),
                     rng.uniform(1.2, 1.8, n), rng.uniform(1.0, 2.0, n)], 1).astype(np.float32)


def test_static_scratch_matches_allocating_entry_point(ctx):
    import torch

    surrogate.install(ctx)
    fn = ctx._lib.lambda_surrogate_eval_static
    # two calls in a row: the second must not see the first call's scratch contents
    for seed, n in ((1, 40000), (2, 1234)):
        q = _queries(n, seed)
        want = ctx.surrogate_eval(q)  # the allocating entry point
        dq = torch.from_numpy(q).cuda()
        dout = torch.full((n, 4), float("nan"), dtype=torch.float32, device="cuda")
        st = fn(ctx._h, C.c_void_p(dq.data_ptr()), n, C.c_void_p(dout.data_ptr()))
        assert st == 0, ctx.last_error
        got = dout.cpu().numpy()
        scale = np.abs(want).max()
        err = np.abs(got - want)
        # same tolerance as the tensor-core inference test: the two paths differ only in
        # where the input encoding is computed (host libm vs device sincosf)
        assert err.max() <= 1e-2 * scale and err.mean() <= 1e-3 * scale, (err.max(), err.mean())


def test_static_scratch_rejects_oversized_batches(ctx):
    import torch

    surrogate.install(ctx)
    fn = ctx._lib.lambda_surrogate_eval_static
    dq = torch.zeros((4, 5), dtype=torch.float32, device="cuda")
    dout = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    st = fn(ctx._h, C.c_void_p(dq.data_ptr()), LIMIT + 1, C.c_void_p(dout.data_ptr()))
    assert st == 1 and "131072" in ctx.last_error
    host = np.zeros((4, 5), np.float32)
    st = fn(ctx._h, C.c_void_p(host.ctypes.data), 4, C.c_void_p(dout.data_ptr()))
    assert st == 1 and "device pointers" in ctx.last_error
