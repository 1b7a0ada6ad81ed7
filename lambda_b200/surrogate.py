"""Thin-film surrogate weights: the BF16 MLP that stands in for the transfer
matrix, trained on the GPU by the library's own kernels and stored next to the
package as data/surrogate_weights.npz (parameters, input range, training report).

  python -m lambda_b200.surrogate [out.npz]   trains (2^24 FP64-labelled samples)
                                               and writes the weights file
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "surrogate_weights.npz")
RANGE_KEYS = ("lambda_nm", "cos_theta", "thickness_nm", "n_film", "n_sub")


def encode(q: np.ndarray, film_range) -> np.ndarray:
    """The network's input encoding of queries [n, 5] = (lambda, cos, d, n_film, n_sub),
    in float32 like the library: (cos 2delta, sin 2delta, cos, n_film, n_sub) with
    2delta = 4 pi n_film d cos(theta_film) / lambda and the last three mapped to [-1, 1]."""
    q = np.asarray(q, np.float32)
    lam, c0, d, nf, ns = (q[:, i] for i in range(5))
    cf = np.sqrt(np.maximum(np.float32(1) - (np.float32(1) - c0 * c0) / (nf * nf), np.float32(0)))
    two_delta = np.float32(4.0 * 3.14159265358979) * nf * d * cf / lam
    lo = {k: np.float32(getattr(film_range, k)[0]) for k in RANGE_KEYS}
    hi = {k: np.float32(getattr(film_range, k)[1]) for k in RANGE_KEYS}

    def norm(v, k):
        return np.float32(2) * (v - lo[k]) / (hi[k] - lo[k]) - np.float32(1)

    return np.stack([np.cos(two_delta), np.sin(two_delta), norm(c0, "cos_theta"), norm(nf, "n_film"),
                     norm(ns, "n_sub")], 1).astype(np.float32)


def load(path: str = WEIGHTS):
    from . import _native as N

    if not os.path.exists(path):
        raise FileNotFoundError(f"{path}: no trained surrogate weights")
    z = np.load(path)
    r = N.FilmRange()
    for k in RANGE_KEYS:
        getattr(r, k)[:] = tuple(float(x) for x in z[k])
    return z["params"].astype(np.float32), r


def install(ctx, path: str = WEIGHTS) -> None:
    """Loads trained weights and their input range into a context."""
    params, r = load(path)
    ctx.surrogate_set(params, r)


def train_and_save(ctx, path: str = WEIGHTS, samples: int = 1 << 24, epochs: int = 24, batch: int = 8192,
                   lr: float = 3e-3, seed: int = 2024) -> dict:
    from . import default_film_range

    rng = default_film_range()
    rep = ctx.surrogate_train(samples=samples, epochs=epochs, batch=batch, lr=lr, seed=seed, film_range=rng)
    params, r = ctx.surrogate_get()
    info = {"samples": samples, "epochs": epochs, "batch": batch, "lr": lr, "seed": seed,
            "train_ms": rep.train_ms, "label_ms": rep.label_ms, "final_loss": rep.final_loss,
            "audit_max_abs_error": rep.max_abs_error, "audit_mean_abs_error": rep.mean_abs_error,
            "audit_samples": rep.audit_samples}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, params=params, report=json.dumps(info),
             **{k: np.array(getattr(r, k)[:], np.float32) for k in RANGE_KEYS})
    return info


if __name__ == "__main__":
    from . import Context

    out = sys.argv[1] if len(sys.argv) > 1 else WEIGHTS
    with Context(0) as c:
        print(json.dumps(train_and_save(c, out)))
