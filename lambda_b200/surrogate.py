"""Thin-film surrogate weights: the trained BF16 MLP that stands in for the
transfer matrix, stored next to the package as surrogate_weights.npz."""

from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "surrogate_weights.npz")


def install(ctx, path: str = WEIGHTS) -> None:
    """Loads trained weights and their input range into a context."""
    from . import _native as N

    if not os.path.exists(path):
        raise FileNotFoundError(f"{path}: no trained surrogate weights")
    z = np.load(path)
    r = N.FilmRange()
    for k in ("lambda_nm", "cos_theta", "thickness_nm", "n_film", "n_sub"):
        getattr(r, k)[:] = tuple(float(x) for x in z[k])
    ctx.surrogate_set(z["params"], r)
