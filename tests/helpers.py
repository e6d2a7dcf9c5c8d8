"""Shared helpers for the parity tests (host side)."""
from __future__ import annotations

import numpy as np

from cudakdtree_b200 import workloads as wl


def make_points(n, D=3, kind="uniform", scalar="float32", seed=0):
    if kind == "uniform":
        p = wl.uniform_points(n, D, seed=seed + 1)
    elif kind == "tie":
        p = wl.tie_heavy(n, D, seed=seed + 11)
    elif kind == "gmm":
        p = wl.gmm_points(n, D, seed=3, sample_seed=seed + 100)
    elif kind == "unique":
        p = wl.unique_ints(n, D, seed=seed + 12)
    elif kind == "same":
        p = np.full((n, D), 0.25, np.float32)
    else:
        raise ValueError(kind)
    if scalar == "int32":
        if kind == "uniform":
            p = (p * 2000 - 1000).astype(np.int32)
        else:
            p = p.astype(np.int32)
    return np.ascontiguousarray(p)


def make_queries(nq, D=3, kind="uniform", scalar="float32", seed=0):
    if kind == "tie":
        rng = np.random.Generator(np.random.MT19937(seed + 77))
        q = rng.integers(-1, 7, size=(nq, D)).astype(np.float32)
    elif kind == "gmm":
        q = wl.gmm_points(nq, D, seed=3, sample_seed=seed + 200)
    else:
        rng = np.random.Generator(np.random.MT19937(seed + 55))
        q = (rng.random((nq, D)) * 1.2 - 0.1).astype(np.float32)
    if scalar == "int32":
        if kind == "uniform":
            q = (q * 2000 - 1000).astype(np.int32)
        else:
            q = q.astype(np.int32)
    return np.ascontiguousarray(q)


def f32_bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)
