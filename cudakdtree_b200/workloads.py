"""Seeded synthetic inputs with the shapes and value distributions of the
five benchmark configurations (the reference publishes no dataset; these
generators stand in for its inputs).

All generators are numpy-only and deterministic for a given seed.
"""
from __future__ import annotations

import numpy as np

# record dtypes (byte layouts described to the C ABI by cudakdtree_b200.Layout)
PAYLOAD_PACKED = np.dtype([("p", np.float32, (3,)), ("payload", np.uint32)])  # 16 B
POINT_DIM3 = np.dtype({"names": ["p", "dim"], "formats": [(np.float32, (3,)), np.int32],
                       "offsets": [0, 12], "itemsize": 16})


def uniform_points(n, D=3, seed=1, dtype=np.float32):
    """U[0,1)^D points (config 1: 1M float3, seed 1; queries seed 2)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.random((n, D), dtype=np.float64).astype(dtype)


def gmm_centres(num_components=64, D=3, seed=3):
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.random((num_components, D))


def gmm_points(n, D=3, num_components=64, sigma=0.01, seed=3, sample_seed=None):
    """Gaussian mixture: centres U[0,1)^D (seed), equal weights, isotropic
    sigma, not clamped (config 2: 10M points seed 3, queries seed 4)."""
    centres = gmm_centres(num_components, D, seed)
    rng = np.random.Generator(np.random.MT19937(seed if sample_seed is None else sample_seed))
    comp = rng.integers(0, num_components, size=n)
    pts = centres[comp] + rng.normal(0.0, sigma, size=(n, D))
    return pts.astype(np.float32)


def mixed_queries(n, frac_mixture=0.7, seed=6, centre_seed=3, D=3):
    """70% from the mixture, 30% uniform (config 4 inference queries)."""
    nm = int(round(n * frac_mixture))
    a = gmm_points(nm, D=D, seed=centre_seed, sample_seed=seed)
    b = uniform_points(n - nm, D=D, seed=seed + 1000)
    q = np.concatenate([a, b])
    rng = np.random.Generator(np.random.MT19937(seed + 2000))
    return q[rng.permutation(n)]


def packed_records(points):
    """{float3 p; uint32 payload} with payload = input index (dim bits 30..31
    left zero for the builder to fill): config 2's 16-byte record."""
    rec = np.zeros(len(points), PAYLOAD_PACKED)
    rec["p"] = points
    rec["payload"] = np.arange(len(points), dtype=np.uint32)
    return rec


def batched_sizes(num_clouds=4096, lo=256, hi=65536, seed=5):
    """Cloud sizes floor(exp(U[ln lo, ln hi])) (config 3)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=num_clouds))).astype(np.int64)


def batched_clouds(num_clouds=4096, queries_per_cloud=1024, seed=5, lo=256, hi=65536):
    """Concatenated points/queries with CSR offsets (config 3): each cloud
    uniform in its own unit cube."""
    sizes = batched_sizes(num_clouds, lo, hi, seed)
    rng = np.random.Generator(np.random.MT19937(seed + 1))
    pts = rng.random((int(sizes.sum()), 3), dtype=np.float64).astype(np.float32)
    qs = rng.random((num_clouds * queries_per_cloud, 3), dtype=np.float64).astype(np.float32)
    offs = np.zeros(num_clouds + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    qoffs = np.arange(num_clouds + 1, dtype=np.int64) * queries_per_cloud
    return pts, offs, qs, qoffs


def wide_float4(n, seed=7):
    """xyz U[0,1), w ~ N(0,1) (config 5, float4 part)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    p = np.empty((n, 4), np.float32)
    p[:, :3] = rng.random((n, 3), dtype=np.float64)
    p[:, 3] = rng.normal(0.0, 1.0, size=n)
    return p


def int3_points(n, seed=8, extent=1 << 20):
    """int3 uniform in [-2^20, 2^20]^3 (config 5, int3 part)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.integers(-extent, extent + 1, size=(n, 3), dtype=np.int64).astype(np.int32)


def tie_heavy(n, D=3, levels=6, seed=11):
    """Coordinates drawn from a handful of values: many exact ties."""
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.integers(0, levels, size=(n, D)).astype(np.float32)


def unique_ints(n, D, seed=12, dtype=np.float32):
    """Shuffled unique integers as coordinates: the tie-free inputs of the
    reference's builders-same-result test (testing/testBuildersSameResult.cu:96-110)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.permutation(n * D).reshape(n, D).astype(dtype)
