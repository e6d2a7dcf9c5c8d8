"""Generates the golden fixtures in this folder by running the reference's
own host code (ingowald/cudaKDTree compiled from its headers into
oracle/_ref/libcukd_ref_host.so by oracle/Makefile).

    python tests/golden/make_golden.py

Fixtures (numpy .npz, inputs regenerated from the seeds stored alongside):

  issue5.npz       testing/issue5.cu: 90,167 points from srand(33)/rand() (the
                   MSVC runtime's LCG, see msvc_rand) scaled to [-100,100]^3;
                   query (-98.4496613, 76.9219055,
                   25.8888512), cut-off 5.  Stores the reference's FCP answer
                   for all three traversals and a digest of its tree.
  same_result.npz  testing/testBuildersSameResult.cu: shuffled unique integers
                   as coordinates, D = 2/3/4, N = 4/10/1000/10000; the
                   reference buildTree_host output.
  ties.npz         tie-heavy inputs (coordinates in {0..5}): the reference's
                   point order (payload) for round-robin and widest-dim builds.
  knn.npz          kNN / FCP answers of the reference traversals on small
                   uniform and tie-heavy inputs, fixed and heap lists.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402


def msvc_rand(seed, count):
    """The C runtime rand() the reference's issue-5 numbers were produced
    with (the values listed in testing/issue5.cu:79-84 match it, glibc's do
    not): the published LCG x = x*214013 + 2531011 (mod 2^32), output
    (x >> 16) & 0x7fff, RAND_MAX = 32767."""
    out = np.empty(count, np.int64)
    x = seed & 0xFFFFFFFF
    for i in range(count):
        x = (x * 214013 + 2531011) & 0xFFFFFFFF
        out[i] = (x >> 16) & 0x7FFF
    return out


def issue5_points():
    """testing/issue5.cu:25-40: float(rand() * (2*100/RAND_MAX) - 100) per
    coordinate, x/y/z of point 0 first, seed 33, 90,167 points."""
    n = 90167
    r = msvc_rand(33, 3 * n).astype(np.float64)
    return (r * (2.0 * 100.0 / 32767.0) - 100.0).astype(np.float32).reshape(n, 3)


ISSUE5_QUERY = np.array([[-98.4496613, 76.9219055, 25.8888512]], np.float32)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def unique_ints(n, D, seed):
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.permutation(n * D).reshape(n, D).astype(np.float32)


def tie_points(n, D, seed):
    rng = np.random.Generator(np.random.MT19937(seed))
    return rng.integers(0, 6, size=(n, D)).astype(np.float32)


def payload_perm_rr(pts):
    rec = np.zeros(len(pts), po.ref_record_dtype(po.REF_F3_PAYLOAD))
    rec["p"] = pts
    rec["payload"] = np.arange(len(pts))
    out, b = po.ref_build_host(po.REF_F3_PAYLOAD, rec)
    return out["payload"].astype(np.int64), b


def payload_perm_explicit(pts):
    rec = np.zeros(len(pts), po.ref_record_dtype(po.REF_F3_PACKED))
    rec["p"] = pts
    rec["payload"] = np.arange(len(pts), dtype=np.uint32)
    out, b = po.ref_build_host(po.REF_F3_PACKED, rec)
    return ((out["payload"] & 0x3FFFFFFF).astype(np.int64), (out["payload"] >> 30).astype(np.int32),
            b)


def main():
    if po.ref_host() is None:
        raise SystemExit("build oracle/_ref first: make -C oracle")

    # ---- issue 5
    pts = issue5_points()
    tree, b = po.ref_build_host(po.REF_F3, pts)
    ids = [po.ref_fcp_host(po.REF_F3, tree, b, ISSUE5_QUERY, m, cutoff=5.0)[0]
           for m in (po.STACK_BASED, po.STACK_FREE, po.CCT)]
    p = tree[ids[0]]
    d2 = np.float32(0)
    for d in range(3):
        diff = np.float32(p[d] - ISSUE5_QUERY[0, d])
        d2 = np.float32(d2 + np.float32(diff * diff))
    np.savez_compressed(os.path.join(HERE, "issue5.npz"), first5=pts[:5], tree_sha256=digest(tree),
                        bounds=b, fcp_ids=np.array(ids, np.int32), fcp_d2=np.float32(d2),
                        query=ISSUE5_QUERY)
    print("issue5: ids", ids, "d2", d2)

    # ---- builders same result (unique ints)
    out = {}
    for D, code in ((2, po.REF_F2), (3, po.REF_F3), (4, po.REF_F4)):
        for n in (4, 10, 1000, 10000):
            inp = unique_ints(n, D, seed=1000 * D + n)
            tr, _ = po.ref_build_host(code, inp)
            out[f"D{D}_N{n}"] = tr
    np.savez_compressed(os.path.join(HERE, "same_result.npz"), **out)
    print("same_result:", len(out), "cases")

    # ---- tie-heavy builds
    out = {}
    for n in (1000, 15763):
        pts = tie_points(n, 3, seed=n)
        perm, _ = payload_perm_rr(pts)
        out[f"rr_N{n}_perm"] = perm.astype(np.int32)
        perm, dims, _ = payload_perm_explicit(pts)
        out[f"ex_N{n}_perm"] = perm.astype(np.int32)
        out[f"ex_N{n}_dims"] = dims.astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "ties.npz"), **out)
    print("ties:", len(out), "arrays")

    # ---- queries
    out = {}
    for kind in ("uniform", "tie"):
        rng = np.random.Generator(np.random.MT19937(77))
        if kind == "uniform":
            pts = rng.random((2000, 3)).astype(np.float32)
            q = (rng.random((300, 3)) * 1.2 - 0.1).astype(np.float32)
        else:
            pts = tie_points(2000, 3, seed=5)
            q = rng.integers(-1, 7, size=(300, 3)).astype(np.float32)
        tree, b = po.ref_build_host(po.REF_F3, pts)
        out[f"{kind}_tree_sha256"] = np.array(digest(tree))
        for m in (po.STACK_BASED, po.STACK_FREE, po.CCT):
            out[f"{kind}_fcp_m{m}"] = po.ref_fcp_host(po.REF_F3, tree, b, q, m)
            for lk, k in ((0, 1), (0, 8), (0, 16), (1, 20), (1, 50)):
                ids, d2, ret = po.ref_knn_host(po.REF_F3, tree, b, q, k, m, list_kind=lk)
                out[f"{kind}_knn_m{m}_l{lk}_k{k}_ids"] = ids
                out[f"{kind}_knn_m{m}_l{lk}_k{k}_d2"] = d2
                out[f"{kind}_knn_m{m}_l{lk}_k{k}_ret"] = ret
    np.savez_compressed(os.path.join(HERE, "knn.npz"), **out)
    print("knn:", len(out), "arrays")


if __name__ == "__main__":
    main()
