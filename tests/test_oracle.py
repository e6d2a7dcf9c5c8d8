"""CPU tests: the oracle (oracle/cukd_oracle.c, a restatement of the
reference's algorithms) pinned against the reference's golden vectors and
against the reference itself (oracle/_ref, compiled from its headers).

These run without a GPU.  The GPU tests then compare the CUDA library with
this oracle.
"""
import hashlib
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _issue5_points():
    from tests.golden.make_golden import issue5_points
    return issue5_points()


# ---------------------------------------------------------------------------
# golden vectors
# ---------------------------------------------------------------------------
def test_issue5_points_match_the_reference_listing():
    """testing/issue5.cu:79-84 lists the first generated points."""
    pts = _issue5_points()
    listed = np.array([[-99.1088562, -87.9879150, 27.7626877],
                       [-38.3892326, 31.5713978, -37.0891457],
                       [-22.0435200, -92.5473785, 89.4833221],
                       [48.5274811, -94.0671997, 80.3888092],
                       [-33.9030113, 34.4157219, 95.2085953]], np.float32)
    assert np.allclose(pts[:5], listed, rtol=0, atol=2e-5)
    assert np.array_equal(pts[:5], _load("issue5.npz")["first5"])


def test_issue5_fcp_golden():
    """testing/issue5.cu:101-107: cut-off 5, closest squared distance
    2.8466301 (the reference prints it; here it is asserted bit-exactly)."""
    g = _load("issue5.npz")
    pts = _issue5_points()
    perm, _, bounds = po.build(pts)
    tree = pts[perm]
    assert _digest(tree) == str(g["tree_sha256"])
    assert np.array_equal(bounds, g["bounds"])
    q = g["query"]
    for m, ref_id in zip((po.STACK_BASED, po.STACK_FREE, po.CCT), g["fcp_ids"]):
        got = po.fcp(tree, q, m, bounds=bounds, cutoff=5.0)
        assert got[0] == ref_id
    p = tree[g["fcp_ids"][0]]
    d2 = np.float32(0)
    for d in range(3):
        diff = np.float32(p[d] - q[0, d])
        d2 = np.float32(d2 + np.float32(diff * diff))
    assert d2 == g["fcp_d2"] == np.float32(2.8466301)


@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("n", [4, 10, 1000, 10000])
def test_builders_same_result_golden(D, n):
    """testing/testBuildersSameResult.cu: unique integer coordinates."""
    from tests.golden.make_golden import unique_ints
    inp = unique_ints(n, D, seed=1000 * D + n)
    perm, _, _ = po.build(inp)
    assert np.array_equal(inp[perm], _load("same_result.npz")[f"D{D}_N{n}"])


@pytest.mark.parametrize("n", [1000, 15763])
def test_tie_heavy_build_golden(n):
    from tests.golden.make_golden import tie_points
    g = _load("ties.npz")
    pts = tie_points(n, 3, seed=n)
    perm, _, _ = po.build(pts)
    assert np.array_equal(perm, g[f"rr_N{n}_perm"])
    perm, dims, _ = po.build(pts, explicit_dim=True)
    assert np.array_equal(perm, g[f"ex_N{n}_perm"])
    assert np.array_equal(dims, g[f"ex_N{n}_dims"])


@pytest.mark.parametrize("kind", ["uniform", "tie"])
def test_queries_golden(kind):
    g = _load("knn.npz")
    rng = np.random.Generator(np.random.MT19937(77))
    if kind == "uniform":
        pts = rng.random((2000, 3)).astype(np.float32)
        q = (rng.random((300, 3)) * 1.2 - 0.1).astype(np.float32)
    else:
        from tests.golden.make_golden import tie_points
        pts = tie_points(2000, 3, seed=5)
        q = rng.integers(-1, 7, size=(300, 3)).astype(np.float32)
    perm, _, bounds = po.build(pts)
    tree = pts[perm]
    assert _digest(tree) == str(g[f"{kind}_tree_sha256"])
    for m in (po.STACK_BASED, po.STACK_FREE, po.CCT):
        assert np.array_equal(po.fcp(tree, q, m, bounds=bounds), g[f"{kind}_fcp_m{m}"])
        for lk, k in ((0, 1), (0, 8), (0, 16), (1, 20), (1, 50)):
            ids, d2, ret = po.knn(tree, q, k, m, bounds=bounds, list_kind=lk)
            key = f"{kind}_knn_m{m}_l{lk}_k{k}"
            assert np.array_equal(ids, g[key + "_ids"]), key
            assert np.array_equal(d2.view(np.uint32), g[key + "_d2"].view(np.uint32)), key
            assert np.array_equal(ret.view(np.uint32), g[key + "_ret"].view(np.uint32)), key


# ---------------------------------------------------------------------------
# live comparison with the reference (oracle/_ref) when it was built here
# ---------------------------------------------------------------------------
needs_ref = pytest.mark.skipif(po.ref_host() is None, reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 31, 100, 2049, 30000])
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("tie", [False, True])
@pytest.mark.parametrize("explicit", [False, True])
def test_build_matches_reference_host(n, D, tie, explicit):
    rng = np.random.Generator(np.random.MT19937(n * 10 + D))
    pts = (rng.integers(0, 6, size=(n, D)) if tie else rng.random((n, D))).astype(np.float32)
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    if explicit:
        code = {2: po.REF_F2_DIM, 3: po.REF_F3_DIM, 4: po.REF_F4_DIM}[D]
        rec = np.zeros(n, po.ref_record_dtype(code))
        rec["p"] = pts
        rec["dim"] = -1
        out, rb = po.ref_build_host(code, rec)
        assert np.array_equal(out["p"], pts[perm])
        assert np.array_equal(out["dim"], dims)
    else:
        code = {2: po.REF_F2, 3: po.REF_F3, 4: po.REF_F4}[D]
        out, rb = po.ref_build_host(code, pts)
        assert np.array_equal(out, pts[perm])
    assert np.array_equal(rb, bounds)


@needs_ref
@pytest.mark.parametrize("tie", [False, True])
@pytest.mark.parametrize("explicit", [False, True])
@pytest.mark.parametrize("cutoff", [np.inf, 0.07])
def test_queries_match_reference_host(tie, explicit, cutoff):
    rng = np.random.Generator(np.random.MT19937(5 + tie + 2 * explicit))
    n, nq = 5000, 2000
    pts = (rng.integers(0, 6, size=(n, 3)) if tie else rng.random((n, 3))).astype(np.float32)
    q = (rng.integers(-1, 7, size=(nq, 3)) if tie else rng.random((nq, 3)) * 1.2 - 0.1)
    q = q.astype(np.float32)
    if tie:
        cutoff = cutoff * 20
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    tree = pts[perm]
    if explicit:
        rec = np.zeros(n, po.ref_record_dtype(po.REF_F3_DIM))
        rec["p"] = tree
        rec["dim"] = dims
        code, d = po.REF_F3_DIM, dims
    else:
        rec, code, d = tree, po.REF_F3, None
    for m in (po.STACK_BASED, po.STACK_FREE, po.CCT):
        assert np.array_equal(po.fcp(tree, q, m, dims=d, bounds=bounds, cutoff=cutoff),
                              po.ref_fcp_host(code, rec, bounds, q, m, cutoff=cutoff))
        for lk, k in ((0, 4), (0, 16), (1, 20), (1, 64)):
            a = po.knn(tree, q, k, m, dims=d, bounds=bounds, cutoff=cutoff, list_kind=lk)
            r = po.ref_knn_host(code, rec, bounds, q, k, m, list_kind=lk, cutoff=cutoff)
            assert np.array_equal(a[0], r[0])
            assert np.array_equal(a[1].view(np.uint32), r[1].view(np.uint32))


@needs_ref
@pytest.mark.parametrize("eps", [0.25, 1.0])
def test_stack_free_eps_matches_reference_host(eps):
    rng = np.random.Generator(np.random.MT19937(9))
    pts = rng.random((5000, 3)).astype(np.float32)
    q = rng.random((2000, 3)).astype(np.float32)
    perm, _, bounds = po.build(pts)
    tree = pts[perm]
    assert np.array_equal(po.fcp(tree, q, po.STACK_FREE, bounds=bounds, eps=eps),
                          po.ref_fcp_host(po.REF_F3, tree, bounds, q, po.STACK_FREE, eps=eps))


# ---------------------------------------------------------------------------
# host-side logic
# ---------------------------------------------------------------------------
def test_subtree_sizes():
    """ArbitraryBinaryTree::numNodesInSubtree (helpers.h:161-177)."""
    for n in range(1, 200):
        for g in range(n):
            size = 0
            stack = [g]
            while stack:
                x = stack.pop()
                if x < n:
                    size += 1
                    stack += [2 * x + 1, 2 * x + 2]
            assert po.subtree_size(g, n) == size


def test_explicit_dims_need_bounds():
    """builder_thrust.h:469-473 throws without world bounds."""
    pts = np.zeros((4, 3), np.float32)
    import ctypes as C
    perm = np.zeros(4, np.int64)
    rc = po.lib().cko_build(0, 3, pts.ctypes.data_as(C.c_void_p), 4, 1,
                            perm.ctypes.data_as(C.c_void_p), None, None)
    assert rc == 2


def test_mlp_oracle_gradient_matches_finite_differences():
    """The MLP oracle's backward pass (the reference point for the GPU
    training kernels) against central finite differences."""
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mo.NP)
    f = rng.normal(0, 1, (16, mo.NIN))
    t = rng.normal(0, 1, 16)
    _, g = mo.loss_and_grad(p, f, t, bf16_act=False)
    for i in [0, 5, mo.OB1 + 3, mo.OW2 + 100, mo.OW2 + 4000, mo.OB2 + 7, mo.OW3 + 9, mo.OB3]:
        e = np.zeros(mo.NP)
        e[i] = 1e-6
        lp, _ = mo.loss_and_grad(p + e, f, t, bf16_act=False)
        lm, _ = mo.loss_and_grad(p - e, f, t, bf16_act=False)
        assert abs((lp - lm) / 2e-6 - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


@pytest.mark.parametrize("quantile", [0.3, 0.8])
def test_mlp_oracle_pinball_gradient_matches_finite_differences(quantile):
    """The pinball-loss gradient (quantile training) against central finite
    differences, away from the kinks (no target within the step of a
    prediction)."""
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, mo.NP)
    f = rng.normal(0, 1, (16, mo.NIN))
    y, _ = mo.forward(p, f, bf16_act=False)
    t = y + rng.choice([-1.0, 1.0], 16) * rng.uniform(0.1, 1.0, 16)
    _, g = mo.loss_and_grad(p, f, t, bf16_act=False, quantile=quantile)
    for i in [0, 5, mo.OB1 + 3, mo.OW2 + 100, mo.OW2 + 4000, mo.OB2 + 7, mo.OW3 + 9, mo.OB3]:
        e = np.zeros(mo.NP)
        e[i] = 1e-6
        lp, _ = mo.loss_and_grad(p + e, f, t, bf16_act=False, quantile=quantile)
        lm, _ = mo.loss_and_grad(p - e, f, t, bf16_act=False, quantile=quantile)
        assert abs((lp - lm) / 2e-6 - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_mlp_oracle_bf16_rounding():
    """The oracle's bf16 rounding (of the tensor-core operands) against
    torch's bfloat16 conversion, ties included."""
    import torch
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 3, 4000), [0.0, 1.0, -2.5, 1.00390625, 1.01171875]])
    x32 = x.astype(np.float32)
    ref = torch.from_numpy(x32).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(mo.bf16(x32).astype(np.float32), ref)


# ---------------------------------------------------------------------------
# the canonical-tree checker (used on trees too large to rebuild on the CPU)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("kind", ["uniform", "tie", "int"])
@pytest.mark.parametrize("explicit", [False, True])
def test_check_tree_accepts_oracle_builds(D, kind, explicit):
    rng = np.random.Generator(np.random.MT19937(D * 7 + len(kind)))
    n = 5003
    if kind == "uniform":
        pts = rng.random((n, D)).astype(np.float32)
    elif kind == "tie":
        pts = rng.integers(0, 4, size=(n, D)).astype(np.float32)
    else:
        pts = rng.integers(-50, 50, size=(n, D)).astype(np.int32)
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    assert po.check_tree(pts[perm], perm, dims if explicit else None,
                         bounds if explicit else None) == 0


@pytest.mark.parametrize("explicit", [False, True])
def test_check_tree_rejects_perturbed_trees(explicit):
    rng = np.random.Generator(np.random.MT19937(3))
    n = 3001
    pts = rng.integers(0, 5, size=(n, 3)).astype(np.float32)  # many ties
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    dm = dims if explicit else None
    bd = bounds if explicit else None
    tree, idx = pts[perm].copy(), perm.copy()
    # two nodes whose points differ
    i, j = 5, 2900
    assert not np.array_equal(tree[i], tree[j])
    t2, x2 = tree.copy(), idx.copy()
    t2[[i, j]] = t2[[j, i]]
    x2[[i, j]] = x2[[j, i]]
    assert po.check_tree(t2, x2, dm, bd) > 0
    # two nodes holding equal points: only the input-index tie-break differs
    eq = [(a, b) for a in range(n) for b in range(a + 1, min(n, a + 400))
          if np.array_equal(tree[a], tree[b]) and a != 0][:1]
    a, b = eq[0]
    x3 = idx.copy()
    x3[[a, b]] = x3[[b, a]]
    assert po.check_tree(tree, x3, dm, bd) > 0
    if explicit:
        d4 = dims.copy()
        d4[17] = (d4[17] + 1) % 3
        assert po.check_tree(tree, idx, d4, bounds) > 0


@pytest.mark.parametrize("explicit", [False, True])
def test_check_kd_accepts_valid_trees_and_rejects_broken_ones(explicit):
    """The k-d validity checker: every canonical tree passes, and so does a
    canonical tree with two equal points exchanged (a different but valid
    tree, which the canonical checker rejects); exchanging points that
    differ, or a wrong explicit dim, is caught."""
    rng = np.random.Generator(np.random.MT19937(11))
    n = 3001
    pts = rng.integers(0, 5, size=(n, 3)).astype(np.float32)
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    dm = dims if explicit else None
    bd = bounds if explicit else None
    tree = pts[perm].copy()
    assert po.check_kd(tree, dm, bd) == 0
    eq = [(a, b) for a in range(1, n) for b in range(a + 1, min(n, a + 400))
          if np.array_equal(tree[a], tree[b])][:1]
    a, b = eq[0]
    idx = perm.astype(np.int64)
    x2 = idx.copy()
    x2[[a, b]] = x2[[b, a]]
    assert po.check_kd(tree, dm, bd) == 0 and po.check_tree(tree, x2, dm, bd) > 0
    t3 = tree.copy()
    t3[[5, 2900]] = t3[[2900, 5]]
    assert not np.array_equal(tree[5], tree[2900])
    assert po.check_kd(t3, dm, bd) > 0
    if explicit:
        d4 = dims.copy()
        d4[17] = (d4[17] + 1) % 3
        assert po.check_kd(tree, d4, bounds) > 0


@needs_ref
@pytest.mark.parametrize("n", [1000, 40000])
def test_check_tree_accepts_reference_host_builds(n):
    """buildTree_host itself (unmodified reference code) passes the check,
    explicit dims and ties included: the checker states the reference's
    canonical order, not only this restatement's."""
    rng = np.random.Generator(np.random.MT19937(n))
    pts = rng.integers(0, 7, size=(n, 3)).astype(np.float32)
    rec = np.zeros(n, po.ref_record_dtype(po.REF_F3_PACKED))
    rec["p"] = pts
    rec["payload"] = np.arange(n, dtype=np.uint32)
    out, rb = po.ref_build_host(po.REF_F3_PACKED, rec)
    idx = (out["payload"] & 0x3FFFFFFF).astype(np.int64)
    dims = (out["payload"] >> 30).astype(np.int32)
    assert po.check_tree(np.ascontiguousarray(out["p"]), idx, dims, rb) == 0
    out2, _ = po.ref_build_host(po.REF_F3_PAYLOAD, rec.view(po.ref_record_dtype(po.REF_F3_PAYLOAD)))
    assert po.check_tree(np.ascontiguousarray(out2["p"]), out2["payload"].astype(np.int64)) == 0
