"""Learned kNN-radius proposal: gradients of the hand-written backward pass
against the CPU oracle (oracle/mlp_oracle.py), results identical to the plain
traversal, and what the trained network gains over the plain method."""
import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from cudakdtree_b200 import workloads as wl
from oracle import mlp_oracle
from oracle import pyoracle as po
from tests.helpers import f32_bits

pytestmark = pytest.mark.gpu

LAYOUT = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)


def _tree(n, seed=3):
    pts = wl.gmm_points(n, seed=seed)
    rec = torch.from_numpy(wl.packed_records(pts).view(np.int32).reshape(n, 4).copy()).cuda()
    wb = ck.build_tree(rec, layout=LAYOUT)
    return pts, rec, wb


@pytest.mark.parametrize("quantile", [0.0, 0.8])
def test_gradients_match_cpu_oracle(quantile):
    _, rec, wb = _tree(20000)
    m = ck.RadiusModel(seed=7, quantile=quantile)
    m.set_grid(rec, LAYOUT, wb)
    q = torch.from_numpy(wl.mixed_queries(3000, seed=11)).cuda()
    f = m.features(q)
    t = torch.randn(3000, generator=torch.Generator().manual_seed(0)).cuda()
    g, p, loss = m.gradients(f, t)
    ref_loss, ref_g = mlp_oracle.loss_and_grad(p, f.cpu().numpy(), t.cpu().numpy(),
                                               quantile=quantile)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    # FP32 accumulation vs float64: relative to the gradient's scale
    scale = np.abs(ref_g).max()
    assert np.max(np.abs(g - ref_g)) <= 2e-4 * scale


def test_training_reduces_loss_and_forward_matches_oracle():
    _, rec, wb = _tree(50000)
    m = ck.RadiusModel(seed=1)
    qtrain = torch.from_numpy(wl.gmm_points(20000, seed=3, sample_seed=21)).cuda()
    m.set_grid(rec, LAYOUT, wb)
    _, _, kth = ck.knn(rec, qtrain, 8, "cct", layout=LAYOUT, world_bounds=wb, with_max=True)
    f = m.features(qtrain)
    t_raw = 0.5 * torch.log(kth)
    t = (t_raw - t_raw.mean()) / t_raw.std(unbiased=False)
    _, _, loss0 = m.gradients(f, t)
    loss = m.train(qtrain, kth, epochs=8, batch=2048, lr=3e-3)
    assert loss < 0.5 * loss0
    # the model's radius prediction is its forward pass de-standardised
    _, p, _ = m.gradients(f, t)
    y, _ = mlp_oracle.forward(p, f.cpu().numpy().astype(np.float64))
    r = m.predict(qtrain).cpu().numpy()
    mean, std = float(t_raw.mean()), float(t_raw.std(unbiased=False))
    assert np.allclose(np.log(r), y * std + mean, rtol=0, atol=2e-3)


@pytest.mark.parametrize("k", [2, 8, 16, 32])
@pytest.mark.parametrize("method", ["stack_based", "stack_free", "cct"])
def test_learned_results_identical_to_plain(k, method):
    n = 200000
    _, rec, wb = _tree(n)
    m = ck.RadiusModel(seed=2)
    m.fit(rec, torch.from_numpy(wl.gmm_points(50000, seed=3, sample_seed=31)).cuda(), k,
          layout=LAYOUT, world_bounds=wb, epochs=6, batch=4096)
    q = torch.from_numpy(wl.mixed_queries(100000, seed=41)).cuda()
    pi, pd = ck.knn(rec, q, k, method, layout=LAYOUT, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(rec, q, k, m, method, layout=LAYOUT, world_bounds=wb)
    assert torch.equal(li, pi)
    assert np.array_equal(f32_bits(ld.cpu().numpy()), f32_bits(pd.cpu().numpy()))
    # and with the reference traversal order everywhere
    ri, rd = ck.knn(rec, q, k, method, layout=LAYOUT, world_bounds=wb, reference_order=True)
    assert torch.equal(li, ri)


def test_learned_radius_with_tiny_scale_falls_back_and_stays_exact():
    """A radius far too small sends (almost) every query to the plain path;
    the results must not change."""
    _, rec, wb = _tree(50000)
    m = ck.RadiusModel(seed=3)
    m.fit(rec, torch.from_numpy(wl.gmm_points(20000, seed=3, sample_seed=5)).cuda(), 16,
          layout=LAYOUT, world_bounds=wb, epochs=2)
    q = torch.from_numpy(wl.mixed_queries(20000, seed=6)).cuda()
    pi, pd = ck.knn(rec, q, 16, layout=LAYOUT, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(rec, q, 16, m, layout=LAYOUT, world_bounds=wb, scale=1e-3)
    assert int(fb[0]) > 19000
    assert torch.equal(li, pi) and torch.equal(ld, pd)


def test_learned_on_tie_heavy_tree_stays_exact():
    """Points on a coarse integer lattice: whole groups of neighbours share
    one squared distance, so the k-th boundary is tied for most queries;
    every tied query must come back in the reference's own order."""
    n = 60000
    pts = wl.tie_heavy(n, levels=12, seed=4) * np.float32(0.05)
    rec = torch.from_numpy(wl.packed_records(pts).view(np.int32).reshape(n, 4).copy()).cuda()
    wb = ck.build_tree(rec, layout=LAYOUT)
    m = ck.RadiusModel(seed=6)
    m.fit(rec, torch.from_numpy(wl.uniform_points(20000, seed=13) * np.float32(0.55)).cuda(),
          16, layout=LAYOUT, world_bounds=wb, epochs=2)
    q = torch.from_numpy(wl.uniform_points(20000, seed=14) * np.float32(0.55)).cuda()
    for method in ("stack_based", "stack_free", "cct"):
        ri, rd = ck.knn(rec, q, 16, method, layout=LAYOUT, world_bounds=wb, reference_order=True)
        for scale in (1.2, 3.0):
            li, ld, fb, _ = ck.knn_learned(rec, q, 16, m, method, layout=LAYOUT,
                                           world_bounds=wb, scale=scale)
            assert torch.equal(li, ri)
            assert np.array_equal(f32_bits(ld.cpu().numpy()), f32_bits(rd.cpu().numpy()))


def test_trained_network_reduces_work():
    """What the trained network gains: every query the learned pass answers
    visits no more nodes than the plain search does (the radius only adds
    culling), fewer on average, with identical answers; the share of
    queries re-run stays small."""
    n = 1000000
    _, rec, wb = _tree(n)
    m = ck.RadiusModel(grid_res=64, seed=4)
    m.fit(rec, torch.from_numpy(wl.mixed_queries(200000, seed=51)).cuda(), 16,
          layout=LAYOUT, world_bounds=wb, epochs=20, batch=4096)
    q = torch.from_numpy(wl.mixed_queries(200000, seed=52)).cuda()
    # the plain fast path with visit counting: an infinite radius scale
    pi, pd, _, v_plain = ck.knn_learned(rec, q, 16, m, layout=LAYOUT, world_bounds=wb,
                                        scale=1e30, visits=True)
    li, ld, fb, v_learn, st = ck.knn_learned(rec, q, 16, m, layout=LAYOUT, world_bounds=wb,
                                             scale=1.2, visits=True, status=True)
    assert torch.equal(li, pi) and torch.equal(ld, pd)
    answered = st == 0
    frac_fallback = 1.0 - answered.double().mean().item()
    assert abs(frac_fallback - int(fb[0]) / q.shape[0]) < 1e-9
    assert torch.all(v_learn[answered] <= v_plain[answered])
    vp = v_plain[answered].double().mean().item()
    vl = v_learn[answered].double().mean().item()
    print(f"fallback {frac_fallback:.3f}  visits of answered queries: plain {vp:.1f} "
          f"learned {vl:.1f}  final loss {m.final_loss:.4f}")
    assert frac_fallback < 0.25
    assert vl < vp


def test_trained_network_predicts_the_kth_distance():
    """What training gives the range traversal: the trained network's radius
    is close to each query's exact k-th distance (so the ball holds few
    more than k points and few queries fall back), where the untrained
    network's is not; both return the plain answers."""
    n = 1000000
    _, rec, wb = _tree(n)
    q = torch.from_numpy(wl.mixed_queries(100000, seed=53)).cuda()
    _, _, kth = ck.knn(rec, q, 16, layout=LAYOUT, world_bounds=wb, with_max=True)
    true_r = torch.sqrt(kth)
    untrained = ck.RadiusModel(grid_res=64, seed=4)
    untrained.set_grid(rec, LAYOUT, wb)
    trained = ck.RadiusModel(grid_res=64, seed=4)
    trained.fit(rec, torch.from_numpy(wl.mixed_queries(200000, seed=51)).cuda(), 16,
                layout=LAYOUT, world_bounds=wb, epochs=20, batch=4096)
    ratio_t = (trained.predict(q) / true_r).log().abs()
    ratio_u = (untrained.predict(q) / true_r).log().abs()
    within_t = (ratio_t < np.log(1.25)).double().mean().item()
    within_u = (ratio_u < np.log(1.25)).double().mean().item()
    print(f"share of radii within 25% of the k-th distance: trained {within_t:.3f} "
          f"untrained {within_u:.3f}")
    assert within_t > 0.8 and within_u < 0.2
    pi, pd = ck.knn(rec, q, 16, layout=LAYOUT, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(rec, q, 16, trained, layout=LAYOUT, world_bounds=wb)
    assert torch.equal(li, pi) and torch.equal(ld, pd)
    assert int(fb[0]) < 0.2 * q.shape[0]


F4_RECORD = np.dtype({"names": ["p", "dim"], "formats": [(np.float32, (4,)), np.int32],
                      "offsets": [0, 16], "itemsize": 32})
F4_LAYOUT = ck.layout_for("float32", 4, stride=32, dim_offset=16, dim_bits=32)


@pytest.mark.parametrize("k", [16, 64])
def test_learned_float4_wide_records_identical_to_plain(k):
    """Config 5's float part: {float4; int dim} records (the reference's
    32-byte layout) with widest-extent dims; a 4-D model (4 coordinates +
    a 4-D grid density) seeds the fused kernel (k = 16) or the heap kernel
    (k = 64); answers equal the plain path's and the reference order's."""
    n = 200000
    pts = wl.wide_float4(n, seed=7)
    rec = np.zeros(n, F4_RECORD)
    rec["p"] = pts
    d = torch.from_numpy(rec.view(np.uint8)).cuda()
    wb = ck.build_tree(d, layout=F4_LAYOUT)
    m = ck.RadiusModel(grid_res=16, seed=3, quantile=0.9, num_dims=4)
    m.fit(d, torch.from_numpy(wl.wide_float4(40000, seed=8)).cuda(), k, layout=F4_LAYOUT,
          world_bounds=wb, epochs=5)
    q = torch.from_numpy(wl.wide_float4(30000, seed=9)).cuda()
    pi, pd = ck.knn(d, q, k, layout=F4_LAYOUT, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(d, q, k, m, layout=F4_LAYOUT, world_bounds=wb)
    assert torch.equal(li, pi)
    assert np.array_equal(f32_bits(ld.cpu().numpy()), f32_bits(pd.cpu().numpy()))
    ri, rd = ck.knn(d, q, k, layout=F4_LAYOUT, world_bounds=wb, reference_order=True)
    assert torch.equal(li, ri)
    assert int(fb[0]) < 0.3 * q.shape[0]


@pytest.mark.parametrize("k", [8, 64])
def test_learned_int3_identical_to_plain(k):
    """Config 5's integer part: int3 points in [-2^20, 2^20]^3, exact int64
    distances; the model learns on integer queries and seeds the integer
    kernel with a radius rounded to an int64 bound."""
    n = 300000
    pts = wl.int3_points(n)
    d = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(d)
    m = ck.RadiusModel(grid_res=32, seed=4, quantile=0.9)
    m.fit(d, torch.from_numpy(wl.int3_points(50000, seed=11)).cuda(), k, world_bounds=wb,
          epochs=5)
    q = torch.from_numpy(wl.int3_points(40000, seed=12)).cuda()
    pi, pd = ck.knn(d, q, k, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(d, q, k, m, world_bounds=wb)
    assert torch.equal(li, pi) and torch.equal(ld, pd)
    ri, rd = ck.knn(d, q, k, world_bounds=wb, reference_order=True)
    assert torch.equal(li, ri) and torch.equal(ld, rd)
    assert int(fb[0]) < 0.3 * q.shape[0]


def test_learned_float2_fused_identical_to_plain():
    n = 300000
    pts = wl.uniform_points(n, D=2, seed=21)
    d = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(d)
    m = ck.RadiusModel(grid_res=128, seed=5, num_dims=2)
    m.fit(d, torch.from_numpy(wl.uniform_points(50000, D=2, seed=22)).cuda(), 16,
          world_bounds=wb, epochs=5)
    q = torch.from_numpy(wl.uniform_points(50000, D=2, seed=23)).cuda()
    pi, pd = ck.knn(d, q, 16, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(d, q, 16, m, world_bounds=wb)
    assert torch.equal(li, pi)
    assert np.array_equal(f32_bits(ld.cpu().numpy()), f32_bits(pd.cpu().numpy()))
