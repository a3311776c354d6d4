"""The learned pruning-radius model (no counterpart in the reference): gradients of the GPU
backward kernels against the CPU restatement (oracle/seed_numpy.py), training quality, exactness of
seeded queries (the radius only prunes), the fallback when a radius is wrong, checkpoints, what the
trained model saves in traversal work, and the per-query radius hint (the exact distances as hint
give the least work any radius can give)."""
import numpy as np
import pytest
import torch

from ebgeometry_b200 import SeedModel, TriMeshSDF
from ebgeometry_b200 import workloads as W
from oracle import seed_numpy as SN

pytestmark = pytest.mark.gpu


def test_gradients_match_cpu_oracle():
    log2t = 10
    lo, hi = np.array([-1.0, -1.0, -1.0]), np.array([1.0, 1.0, 1.0])
    m = SeedModel.create(log2_table=log2t, base_resolution=4, max_resolution=64, lo=lo, hi=hi, rng_seed=3)
    T = 16 * (1 << log2t) * 2
    rng = np.random.default_rng(0)
    table = rng.uniform(-0.5, 0.5, T).astype(np.float32)
    params = np.zeros(SN.NPARAM, np.float32)
    params[SN.W1:SN.B1] = rng.uniform(-0.4, 0.4, 64 * 32)
    params[SN.B1:SN.W2] = rng.uniform(-0.1, 0.1, 64)
    params[SN.W2:SN.B2] = rng.uniform(-0.3, 0.3, 64 * 64)
    params[SN.B2:SN.W3] = rng.uniform(-0.1, 0.1, 64)
    params[SN.W3:SN.B3] = rng.uniform(-0.3, 0.3, 64 * 64)
    params[SN.B3:SN.W4] = rng.uniform(-0.1, 0.1, 64)
    params[SN.W4:SN.B4] = rng.uniform(-0.3, 0.3, 64)
    params[SN.B4] = 0.05
    m.set_params(table, params)
    pts = rng.uniform(-1.1, 1.1, (96, 3)).astype(np.float32)  # a few outside the domain (clamped)
    tgt = rng.uniform(-0.8, 0.8, 96).astype(np.float32)
    loss, gt, gp = m.gradients(pts, tgt, 0.05, T)
    res, dense = SN.levels(4, 64, log2t)
    scale = (1.0 / (hi - lo)).astype(np.float32).astype(np.float64)
    lref, gt_ref, gp_ref, _ = SN.loss_and_grads(pts.astype(np.float64), tgt.astype(np.float64), table, params,
                                                lo.astype(np.float32).astype(np.float64), scale, res, dense, log2t, 0.05)
    assert loss == pytest.approx(lref, rel=2e-2)
    # BF16 operands in the backward products: agreement to ~1% of the gradient norm, per block
    for name, a, b in (("W1", SN.W1, SN.B1), ("b1", SN.B1, SN.W2), ("W2", SN.W2, SN.B2), ("b2", SN.B2, SN.W3),
                       ("W3", SN.W3, SN.B3), ("b3", SN.B3, SN.W4), ("w4", SN.W4, SN.B4), ("b4", SN.B4, SN.NPARAM)):
        ref = gp_ref[a:b]
        rel = np.linalg.norm(gp[a:b] - ref) / max(np.linalg.norm(ref), 1e-12)
        assert rel < 3e-2, (name, rel)
    rel = np.linalg.norm(gt - gt_ref) / np.linalg.norm(gt_ref)
    assert rel < 3e-2, ("table", rel)


@pytest.fixture(scope="module")
def trained():
    v, f = W.displaced_icosphere(5, 1)
    mesh = TriMeshSDF(v, f)
    seed = SeedModel.train(mesh, num_samples=1 << 21, steps=600, batch=1 << 16, rng_seed=1,
                           lo=[-1.25] * 3, hi=[1.25] * 3)
    return mesh, seed


def test_training_quality(trained):
    mesh, seed = trained
    r = seed.report()
    assert r["coverage"] >= 0.99
    assert r["mean_abs_err"] < 0.02
    assert r["train_samples"] == 1 << 21
    # the model as a far-field surrogate: its error, judged by the exact method, is reported
    assert np.isfinite(r["max_abs_err_far"])


def test_seeded_queries_are_exact_and_cheaper(trained):
    mesh, seed = trained
    p = torch.from_numpy(np.concatenate([W.grid_points(96, -1.25, 1.25),
                                         W.band_points(*W.displaced_icosphere(5, 1), 100000, 4)])).cuda()
    d0, s0 = mesh.stats(p)
    d1, s1 = mesh.stats(p, seed=seed)
    d0, d1 = d0.cpu().numpy(), d1.cpu().numpy()
    err = np.abs(d0 - d1)
    assert err.max() <= 1e-6 * mesh.diagonal
    out = np.abs(d0) > 1e-4 * mesh.diagonal
    assert np.all(np.sign(d0[out]) == np.sign(d1[out]))
    assert np.mean(d0 == d1) > 0.999
    # what the trained network gains over the plain traversal (printed; -s shows it): it must never
    # cost work, and its radius must hold for almost every query
    gain = {k: 1.0 - s1[k] / max(s0[k], 1) for k in ("nodes_visited", "leaves_visited", "triangles_tested")}
    print("seed gain (fraction of traversal work saved):", gain, "fallbacks:", s1["seed_fallbacks"])
    assert s1["nodes_visited"] <= 1.02 * s0["nodes_visited"], (s0, s1)
    assert s1["triangles_tested"] <= 1.02 * s0["triangles_tested"], (s0, s1)
    assert s1["seed_fallbacks"] < 0.02 * p.shape[0]


def test_wrong_radius_falls_back(trained):
    mesh, seed = trained
    bad = SeedModel.create(log2_table=12, base_resolution=4, max_resolution=32, lo=[-1.25] * 3, hi=[1.25] * 3)
    table, params = bad.get_params(16 * (1 << 12) * 2)
    params[:] = 0.0  # predicts 0 everywhere: the radius is only the distance to the packet centroid
    bad.set_params(params=params)
    p = torch.from_numpy(W.uniform_points(20000, 5)).cuda()
    d0 = mesh.signed_distance(p).cpu().numpy()
    d1, st = mesh.stats(p, seed=bad)
    d1 = d1.cpu().numpy()
    assert np.abs(d0 - d1).max() <= 1e-6 * mesh.diagonal
    assert np.mean(d0 == d1) > 0.999
    assert st["seed_fallbacks"] > 10000  # most radii held no triangle and were traversed again


def test_checkpoint_roundtrip(trained, tmp_path):
    mesh, seed = trained
    path = tmp_path / "seed.bin"
    seed.save(path)
    again = SeedModel.load(path)
    p = torch.from_numpy(W.uniform_points(5000, 6)).cuda()
    assert torch.equal(seed.predict(p), again.predict(p))
    assert again.report()["alpha"] == seed.report()["alpha"]


def test_radius_hint_exact_distances(trained):
    mesh, _ = trained
    p = torch.from_numpy(W.grid_points(64, -1.25, 1.25)).cuda()
    d0, s0 = mesh.stats(p)
    hint = d0.abs() * (1 + 1e-5) + 1e-6
    d1, s1 = mesh.stats(p, radius_hint=hint)
    assert torch.equal(d0, d1)
    assert s1["seed_fallbacks"] == 0
    assert s1["nodes_visited"] <= s0["nodes_visited"]
    print("exact-radius gain:", 1 - s1["nodes_visited"] / s0["nodes_visited"], 1 - s1["triangles_tested"] / s0["triangles_tested"])
    # a hint below |d| only costs a second traversal
    d2, s2 = mesh.stats(p, radius_hint=hint * 0.5)
    assert torch.equal(d0, d2) and s2["seed_fallbacks"] > 0
