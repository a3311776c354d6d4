"""The learned pruning-radius model (no counterpart in the reference): gradients of the GPU
backward kernels against the CPU restatement (oracle/seed_numpy.py), training quality, exactness of
seeded queries (the model's radius only prunes: queries start from per-cell entry cuts of the tree),
the traversal work the trained model must save, the fallback when a radius is wrong, the attach
options (radius from the model, none or exact; anchors on or off) giving identical answers, a refit
dropping the cuts, checkpoints, and the per-query radius hint (the exact distances as hint give the
least work any radius can give)."""
import numpy as np
import pytest
import torch

from ebgeometry_b200 import EbgError, SeedModel, TriMeshSDF
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
    assert loss == pytest.approx(lref, rel=1e-3)
    # The oracle rounds to BF16 where the kernels do (weights, activations, and the deltas that enter
    # the gradient products as tensor-core operands), so what remains is FP32 accumulation order
    # and the odd BF16 rounding that lands on the other side of a tie because the device's FP32
    # input differs from the oracle's FP64 one in the last bits: 5e-3 of each block's norm.
    for name, a, b in (("W1", SN.W1, SN.B1), ("b1", SN.B1, SN.W2), ("W2", SN.W2, SN.B2), ("b2", SN.B2, SN.W3),
                       ("W3", SN.W3, SN.B3), ("b3", SN.B3, SN.W4), ("w4", SN.W4, SN.B4), ("b4", SN.B4, SN.NPARAM)):
        ref = gp_ref[a:b]
        rel = np.linalg.norm(gp[a:b] - ref) / max(np.linalg.norm(ref), 1e-12)
        print(f"gradient block {name}: relative error {rel:.2e}")
        assert rel < 5e-3, (name, rel)
    rel = np.linalg.norm(gt - gt_ref) / np.linalg.norm(gt_ref)
    print(f"gradient table: relative error {rel:.2e}")
    assert rel < 5e-3, ("table", rel)


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


def _workload(n_grid=96, n_band=100000):
    v, f = W.displaced_icosphere(5, 1)
    return torch.from_numpy(np.concatenate([W.grid_points(n_grid, -1.25, 1.25), W.band_points(v, f, n_band, 4)])).cuda()


def _packet_work(s):
    """What a packet's warp executes, per packet: stack pops, interior nodes, oriented boxes and
    triangle passes."""
    pk = max(s["packets"], 1)
    return {k: s[k] / pk for k in ("packet_pops", "packet_nodes", "packet_boxes", "packet_triangles")}


def test_seeded_queries_are_exact_and_cheaper(trained):
    mesh, seed = trained
    p = _workload()
    d0, s0 = mesh.stats(p)
    d1, s1 = mesh.stats(p, seed=seed)
    # the seeded traversal returns the plain traversal's answers, bit for bit (also when the plain
    # path's option of a shared-memory top tree is passed, which seeded packets do not use)
    assert torch.equal(d0, d1)
    assert torch.equal(mesh.signed_distance(p, seed=seed, top_nodes=21), d0)
    w0, w1 = _packet_work(s0), _packet_work(s1)
    print("packet work plain:", w0, "seeded:", w1, "cut packets:", s1["cut_packets"] / s1["packets"],
          "fallbacks:", s1["seed_fallbacks"])
    # what the trained model must save: most packets start from a cut, and the warps open far fewer
    # interior nodes and test fewer boxes and triangles
    assert s1["cut_packets"] >= 0.8 * s1["packets"]
    assert w1["packet_nodes"] <= 0.6 * w0["packet_nodes"], (w0, w1)
    assert w1["packet_boxes"] <= 0.9 * w0["packet_boxes"], (w0, w1)
    assert w1["packet_triangles"] <= 0.95 * w0["packet_triangles"], (w0, w1)
    assert s1["seed_fallbacks"] < 0.01 * p.shape[0]


def test_seeded_fp64_queries_equal_plain(trained):
    """FP64 points, every query re-evaluated in FP64: with the model attached, FP64 packets whose
    bounds lie within their cell's radius start from the cell's cut, the rest from the root; the
    results equal the plain FP64 call's bit for bit, near the surface and far from it."""
    mesh, seed = trained
    v, f = W.displaced_icosphere(5, 1)
    p = np.concatenate([W.grid_points(48, -1.25, 1.25), W.band_points(v, f, 50000, 5)]).astype(np.float64)
    pd = torch.from_numpy(p).cuda()
    d0 = mesh.signed_distance(pd)
    d1 = mesh.signed_distance(pd, seed=seed)
    torch.cuda.synchronize()
    mesh.check_status()
    assert d0.dtype == torch.float64 and torch.equal(d0, d1)


def test_seeded_queries_outside_the_models_domain(trained):
    """Points outside the model's domain ([-1.25, 1.25]^3 here) and packets straddling its edge
    have no cell: they start from the root, and every result equals the plain traversal's."""
    mesh, seed = trained
    rng = np.random.default_rng(71)
    far = rng.uniform(-4.0, 4.0, size=(200000, 3)).astype(np.float32)
    edge = rng.uniform(1.1, 1.4, size=(50000, 3)).astype(np.float32) * rng.choice([-1.0, 1.0], size=(50000, 3)).astype(np.float32)
    p = torch.from_numpy(np.concatenate([far, edge])).cuda()
    d0 = mesh.signed_distance(p)
    d1, st = mesh.stats(p, seed=seed)
    assert torch.equal(d0, d1)
    assert st["cut_packets"] < st["packets"]  # some packets had no cell to start from


def test_seeded_queries_in_a_cuda_graph(trained):
    """The seeded query path (ordering, the cut-started traversal with its bulk copies, the
    cut-started FP64 band pass) issues only stream-ordered work: captured once in a CUDA graph and
    replayed, it gives the plain traversal's results."""
    mesh, seed = trained
    p = _workload(48, 20000)
    d0 = mesh.signed_distance(p)
    out = torch.empty_like(d0)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            mesh.signed_distance(p, out=out, seed=seed, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        mesh.signed_distance(p, out=out, seed=seed, stream=s)
    out.zero_()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    mesh.check_status()
    assert torch.equal(out, d0)


def test_wrong_radius_falls_back(trained):
    mesh, seed = trained
    bad = SeedModel.create(log2_table=12, base_resolution=4, max_resolution=32, lo=[-1.25] * 3, hi=[1.25] * 3)
    table, params = bad.get_params(16 * (1 << 12) * 2)
    params[:] = 0.0  # predicts 0 everywhere: each cell's radius is only the cell's half-diagonal
    bad.set_params(params=params)
    p = torch.from_numpy(W.grid_points(64, -1.25, 1.25)).cuda()  # packets compact enough to fit cells
    d0 = mesh.signed_distance(p)
    try:
        mesh.attach_seed(bad, anchors=False)
        d1, st = mesh.stats(p, seed=bad)
        assert torch.equal(d0, d1)
        assert st["cut_packets"] > 0
        assert st["seed_fallbacks"] > 0  # radii that held no triangle: traversed again from the root
    finally:
        mesh.attach_seed(seed)


def test_attach_options_give_identical_answers(trained):
    mesh, seed = trained
    p = _workload(48, 20000)
    d0 = mesh.signed_distance(p)
    try:
        for mode in (0, 1, 2):
            for anchors in (True, False):
                rep = mesh.attach_seed(seed, cells_per_axis=24, max_entries=40, radius_mode=mode, anchors=anchors)
                assert rep["cells"] == 24 ** 3 and rep["max_entries"] == 40
                assert torch.equal(mesh.signed_distance(p, seed=seed), d0), (mode, anchors)
    finally:
        mesh.attach_seed(seed)


def test_unattached_model_is_rejected_and_refit_drops_cuts():
    v, f = W.displaced_icosphere(3, 2)
    mesh = TriMeshSDF(v, f)
    seed = SeedModel.train(mesh, num_samples=1 << 16, steps=50, batch=1 << 12, rng_seed=2, attach=False)
    p = torch.from_numpy(W.uniform_points(5000, 3)).cuda()
    with pytest.raises(EbgError):
        mesh.signed_distance(p, seed=seed)
    mesh.attach_seed(seed)
    d = mesh.signed_distance(p, seed=seed)
    assert torch.equal(d, mesh.signed_distance(p))
    mesh.refit(v)  # the cuts were cut from the old boxes: a refit drops them
    with pytest.raises(EbgError):
        mesh.signed_distance(p, seed=seed)
    mesh.attach_seed(seed)
    assert torch.equal(mesh.signed_distance(p, seed=seed), d)


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
