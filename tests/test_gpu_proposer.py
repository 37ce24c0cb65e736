"""Learned tile proposer: its hand-written kernels against the numpy oracle
(oracle/cnn_oracle.py), and the tile-masked alignment against the full one.

Tolerances (FP32 kernels against FP64 numpy): forward values and gradients
within 1e-4 of the largest magnitude of the compared array; tile scores and
their argmax exact (the oracle is fed the device's own logits); bf16
activation storage within 3e-2.  Masked runs: bit-exact against the
unmasked run whenever the mask holds every tile the full path uses.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import parflexdtw_b200 as pf  # noqa: E402
from parflexdtw_b200 import _lib, workloads as W  # noqa: E402
from parflexdtw_b200.prune import (FPP, STRIDES, TileProposer, _needs_fallback,  # noqa: E402
                                   _p, _pruned_near_path, tiles_on_path)
from oracle import cnn_oracle as CO  # noqa: E402

STD = [(1, 1), (1, 2), (2, 1)]
WTS = [2.0, 3.0, 3.0]
TOL = 1e-4


def close(a, b, tol=TOL):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= tol * scale


def test_pooled_cost_vs_oracle():
    rng = np.random.default_rng(0)
    F1, F2 = W.warped_pair(rng, 1003, 1210)
    f1, f2 = torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda()
    got = TileProposer.pooled_cost(f1, f2, center=False).cpu().numpy()
    ref = CO.pooled_cost(CO.pool_features(F1, 16), CO.pool_features(F2, 16))
    assert got.shape == ref.shape == (63, 76)
    assert np.abs(got - ref).max() < 1e-5
    # the pooled map is the block mean of the full cost matrix
    C = W.cost_matrix_det(F1, F2)
    assert abs(got[3, 5] - C[48:64, 80:96].mean()) < 1e-5
    cen = TileProposer.pooled_cost(f1, f2).cpu().numpy()
    assert np.abs(cen - CO.center(ref)).max() < 1e-3


@pytest.mark.parametrize("cin,cout,stride,relu,H,W", [(1, 32, 2, 1, 37, 51), (32, 32, 2, 1, 19, 23),
                                                      (32, 1, 1, 0, 17, 30), (3, 5, 1, 1, 16, 16),
                                                      (1, 32, 4, 1, 70, 61), (2, 3, 4, 0, 9, 13)])
def test_conv_forward_backward_vs_oracle(cin, cout, stride, relu, H, W):
    rng = np.random.default_rng(cin * 100 + cout)
    x = rng.standard_normal((cin, H, W)).astype(np.float32)
    w = (rng.standard_normal((cout, cin, 3, 3)) * 0.3).astype(np.float32)
    b = (rng.standard_normal(cout) * 0.1).astype(np.float32)
    xd, wd, bd = (torch.from_numpy(a).cuda() for a in (x, w, b))
    Ho, Wo = (H - 1) // stride + 1, (W - 1) // stride + 1
    y = torch.empty((cout, Ho, Wo), dtype=torch.float32, device="cuda")
    lib = _lib.load()
    s = pf.plan.current_stream_ptr()
    _lib.check(lib.pfx_conv3x3_forward(_p(xd), 0, cin, H, W, _p(wd), _p(bd), cout, stride, relu,
                                       _p(y), 0, s))
    yref = CO.conv3x3(x, w, b, stride, relu)
    assert close(y.cpu().numpy(), yref)
    dy = rng.standard_normal(yref.shape).astype(np.float32)
    dyd = torch.from_numpy(dy).cuda()
    dx = torch.empty_like(xd)
    dw = torch.zeros_like(wd)
    db = torch.zeros_like(bd)
    _lib.check(lib.pfx_conv3x3_backward(_p(xd), cin, H, W, _p(wd), cout, stride, _p(y), relu,
                                        _p(dyd), _p(dx), _p(dw), _p(db), s))
    rdx, rdw, rdb = CO.conv3x3_backward(x, w, stride, y.cpu().numpy(), relu, dy)
    assert close(dx.cpu().numpy(), rdx)
    assert close(dw.cpu().numpy(), rdw)
    assert close(db.cpu().numpy(), rdb)
    # bf16 storage of the output (inference)
    yb = torch.empty((cout, Ho, Wo), dtype=torch.bfloat16, device="cuda")
    _lib.check(lib.pfx_conv3x3_forward(_p(xd), 0, cin, H, W, _p(wd), _p(bd), cout, stride, relu,
                                       _p(yb), 1, s))
    assert close(yb.float().cpu().numpy(), yref, 3e-2)


def test_network_gradients_vs_oracle():
    """Loss and every parameter gradient of the whole proposer (three convs,
    tile max, weighted BCE) against the numpy chain on the same input."""
    rng = np.random.default_rng(3)
    F1, F2 = W.warped_pair(rng, 2600, 3100, pad_frac=0.1)
    N, M, L = F1.shape[1], F2.shape[1], 500
    net = TileProposer(seed=1)
    pooled = net.pooled_cost(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda())
    hop = L - 1
    n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
    label = (rng.random((n1, n2)) < 0.3).astype(np.uint8)
    loss, grads = net.gradients(pooled, label, N, M, L, pos_weight=3.0)
    P = {k: v.cpu().numpy().astype(np.float64) for k, v in net.params.items()}
    x0 = pooled.cpu().numpy()[None].astype(np.float64)
    a1 = CO.conv3x3(x0, P["w1"], P["b1"], STRIDES[0], 1)
    a2 = CO.conv3x3(a1, P["w2"], P["b2"], STRIDES[1], 1)
    a3 = CO.conv3x3(a2, P["w3"], P["b3"], STRIDES[2], 0)
    logits = net.forward(pooled).cpu().numpy()
    assert close(logits, a3[0])
    score, arg = CO.tile_max(logits, n1, n2, hop, L, N, M, FPP)
    s_dev, a_dev, _ = net.tile_scores(net.forward(pooled), N, M, L)
    assert np.array_equal(s_dev.cpu().numpy(), score.astype(np.float32))
    assert np.array_equal(a_dev.cpu().numpy(), arg)
    rl, ds = CO.bce(score, label.reshape(-1), 3.0)
    assert abs(float(loss.item()) - rl) <= 1e-5 * abs(rl)
    d3 = np.zeros_like(a3[0]).reshape(-1)
    np.add.at(d3, arg, ds)
    d3 = d3.reshape(1, *a3.shape[1:])
    dx2, dw3, db3 = CO.conv3x3_backward(a2, P["w3"], STRIDES[2], a3, 0, d3)
    dx1, dw2, db2 = CO.conv3x3_backward(a1, P["w2"], STRIDES[1], a2, 1, dx2)
    _, dw1, db1 = CO.conv3x3_backward(x0, P["w1"], STRIDES[0], a1, 1, dx1)
    for k, ref in (("w3", dw3), ("b3", db3), ("w2", dw2), ("b2", db2), ("w1", dw1), ("b1", db1)):
        assert close(grads[k].cpu().numpy(), ref, 1e-3), k


def test_adam_and_training_lower_the_loss():
    rng = np.random.default_rng(5)
    pairs = [W.warped_pair(rng, n, int(n * 1.1), pad_frac=0.1) for n in (2500, 3300)]
    net = TileProposer(seed=2)
    net.init_optimizer()
    data = []
    for F1, F2 in pairs:
        N, M = F1.shape[1], F2.shape[1]
        best, wp = pf.parflex(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, L=400, profile_dir=None)
        data.append((net.pooled_cost(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda()),
                     tiles_on_path(wp, N, M, 400), N, M))
    losses = []
    for ep in range(30):
        tot = 0.0
        for pooled, lab, N, M in data:
            loss, g = net.gradients(pooled, lab, N, M, 400, pos_weight=4.0)
            net.step(g, lr=3e-3)
            tot += float(loss.item())
        losses.append(tot)
    assert losses[-1] < 0.7 * losses[0], losses[::5]
    # one Adam update against its formula
    p = torch.tensor([1.0, -2.0], device="cuda")
    gr = torch.tensor([0.5, 0.25], device="cuda")
    m = torch.zeros(2, device="cuda")
    v = torch.zeros(2, device="cuda")
    _lib.check(_lib.load().pfx_adam_step(_p(p), _p(gr), _p(m), _p(v), 2, 0.1, 0.9, 0.999, 1e-8, 1,
                                         pf.plan.current_stream_ptr()))
    ref = np.array([1.0, -2.0]) - 0.1 * np.sign([0.5, 0.25])
    assert np.abs(p.cpu().numpy() - ref).max() < 1e-6


def test_tile_mask_with_full_tiles_is_exact():
    rng = np.random.default_rng(7)
    F1, F2 = W.warped_pair(rng, 3000, 3400, pad_frac=0.1)
    N, M, L = F1.shape[1], F2.shape[1], 400
    f1, f2 = torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda()
    plan = pf.Plan(N, M, L, STD, WTS)
    plan.load_features(f1, f2)
    plan.run(None, 0.1)
    best, end, _, n = plan.result()
    wp = plan.path(n)
    D_full = plan.host("D_ARR")
    # all tiles set: identical to the unmasked run
    plan.set_tile_mask(np.ones((plan.n1, plan.n2), np.uint8))
    plan.load_features(f1, f2)
    plan.run(None, 0.1)
    b2, e2, _, n2 = plan.result()
    assert b2 == best and e2 == end and np.array_equal(plan.path(n2), wp)
    assert np.array_equal(plan.host("D_ARR"), D_full)
    # the path's tiles and a ring of one tile: same path, fewer tiles
    lab = tiles_on_path(wp, N, M, L).astype(bool)
    ring = np.pad(lab, 1)
    dil = np.zeros_like(lab)
    for di in range(3):
        for dj in range(3):
            dil |= ring[di:di + lab.shape[0], dj:dj + lab.shape[1]]
    assert dil.sum() < lab.size
    for mask in (dil, torch.from_numpy(dil.astype(np.uint8)).cuda()):
        plan.set_tile_mask(mask)
        plan.set_warps(16)
        plan.load_features(f1, f2)
        plan.run(None, 0.1)
        b3, e3, _, n3 = plan.result()
        assert b3 == best and e3 == end and np.array_equal(plan.path(n3), wp)
        assert not _needs_fallback(plan.path(n3), dil, N, M, L)
    plan.set_tile_mask(None)


def test_parflex_pruned_equals_full_and_falls_back():
    rng = np.random.default_rng(8)
    F1, F2 = W.warped_pair(rng, 4200, 4600, pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    best, wp = pf.parflex(C, STD, WTS, 0.1, L=500, profile_dir=None)
    # an untrained network proposes little: the fallback must give the full path
    net = TileProposer(seed=4)
    b1, wp1, info = pf.parflex_pruned(F1, F2, STD, WTS, 0.1, 500, proposer=net, threshold=50.0)
    assert info["fallback"] and b1 == best and np.array_equal(wp1, wp)
    # a threshold that keeps everything: no fallback, same result
    b2, wp2, info2 = pf.parflex_pruned(F1, F2, STD, WTS, 0.1, 500, proposer=net, threshold=-1e30)
    assert not info2["fallback"] and info2["tiles_run"] == info2["tiles_total"]
    assert b2 == best and np.array_equal(wp2, wp)


@pytest.mark.parametrize("cost", ["tile", "slabs"])
def test_batch_masks_and_pruned_batch_exact(oracle_mod, cost):
    """Masked batches: all-ones masks and path-dilated masks reproduce the
    unmasked results bit for bit; PrunedBatch (any proposer) returns the
    full-tile results, through its fallback when needed.  With the cost
    built inside stage 1 ("tile") or by separate cost kernels ("slabs")."""
    from parflexdtw_b200.batch import Batch
    rng = np.random.default_rng(12)
    sizes = [(2600, 2900), (1800, 1500), (3100, 3300)]
    pairs = [W.warped_pair(rng, n, m, pad_frac=0.1) for n, m in sizes]
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    L = 300
    refs = [oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, L)
            for F1, F2 in pairs]
    b = Batch(shapes, L, STD, WTS, 12, warps=4, cost=cost)
    assert b.cost_in_kernel == (cost == "tile")
    b.load(pairs)
    grids = [(-(-(n - 1) // (L - 1)), -(-(m - 1) // (L - 1))) for n, m in shapes]
    ones = torch.ones(sum(a * c for a, c in grids), dtype=torch.uint8, device="cuda")
    b.set_masks(ones)
    b.run(0.1, use_graph=False)
    best, end, lens = b.results()
    paths = b.paths(lens)
    for i, r in enumerate(refs):
        assert best[i] == r["best_cost"] and np.array_equal(paths[i].T, r["wp"])
    dil, labs = [], []
    for (n, m), r in zip(shapes, refs):
        lab = tiles_on_path(r["wp"], n, m, L).astype(bool)
        labs.append(lab.reshape(-1))
        p = np.pad(lab, 1)
        d = np.zeros_like(lab)
        for di in range(3):
            for dj in range(3):
                d |= p[di:di + lab.shape[0], dj:dj + lab.shape[1]]
        dil.append(d.reshape(-1))
    masks = torch.from_numpy(np.concatenate(dil).astype(np.uint8)).cuda()
    assert int(masks.sum()) < masks.numel()
    b.set_masks(masks)
    for use_graph in (False, True):
        b.run(0.1, use_graph=use_graph)
        best, end, lens = b.results()
        paths = b.paths(lens)
        for i, r in enumerate(refs):
            assert best[i] == r["best_cost"] and np.array_equal(paths[i].T, r["wp"])
    # completion after a masked run reuses the kept tiles and leaves the
    # batch's masked state (queues, graph) intact
    rng = np.random.default_rng(3)
    sparse = torch.from_numpy((rng.random(masks.numel()) < 0.4).astype(np.uint8)).cuda()
    # the device path check and row-layout paths against the host statement
    # (masks of the path tiles alone: the paths pass near pruned tiles)
    on_path = torch.from_numpy(np.concatenate(labs).astype(np.uint8)).cuda()
    b.set_masks(on_path)
    b.run(0.1, use_graph=False)
    near, flags = b.check_paths(32)
    _, end_s, lens_s = b.results()
    rows = b.paths_rows(lens_s)
    pts = b.paths(lens_s)
    near, flags, sp = near.cpu().numpy(), flags.cpu().numpy(), on_path.cpu().numpy()
    offs = np.concatenate([[0], np.cumsum([a * c for a, c in grids])])
    n_near = 0
    for i, (n, m) in enumerate(shapes):
        assert np.array_equal(rows[i], pts[i].T)
        mk = sp[offs[i]:offs[i + 1]].reshape(grids[i]).astype(bool)
        want = _pruned_near_path(rows[i], mk, n, m, L, 32)
        got = near[offs[i]:offs[i + 1]].reshape(grids[i]).astype(bool)
        assert np.array_equal(got, want)
        assert bool(flags[i]) == bool(want.any())
        n_near += int(want.sum())
    assert n_near > 0
    # adding tiles in steps: the path tiles' neighbourhood, then the rest
    b.set_masks(sparse)
    b.run(0.1, use_graph=True)
    for i, r in enumerate(refs):
        bc, wp = b.complete(i, 0.1, dil[i].reshape(grids[i]))
        assert bc == r["best_cost"] and np.array_equal(wp.T, r["wp"])
        bc, wp = b.complete(i, 0.1)
        assert bc == r["best_cost"] and np.array_equal(wp.T, r["wp"])
    for m in (sparse, masks):
        b.set_masks(m)
        b.run(0.1, use_graph=True)
        for i, r in enumerate(refs):
            bc, wp = b.complete(i, 0.1)
            assert bc == r["best_cost"] and np.array_equal(wp.T, r["wp"])
    b.run(0.1, use_graph=True)
    best, end, lens = b.results()
    paths = b.paths(lens)
    for i, r in enumerate(refs):
        assert best[i] == r["best_cost"] and np.array_equal(paths[i].T, r["wp"])
    b.close()
    net = TileProposer(seed=6)
    for thr in (-1e30, 1e30):  # everything kept / nothing kept (all fall back)
        pb = pf.PrunedBatch(shapes, L, STD, WTS, 12, proposer=net, threshold=thr, cost=cost)
        pb.load(pairs)
        out, info = pb.run(0.1)
        for (bc, wp), r in zip(out, refs):
            assert bc == r["best_cost"] and np.array_equal(wp, r["wp"])
        assert (info["fallbacks"] == 3) == (thr > 0)
        pb.close()


def test_pruned_batch_cost_fma_equals_full_tiles(oracle_mod):
    """Learned pruning over an FMA-cost batch: every path equals the full-tile
    FMA-cost result, which equals the oracle's on the oracle's fma-chain cost."""
    from parflexdtw_b200.batch import Batch
    rng = np.random.default_rng(44)
    sizes = [(2600, 2900), (1800, 1500), (3100, 3300)]
    pairs = [W.warped_pair(rng, n, m, pad_frac=0.1) for n, m in sizes]
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    L = 300
    refs = [oracle_mod.parflex_full(oracle_mod.cost_matrix_fma(F1, F2), STD, WTS, 0.1, L)
            for F1, F2 in pairs]
    full = Batch(shapes, L, STD, WTS, 12, cost_fma=True)
    full.load(pairs)
    full.run(0.1)
    best, end, lens = full.results()
    paths = full.paths(lens)
    for i, r in enumerate(refs):
        assert best[i] == r["best_cost"] and np.array_equal(paths[i].T, r["wp"])
    full.close()
    pb = pf.PrunedBatch(shapes, L, STD, WTS, 12, proposer=TileProposer.load(), cost_fma=True)
    pb.load(pairs)
    for _ in range(2):
        out, info = pb.run(0.1)
        for (bc, wp), r in zip(out, refs):
            assert bc == r["best_cost"] and np.array_equal(wp, r["wp"])
    pb.close()


def test_pruned_batch_host_pairs_upload_in_the_graph():
    """run(host_pairs=...) uploads each pair's page-locked features on its
    proposer stream inside the recorded graph: the results equal those of
    load() + run(), on the first (eager) run and on replays, and new contents
    of the same host buffers are picked up by the replay."""
    rng = np.random.default_rng(52)
    sizes = [(2600, 2900), (1800, 1500), (3100, 3300)]
    sets = [[W.warped_pair(rng, n, m) for n, m in sizes] for _ in range(2)]  # same shapes
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in sets[0]]
    L = 300
    net = TileProposer.load()
    want = []
    pb = pf.PrunedBatch(shapes, L, STD, WTS, 12, proposer=net)
    for pairs in sets:
        pb.load(pairs)
        out, _ = pb.run(0.1)
        want.append(out)
    pinned = [(torch.from_numpy(F1).pin_memory(), torch.from_numpy(F2).pin_memory())
              for F1, F2 in sets[0]]
    for k in (0, 0, 1, 0):
        for (h1, h2), (F1, F2) in zip(pinned, sets[k]):
            h1.copy_(torch.from_numpy(F1))
            h2.copy_(torch.from_numpy(F2))
        out, _ = pb.run(0.1, host_pairs=pinned)
        for (b1, w1), (b2, w2) in zip(out, want[k]):
            assert b1 == b2 and np.array_equal(w1, w2), k
    with pytest.raises(ValueError):
        pb.run(0.1, host_pairs=[(torch.from_numpy(F1), torch.from_numpy(F2))
                                for F1, F2 in sets[0]])  # not page-locked
    pb.close()


def test_trained_proposer_gain_on_held_out_pairs():
    """What the shipped, trained network gains over the method without it.

    Held-out pairs (a seed outside the training seeds 12345..17344 of
    train_proposer.py, drawn like the training pairs: N ~ U(20000, 30000),
    M = N x U(0.7, 1.4), 0-10 % unrelated padding per end), L = 2000.  The
    full-tile FP64 method gives the reference answer: every pruned result must
    equal its best cost and path bit for bit.  The trained proposer must skip more than
    half of the tiles, counting every tile its expansions and fallbacks ran;
    an untrained network of the same layout at the same threshold, which the
    same fallback keeps exact, must run more tiles than the trained one."""
    from parflexdtw_b200.batch import Batch
    from parflexdtw_b200.train_proposer import make_pairs
    L = 2000
    pairs = make_pairs(8, 90210, lo=20000, hi=30000)
    shapes = [(F1.shape[1], F2.shape[1]) for F1, F2 in pairs]
    full = Batch(shapes, L, STD, WTS, 12)
    full.load(pairs)
    full.run(0.1, use_graph=False)
    best, end, lens = full.results()
    paths = full.paths(lens)
    full.close()
    assert end[:, 6].all()
    trained = TileProposer.load()
    runs = {}
    for name, net in (("trained", trained), ("untrained", TileProposer(seed=3))):
        pb = pf.PrunedBatch(shapes, L, STD, WTS, 12, proposer=net, threshold=trained.threshold)
        pb.load(pairs)
        out, info = pb.run(0.1)
        pb.close()
        for i, (bc, wp) in enumerate(out):
            assert bc == best[i] and np.array_equal(wp, paths[i].T), (name, i, info)
        runs[name] = info
    t, u = runs["trained"], runs["untrained"]
    print(f"trained: {t['tiles_run']}/{t['tiles_total']} tiles run, proposed "
          f"{t['tiles_proposed']}, {t['expanded']} expanded, {t['fallbacks']} fallbacks; "
          f"untrained: {u['tiles_run']} tiles run, {u['fallbacks']} fallbacks")
    assert t["skipped_fraction"] > 0.5, t
    assert t["tiles_run"] < 0.5 * t["tiles_total"], t
    assert u["tiles_run"] > t["tiles_run"], (t, u)


@pytest.mark.parametrize("H,W,relu", [(19, 23, 1), (70, 61, 0), (33, 130, 1), (1, 5, 1)])
def test_conv_tensor_core_layer_vs_oracle(H, W, relu):
    """The 32 -> 32-channel stride-2 layer with bf16 activations in and out
    runs on the tensor cores (k_conv3x3_mma32, weights split into bf16 high and
    low parts): within bf16 output rounding of the oracle's convolution of the
    same bf16 inputs, and of the CUDA-core kernel's FP32-output result, on maps
    whose output tiles are partial."""
    rng = np.random.default_rng(H * 1000 + W)
    x = rng.standard_normal((32, H, W)).astype(np.float32)
    w = (rng.standard_normal((32, 32, 3, 3)) * 0.1).astype(np.float32)
    b = (rng.standard_normal(32) * 0.1).astype(np.float32)
    xb = torch.from_numpy(x).cuda().to(torch.bfloat16)
    xr = xb.float().cpu().numpy()  # the bf16 inputs, exactly
    wd, bd = torch.from_numpy(w).cuda(), torch.from_numpy(b).cuda()
    Ho, Wo = (H - 1) // 2 + 1, (W - 1) // 2 + 1
    y = torch.full((32, Ho, Wo), float("nan"), dtype=torch.bfloat16, device="cuda")
    lib = _lib.load()
    s = pf.plan.current_stream_ptr()
    _lib.check(lib.pfx_conv3x3_forward(_p(xb), 1, 32, H, W, _p(wd), _p(bd), 32, 2, relu,
                                       _p(y), 1, s))
    got = y.float().cpu().numpy()
    assert np.isfinite(got).all()
    yref = CO.conv3x3(xr, w, b, 2, relu)
    assert close(got, yref, 1e-2)
    # the CUDA-core kernel on the same inputs, FP32 output
    yf = torch.empty((32, Ho, Wo), dtype=torch.float32, device="cuda")
    _lib.check(lib.pfx_conv3x3_forward(_p(xb), 1, 32, H, W, _p(wd), _p(bd), 32, 2, relu,
                                       _p(yf), 0, s))
    assert close(yf.cpu().numpy(), yref)
    assert close(got, yf.cpu().numpy(), 1e-2)


def test_center_features_and_first_layer_vs_materialised_map():
    """pfx_pooled_center_features makes A^T B the centred, standardised map that
    pfx_pooled_center makes from 1 - A^T B (the pooled cost is bilinear), and
    pfx_conv3x3_forward_features gives the first layer of that map without
    storing it: both within FP32 rounding of the materialised path."""
    from parflexdtw_b200 import _lib
    from parflexdtw_b200.plan import current_stream_ptr
    rng = np.random.default_rng(5)
    F1, F2 = W.warped_pair(rng, 3301, 2950, pad_frac=0.1)
    f1, f2 = torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda()
    lib, s = _lib.load(), current_stream_ptr()
    d, N, M = 12, F1.shape[1], F2.shape[1]
    P1, P2 = -(-N // 16), -(-M // 16)
    A = torch.empty(d * P1, dtype=torch.float32, device="cuda")
    B = torch.empty(d * P2, dtype=torch.float32, device="cuda")
    _lib.check(lib.pfx_pool_features(f1.data_ptr(), d, N, 16, A.data_ptr(), s))
    _lib.check(lib.pfx_pool_features(f2.data_ptr(), d, M, 16, B.data_ptr(), s))
    want = TileProposer.pooled_cost(f1, f2)  # materialised, centred, standardised
    mom = torch.empty(int(lib.pfx_pooled_center_scratch(P1, P2)), dtype=torch.uint8,
                      device="cuda")
    _lib.check(lib.pfx_pooled_center_features(A.data_ptr(), B.data_ptr(), d, P1, P2,
                                              mom.data_ptr(), s))
    got = (A.reshape(d, P1).double().T @ B.reshape(d, P2).double()).float()
    assert close(got.cpu().numpy(), want.cpu().numpy(), 1e-4)
    # the centred map of the CPU oracle, computed in FP64
    ref = CO.center(CO.pooled_cost(CO.pool_features(F1, 16), CO.pool_features(F2, 16)))
    assert close(got.cpu().numpy(), ref, 1e-4)
    net = TileProposer.load()
    w, b = net.params["w1"], net.params["b1"]
    Ho, Wo = (P1 - 1) // 4 + 1, (P2 - 1) // 4 + 1
    y_feat = torch.empty((32, Ho, Wo), dtype=torch.float32, device="cuda")
    y_map = torch.empty_like(y_feat)
    _lib.check(lib.pfx_conv3x3_forward_features(A.data_ptr(), B.data_ptr(), d, P1, P2,
                                                w.data_ptr(), b.data_ptr(), 32, 4, 1,
                                                y_feat.data_ptr(), 0, s))
    _lib.check(lib.pfx_conv3x3_forward(want.data_ptr(), 0, 1, P1, P2, w.data_ptr(), b.data_ptr(),
                                       32, 4, 1, y_map.data_ptr(), 0, s))
    assert close(y_feat.cpu().numpy(), y_map.cpu().numpy(), 1e-4)


def test_propose_into_and_graph_replay_match_propose():
    """The preallocated, graph-captured proposer pass of PrunedBatch gives the
    masks of the allocating per-pair path (propose), on the eager first run
    and on later graph replays with other features in the same buffers.  The
    pass builds the network's input from the features instead of the stored
    map (FP32 rounding differs), so a tile whose score lies within 1e-3 of
    the threshold may go either way; every other tile must agree."""
    rng = np.random.default_rng(21)
    sizes = [(5200, 6100), (4100, 3900), (6000, 5300)]
    sets = [[W.warped_pair(rng, n, m) for n, m in sizes] for _ in range(2)]
    L = 500
    net = TileProposer.load()

    def per_pair(pairs):
        masks, clear = [], []
        for F1, F2 in pairs:
            f1, f2 = torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda()
            m, sc = net.propose(net.pooled_cost(f1, f2), f1.shape[1], f2.shape[1], L,
                                dilation=0)
            m1, _ = net.propose(net.pooled_cost(f1, f2), f1.shape[1], f2.shape[1], L)
            masks.append(m1.reshape(-1).cpu().numpy())
            # a dilated mask is decided by the scores in each tile's 3 x 3 neighbourhood
            near = np.abs(sc.cpu().numpy() - net.threshold) <= 1e-3
            p = np.pad(near, 1)
            nb = np.zeros_like(near)
            for di in range(3):
                for dj in range(3):
                    nb |= p[di:di + near.shape[0], dj:dj + near.shape[1]]
            clear.append(~nb.reshape(-1))
        return np.concatenate(masks), np.concatenate(clear)

    want = [per_pair(p) for p in sets]
    assert all(c.mean() > 0.9 for _, c in want)
    pb = pf.PrunedBatch(sizes, L, STD, WTS, 12, proposer=net)
    results = []
    for k in (0, 1, 0):
        pb.load(sets[k])
        out, _ = pb.run(0.1)
        m, clear = want[k]
        got = pb.last_masks.cpu().numpy()
        assert np.array_equal(got[clear], m[clear]), k
        results.append(out)
    for (b1, w1), (b3, w3) in zip(results[0], results[2]):
        assert b1 == b3 and np.array_equal(w1, w3)
    pb.close()
