"""The ray-cost MLP's tcgen05 kernels against the CPU oracle (oracle/mlp_np.py), its
training on the tracer's own per-ray logs, and the cost-binned launch order.

Tolerances: with dyadic inputs and weights every fp32 sum is exact, so predictions are
compared bit for bit (a wrong operand layout shows as O(1) errors). With encoded rays the
GPU and the oracle can round an activation to different bf16 neighbours after a last-bit
difference in an fp32 sum; errors are then bounded relative to the largest value."""
import numpy as np
import pytest
import torch

from ever_b200 import scheduler as SCH
from ever_b200 import synthetic as S
from ever_b200 import tracer as T
from oracle import mlp_np as M

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _dyadic_problem(R, seed):
    """Inputs in {-1,0,1}/4, weights in {-1,0,1}/8, biases k/32: all fp32 sums exact."""
    rng = np.random.default_rng(seed)
    feat = np.zeros((R, 64), np.float32)
    feat[:, :39] = rng.integers(-1, 2, (R, 39)) * 0.25
    w1 = np.zeros((64, 64), np.float32)
    w1[:, :39] = rng.integers(-1, 2, (64, 39)) * 0.125
    w2 = (rng.integers(-1, 2, (64, 64)) * 0.125).astype(np.float32)
    w3 = np.zeros((16, 64), np.float32)
    w3[:2] = rng.integers(-1, 2, (2, 64)) * 0.125
    b1 = rng.integers(-8, 9, 64) / 32.0
    b2 = rng.integers(-8, 9, 64) / 32.0
    b3 = np.zeros(16)
    b3[:2] = rng.integers(-8, 9, 2) / 32.0
    p = M.pack(w1, w2, w3, b1, b2, b3)
    target = (rng.integers(-16, 17, (R, 2)) / 16.0).astype(np.float32)
    return p, feat, target


def _block_errors(g, ref):
    blocks = dict(W1=(M.OFF_W1, M.OFF_W2), W2=(M.OFF_W2, M.OFF_W3), W3=(M.OFF_W3, M.OFF_B1), b1=(M.OFF_B1, M.OFF_B2),
                  b2=(M.OFF_B2, M.OFF_B3), b3=(M.OFF_B3, M.NPARAMS))
    return {k: float(np.abs(g[a:b] - ref[a:b]).max() / max(np.abs(ref[a:b]).max(), 1e-30))
            for k, (a, b) in blocks.items()}


@pytest.mark.parametrize("R", [1, 127, 128, 1000, 40_000])
def test_predictions_bit_exact_on_dyadic_inputs(R):
    dev = _dev()
    p, feat, _ = _dyadic_problem(R, R)
    cm = SCH.CostModel(params=p, device=dev)
    pred, _ = cm.predict(feat=torch.tensor(feat, device=dev))
    torch.cuda.synchronize()
    cm.check()
    np.testing.assert_array_equal(pred.cpu().numpy(), M.predict(p, feat))


@pytest.mark.parametrize("R", [128, 1024, 65_536])
def test_gradients_on_dyadic_inputs(R):
    dev = _dev()
    p, feat, target = _dyadic_problem(R, 7 + R)
    cm = SCH.CostModel(params=p, device=dev)
    grads, loss = cm.gradients(None, None, torch.tensor(target, device=dev), feat=torch.tensor(feat, device=dev),
                               weights=(1.0, 0.5))
    torch.cuda.synchronize()
    cm.check()
    ref, ref_loss = M.gradients(p, feat, target, 1.0, 0.5)
    err = _block_errors(grads.cpu().numpy().astype(np.float64), ref)
    assert max(err.values()) < 1e-5, err
    assert abs(float(loss.item()) - ref_loss) < 1e-5 * max(1.0, ref_loss)
    # padding stays untouched: no gradient reaches W1's input columns 39..63 or W3's rows 2..15
    g = grads.cpu().numpy()
    assert np.all(g[M.OFF_W1:M.OFF_W2].reshape(64, 64)[:, 39:] == 0)
    assert np.all(g[M.OFF_W3:M.OFF_B1].reshape(16, 64)[2:] == 0)


def _ray_problem(R, seed):
    rng = np.random.default_rng(seed)
    ro = rng.normal(0, 3, (R, 3)).astype(np.float32)
    rd = rng.normal(0, 1, (R, 3)).astype(np.float32)
    p = M.init_params(seed)
    p[M.OFF_B1:M.OFF_B3] = rng.normal(0, 0.1, M.OFF_B3 - M.OFF_B1)
    target = rng.normal(0, 1, (R, 2)).astype(np.float32)
    return p, ro, rd, target


@pytest.mark.parametrize("train", [False, True])
def test_tensor_core_wait_that_runs_out_is_reported_and_the_next_call_succeeds(train):
    # A wait bound of a few clocks makes the first completion wait give up while the MMAs are
    # still running: the kernel raises the error word, lets the MMAs in flight finish (at the
    # full bound) and frees its tensor memory, so the context stays usable and a call with
    # the default bound right after gives the exact results.
    dev = _dev()
    p, feat, target = _dyadic_problem(4096, 7)
    cm = SCH.CostModel(params=p, device=dev)
    x = torch.tensor(feat, device=dev)
    run = (lambda: cm.gradients(None, None, torch.tensor(target, device=dev), feat=x)) if train else (
        lambda: cm.predict(feat=x))
    cm.set_wait_clocks(4)
    run()
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match="timed out"):
        cm.check()
    cm.clear_error()
    cm.set_wait_clocks(0)
    out = run()
    torch.cuda.synchronize()
    cm.check()
    if train:
        ref, _ = M.gradients(p, feat, target, 1.0, 1.0)
        assert max(_block_errors(out[0].cpu().numpy().astype(np.float64), ref).values()) < 1e-5
    else:
        np.testing.assert_array_equal(out[0].cpu().numpy(), M.predict(p, feat))


def test_predictions_on_encoded_rays_match_oracle():
    dev = _dev()
    p, ro, rd, _ = _ray_problem(30_000, 3)
    cm = SCH.CostModel(centre=(0.5, -0.25, 0.1), scale=2.0, params=p, device=dev)
    pred, _ = cm.predict(torch.tensor(ro, device=dev), torch.tensor(rd, device=dev))
    torch.cuda.synchronize()
    ref = M.predict(p, M.encode(ro, rd, (0.5, -0.25, 0.1), 0.5))
    err = np.abs(pred.cpu().numpy() - ref)
    scale = np.abs(ref).max()
    assert err.max() < 2e-2 * scale, (err.max(), scale)
    assert np.median(err) < 1e-4 * scale


def test_gradients_on_encoded_rays_match_oracle_and_fp64():
    dev = _dev()
    p, ro, rd, target = _ray_problem(20_000, 4)
    cm = SCH.CostModel(scale=2.0, params=p, device=dev)
    args = (torch.tensor(ro, device=dev), torch.tensor(rd, device=dev), torch.tensor(target, device=dev))
    grads, loss = cm.gradients(*args, weights=(1.0, 0.25))
    g1 = grads.clone()
    grads, _ = cm.gradients(*args, weights=(1.0, 0.25))
    torch.cuda.synchronize()
    cm.check()
    assert torch.equal(g1, grads)  # deterministic: per-CTA partials summed in CTA order
    g = grads.cpu().numpy().astype(np.float64)
    feat = M.encode(ro, rd, (0, 0, 0), 0.5)
    ref, ref_loss = M.gradients(p, feat, target, 1.0, 0.25)
    ref64, _ = M.gradients(p.astype(np.float64), feat.astype(np.float64), target.astype(np.float64), 1.0, 0.25,
                           rounding=False)
    err = _block_errors(g, ref)
    err64 = _block_errors(g, ref64)
    print("max error relative to block max: vs bf16 oracle", err, "vs fp64", err64)
    assert max(err.values()) < 1e-2, err
    assert max(err64.values()) < 5e-2, err64
    assert abs(float(loss.item()) - ref_loss) < 1e-4 * ref_loss


def test_sample_indices_select_rays():
    dev = _dev()
    p, ro, rd, target = _ray_problem(5000, 5)
    cm = SCH.CostModel(scale=2.0, params=p, device=dev)
    ro_t, rd_t, tg = (torch.tensor(a, device=dev) for a in (ro, rd, target))
    idx = torch.randperm(5000, device=dev)[:1700].to(torch.int32)
    g_idx = cm.gradients(ro_t, rd_t, tg, sample_idx=idx)[0].clone()
    l = idx.long()
    g_sub = cm.gradients(ro_t[l].contiguous(), rd_t[l].contiguous(), tg[l].contiguous())[0]
    torch.cuda.synchronize()
    assert torch.equal(g_idx, g_sub)


def test_adam_step_matches_formula():
    dev = _dev()
    p, ro, rd, target = _ray_problem(4096, 6)
    cm = SCH.CostModel(scale=2.0, params=p, device=dev)
    g, _ = cm.gradients(torch.tensor(ro, device=dev), torch.tensor(rd, device=dev), torch.tensor(target, device=dev))
    g = g.cpu().numpy().astype(np.float64)
    cm.adam_step(lr=1e-2)
    torch.cuda.synchronize()
    m = 0.1 * g
    v = 0.001 * g * g
    want = p - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    np.testing.assert_allclose(cm.params.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(cm.w1.float().cpu().numpy(), M.bf16(cm.params.cpu().numpy()[:4096]))


# ------------------------------------------------------------ training on tracer logs
def _scene_tensors(dev, sc):
    return T.Scene(*(torch.tensor(np.ascontiguousarray(a), device=dev) for a in
                     (sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), sc.features)))


def _orbit_logs(dev, scene, n_views=8, w=96, h=72):
    views = []
    for eye in S.orbit(4.0, n_views):
        ro, rd = S.look_at_rays(S.Camera(eye, w, h, 50.0))
        ro, rd = torch.tensor(ro, device=dev), torch.tensor(rd, device=dev)
        f = T.forward(scene, ro, rd, max_iters=500, log_events=False, ray_stats=True)
        views.append((ro, rd, f.ray_stats.clone(), f.out.clone()))
    return views


def _fog_ball(n=5000, seed=12):
    """Ellipsoids uniform in the unit ball with low densities: rays seldom saturate, so a
    ray's event count follows its chord through the ball, a smooth function of the line."""
    sc = S.uniform_scene(4 * n, 1, seed)
    keep = np.flatnonzero(np.linalg.norm(sc.mean, axis=1) < 1.0)[:n]
    sc = sc.subset(keep)
    sc.density = (sc.density * 0.002).astype(np.float32)
    return sc


def test_training_on_tracer_logs_learns_ray_cost():
    dev = _dev()
    views = _orbit_logs(dev, _scene_tensors(dev, _fog_ball()))
    train, held = views[:6], views[6:]
    cat = lambda vs, i: torch.cat([v[i] for v in vs])
    ro, rd, st = cat(train, 0), cat(train, 1), cat(train, 2)
    tg = SCH.cost_targets(st, ro, rd, scale=2.0)
    cm = SCH.CostModel(scale=2.0, seed=1, device=dev)
    losses = cm.fit(ro, rd, tg, epochs=40, batch=8192, lr=3e-3).cpu().numpy()
    cm.check()
    assert np.isfinite(losses).all()
    assert losses[-20:].mean() < 0.2 * losses[:5].mean(), (losses[:5], losses[-20:])
    hro, hrd, hst = cat(held, 0), cat(held, 1), cat(held, 2)
    pred, _ = cm.predict(hro, hrd)
    truth = torch.log1p(hst[:, 0])
    r2 = 1 - float(((pred[:, 0] - truth) ** 2).mean() / truth.var())
    print("fog ball: held-out R^2 of log(1 + events):", r2, "mean events", float(hst[:, 0].mean()))
    assert r2 > 0.6


def _lane_slots(cost, order):
    """Sum over 32-ray packets of 32 x the costliest ray, over the total cost: lane-steps a
    SIMT warp occupies per useful step (1 = perfectly balanced packets)."""
    c = cost[order.long()] if order is not None else cost
    pad = (-c.numel()) % 32
    c = torch.cat([c, c.new_zeros(pad)]).view(-1, 32)
    return float(c.max(1).values.sum() * 32 / cost.sum())


def _bins_of(x, thr):
    return ((x > thr[0]).int() + (x > thr[1]).int() + (x > thr[2]).int()).to(torch.uint8)


def test_cost_binned_orders_keep_images_bit_identical_and_balance_packets():
    """Clustered sheets: the order changes which lanes share a packet, never a result.
    Packets ordered by true cost bins are better balanced than coherent tiles, which are
    far better balanced than scanline packets; the learned bins keep the coherent tiles'
    balance within a few percent (per-ray cost in this scene is mostly which sheets a ray
    happens to cross, which a function of the line alone cannot predict)."""
    dev = _dev()
    sc = S.clustered_scene(40_000, 1, seed=11, n_clusters=200)
    scene = _scene_tensors(dev, sc)
    views = _orbit_logs(dev, scene)
    cat = lambda vs, i: torch.cat([v[i] for v in vs])
    ro, rd, st = cat(views[:6], 0), cat(views[:6], 1), cat(views[:6], 2)
    cm = SCH.CostModel(scale=2.0, seed=1, device=dev)
    cm.fit(ro, rd, SCH.cost_targets(st, ro, rd, scale=2.0), epochs=40, batch=8192, lr=3e-3)
    thr = SCH.quantile_thresholds(cm.predict(ro, rd)[0][:, 0])
    true_thr = SCH.quantile_thresholds(torch.log1p(st[:, 0]))
    for hro, hrd, hst, hout in views[6:]:
        _, bins = cm.predict(hro, hrd, thresholds=thr)
        order = SCH.binned_order(hro, hrd, bins)
        assert torch.equal(torch.sort(order).values, torch.arange(hro.shape[0], device=dev, dtype=torch.int32))
        b = bins[order.long()].int()
        assert bool((b[1:] <= b[:-1]).all())  # costlier bins first
        true_order = SCH.binned_order(hro, hrd, _bins_of(torch.log1p(hst[:, 0]), true_thr))
        for o in (order, true_order):
            f = T.forward(scene, hro, hrd, max_iters=500, ray_stats=True, ray_order=o)
            assert torch.equal(f.out, hout) and torch.equal(f.ray_stats, hst)  # bit-identical images
        cost = hst[:, 0]
        s = dict(plain=_lane_slots(cost, None), coherent=_lane_slots(cost, T.ray_order(hro, hrd)),
                 learned=_lane_slots(cost, order), true=_lane_slots(cost, true_order))
        print("lane slots per useful step:", s)
        assert s["true"] < s["coherent"] < s["plain"]
        assert s["learned"] < s["plain"] and s["learned"] < 1.05 * s["coherent"]


@pytest.mark.parametrize("graph", [False, True])
def test_batched_tracer_with_learned_scheduler_matches_unscheduled(graph):
    from ever_b200.batched import BatchedTracer
    dev = _dev()
    sc = S.clustered_scene(20_000, 1, seed=13, n_clusters=100)
    arrs = tuple(torch.tensor(np.ascontiguousarray(a), device=dev) for a in
                 (sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), sc.features))
    views = [(0, *S.look_at_rays_device(S.Camera(e, w, h, 50.0), dev))
             for e, (w, h) in zip(S.orbit(4.0, 3), [(64, 48), (40, 30), (33, 17)])]
    cm = SCH.CostModel(scale=2.0, seed=3, device=dev)
    plain = BatchedTracer([arrs], views, graph=False)
    sched = BatchedTracer([arrs], views, graph=graph, scheduler=(cm, [2.0, 2.5, 3.0]))
    g = torch.full((plain.R, 5), 0.1, device=dev)
    plain.step(g)
    sched.step(g)
    torch.cuda.synchronize()
    assert torch.equal(plain.out, sched.out) and torch.equal(plain.iters, sched.iters)
    assert torch.equal(plain.drayo, sched.drayo) and torch.equal(plain.drayd, sched.drayd)
    for a, b in zip(plain.grads, sched.grads):
        for x, y in zip([a.mean, a.density, a.features], [b.mean, b.density, b.features]):
            assert float((x - y).abs().max()) <= 1e-4 * float(y.abs().max()) + 1e-12
    assert int(sched.bins.max()) <= 3
    cm.check()
