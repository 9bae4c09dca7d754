"""The learned depth hint on an orbit of clustered ellipsoids: the cost model, trained on the
tracer's logs of some views, predicts where each ray of the other views stops; the forward's
frustum phase walks only up to there, and the rounds continue any ray that goes on.
- the held-out R^2 of the depth output is positive, so the gate switches the hint on;
- forward + backward with the hint give the same images, event counts and gradients, bit
  for bit, as the coherent order alone;
- with the hint the views trace faster than with the coherent order alone (median of
  interleaved passes);
- with the gate off, plan() gives the coherent order and no hint."""
import numpy as np
import pytest
import torch

from ever_b200 import scheduler as SCH
from ever_b200 import synthetic as S
from ever_b200 import tracer as T

pytestmark = pytest.mark.gpu


def test_learned_depth_hint_is_exact_and_faster_than_coherent_alone():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dev = torch.device("cuda:0")
    sc, cams = S.workload_orbit(n=1_000_000, n_views=16, width=960, height=540)
    arrs = [torch.tensor(np.ascontiguousarray(a), device=dev) for a in
            (sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), sc.features)]
    scene = T.Scene(*arrs)
    rays = [S.look_at_rays_device(c, dev) for c in cams]
    train, test = list(range(0, 16, 2)), list(range(1, 16, 2))  # every other view held out
    stats = {}
    for v in range(16):
        ro, rd = rays[v]
        stats[v] = T.forward(scene, ro, rd, 0.0, 1000.0, 500, log_events=False, ray_stats=True,
                             ray_order=T.ray_order(ro, rd)).ray_stats.clone()
    cm = SCH.CostModel(scale=2.0, seed=1, device=dev)
    ro_tr = torch.cat([rays[v][0] for v in train])
    rd_tr = torch.cat([rays[v][1] for v in train])
    cm.fit(ro_tr, rd_tr, SCH.cost_targets(torch.cat([stats[v] for v in train]), ro_tr, rd_tr, scale=2.0),
           epochs=3, batch=65536, lr=3e-3)
    cm.check()
    r2 = [SCH.heldout_r2(cm, *rays[v], stats[v], scale=2.0) for v in test]
    r2_depth = float(np.mean([x[1] for x in r2]))
    gate = SCH.Gate(float(np.mean([x[0] for x in r2])), r2_depth)
    assert r2_depth > 0.0 and gate.depth, r2

    gout = torch.full((rays[0][0].shape[0], 5), 0.1, device=dev)

    def step(v, use_hint):
        ro, rd = rays[v]
        order, hint = SCH.plan(cm, ro, rd, gate if use_hint else SCH.Gate(-1.0, -1.0), scale=2.0)
        f = T.forward(scene, ro, rd, 0.0, 1000.0, 500, ray_order=order, depth_hint=hint)
        slots = T.backward_order(f, order, 0)
        g = T.backward(scene, ro, rd, f, gout, 0.0, 1000.0, 500, ray_order=order, slot_order=slots)
        return f, g, hint

    for v in test:
        fa, ga, ha = step(v, False)
        fb, gb, hb = step(v, True)
        assert ha is None and hb is not None
        assert int(fb.status.item()) == 0
        assert torch.equal(fa.out, fb.out) and torch.equal(fa.iters, fb.iters)
        for x, y in zip((ga.mean, ga.scale, ga.quat, ga.density, ga.features, ga.rayo, ga.rayd),
                        (gb.mean, gb.scale, gb.quat, gb.density, gb.features, gb.rayo, gb.rayd)):
            assert float((x - y).abs().max()) <= 1e-5 * float(y.abs().max()) + 1e-12  # atomics: order only

    def timed(use_hint):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for v in test:
            step(v, use_hint)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    timed(False), timed(True)
    ms = {False: [], True: []}
    for _ in range(3):
        for h in (False, True):
            ms[h].append(timed(h))
    speedup = float(np.median(ms[False]) / np.median(ms[True]))
    print(f"learned depth hint vs coherent order alone: {speedup:.3f}x, held-out R^2 depth {r2_depth:.3f}")
    assert speedup > 1.0, (speedup, ms)
