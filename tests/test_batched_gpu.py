"""Batched persistent tracing (several scenes, views of mixed sizes, one forward and one
backward launch, optionally replayed from a CUDA graph) against per-view single launches."""
import numpy as np
import pytest
import torch

from ever_b200 import synthetic as S
from ever_b200 import tracer as T
from ever_b200.batched import BatchedTracer

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _setup(dev):
    scenes_np = [S.clustered_scene(3000, 3, seed=50, n_clusters=20), S.uniform_scene(5000, 3, seed=51)]
    scenes = [tuple(torch.tensor(np.ascontiguousarray(a), device=dev) for a in
                    (s.mean, s.scale, s.quat, s.density.reshape(-1), s.features)) for s in scenes_np]
    cams = [(0, S.Camera(S.sphere_point(4.0, 60), 40, 30, 50.0)), (1, S.Camera(S.sphere_point(3.0, 61), 33, 17, 60.0)),
            (0, S.Camera(S.sphere_point(4.0, 62), 64, 36, 50.0)), (1, S.Camera(S.sphere_point(3.0, 63), 8, 8, 40.0))]
    views = []
    for si, cam in cams:
        ro, rd = S.look_at_rays(cam)
        views.append((si, torch.tensor(ro, device=dev), torch.tensor(rd, device=dev)))
    return scenes, views


def _reference(scenes, views, gout_views, tune):
    """Per-view single launches; prim gradients summed over the views of each scene."""
    outs, grads = [], [None] * len(scenes)
    for (si, ro, rd), go in zip(views, gout_views):
        sc = T.Scene(*scenes[si])
        fwd = T.forward(sc, ro, rd, tune=tune)
        g = T.backward(sc, ro, rd, fwd, go, tune=tune)
        outs.append((fwd.out.clone(), fwd.iters.clone(), fwd.states.clone(), g.rayo.clone(), g.rayd.clone()))
        gs = [g.mean, g.scale, g.quat, g.density, g.features]
        grads[si] = gs if grads[si] is None else [a + b for a, b in zip(grads[si], gs)]
    return outs, grads


def _rel(a, b):
    return float((a - b).abs().max() / (b.abs().max() + 1e-12))


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("kbuf,block", [(16, 128), (8, 64), (32, 256)])
def test_batched_matches_single_view_launches(graph, kbuf, block):
    dev = _dev()
    scenes, views = _setup(dev)
    tune = T.Tune(kbuf=kbuf, block=block)
    bt = BatchedTracer(scenes, views, tune=tune, graph=graph)
    gen = torch.Generator(device=dev).manual_seed(0)
    gout = torch.randn((bt.R, 5), device=dev, generator=gen)
    bt.step(gout)
    torch.cuda.synchronize()
    gout_views = [gout[bt.view_slice(v)] for v in range(len(views))]
    ref_outs, ref_grads = _reference(scenes, views, gout_views, tune)
    for v, (out, iters, states, dro, drd) in enumerate(ref_outs):
        sl = bt.view_slice(v)
        assert torch.equal(bt.out[sl], out) and torch.equal(bt.iters[sl], iters) and torch.equal(bt.states[sl], states)
        assert torch.equal(bt.drayo[sl], dro) and torch.equal(bt.drayd[sl], drd)
    for si, g in enumerate(bt.grads):
        for a, b in zip([g.mean, g.scale, g.quat, g.density, g.features], ref_grads[si]):
            assert _rel(a, b) < 1e-4
    assert int(bt.status.item()) == 0


def test_graph_replay_follows_in_place_updates():
    dev = _dev()
    scenes, views = _setup(dev)
    bt = BatchedTracer(scenes, views, graph=True)
    gout = torch.ones((bt.R, 5), device=dev)
    bt.step(gout)
    first = bt.out.clone()
    with torch.no_grad():
        scenes[0][3].mul_(0.5)  # densities of scene 0, updated in place as an optimizer would
        scenes[1][0].add_(0.01)  # means of scene 1
    bt.step(gout)
    torch.cuda.synchronize()
    assert not torch.equal(first, bt.out)
    eager = BatchedTracer(scenes, views, graph=False)
    eager.step(gout)
    torch.cuda.synchronize()
    assert torch.equal(eager.out, bt.out) and torch.equal(eager.iters, bt.iters)
