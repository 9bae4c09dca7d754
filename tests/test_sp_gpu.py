"""The reference's object API (ever_b200.sp) and the persistent BVH (refit): the same
kernels as trace_rays, so outputs are compared bit for bit."""
import numpy as np
import pytest
import torch

from ever_b200 import sp
from ever_b200 import synthetic as S
from ever_b200 import tracer as T
from ever_b200.fast_ellipsoid_splinetracer import trace_rays

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _setup(dev, n=20_000, deg=1, seed=40):
    sc = S.clustered_scene(n, deg, seed=seed, n_clusters=80)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    p = dict(mean=t(sc.mean), scale=t(sc.scale), quat=t(sc.quat), density=t(sc.density), features=t(sc.features))
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(4.0, seed), 64, 48, 50.0))
    return p, t(ro), t(rd)


def _sp(dev, p):
    ctx = sp.OptixContext(dev)
    prims = sp.Primitives(dev)
    half = torch.cat([p["mean"], p["scale"], p["quat"]], 1).half()
    prims.add_primitives(p["mean"], p["scale"], p["quat"], half, p["density"], p["features"])
    return ctx, prims, sp.GAS(ctx, dev, prims, True, False, True), sp.Forward(ctx, dev, prims, False)


def test_object_api_matches_trace_rays():
    dev = _dev()
    p, ro, rd = _setup(dev)
    ctx, prims, gas, fwd = _sp(dev, p)
    out = fwd.trace_rays(gas, ro, rd, 0.0, 1000.0, 200, 3.0)
    ref, extras = trace_rays(p["mean"], p["scale"], p["quat"], p["density"], p["features"], ro, rd, 0.0, 1000.0, 3,
                             None, None, 200, True)
    assert torch.equal(out["color"], ref[:, :4])
    assert torch.equal(out["saved"].iters, extras["iters"])
    assert torch.equal(out["tri_collection"], extras["tri_collection"])
    assert torch.equal(out["saved"].touch_count, extras["touch_count"])
    assert out["saved"].states.shape == (ro.shape[0], 16) and out["initial_drgb"].shape == (ro.shape[0], 4)


def test_update_model_swaps_colours():
    dev = _dev()
    p, ro, rd = _setup(dev)
    ctx, prims, gas, fwd = _sp(dev, p)
    fwd.trace_rays(gas, ro, rd, 0.0, 1000.0, 200)
    new_feat = (p["features"] * -0.7 + 0.1).contiguous()
    prims.set_features(new_feat)
    fwd.update_model(prims)
    out = fwd.trace_rays(gas, ro, rd, 0.0, 1000.0, 200)
    ref = trace_rays(p["mean"], p["scale"], p["quat"], p["density"], new_feat, ro, rd, 0.0, 1000.0, 3, None, None, 200)
    assert torch.equal(out["color"], ref[:, :4])


def test_refit_follows_moved_ellipsoids_exactly():
    dev = _dev()
    p, ro, rd = _setup(dev)
    scene = T.Scene(p["mean"], p["scale"], p["quat"], p["density"].reshape(-1), p["features"])
    gen = torch.Generator(device=dev).manual_seed(3)
    with torch.no_grad():  # an optimiser step: every parameter moves a little, in place
        p["mean"].add_(torch.randn(p["mean"].shape, device=dev, generator=gen) * 0.01)
        p["scale"].mul_(1 + 0.05 * torch.rand(p["scale"].shape, device=dev, generator=gen))
        p["quat"].add_(torch.randn(p["quat"].shape, device=dev, generator=gen) * 0.02)
        p["density"].mul_(1.1)
        p["features"].add_(0.05)
    scene.refit()
    a = T.forward(scene, ro, rd, max_iters=200)
    fresh = T.Scene(p["mean"], p["scale"], p["quat"], p["density"].reshape(-1), p["features"])
    b = T.forward(fresh, ro, rd, max_iters=200)
    assert torch.equal(a.out, b.out) and torch.equal(a.iters, b.iters) and torch.equal(a.states, b.states)
    # the GAS object refits the same way
    ctx, prims, gas, fwd = _sp(dev, p)
    with torch.no_grad():
        p["mean"].add_(0.02)
    gas.refit()
    out = fwd.trace_rays(gas, ro, rd, 0.0, 1000.0, 200)
    ref = trace_rays(p["mean"], p["scale"], p["quat"], p["density"], p["features"], ro, rd, 0.0, 1000.0, 3, None, None,
                     200)
    assert torch.equal(out["color"], ref[:, :4])


def test_initial_density_outputs():
    dev = _dev()
    p, ro, rd = _setup(dev, n=5000, deg=0, seed=41)
    ro = p["mean"][7].expand_as(ro).contiguous()  # rays start at an ellipsoid's centre, inside it
    ctx, prims, gas, fwd = _sp(dev, p)
    out = fwd.trace_rays(gas, ro, rd, 0.0, 1000.0, 200)
    cnt = int(out["initial_touch_count"][0])
    inds = out["initial_touch_inds"][:cnt].long()
    assert cnt >= 1 and 7 in inds.tolist()
    # rays share the origin: each ray's initial density is the density sum of the members
    want = float(p["density"].reshape(-1)[inds].sum())
    got = out["initial_drgb"][:, 0]
    assert torch.allclose(got, torch.full_like(got, want), rtol=1e-5)
