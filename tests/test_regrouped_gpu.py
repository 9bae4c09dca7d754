"""The regrouped forward (ever_trace_forward_regrouped: rays still active after a gather
round are packed into full warps for the next pass) against the single-kernel forward
(ever_trace_forward): every output must be bit-identical, including the event sequences,
for all k-buffer sizes, block sizes, launch orders and the truncation / tmin / tmax /
start-inside cases."""
import numpy as np
import pytest
import torch

from ever_b200 import synthetic as S
from ever_b200 import tracer as T

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _scene(dev, sc):
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    return T.Scene(t(sc.mean), t(sc.scale), t(sc.quat), t(sc.density), t(sc.features))


def _both(scene, ro, rd, max_iters=500, tmin=0.0, tmax=1000.0, order=None, tune=None):
    # regroup_min=1: every pass hands its remaining rays on, whatever their number (the
    # default keeps small launches in one pass)
    tune = tune or T.Tune(regroup_min=1)
    kw = dict(touch_count=True, ray_stats=True, ray_order=order, tune=tune)
    a = T.forward(scene, ro, rd, tmin, tmax, max_iters, regrouped=False, **kw)
    b = T.forward(scene, ro, rd, tmin, tmax, max_iters, regrouped=True, **kw)
    for k in ("out", "states", "last_dirac", "iters", "touch_count", "ray_stats", "status"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    if max_iters > 0:
        ta = T.reference_tri_collection(scene, a, max_iters, order)
        tb = T.reference_tri_collection(scene, b, max_iters, order)
        assert torch.equal(ta, tb), "event sequences differ"
    return a


def _thin_scene(n, deg, seed):
    # a faint uniform cloud: rays consume ~150 events (up to ~340), so every k-buffer size
    # needs several gather rounds and all three passes carry rays
    sc = S.uniform_scene(n, deg, seed)
    sc.density[:] = sc.density * 0.02
    return sc


@pytest.mark.parametrize("kbuf,block", [(16, 128), (8, 64), (32, 256), (16, 256), (8, 128)])
@pytest.mark.parametrize("ordered", [False, True])
def test_regrouped_equals_single_kernel(kbuf, block, ordered):
    dev = _dev()
    scene = _scene(dev, _thin_scene(20_000, 2, 51))
    ro, rd = S.look_at_rays_device(S.Camera(S.sphere_point(3.0, 51), 45, 37, 40.0), dev)  # 1665 rays
    order = T.ray_order(ro, rd) if ordered else None
    a = _both(scene, ro, rd, order=order, tune=T.Tune(kbuf, block, 0, regroup_min=1))
    assert int(a.iters.max()) > 2 * kbuf  # rays reach the last pass
    assert int((a.iters < kbuf).sum()) > 0  # and others finish in the first


def test_regrouped_clustered_scene():
    dev = _dev()
    scene = _scene(dev, S.clustered_scene(20_000, 3, seed=52, n_clusters=40))
    ro, rd = S.look_at_rays_device(S.Camera(S.sphere_point(3.0, 52), 33, 29, 50.0), dev)
    _both(scene, ro, rd, order=T.ray_order(ro, rd))


@pytest.mark.parametrize("max_iters", [0, 1, 3, 16, 17, 33, 48])
def test_regrouped_truncation(max_iters):
    dev = _dev()
    scene = _scene(dev, _thin_scene(10_000, 3, 52))
    ro, rd = S.look_at_rays_device(S.Camera(S.sphere_point(3.0, 52), 33, 29, 40.0), dev)
    _both(scene, ro, rd, max_iters=max_iters, order=T.ray_order(ro, rd))


def test_regrouped_tmin_tmax_and_rays_starting_inside():
    dev = _dev()
    sc = S.uniform_scene(3000, 1, seed=53)
    scene = _scene(dev, sc)
    # camera inside the ellipsoid cloud: rays start inside ellipsoids
    ro, rd = S.look_at_rays_device(S.Camera(np.array([0.1, -0.2, 0.3]), 31, 19, 70.0), dev)
    for tmin, tmax in ((0.0, 1000.0), (0.05, 1000.0), (0.0, 0.7), (0.2, 1.1)):
        _both(scene, ro, rd, tmin=tmin, tmax=tmax)


def test_regrouped_empty_and_tiny():
    dev = _dev()
    z = lambda *s: torch.zeros(s, device=dev)
    empty = T.Scene(z(0, 3), z(0, 3), z(0, 4), z(0, 1), z(0, 1, 3))
    ro, rd = S.look_at_rays_device(S.Camera(np.array([0.0, 0.0, 3.0]), 7, 5, 50.0), dev)
    a = _both(empty, ro, rd)
    assert torch.equal(a.out, torch.zeros_like(a.out))
    scene = _scene(dev, S.uniform_scene(200, 0, seed=54))
    _both(scene, ro[:1].contiguous(), rd[:1].contiguous())  # one ray
    _both(scene, ro[:33].contiguous(), rd[:33].contiguous())  # one full warp and one lane
    r0 = T.forward(scene, ro[:0], rd[:0], regrouped=True)
    assert r0.out.shape == (0, 5)


def test_regrouped_many_rays():
    # 307,200 rays: 9,600 warp masks, more than one step of the compaction scan
    dev = _dev()
    scene = _scene(dev, _thin_scene(5000, 0, 55))
    ro, rd = S.look_at_rays_device(S.Camera(S.sphere_point(3.0, 55), 640, 480, 45.0), dev)
    a = _both(scene, ro, rd, order=T.ray_order(ro, rd))
    assert int((a.iters > 32).sum()) > 10_000


@pytest.mark.parametrize("regroup_min", [0, 1000, 100_000])
def test_regrouped_split_threshold(regroup_min):
    # 0 (four times the resident lanes: here one pass), and thresholds that split only the
    # first pass or none: the results never change
    dev = _dev()
    scene = _scene(dev, _thin_scene(20_000, 2, 56))
    ro, rd = S.look_at_rays_device(S.Camera(S.sphere_point(3.0, 56), 45, 37, 40.0), dev)
    _both(scene, ro, rd, order=T.ray_order(ro, rd), tune=T.Tune(16, 128, 0, regroup_min=regroup_min))
