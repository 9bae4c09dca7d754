"""Camera traces (ever_trace_forward_camera / ever_trace_backward_camera): the rays are made
inside the kernels, so the results must equal trace_rays on ever_camera_rays' rays bit for
bit (per-pixel outputs, event sequences, ray gradients) and up to the summation order of
the float atomics for the ellipsoid gradients. Also checked directly against the oracle."""
import math

import numpy as np
import pytest
import torch

from ever_b200 import camera as CAM
from ever_b200 import synthetic as S
from ever_b200 import tracer as T
from ever_b200.fast_ellipsoid_splinetracer import trace_rays
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _look_at(eye):
    """Camera-to-world 3x4 (x right, y down, z forward) looking at the origin."""
    eye = np.asarray(eye, np.float64)
    f = -eye / np.linalg.norm(eye)
    r = np.cross(f, [0.0, 0.0, 1.0])
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    m = np.zeros((3, 4))
    m[:, 0], m[:, 1], m[:, 2], m[:, 3] = r, d, f, eye
    return m


def _camera(w, h, eye=(0.6, -3.2, 1.1), fov=55.0, cx=None, cy=None):
    f = 0.5 * h / math.tan(math.radians(fov) / 2)
    return CAM.Camera(w, h, f, f * 1.05, _look_at(eye), cx, cy)


def _params(dev, n, deg, seed, clustered=False):
    sc = S.clustered_scene(n, deg, seed=seed, n_clusters=60) if clustered else S.uniform_scene(n, deg, seed)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    return sc, dict(mean=t(sc.mean), scale=t(sc.scale), quat=t(sc.quat), density=t(sc.density),
                    features=t(sc.features))


def _jitter(cam, dev, on, seed=3):
    if not on:
        return None
    g = torch.Generator(device=dev).manual_seed(seed)
    return torch.rand((cam.num_pixels, 2), generator=g, device=dev)


def _slot_pixels_np(w, h):
    # 8x4 pixel tiles; 64x64-pixel supertiles row-major; tiles in a supertile in Morton order
    ux_n, uy_n = (w + 63) // 64, (h + 63) // 64
    s = np.arange(ux_n * uy_n * 4096)
    u, t, l = s // 4096, (s // 32) % 128, s % 32
    bit = lambda v, i: (v >> i) & 1
    tx = bit(t, 0) | bit(t, 2) << 1 | bit(t, 4) << 2
    ty = bit(t, 1) | bit(t, 3) << 1 | bit(t, 5) << 2 | bit(t, 6) << 3
    col = (u % ux_n) * 64 + tx * 8 + l % 8
    row = (u // ux_n) * 64 + ty * 4 + l // 8
    return np.where((col < w) & (row < h), row * w + col, -1)


@pytest.mark.parametrize("w,h", [(37, 23), (64, 48), (1, 1), (8, 4), (9, 5), (130, 70)])
def test_slot_pixels_are_the_tile_order(w, h):
    dev = _dev()
    cam = _camera(w, h)
    sp = CAM.slot_pixels(cam, dev).cpu().numpy()
    want = _slot_pixels_np(w, h)
    assert np.array_equal(sp, want)
    valid = sp[sp >= 0]
    assert np.array_equal(np.sort(valid), np.arange(w * h)), "every pixel in exactly one slot"


@pytest.mark.parametrize("jitter", [False, True])
@pytest.mark.parametrize("kbuf,block", [(16, 128), (8, 64), (32, 256)])
def test_camera_forward_matches_trace_of_camera_rays(jitter, kbuf, block):
    dev = _dev()
    _, p = _params(dev, 4000, 3, seed=21)
    cam = _camera(45, 31)
    jit = _jitter(cam, dev, jitter)
    scene = T.Scene(p["mean"], p["scale"], p["quat"], p["density"], p["features"])
    tune = T.Tune(kbuf, block, 0)
    ro, rd = CAM.camera_rays(cam.width, cam.height, cam.fx, cam.fy, cam.c2w, jitter=jit, device=dev)
    want = T.forward(scene, ro, rd, 0.0, 1000.0, 500, touch_count=True, ray_stats=True, tune=tune)
    got = CAM.forward(scene, cam, jit, 0.0, 1000.0, 500, touch_count=True, ray_stats=True, tune=tune)
    for k in ("out", "states", "last_dirac", "iters", "ray_stats", "touch_count"):
        assert torch.equal(getattr(got, k), getattr(want, k)), k
    assert int(got.status.item()) == 0 and int(want.status.item()) == 0
    tri_w = T.reference_tri_collection(scene, want, 500)
    tri_g = CAM.tri_collection(scene, cam, got, 500)
    assert torch.equal(tri_g, tri_w)
    assert int(got.iters.sum()) > 1000  # the view sees the scene


def test_camera_forward_matches_oracle():
    dev = _dev()
    sc, p = _params(dev, 1500, 3, seed=22)
    cam = _camera(29, 19, cx=13.25, cy=10.5)
    scene = T.Scene(p["mean"], p["scale"], p["quat"], p["density"], p["features"])
    got = CAM.forward(scene, cam, None, 0.0, 1000.0, 500)
    tri = CAM.tri_collection(scene, cam, got, 500).reshape(500, -1).cpu().numpy()
    ro, rd = CAM.camera_rays(cam.width, cam.height, cam.fx, cam.fy, cam.c2w, cx=cam.cx, cy=cam.cy, device=dev)
    ref = O.trace(O.Scene(sc.mean, sc.scale, sc.quat, sc.density, sc.features), ro.cpu().numpy(),
                  rd.cpu().numpy(), 0.0, 1000.0, 500)
    iters = got.iters.cpu().numpy()
    assert np.array_equal(iters, ref.iters)
    for j in range(iters.size):
        assert np.array_equal(tri[:iters[j], j], ref.events[:iters[j], j]), f"pixel {j}"
    np.testing.assert_allclose(got.out.cpu().numpy(), ref.out, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("ordered", [False, True])
@pytest.mark.parametrize("jitter", [False, True])
def test_camera_backward_matches_trace_of_camera_rays(ordered, jitter):
    dev = _dev()
    _, p = _params(dev, 6000, 2, seed=23, clustered=True)
    cam = _camera(53, 27, eye=(3.0, 1.5, 1.0))
    jit = _jitter(cam, dev, jitter)
    scene = T.Scene(p["mean"], p["scale"], p["quat"], p["density"], p["features"])
    ro, rd = CAM.camera_rays(cam.width, cam.height, cam.fx, cam.fy, cam.c2w, jitter=jit, device=dev)
    fw = T.forward(scene, ro, rd, 0.0, 1000.0, 500)
    fc = CAM.forward(scene, cam, jit, 0.0, 1000.0, 500)
    assert torch.equal(fc.out, fw.out)
    gout = torch.randn((cam.num_pixels, 5), generator=torch.Generator(device=dev).manual_seed(9), device=dev)
    wct = torch.randn((1, 4, 4), generator=torch.Generator(device=dev).manual_seed(10), device=dev)
    want = T.backward(scene, ro, rd, fw, gout, 0.0, 1000.0, 500, wcts=wct, want_means2d=True)
    order = CAM.backward_order(cam, fc) if ordered else None
    if ordered:
        o = order.cpu().numpy()
        assert np.array_equal(np.sort(o), np.arange(CAM.camera_slots(cam)))
    got = CAM.backward(scene, cam, fc, gout, jit, 0.0, 1000.0, 500, wcts=wct, want_means2d=True,
                       want_ray_grads=True, slot_order=order)
    # per-ray work has no atomics: ray gradients are bit-identical
    assert torch.equal(got.rayo, want.rayo) and torch.equal(got.rayd, want.rayd)
    for k in ("mean", "scale", "quat", "density", "features", "means2d"):
        a, b = getattr(got, k), getattr(want, k)
        tol = 1e-5 * max(1.0, float(b.abs().max()))
        assert float((a - b).abs().max()) <= tol, k
    assert float(want.mean.abs().max()) > 0


def test_camera_backward_without_ray_gradients():
    dev = _dev()
    _, p = _params(dev, 3000, 0, seed=24)
    cam = _camera(33, 17)
    scene = T.Scene(p["mean"], p["scale"], p["quat"], p["density"], p["features"])
    fc = CAM.forward(scene, cam, None)
    gout = torch.ones((cam.num_pixels, 5), device=dev)
    a = CAM.backward(scene, cam, fc, gout, want_ray_grads=True)
    b = CAM.backward(scene, cam, fc, gout, want_ray_grads=False)
    assert b.rayo is None and b.rayd is None
    for k in ("mean", "scale", "quat", "density", "features"):
        x, y = getattr(a, k), getattr(b, k)
        assert float((x - y).abs().max()) <= 1e-5 * max(1.0, float(x.abs().max())), k


def test_trace_camera_autograd_matches_trace_rays():
    dev = _dev()
    _, p = _params(dev, 5000, 3, seed=25, clustered=True)
    cam = _camera(40, 30, eye=(-2.5, 2.5, 1.5))
    jit = _jitter(cam, dev, True, seed=8)
    a = {k: v.clone().requires_grad_(True) for k, v in p.items()}
    b = {k: v.clone().requires_grad_(True) for k, v in p.items()}
    out_c, ex_c = CAM.trace_camera(a["mean"], a["scale"], a["quat"], a["density"], a["features"], cam,
                                   0.0, 1000.0, return_extras=True, jitter=jit)
    ro, rd = CAM.camera_rays(cam.width, cam.height, cam.fx, cam.fy, cam.c2w, jitter=jit, device=dev)
    out_r, ex_r = trace_rays(b["mean"], b["scale"], b["quat"], b["density"], b["features"], ro, rd, 0.0, 1000.0,
                             return_extras=True)
    assert torch.equal(out_c, out_r)
    assert torch.equal(ex_c["tri_collection"], ex_r["tri_collection"])
    assert torch.equal(ex_c["touch_count"], ex_r["touch_count"])
    g = torch.randn_like(out_r)
    (out_c * g).sum().backward()
    (out_r * g).sum().backward()
    for k in p:
        x, y = a[k].grad, b[k].grad
        assert float((x - y).abs().max()) <= 1e-5 * max(1.0, float(y.abs().max())), k


def test_camera_trace_truncation_and_empty_cases():
    dev = _dev()
    _, p = _params(dev, 2000, 0, seed=26)
    scene = T.Scene(p["mean"], p["scale"], p["quat"], p["density"], p["features"])
    cam = _camera(21, 13)
    ro, rd = CAM.camera_rays(cam.width, cam.height, cam.fx, cam.fy, cam.c2w, device=dev)
    for mi in (0, 1, 3):  # max_iters truncation, as trace_rays
        got = CAM.forward(scene, cam, None, 0.0, 1000.0, mi)
        want = T.forward(scene, ro, rd, 0.0, 1000.0, mi)
        assert torch.equal(got.out, want.out) and torch.equal(got.iters, want.iters)
    # an empty image launches nothing
    empty = CAM.forward(scene, _camera(0, 7), None)
    assert empty.out.shape == (0, 5)
    # a scene without ellipsoids: transparent pixels, zero gradients
    z = torch.zeros((0, 3), device=dev)
    s0 = T.Scene(z, z.clone(), torch.zeros((0, 4), device=dev), torch.zeros((0, 1), device=dev),
                 torch.zeros((0, 1, 3), device=dev))
    f0 = CAM.forward(s0, cam, None)
    assert torch.equal(f0.out, torch.zeros_like(f0.out))
    g0 = CAM.backward(s0, cam, f0, torch.ones_like(f0.out), want_ray_grads=True)
    assert torch.equal(g0.rayd, torch.zeros_like(g0.rayd))


@pytest.mark.parametrize("kbuf,block", [(16, 128), (8, 64), (16, 256)])
@pytest.mark.parametrize("jitter", [False, True])
def test_camera_regrouped_equals_single_kernel(kbuf, block, jitter):
    # the camera forward in packed passes (every pass splits: regroup_min=1) against the
    # single camera kernel, on a faint cloud where rays need many gather rounds
    dev = _dev()
    sc = S.uniform_scene(20_000, 2, 61)
    sc.density[:] = sc.density * 0.02
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    scene = T.Scene(t(sc.mean), t(sc.scale), t(sc.quat), t(sc.density), t(sc.features))
    cam = _camera(70, 45, eye=(2.0, -2.0, 1.2), fov=40.0)
    jit = _jitter(cam, dev, jitter)
    tune = T.Tune(kbuf, block, 0, regroup_min=1)
    a = CAM.forward(scene, cam, jit, 0.0, 1000.0, 500, touch_count=True, ray_stats=True, tune=tune, regrouped=False)
    b = CAM.forward(scene, cam, jit, 0.0, 1000.0, 500, touch_count=True, ray_stats=True, tune=tune, regrouped=True)
    for k in ("out", "states", "last_dirac", "iters", "ray_stats", "touch_count", "status"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    assert torch.equal(CAM.tri_collection(scene, cam, a, 500), CAM.tri_collection(scene, cam, b, 500))
    assert int(a.iters.max()) > 2 * kbuf
