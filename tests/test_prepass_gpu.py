"""GPU checks of the colour pre-pass (ever_sh_prepass*) and camera rays (ever_camera_rays)
against the CPU oracle (oracle/prepass_np.py): colours and features within 1e-5 relative,
feature gradients against fp64 autograd through the oracle within 1e-5 of the max, rays
within 1e-6."""
import math

import numpy as np
import pytest
import torch

from ever_b200 import camera as CAM
from ever_b200 import eval_sh as E
from oracle import prepass_np as P

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _scene(n, K, seed):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    feats = (rng.normal(size=(n, K, 3)) * 0.4).astype(np.float32)
    cam = np.array([0.5, -4.0, 1.5], np.float32)
    return means, feats, cam


@pytest.mark.parametrize("deg,K", [(0, 1), (0, 16), (1, 4), (2, 9), (3, 16)])
def test_eval_sh_and_trainer_features_match_oracle(deg, K):
    dev = _dev()
    means, feats, cam = _scene(5000, K, deg)
    t = lambda a: torch.tensor(a, device=dev)
    col = E.eval_sh(t(means), t(feats), t(cam), deg)
    fea = E.sh_features(t(means), t(feats), t(cam), deg)
    m64, f64, c64 = (torch.tensor(a, dtype=torch.float64) for a in (means, feats, cam))
    want_col = P.eval_sh(m64, f64, c64, deg).numpy()
    want_fea = P.sh_features(m64, f64, c64, deg).numpy()
    np.testing.assert_allclose(col.cpu().numpy(), want_col, rtol=1e-5, atol=1e-6)
    assert fea.shape == (5000, 1, 3)
    np.testing.assert_allclose(fea.cpu().numpy(), want_fea, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("deg", [1, 3])
def test_feature_gradients_match_fp64_autograd(deg, fused):
    dev = _dev()
    means, feats, cam = _scene(3000, 16, 10 + deg)
    rng = np.random.default_rng(3)
    g = rng.normal(size=(3000, 3)).astype(np.float32)
    g[:100] = 0.0  # ellipsoids without gradient: skipped, zero rows
    ft = torch.tensor(feats, device=dev, requires_grad=True)
    fn = E.sh_features if fused else E.eval_sh
    out = fn(torch.tensor(means, device=dev), ft, torch.tensor(cam, device=dev), deg)
    (out.reshape(-1, 3) * torch.tensor(g, device=dev)).sum().backward()
    f64 = torch.tensor(feats, dtype=torch.float64, requires_grad=True)
    ofn = P.sh_features if fused else P.eval_sh
    o64 = ofn(torch.tensor(means, dtype=torch.float64), f64, torch.tensor(cam, dtype=torch.float64), deg)
    (o64.reshape(-1, 3) * torch.tensor(g, dtype=torch.float64)).sum().backward()
    got, want = ft.grad.cpu().double().numpy(), f64.grad.numpy()
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    assert np.all(got[:100] == 0) and np.all(got[:, (deg + 1) ** 2:] == 0)


def test_tiny_colour_gradients_are_skipped_like_the_reference():
    dev = _dev()
    means, feats, cam = _scene(64, 4, 7)
    t = lambda a: torch.tensor(a, device=dev)
    ft = t(feats).requires_grad_(True)
    out = E.eval_sh(t(means), ft, t(cam), 1)
    g = torch.full_like(out, 5e-9)  # below the 1e-8 threshold in every channel
    g[0, 1] = 2e-8
    out.backward(g)
    assert torch.all(ft.grad[1:] == 0) and torch.any(ft.grad[0] != 0)


class _View:
    def __init__(self, w, h, fovx, fovy, wvt):
        self.image_width, self.image_height, self.FoVx, self.FoVy = w, h, fovx, fovy
        self.world_view_transform = wvt


@pytest.mark.parametrize("jitter", [False, True])
def test_camera_rays_match_oracle(jitter):
    dev = _dev()
    w, h = 333, 211
    ang = 0.7
    R = np.array([[math.cos(ang), -math.sin(ang), 0], [math.sin(ang), math.cos(ang), 0], [0, 0, 1]])
    R = R @ np.array([[1, 0, 0], [0, math.cos(0.4), -math.sin(0.4)], [0, math.sin(0.4), math.cos(0.4)]])
    c2w = np.eye(4)
    c2w[:3, :3] = R
    c2w[:3, 3] = [0.5, -3.0, 2.0]
    wvt = torch.tensor(np.linalg.inv(c2w).T, dtype=torch.float32)  # row-vector convention
    view = _View(w, h, math.radians(55), math.radians(40), wvt)
    gen = torch.Generator(device=dev).manual_seed(5)
    ro, rd = CAM.camera2rays(view, random=jitter, generator=gen)
    off = None
    if jitter:
        off = torch.rand((w * h, 2), generator=torch.Generator(device=dev).manual_seed(5), device=dev).cpu().numpy()
    fx, fy = P.focal(w, view.FoVx), P.focal(h, view.FoVy)
    c2w_used = np.linalg.inv(wvt.double().numpy().T)
    wro, wrd = P.camera_rays(w, h, fx, fy, c2w_used, off)
    np.testing.assert_allclose(ro.cpu().numpy(), wro, atol=1e-6)
    np.testing.assert_allclose(rd.cpu().numpy(), wrd, atol=1e-6)
