"""CPU checks of the colour pre-pass / camera ray oracle (oracle/prepass_np.py) and of the
host validation of their C entry points. No GPU calls."""
import ctypes
import math

import numpy as np
import torch

from ever_b200 import _native as N
from oracle import prepass_np as P


def test_sh_known_answers():
    f = np.zeros((3, 16, 3))
    f[:, 0] = [1.0, -2.0, 0.5]
    f[:, 2] = 1.0  # the z-linear coefficient
    d = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, -1.0], [1.0, 0.0, 0.0]])
    c0 = P.sh_colour(0, f, d)
    np.testing.assert_allclose(c0, P.C0 * f[:, 0] + 0.5)
    c1 = P.sh_colour(1, f, d)
    np.testing.assert_allclose(c1[0], P.C0 * f[0, 0] + 0.5 + P.C1)  # +z sees +C1
    np.testing.assert_allclose(c1[1], P.C0 * f[1, 0] + 0.5 - P.C1)
    np.testing.assert_allclose(c1[2], P.C0 * f[2, 0] + 0.5)
    # higher degrees are linear in the features with the reference constants
    rng = np.random.default_rng(0)
    dd = rng.normal(size=(5, 3))
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    for deg in range(4):
        nb = (deg + 1) ** 2
        for k in range(nb):
            e = np.zeros((5, 16, 3))
            e[:, k, 1] = 1.0
            col = P.sh_colour(deg, e, dd) - 0.5
            assert np.all(col[:, 0] == 0) and np.all(col[:, 2] == 0)
        e = np.zeros((5, 16, 3))
        e[:, nb:, :] = 7.0  # coefficients beyond the degree do not count
        np.testing.assert_allclose(P.sh_colour(deg, e, dd), 0.5)


def test_trainer_chain_and_its_gradient():
    rng = np.random.default_rng(1)
    means = torch.tensor(rng.normal(size=(50, 3)), dtype=torch.float64)
    feats = torch.tensor(rng.normal(size=(50, 16, 3)) * 0.5, dtype=torch.float64, requires_grad=True)
    cam = torch.tensor([0.3, -4.0, 1.0], dtype=torch.float64)
    out = P.sh_features(means, feats, cam, 3)
    col = P.eval_sh(means, feats, cam, 3)
    want = (torch.nn.functional.softplus(col, beta=10) - 0.5) / P.C0
    torch.testing.assert_close(out.reshape(-1, 3), want)
    g = torch.randn(out.shape, dtype=torch.float64)
    (out * g).sum().backward()
    # closed form: dL/df_k = B_k(dir) * sigmoid(10 c) * g / C0
    dirs = P.directions(means, cam)
    with torch.no_grad():
        gc = torch.sigmoid(10 * col) * g.reshape(-1, 3) / P.C0
        for k in range(16):
            e = torch.zeros(50, 16, 3, dtype=torch.float64)
            e[:, k, :] = 1.0
            bk = P.sh_colour(3, e, dirs)[:, 0:1] - 0.5
            torch.testing.assert_close(feats.grad[:, k, :], bk * gc)


def test_camera_rays_oracle_geometry():
    w, h = 64, 48
    fx, fy = P.focal(w, math.radians(60)), P.focal(h, math.radians(45))
    ang = 0.3
    R = np.array([[math.cos(ang), 0, math.sin(ang)], [0, 1, 0], [-math.sin(ang), 0, math.cos(ang)]])
    c2w = np.concatenate([R, np.array([[1.0], [2.0], [3.0]])], 1)
    ro, rd = P.camera_rays(w, h, fx, fy, c2w)
    assert ro.shape == (w * h, 3) and np.allclose(ro, [1, 2, 3])
    np.testing.assert_allclose(np.linalg.norm(rd, axis=1), 1.0)
    # the pixel-corner offset (0, 0) of the centre pixel looks along the camera's +z axis
    off = np.full((w * h, 2), 0.5)
    off[(h // 2) * w + w // 2] = [0.0, 0.0]
    _, rd2 = P.camera_rays(w, h, fx, fy, c2w, off)
    np.testing.assert_allclose(rd2[(h // 2) * w + w // 2], R[:, 2], atol=1e-12)
    # row-major: along a row the x offset grows
    np.testing.assert_allclose((rd[1] @ R)[0] > (rd[0] @ R)[0], True)


def test_prepass_and_camera_abi_validation():
    lib = N.load()
    assert lib.ever_sh_prepass(None, None, 5, 16, 3, None, 1, None, None) == 1
    assert b"null" in lib.ever_last_error()
    assert lib.ever_sh_prepass(None, None, 5, 4, 2, None, 1, None, None) == 1
    assert b"sh_degree" in lib.ever_last_error()
    assert lib.ever_sh_prepass(None, None, 5, 16, 3, None, 2, None, None) == 1
    assert b"mode" in lib.ever_last_error()
    assert lib.ever_sh_prepass(None, None, 0, 16, 3, None, 1, None, None) == 0  # nothing to do
    assert lib.ever_sh_prepass_backward(None, None, 5, 16, 3, None, 0, None, None, None) == 1
    assert lib.ever_camera_rays(None, None, None, None, None) == 1
    cam = N.EverCamera()
    cam.width, cam.height, cam.fx, cam.fy = 4, 4, 0.0, 1.0
    assert lib.ever_camera_rays(ctypes.byref(cam), None, None, None, None) == 1
    assert b"focal" in lib.ever_last_error()
    cam.fx = 1.0
    assert lib.ever_camera_rays(ctypes.byref(cam), None, None, None, None) == 1
    cam.width = cam.height = 0
    assert lib.ever_camera_rays(ctypes.byref(cam), None, None, None, None) == 0
