"""CPU oracle of the colour pre-pass and of camera ray generation (test infrastructure only:
imported by tests/, never by the product path).

SH evaluation restates the hard-coded SH polynomials of the reference (tests/eval_sh.py
`eval_sh_py`, splinetracers/slang/sh.slang:49-100) for features laid out (N, K, 3); the
colour is the SH sum plus 0.5. The trainer's chain (integration_utils/gaussian_renderer/
ever.py:178-180) adds softplus(beta=10) and RGB2SH. Camera rays restate
integration_utils/gaussian_renderer/ever.py:29-74 and 105-118. The functions use only
arithmetic and indexing, so they run on numpy arrays and on torch tensors (the tests take
fp64 autograd gradients through them).
"""
from __future__ import annotations

import math

import numpy as np

C0 = 0.28209479177387814
C1 = 0.4886025119029199
C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
      1.445305721320277, -0.5900435899266435]


def sh_colour(deg, feats, dirs):
    """feats (N, K, 3), dirs (N, 3) unit -> (N, 3) colour = SH sum + 0.5."""
    f = lambda k: feats[:, k, :]
    x, y, z = dirs[:, 0:1], dirs[:, 1:2], dirs[:, 2:3]
    r = C0 * f(0)
    if deg > 0:
        r = r - C1 * y * f(1) + C1 * z * f(2) - C1 * x * f(3)
    if deg > 1:
        xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
        r = (r + C2[0] * xy * f(4) + C2[1] * yz * f(5) + C2[2] * (2.0 * zz - xx - yy) * f(6) + C2[3] * xz * f(7) +
             C2[4] * (xx - yy) * f(8))
    if deg > 2:
        r = (r + C3[0] * y * (3 * xx - yy) * f(9) + C3[1] * xy * z * f(10) + C3[2] * y * (4 * zz - xx - yy) * f(11) +
             C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * f(12) + C3[4] * x * (4 * zz - xx - yy) * f(13) +
             C3[5] * z * (xx - yy) * f(14) + C3[6] * x * (xx - 3 * yy) * f(15))
    return r + 0.5


def directions(means, cam):
    v = means - cam.reshape(1, 3)
    n = (v * v).sum(1, keepdims=True) ** 0.5 if isinstance(v, np.ndarray) else (v * v).sum(1, keepdim=True) ** 0.5
    return v / n


def softplus10(x):
    """torch.nn.functional.softplus(x, beta=10) (threshold 20)."""
    if isinstance(x, np.ndarray):
        return np.where(10 * x > 20, x, np.log1p(np.exp(np.minimum(10 * x, 20))) / 10)
    import torch
    return torch.where(10 * x > 20, x, torch.log1p(torch.exp(torch.clamp(10 * x, max=20))) / 10)


def rgb2sh(rgb):
    return (rgb - 0.5) / C0


def eval_sh(means, feats, cam, deg):
    return sh_colour(deg, feats, directions(means, cam))


def sh_features(means, feats, cam, deg):
    """The trainer's tracer input: RGB2SH(softplus(eval_sh, beta=10)), (N, 1, 3)."""
    return rgb2sh(softplus10(eval_sh(means, feats, cam, deg))).reshape(-1, 1, 3)


def camera_rays(width, height, fx, fy, c2w, offsets=None):
    """(rayo, rayd) float64, row-major pixels; offsets (H*W, 2) or pixel centres."""
    c2w = np.asarray(c2w, np.float64).reshape(-1, 4)[:3]
    row, col = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    row, col = row.reshape(-1).astype(np.float64), col.reshape(-1).astype(np.float64)
    ox, oy = (0.5, 0.5) if offsets is None else (offsets[:, 0], offsets[:, 1])
    d = np.stack([(col + ox - width / 2) / fx, (row + oy - height / 2) / fy, np.ones_like(col)], 1)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    rayd = d @ c2w[:, :3].T
    rayo = np.broadcast_to(c2w[:, 3], rayd.shape)
    return rayo, rayd


def focal(size, fov):
    return 0.5 * size / math.tan(0.5 * fov)
