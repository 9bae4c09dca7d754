"""Seeded synthetic scenes and pinhole cameras for the trace workloads.

Distributions (all float32):
  uniform scene   means U[-1,1]^3, scales exp(U[ln .02, ln .2]) per axis, quats
                  normalise(N(0,1)^4), densities exp(U[ln .1, ln 50]),
                  SH features N(0, 0.5) at degree 0 or N(0, 0.3) at degree 3.
  clustered scene 2,000 thin sheets with centres U[-2,2]^3, each a random orthonormal
                  frame with in-plane offsets N(0, 0.3^2) and normal offsets
                  N(0, 0.01^2); ellipsoids assigned uniformly to sheets; scales
                  exp(U[ln .002, ln .05]); densities exp(U[ln 1, ln 200]); SH degree 3
                  features N(0, 0.3).
Cameras are pinholes looking at the origin; rays are one per pixel, row-major,
unit directions. These stand in for trained scenes, which the reference does not ship.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class SceneArrays:
    mean: np.ndarray      # (N,3)
    scale: np.ndarray     # (N,3)
    quat: np.ndarray      # (N,4) (r,x,y,z)
    density: np.ndarray   # (N,1)
    features: np.ndarray  # (N,K,3)

    @property
    def N(self):
        return self.mean.shape[0]

    def subset(self, idx):
        return SceneArrays(self.mean[idx], self.scale[idx], self.quat[idx], self.density[idx],
                           self.features[idx])


def _loguniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size)).astype(np.float32)


def _quats(rng, n):
    q = rng.standard_normal((n, 4))
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


def uniform_scene(n, sh_degree=0, seed=0) -> SceneArrays:
    rng = np.random.default_rng(seed)
    K = (sh_degree + 1) ** 2
    sd = 0.5 if sh_degree == 0 else 0.3
    return SceneArrays(
        mean=rng.uniform(-1, 1, (n, 3)).astype(np.float32),
        scale=_loguniform(rng, 0.02, 0.2, (n, 3)),
        quat=_quats(rng, n),
        density=_loguniform(rng, 0.1, 50.0, (n, 1)),
        features=(rng.standard_normal((n, K, 3)) * sd).astype(np.float32),
    )


def clustered_scene(n, sh_degree=3, seed=2, n_clusters=2000, extent=0.3, thickness=0.01) -> SceneArrays:
    rng = np.random.default_rng(seed)
    K = (sh_degree + 1) ** 2
    centres = rng.uniform(-2, 2, (n_clusters, 3))
    frames = np.linalg.qr(rng.standard_normal((n_clusters, 3, 3)))[0]  # random orthonormal frames
    which = rng.integers(0, n_clusters, n)
    local = rng.standard_normal((n, 3)) * np.array([extent, extent, thickness])
    mean = centres[which] + np.einsum("nij,nj->ni", frames[which], local)
    return SceneArrays(
        mean=mean.astype(np.float32),
        scale=_loguniform(rng, 0.002, 0.05, (n, 3)),
        quat=_quats(rng, n),
        density=_loguniform(rng, 1.0, 200.0, (n, 1)),
        features=(rng.standard_normal((n, K, 3)) * 0.3).astype(np.float32),
    )


@dataclass
class Camera:
    eye: np.ndarray
    width: int
    height: int
    fov_y_deg: float


def look_at_rays(cam: Camera):
    """(H*W,3) origins and unit directions, row-major, y down, looking at the origin."""
    eye = np.asarray(cam.eye, np.float64)
    fwd = -eye / np.linalg.norm(eye)
    up = np.array([0.0, 0.0, 1.0]) if abs(fwd[2]) < 0.99 else np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    f = 0.5 * cam.height / np.tan(0.5 * np.deg2rad(cam.fov_y_deg))
    j, i = np.meshgrid(np.arange(cam.width) + 0.5, np.arange(cam.height) + 0.5)
    x = (j - 0.5 * cam.width) / f
    y = (i - 0.5 * cam.height) / f
    d = fwd[None, None] + x[..., None] * right[None, None] - y[..., None] * upv[None, None]
    d = d.reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.broadcast_to(eye, d.shape)
    return np.ascontiguousarray(o, np.float32), np.ascontiguousarray(d, np.float32)


def pinhole(cam: Camera):
    """The look-at camera as (width, height, f, c2w 3x4) of a pinhole with the principal
    point at the image centre (x right, y down, z forward): the rays of look_at_rays."""
    eye = np.asarray(cam.eye, np.float64)
    fwd = -eye / np.linalg.norm(eye)
    up = np.array([0.0, 0.0, 1.0]) if abs(fwd[2]) < 0.99 else np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    f = 0.5 * cam.height / np.tan(0.5 * np.deg2rad(cam.fov_y_deg))
    c2w = np.stack([right, -upv, fwd, eye], axis=1)
    return cam.width, cam.height, f, c2w


def look_at_rays_device(cam: Camera, device):
    """look_at_rays computed with torch on `device` (float64, then float32): same rays up to
    the last float32 bit, without the host round trip for large views."""
    import torch
    eye = torch.tensor(np.asarray(cam.eye, np.float64), device=device)
    fwd = -eye / eye.norm()
    up = torch.tensor([0.0, 0.0, 1.0] if abs(float(fwd[2])) < 0.99 else [0.0, 1.0, 0.0], dtype=torch.float64,
                      device=device)
    right = torch.linalg.cross(fwd, up)
    right = right / right.norm()
    upv = torch.linalg.cross(right, fwd)
    f = 0.5 * cam.height / np.tan(0.5 * np.deg2rad(cam.fov_y_deg))
    i, j = torch.meshgrid(torch.arange(cam.height, dtype=torch.float64, device=device) + 0.5,
                          torch.arange(cam.width, dtype=torch.float64, device=device) + 0.5, indexing="ij")
    x = ((j - 0.5 * cam.width) / f).reshape(-1, 1)
    y = ((i - 0.5 * cam.height) / f).reshape(-1, 1)
    d = fwd[None] + x * right[None] - y * upv[None]
    d = d / d.norm(dim=1, keepdim=True)
    o = eye[None].expand_as(d)
    return o.float().contiguous(), d.float().contiguous()


def sphere_point(radius, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(3)
    return radius * v / np.linalg.norm(v)


def orbit(radius, n_views, elevation_deg=20.0):
    el = np.deg2rad(elevation_deg)
    az = 2 * np.pi * np.arange(n_views) / n_views
    return [radius * np.array([np.cos(a) * np.cos(el), np.sin(a) * np.cos(el), np.sin(el)]) for a in az]


# ---------------------------------------------------------------- named workloads
def workload_small(seed=0):
    """1,000 uniform ellipsoids, SH0, one 64x64 view from (0,0,3), 60 deg FOV, forward only."""
    sc = uniform_scene(1000, 0, seed)
    return sc, [Camera(np.array([0.0, 0.0, 3.0]), 64, 64, 60.0)]


def workload_mid(seed=1, n=100_000, width=800, height=800):
    """100,000 uniform ellipsoids, SH3, one 800x800 view from a seeded point at radius 3."""
    sc = uniform_scene(n, 3, seed)
    return sc, [Camera(sphere_point(3.0, seed), width, height, 60.0)]


def workload_scene(seed=2, n=1_000_000, width=1920, height=1080):
    """1M clustered ellipsoids, SH3, one 1920x1080 view, 50 deg FOV, camera at radius 4."""
    sc = clustered_scene(n, 3, seed)
    return sc, [Camera(sphere_point(4.0, seed), width, height, 50.0)]


def workload_batched(scale=1.0):
    """Three clustered scenes (50k, 500k, 2M; seeds 30-32) and 16 cameras of mixed size."""
    sizes = [int(50_000 * scale), int(500_000 * scale), int(2_000_000 * scale)]
    scenes = [clustered_scene(n, 3, 30 + i) for i, n in enumerate(sizes)]
    rng = np.random.default_rng(33)
    res = [(320, 240), (640, 480), (1280, 720), (1920, 1080)] * 4
    order = rng.permutation(16)
    res = [res[i] for i in order]
    assign = [0] * 4 + [1] * 6 + [2] * 6
    cams = []
    for k in range(16):
        w, h = res[k]
        cams.append((assign[k], Camera(sphere_point(4.0, 100 + k), w, h, 50.0)))
    return scenes, cams


def workload_orbit(n=3_000_000, n_views=64, width=1920, height=1080, seed=4):
    """3M clustered ellipsoids, SH3, a 64-view orbit at radius 4."""
    sc = clustered_scene(n, 3, seed)
    return sc, [Camera(e, width, height, 50.0) for e in orbit(4.0, n_views)]
