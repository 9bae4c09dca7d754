"""Camera ray generation on the device (ever_camera_rays).

`camera2rays(view, random=False)` follows the trainer's camera2rays / get_ray_directions /
get_rays (integration_utils/gaussian_renderer/ever.py:29-74, 105-118): one ray per pixel,
row-major, pinhole focal lengths from the view's fields of view, principal point at the
image centre, directions normalised in the camera frame and rotated to the world,
origins at the camera centre. `view` needs image_width, image_height, FoVx, FoVy and
world_view_transform (4x4, row-vector convention: camera-to-world = inv(wvt.T)).
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _native as N


def camera_rays(width, height, fx, fy, c2w, cx=None, cy=None, jitter=None, device=None):
    """(rayo, rayd), each (width*height, 3) float32 on `device`. c2w: 3x4 (or 4x4)
    camera-to-world matrix. jitter: optional (width*height, 2) per-pixel offsets."""
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    m = torch.as_tensor(c2w, dtype=torch.float64).cpu().reshape(-1, 4)[:3]
    cam = N.EverCamera()
    cam.width, cam.height = int(width), int(height)
    cam.fx, cam.fy = float(fx), float(fy)
    cam.cx = float(width) / 2 if cx is None else float(cx)
    cam.cy = float(height) / 2 if cy is None else float(cy)
    cam.c2w = (ctypes.c_float * 12)(*[float(v) for v in m.reshape(-1)])
    R = int(width) * int(height)
    rayo = torch.empty((R, 3), dtype=torch.float32, device=device)
    rayd = torch.empty((R, 3), dtype=torch.float32, device=device)
    if jitter is not None:
        jitter = jitter.to(device=device, dtype=torch.float32).contiguous()
        if jitter.numel() != 2 * R:
            raise RuntimeError("jitter must hold (width*height, 2) offsets")
    with torch.cuda.device(device):
        N.check(N.load().ever_camera_rays(ctypes.byref(cam), N.ptr(jitter), N.ptr(rayo), N.ptr(rayd),
                                          ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)))
    return rayo, rayd


def camera2rays(view, random=False, generator=None, device=None):
    """The trainer's camera2rays for a 3DGS-style view (random: uniform per-pixel jitter)."""
    w, h = int(view.image_width), int(view.image_height)
    fx = 0.5 * w / math.tan(0.5 * float(view.FoVx))
    fy = 0.5 * h / math.tan(0.5 * float(view.FoVy))
    wvt = torch.as_tensor(view.world_view_transform, dtype=torch.float64).cpu()
    c2w = torch.linalg.inv(wvt.T)
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    jitter = None
    if random:
        jitter = torch.rand((w * h, 2), generator=generator, device=device)
    return camera_rays(w, h, fx, fy, c2w, jitter=jitter, device=device)
