"""Trained scenes from binary PLY files (ever_ply_count / ever_ply_read).

Reads the reference's scene file layout and applies its conversion
(splinetracers/fast_ellipsoid_splinetracer/ply_file_loader.cc:166-293): returns the
tracer's inputs mean (N,3), scale (N,3), quat (N,4), density (N,1) and features (N,16,3).
"""
from __future__ import annotations

import os

import torch

from . import _native as N


def read_scene(path, device=None):
    lib = N.load()
    p = os.fsencode(os.fspath(path))
    n = int(lib.ever_ply_count(p))
    if n < 0:
        raise RuntimeError(lib.ever_last_error().decode(errors="replace"))
    pin = torch.cuda.is_available()
    host = dict(mean=torch.empty((n, 3)), scale=torch.empty((n, 3)), quat=torch.empty((n, 4)),
                density=torch.empty((n, 1)), features=torch.empty((n, 16, 3)))
    if pin:
        host = {k: v.pin_memory() for k, v in host.items()}
    N.check(lib.ever_ply_read(p, n, N.ptr(host["mean"]), N.ptr(host["scale"]), N.ptr(host["quat"]),
                              N.ptr(host["density"]), N.ptr(host["features"])))
    if device is None:
        return host
    return {k: v.to(device, non_blocking=True) for k, v in host.items()}
