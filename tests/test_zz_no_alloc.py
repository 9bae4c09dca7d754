"""ever_ray_order_static: the coherent ray order for callers that cannot allocate device
memory (a viewer's frame loop that must never block on the allocator, a binding from a
runtime that cannot pass this library a workspace). It must give exactly what the
workspace version ever_ray_order gives, call after call, although every call reuses
one static scratch array that still holds the previous call's data.

This file is collected last on purpose, so that a run stopping at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from ever_b200 import _native as N
from ever_b200 import synthetic as S

MAX_RAYS = 1 << 21


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_static_ray_order_rejects_too_many_rays():
    lib = N.load()
    rc = lib.ever_ray_order_static(None, None, MAX_RAYS + 1, None, None)
    assert rc == 1
    assert b"out of range" in lib.ever_last_error()
    assert lib.ever_ray_order_static(None, None, 0, None, None) == 0
    # exactly the maximum passes the scratch-layout check (it fails later, on the null pointers)
    assert lib.ever_ray_order_static(None, None, MAX_RAYS, None, None) == 1
    assert b"null pointer" in lib.ever_last_error()


@pytest.mark.gpu
def test_static_ray_order_matches_workspace_version():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = N.load()
    dev = torch.device("cuda:0")
    # consecutive calls of different sizes: the static array keeps the previous call's contents
    # the last size is exactly the documented maximum: keys, values and histogram fill the array
    for W, H, seed in [(640, 480, 1), (1920, 1080, 2), (320, 240, 3), (2048, 1024, 4)]:
        ro, rd = S.look_at_rays(S.Camera(S.sphere_point(4.0, seed), W, H, 50.0))
        rayo = torch.tensor(ro, device=dev)
        rayd = torch.tensor(rd, device=dev)
        R = rayo.shape[0]
        ref = torch.empty(R, dtype=torch.int32, device=dev)
        ws = torch.empty(max(int(lib.ever_ray_order_workspace_bytes(R)), 256), dtype=torch.uint8, device=dev)
        N.check(lib.ever_ray_order(N.ptr(rayo), N.ptr(rayd), R, N.ptr(ws), int(ws.numel()), N.ptr(ref), _stream()))
        got = torch.full((R,), -1, dtype=torch.int32, device=dev)
        N.check(lib.ever_ray_order_static(N.ptr(rayo), N.ptr(rayd), R, N.ptr(got), _stream()))
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (W, H)
        assert np.array_equal(np.sort(got.cpu().numpy()), np.arange(R))
