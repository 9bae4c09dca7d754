"""Per-ellipsoid SH colour from the camera centre, and the trainer's fused colour pre-pass.

`eval_sh(means, features, rayo, sh_degree)` has the reference's signature and autograd
behaviour (eval_sh.py:28-82 of the reference, sh_kernel.slang:21-99): (N,3) colours, SH of
degree `sh_degree` in the direction from the camera centre `rayo` to each mean, plus 0.5;
the backward gives the feature gradient only.

`sh_features(means, features, cam_pos, sh_degree)` is what the trainer feeds the tracer
(integration_utils/gaussian_renderer/ever.py:178-180): RGB2SH(softplus(eval_sh(...), beta=10))
as (N,1,3), computed in one kernel (and one backward kernel) instead of three passes.
"""
from __future__ import annotations

import ctypes
from typing import Any

import torch
from torch.autograd import Function

from . import _native as N


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _check(means, features, cam, sh_degree):
    for name, t in (("means", means), ("features", features), ("ray_origin", cam)):
        if not t.is_cuda or t.dtype != torch.float32:
            raise RuntimeError(f"{name} must be a float32 CUDA tensor")
    if means.dim() != 2 or means.shape[1] != 3:
        raise RuntimeError("means must have shape (N, 3)")
    if features.dim() != 3 or features.shape[0] != means.shape[0] or features.shape[2] != 3:
        raise RuntimeError("features must have shape (N, K, 3)")
    if cam.numel() != 3:
        raise RuntimeError("ray_origin must hold 3 floats")
    if not 0 <= int(sh_degree) <= 3 or (int(sh_degree) + 1) ** 2 > features.shape[1]:
        raise RuntimeError(f"sh_degree {sh_degree} needs (sh_degree+1)^2 <= K = {features.shape[1]}")


def _run(means, features, cam, sh_degree, mode, grad_out=None):
    lib = N.load()
    n, k = means.shape[0], features.shape[1]
    with torch.cuda.device(means.device):
        if grad_out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device=means.device)
            N.check(lib.ever_sh_prepass(N.ptr(means), N.ptr(features), n, k, int(sh_degree), N.ptr(cam), mode,
                                        N.ptr(out), _stream(means.device)))
        else:
            out = torch.empty_like(features)
            N.check(lib.ever_sh_prepass_backward(N.ptr(means), N.ptr(features), n, k, int(sh_degree), N.ptr(cam),
                                                 mode, N.ptr(grad_out), N.ptr(out), _stream(means.device)))
    return out


class _Prepass(Function):
    @staticmethod
    def forward(ctx: Any, means, features, rayo, sh_degree, mode):
        means = means.detach().contiguous()
        features = features.detach().contiguous()
        cam = rayo.detach().reshape(3).contiguous()
        _check(means, features, cam, sh_degree)
        ctx.sh_degree, ctx.mode = int(sh_degree), int(mode)
        ctx.save_for_backward(means, features, cam)
        return _run(means, features, cam, sh_degree, mode)

    @staticmethod
    def backward(ctx, grad_out):
        means, features, cam = ctx.saved_tensors
        g = _run(means, features, cam, ctx.sh_degree, ctx.mode, grad_out.contiguous().float())
        return None, g, None, None, None


class EvalSH(Function):
    """The reference's EvalSH: (means, features, rayo, sh_degree) -> (N,3) colours."""

    @staticmethod
    def forward(ctx: Any, means, features, rayo, sh_degree):
        return _Prepass.forward(ctx, means, features, rayo, sh_degree, 0)

    @staticmethod
    def backward(ctx, grad_out):
        return _Prepass.backward(ctx, grad_out)[:4]


def eval_sh(means, features, rayo, sh_degree):
    return EvalSH.apply(means, features, rayo, sh_degree)


def sh_features(means, features, cam_pos, sh_degree):
    """RGB2SH(softplus(eval_sh(means, features, cam_pos, sh_degree), beta=10)).reshape(-1, 1, 3)."""
    return _Prepass.apply(means, features, cam_pos, sh_degree, 1).reshape(-1, 1, 3)
