"""Drop-in for splinetracers.fast_ellipsoid_splinetracer (N-Demir/ever).

Same entry point, arguments, output layout and autograd behaviour as
splinetracers/fast_ellipsoid_splinetracer.py:37-256:

    trace_rays(mean, scale, quat, density, features, rayo, rayd, tmin=0.0, tmax=1000,
               max_prim_size=3, dL_dmeans2D=None, wcts=None, max_iters=500,
               return_extras=False)
    -> (R,5) [R, G, B, opacity, distortion]  (or (out, extras) with return_extras)

`trace_rays.uses_density` is True, as callers test it (ever.py:184). The backward
returns the 14 gradient slots of SplineTracer.backward (:204-219) with the same
clipping. Everything runs in libever_b200.so: an LBVH built on the device per call
(the reference rebuilds its GAS per call as well, :66-71), a CUDA traversal/integration
kernel and a CUDA reverse-replay backward.

Colour: by default (sh_degree=None) every event takes the ellipsoid's DC colour
C0 * f0 + 0.5 whatever the size K of features (N,K,3), exactly as the reference's forward
(shaders.slang:72-75: get_sh(sh_feats, 0), eval_sh_col0), and the backward differentiates
that colour: feature gradients of the coefficients k >= 1 are zero. The reference's
backward instead differentiates SH of degree sqrt(K)-1 along rayd
(backwards_kernel.slang:162, 238) against the DC-built states, so for K > 1 its feature
gradients are those of a colour its forward never computed; this drop-in returns the
gradients of the image it returned. Opt in to view-dependent colour with sh_degree=d
(1..3, needs (d+1)^2 <= K): SH of degree d evaluated along the raw ray direction rayd in
both passes.

Status: the kernels never trap; overflows of fixed-size device structures raise flags in
a status word, returned as extras["status"] with return_extras=True (see the EVER_STATUS_*
flags in include/ever_b200.h).

Launch order: by default the rays are first sorted into a coherent order on the device
(ray_order="auto", see ever_ray_order in include/ever_b200.h) so that each warp's packet
covers a compact patch of directions; pass ray_order=None for the given order or an
int32 permutation of your own. Results never depend on it.
"""
from __future__ import annotations

from typing import Any

import torch
from torch.autograd import Function

from . import tracer as T

_SIDE_STREAMS: dict = {}


def _side_stream(device) -> torch.cuda.Stream:
    """One side stream per device for work that overlaps the BVH build."""
    key = torch.device(device).index
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = torch.cuda.Stream(device)
    return _SIDE_STREAMS[key]

__all__ = ["SplineTracer", "trace_rays", "SavedForBackward"]


class SavedForBackward:
    """Mirror of the reference's fesSavedForBackward (py_binding.cpp:151-193)."""

    def __init__(self, states, diracs, iters, touch_count, faces=None):
        self.states = states
        self.diracs = diracs
        self.iters = iters
        self.touch_count = touch_count
        self.faces = faces if faces is not None else torch.zeros_like(iters)


class SplineTracer(Function):
    @staticmethod
    def forward(
        ctx: Any,
        mean: torch.Tensor,
        scale: torch.Tensor,
        quat: torch.Tensor,
        density: torch.Tensor,
        color: torch.Tensor,
        rayo: torch.Tensor,
        rayd: torch.Tensor,
        tmin: float,
        tmax: float,
        max_prim_size: float,
        mean2D: torch.Tensor,
        wcts: torch.Tensor,
        max_iters: int,
        return_extras: bool = False,
        sh_degree: int | None = None,
        tune: T.Tune | None = None,
        ray_order="auto",
    ):
        ctx.device = rayo.device
        if tune is None:  # the autotuner's cached pick for this workload, if it ran on it
            from .autotune import cached_tune
            pick = cached_tune(mean.shape[0], rayo.shape[0], color.shape[1], rayo.device)
            if pick is not None:
                # the full stack depth stays: the pick's depth was clean on the tuned scene, and
                # a deeper tree in the same size bucket must not lose subtrees
                tune = T.Tune(kbuf=pick.kbuf, block=pick.block, traversal=pick.traversal)
                if not pick.ordered and isinstance(ray_order, str):
                    ray_order = None
        if isinstance(ray_order, str) and ray_order != "auto":
            raise RuntimeError(f"ray_order must be 'auto', None or an int32 tensor, got {ray_order!r}")
        if isinstance(ray_order, str) and rayo.shape[0] > 0 and rayo.is_cuda:
            # the coherent ray order needs only the rays: it runs on a side stream while the
            # BVH is built on the caller's stream
            main = torch.cuda.current_stream(rayo.device)
            side = _side_stream(rayo.device)
            side.wait_stream(main)
            with torch.cuda.stream(side):
                ray_order = T.ray_order(rayo, rayd)
            rayo.record_stream(side)
            rayd.record_stream(side)
            scene = T.Scene(mean, scale, quat, density, color, dc_only=not sh_degree)
            main.wait_stream(side)
            ray_order.record_stream(main)
        else:
            scene = T.Scene(mean, scale, quat, density, color, dc_only=not sh_degree)
            if isinstance(ray_order, str):
                ray_order = None
        needs_grad = any(ctx.needs_input_grad[:7]) or (mean2D is not None and ctx.needs_input_grad[10])
        fwd = T.forward(scene, rayo, rayd, tmin, tmax, max_iters, sh_degree,
                        log_events=needs_grad or return_extras, touch_count=return_extras, ray_order=ray_order,
                        tune=tune)
        ctx.ray_order = ray_order
        ctx.scene = scene
        ctx.fwd = fwd
        ctx.tmin, ctx.tmax, ctx.max_iters = tmin, tmax, max_iters
        ctx.max_prim_size = max_prim_size
        ctx.sh_degree = sh_degree
        ctx.tune = tune
        ctx.has_wcts = wcts is not None
        ctx.density_shape = density.shape
        ctx.save_for_backward(rayo, rayd, wcts)
        out = fwd.out
        if return_extras:
            saved = SavedForBackward(fwd.states, fwd.last_dirac, fwd.iters, fwd.touch_count)
            return out, dict(
                tri_collection=T.reference_tri_collection(scene, fwd, max_iters, ray_order)
                if fwd.event_log is not None
                else torch.zeros(rayo.shape[0] * max_iters, dtype=torch.int32, device=rayo.device),
                iters=fwd.iters,
                opacity=out[:, 3],
                touch_count=fwd.touch_count,
                distortion_loss=out[:, 4],
                saved=saved,
                # (1,) int32 OR of the EVER_STATUS_* flags the kernels raised (0: clean). Not a
                # reference key: 1 = a traversal stack overflowed (a BVH subtree was skipped),
                # 2 = the event log was too short, 4 = more than 16 ellipsoids contain a ray
                # start (still summed). Read it without a host sync until you need it.
                status=fwd.status,
            )
        return out

    @staticmethod
    def backward(ctx, grad_output: torch.Tensor, *unused):
        rayo, rayd, wcts = ctx.saved_tensors
        # replay order: rays grouped by the number of events the forward consumed (longest
        # first), so a warp's 32 reverse replays run for the same number of steps
        slot_order = T.backward_order(ctx.fwd, ctx.ray_order, 0) if rayo.shape[0] > 0 else None
        g = T.backward(ctx.scene, rayo, rayd, ctx.fwd, grad_output, ctx.tmin, ctx.tmax, ctx.max_iters,
                       ctx.sh_degree, wcts=wcts, want_means2d=ctx.has_wcts, ray_order=ctx.ray_order, tune=ctx.tune,
                       slot_order=slot_order)
        # the event log and scene workspace are not needed again: give them back to the allocator
        ctx.fwd = None
        ctx.scene = None
        return (
            g.mean,
            g.scale,
            g.quat,
            g.density.reshape(ctx.density_shape),
            g.features,
            g.rayo,
            g.rayd,
            None,
            None,
            None,
            g.means2d,
            None,
            None,
            None,
            None,
            None,
            None,
        )


def trace_rays(
    mean: torch.Tensor,
    scale: torch.Tensor,
    quat: torch.Tensor,
    density: torch.Tensor,
    features: torch.Tensor,
    rayo: torch.Tensor,
    rayd: torch.Tensor,
    tmin: float = 0.0,
    tmax: float = 1000,
    max_prim_size: float = 3,
    dL_dmeans2D=None,
    wcts=None,
    max_iters: int = 500,
    return_extras: bool = False,
    sh_degree: int | None = None,
    tune: T.Tune | None = None,
    ray_order="auto",
):
    return SplineTracer.apply(mean, scale, quat, density, features, rayo, rayd, tmin, tmax, max_prim_size,
                              dL_dmeans2D, wcts, max_iters, return_extras, sh_degree, tune, ray_order)


trace_rays.uses_density = True
