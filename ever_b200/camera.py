"""Camera rays on the device: as arrays (ever_camera_rays) or made inside the trace
(ever_trace_forward_camera / ever_trace_backward_camera).

`camera2rays(view, random=False)` follows the trainer's camera2rays / get_ray_directions /
get_rays (integration_utils/gaussian_renderer/ever.py:29-74, 105-118): one ray per pixel,
row-major, pinhole focal lengths from the view's fields of view, principal point at the
image centre, directions normalised in the camera frame and rotated to the world,
origins at the camera centre. `view` needs image_width, image_height, FoVx, FoVy and
world_view_transform (4x4, row-vector convention: camera-to-world = inv(wvt.T)).

`trace_camera(mean, scale, quat, density, features, camera, ...)` is camera2rays followed
by trace_rays (ever.py:105-121, 189-205) in one differentiable call whose kernels make
each pixel's ray themselves: no (R,6) ray arrays, no ray sort (warps take 8x4 pixel
tiles), and the same results bit for bit as trace_rays on camera_rays' rays.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Any

import torch
from torch.autograd import Function

from . import _native as N
from . import tracer as T


@dataclass
class Camera:
    """Pinhole camera: image size, focal lengths and principal point in pixels, and the
    camera-to-world matrix (3x4 or 4x4; rayd = c2w[:3,:3] d, rayo = c2w[:3,3])."""
    width: int
    height: int
    fx: float
    fy: float
    c2w: Any
    cx: float | None = None
    cy: float | None = None

    def c(self) -> N.EverCamera:
        m = torch.as_tensor(self.c2w, dtype=torch.float64).cpu().reshape(-1, 4)[:3]
        cam = N.EverCamera()
        cam.width, cam.height = int(self.width), int(self.height)
        cam.fx, cam.fy = float(self.fx), float(self.fy)
        cam.cx = float(self.width) / 2 if self.cx is None else float(self.cx)
        cam.cy = float(self.height) / 2 if self.cy is None else float(self.cy)
        cam.c2w = (ctypes.c_float * 12)(*[float(v) for v in m.reshape(-1)])
        return cam

    @property
    def num_pixels(self) -> int:
        return int(self.width) * int(self.height)

    @staticmethod
    def from_view(view) -> "Camera":
        """The camera of a 3DGS-style view, as the trainer's camera2rays sees it."""
        w, h = int(view.image_width), int(view.image_height)
        fx = 0.5 * w / math.tan(0.5 * float(view.FoVx))
        fy = 0.5 * h / math.tan(0.5 * float(view.FoVy))
        wvt = torch.as_tensor(view.world_view_transform, dtype=torch.float64).cpu()
        return Camera(w, h, fx, fy, torch.linalg.inv(wvt.T))


def _device(device):
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _jitter(jitter, R, device):
    if jitter is None:
        return None
    jitter = jitter.to(device=device, dtype=torch.float32).contiguous()
    if jitter.numel() != 2 * R:
        raise RuntimeError("jitter must hold (width*height, 2) offsets")
    return jitter


def camera_rays(width, height, fx, fy, c2w, cx=None, cy=None, jitter=None, device=None):
    """(rayo, rayd), each (width*height, 3) float32 on `device`. c2w: 3x4 (or 4x4)
    camera-to-world matrix. jitter: optional (width*height, 2) per-pixel offsets."""
    device = _device(device)
    camera = Camera(width, height, fx, fy, c2w, cx, cy)
    cam = camera.c()
    R = camera.num_pixels
    rayo = torch.empty((R, 3), dtype=torch.float32, device=device)
    rayd = torch.empty((R, 3), dtype=torch.float32, device=device)
    jitter = _jitter(jitter, R, device)
    with torch.cuda.device(device):
        N.check(N.load().ever_camera_rays(ctypes.byref(cam), N.ptr(jitter), N.ptr(rayo), N.ptr(rayd),
                                          _stream(device)))
    return rayo, rayd


def camera2rays(view, random=False, generator=None, device=None):
    """The trainer's camera2rays for a 3DGS-style view (random: uniform per-pixel jitter)."""
    camera = Camera.from_view(view)
    device = _device(device)
    jitter = None
    if random:
        jitter = torch.rand((camera.num_pixels, 2), generator=generator, device=device)
    return camera_rays(camera.width, camera.height, camera.fx, camera.fy, camera.c2w, jitter=jitter, device=device)


def camera_slots(camera: Camera) -> int:
    """Launch slots of a camera trace: 32 per 8x4 pixel tile."""
    n = N.load().ever_camera_slots(ctypes.byref(camera.c()))
    if n < 0:
        N.check(1)
    return int(n)


def slot_pixels(camera: Camera, device=None) -> torch.Tensor:
    """(slots,) int32: the pixel each slot of a camera trace traces, -1 for padding."""
    device = _device(device)
    out = torch.empty(camera_slots(camera), dtype=torch.int32, device=device)
    with torch.cuda.device(device):
        N.check(N.load().ever_camera_slot_pixels(ctypes.byref(camera.c()), N.ptr(out), _stream(device)))
    return out


def forward(scene: T.Scene, camera: Camera, jitter=None, tmin=0.0, tmax=1000.0, max_iters=500, sh_degree=None,
            log_events=True, touch_count=False, ray_stats=False, tune: T.Tune | None = None,
            regrouped: bool = True) -> T.ForwardResult:
    """Forward trace of the camera's pixels; results by pixel, event-log columns by slot.
    regrouped: with k-buffers of up to 16 events, pack the pixels still active after the
    first gather rounds into full warps (ever_trace_forward_camera_regrouped; same results)."""
    device = scene.device
    R, S = camera.num_pixels, camera_slots(camera)
    jitter = _jitter(jitter, R, device)
    f32 = dict(dtype=torch.float32, device=device)
    res = T.ForwardResult(
        out=torch.empty((R, 5), **f32), states=torch.empty((R, 16), **f32), last_dirac=torch.empty((R, 4), **f32),
        iters=torch.empty(R, dtype=torch.int32, device=device),
        event_log=(torch.empty((S, max(int(max_iters), 0)), dtype=torch.int32, device=device)
                   if log_events else None),
        touch_count=(torch.zeros(scene.num_prims, dtype=torch.int32, device=device) if touch_count else None),
        ray_stats=(torch.empty((R, 2), **f32) if ray_stats else None),
        status=torch.zeros(1, dtype=torch.int32, device=device))
    o = N.EverForwardOut()
    o.out, o.states, o.last_dirac, o.iters = N.ptr(res.out), N.ptr(res.states), N.ptr(res.last_dirac), N.ptr(res.iters)
    o.event_log = N.ptr(res.event_log)
    o.log_cap = 0 if res.event_log is None else res.event_log.shape[1]
    o.touch_count = N.ptr(res.touch_count)
    o.ray_stats = N.ptr(res.ray_stats)
    o.status = N.ptr(res.status)
    args = T.trace_args(tmin, tmax, max_iters, sh_degree)
    tune = tune or T.Tune()
    lib = N.load()
    with torch.cuda.device(device):
        if regrouped and tune.kbuf <= 16:
            ws = torch.empty(max(int(lib.ever_trace_forward_workspace_bytes(S)), 256), dtype=torch.uint8,
                             device=device)
            N.check(lib.ever_trace_forward_camera_regrouped(ctypes.byref(scene.c), ctypes.byref(camera.c()),
                                                            N.ptr(jitter), ctypes.byref(args), ctypes.byref(tune.c()),
                                                            ctypes.byref(o), N.ptr(ws), int(ws.numel()),
                                                            _stream(device)))
        else:
            N.check(lib.ever_trace_forward_camera(ctypes.byref(scene.c), ctypes.byref(camera.c()), N.ptr(jitter),
                                                  ctypes.byref(args), ctypes.byref(tune.c()), ctypes.byref(o),
                                                  _stream(device)))
    return res


def backward_order(camera: Camera, fwd: T.ForwardResult, shift: int = 0) -> torch.Tensor:
    """Backward launch order over a camera trace's slots (longest replays first)."""
    device = fwd.iters.device
    S = camera_slots(camera)
    lib = N.load()
    need = int(lib.ever_ray_order_workspace_bytes(S))
    ws = torch.empty(max(need, 256), dtype=torch.uint8, device=device)
    order = torch.empty(S, dtype=torch.int32, device=device)
    with torch.cuda.device(device):
        N.check(lib.ever_camera_backward_slot_order(ctypes.byref(camera.c()), N.ptr(fwd.iters), int(shift),
                                                    N.ptr(ws), int(ws.numel()), N.ptr(order), _stream(device)))
    return order


def backward(scene: T.Scene, camera: Camera, fwd: T.ForwardResult, grad_out, jitter=None, tmin=0.0, tmax=1000.0,
             max_iters=500, sh_degree=None, wcts=None, want_means2d=False, want_ray_grads=False,
             tune: T.Tune | None = None, slot_order=None) -> T.Gradients:
    """Backward of forward(); ray gradients (by pixel) only with want_ray_grads."""
    device = scene.device
    if fwd.event_log is None:
        raise RuntimeError("backward needs the forward's event log (log_events=True)")
    R = camera.num_pixels
    jitter = _jitter(jitter, R, device)
    grad_out = grad_out.contiguous()
    n = scene.num_prims
    m, s, q, d, f = scene.tensors
    f32 = dict(dtype=torch.float32, device=device)
    g = T.Gradients(torch.empty((n, 3), **f32), torch.empty((n, 3), **f32), torch.empty((n, 4), **f32),
                    torch.empty(n, **f32), torch.empty(f.shape, **f32),
                    torch.empty((R, 3), **f32) if want_ray_grads else None,
                    torch.empty((R, 3), **f32) if want_ray_grads else None,
                    torch.zeros((n, 2), **f32) if want_means2d else None)
    lib = N.load()
    need = lib.ever_backward_workspace_bytes(n, scene.sh_coeffs)
    ws = torch.empty(max(int(need), 256), dtype=torch.uint8, device=device)
    wct, num_wct = None, 0
    if wcts is not None and want_means2d:
        wct = wcts.detach().to(device=device, dtype=torch.float32).contiguous().reshape(-1, 4, 4)
        num_wct = wct.shape[0]
    if slot_order is not None:
        T._check_tensor("slot_order", slot_order, device, None, torch.int32)
    o = N.EverBackwardOut()
    o.dmean, o.dscale, o.dquat, o.ddensity = N.ptr(g.mean), N.ptr(g.scale), N.ptr(g.quat), N.ptr(g.density)
    o.dfeatures, o.drayo, o.drayd, o.dmeans2d = N.ptr(g.features), N.ptr(g.rayo), N.ptr(g.rayd), N.ptr(g.means2d)
    args = T.trace_args(tmin, tmax, max_iters, sh_degree)
    with torch.cuda.device(device):
        N.check(lib.ever_trace_backward_camera(
            ctypes.byref(scene.c), ctypes.byref(camera.c()), N.ptr(jitter), ctypes.byref(args), N.ptr(grad_out),
            N.ptr(fwd.states), N.ptr(fwd.iters), N.ptr(fwd.event_log), fwd.event_log.shape[1], N.ptr(wct), num_wct,
            N.ptr(m), N.ptr(s), N.ptr(q), N.ptr(ws), int(ws.numel()), N.ptr(slot_order),
            ctypes.byref((tune or T.Tune()).c()), ctypes.byref(o), _stream(device)))
    return g


def tri_collection(scene: T.Scene, camera: Camera, fwd: T.ForwardResult, max_iters: int) -> torch.Tensor:
    """The reference's tri_collection (R*max_iters,) by pixel, from a camera trace's log."""
    R = camera.num_pixels
    log = fwd.event_log
    if log is None or R == 0 or max_iters <= 0:
        return torch.zeros(R * max(int(max_iters), 0), dtype=torch.int32, device=scene.device)
    tri = torch.empty(R * int(max_iters), dtype=torch.int32, device=scene.device)
    with torch.cuda.device(scene.device):
        N.check(N.load().ever_camera_event_log_to_reference(ctypes.byref(scene.c), ctypes.byref(camera.c()),
                                                            N.ptr(log), log.shape[1], N.ptr(fwd.iters), N.ptr(tri),
                                                            int(max_iters), _stream(scene.device)))
    return tri


class CameraTracer(Function):
    @staticmethod
    def forward(ctx, mean, scale, quat, density, features, camera, jitter, tmin, tmax, max_prim_size, mean2D,
                wcts, max_iters, return_extras, sh_degree, tune):
        scene = T.Scene(mean, scale, quat, density, features)
        needs_grad = any(ctx.needs_input_grad[:5]) or (mean2D is not None and ctx.needs_input_grad[10])
        fwd = forward(scene, camera, jitter, tmin, tmax, max_iters, sh_degree, log_events=needs_grad or return_extras,
                      touch_count=return_extras, tune=tune)
        ctx.scene, ctx.fwd, ctx.camera = scene, fwd, camera
        ctx.tmin, ctx.tmax, ctx.max_iters, ctx.sh_degree, ctx.tune = tmin, tmax, max_iters, sh_degree, tune
        ctx.has_wcts = wcts is not None
        ctx.density_shape = density.shape
        ctx.save_for_backward(jitter, wcts)
        out = fwd.out
        if return_extras:
            from .fast_ellipsoid_splinetracer import SavedForBackward
            R = camera.num_pixels
            return out, dict(
                tri_collection=tri_collection(scene, camera, fwd, max_iters) if fwd.event_log is not None
                else torch.zeros(R * max_iters, dtype=torch.int32, device=mean.device),
                iters=fwd.iters, opacity=out[:, 3], touch_count=fwd.touch_count, distortion_loss=out[:, 4],
                saved=SavedForBackward(fwd.states, fwd.last_dirac, fwd.iters, fwd.touch_count))
        return out

    @staticmethod
    def backward(ctx, grad_output, *unused):
        jitter, wcts = ctx.saved_tensors
        order = backward_order(ctx.camera, ctx.fwd) if ctx.camera.num_pixels > 0 else None
        g = backward(ctx.scene, ctx.camera, ctx.fwd, grad_output, jitter, ctx.tmin, ctx.tmax, ctx.max_iters,
                     ctx.sh_degree, wcts=wcts, want_means2d=ctx.has_wcts, tune=ctx.tune, slot_order=order)
        ctx.fwd = None
        ctx.scene = None
        return (g.mean, g.scale, g.quat, g.density.reshape(ctx.density_shape), g.features, None, None, None, None,
                None, g.means2d, None, None, None, None, None)


def trace_camera(mean, scale, quat, density, features, camera: Camera, tmin: float = 0.0, tmax: float = 1000,
                 max_prim_size: float = 3, dL_dmeans2D=None, wcts=None, max_iters: int = 500,
                 return_extras: bool = False, sh_degree: int | None = None, tune: T.Tune | None = None,
                 jitter=None):
    """trace_rays(..., *camera_rays(camera), ...) with the rays made in the kernels: (R,5)
    by pixel, row-major. jitter: optional (R,2) per-pixel offsets (pixel centres if None)."""
    return CameraTracer.apply(mean, scale, quat, density, features, camera, jitter, tmin, tmax, max_prim_size,
                              dL_dmeans2D, wcts, max_iters, return_extras, sh_degree, tune)
