"""Host-side objects over the C ABI: scene build, forward and backward launches.

PyTorch provides device memory and the current CUDA stream; all compute runs in
libever_b200.so. Nothing here synchronises the host.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _native as N


def _check_tensor(name, t, device, last_dim=None, dtype=torch.float32):
    # mirrors the TORCH_CHECKs of py_binding.cpp:33-61
    if not isinstance(t, torch.Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if t.device != device:
        raise RuntimeError(f"{name} must be on the same device")
    if t.dtype != dtype:
        raise RuntimeError(f"{name} must have float32 type" if dtype == torch.float32 else f"{name} must be {dtype}")
    if last_dim is not None and t.shape[-1] != last_dim:
        raise RuntimeError(f"{name} must have last dimension with size {last_dim}")


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


@dataclass
class Tune:
    kbuf: int = 16
    block: int = 128
    traversal: int = 0  # 0: warp packets with the frustum phase, 1: one walk per ray, 2: packets, rounds only
    regroup_min: int = 0  # regrouped forward: rays below which a pass runs every remaining round (0: auto)
    stack_depth: int = 0  # traversal stack entries in use, 8..64 (0: 64)

    def c(self):
        t = N.EverTune()
        t.kbuf, t.block, t.traversal, t.regroup_min = self.kbuf, self.block, self.traversal, self.regroup_min
        t.stack_depth = self.stack_depth
        return t


class Scene:
    """An LBVH over the ellipsoids plus Morton-ordered records, in one device workspace.

    Counterpart of the reference's Primitives + GAS pair (py_binding.cpp:94-149); built
    on the device with no host synchronisation. Keeps references to the input tensors.
    """

    def __init__(self, mean, scale, quat, density, features, dc_only: bool = False):
        """dc_only: keep only each ellipsoid's DC colour (ever_scene_build_dc); traces of
        sh_degree > 0 on the scene are then refused."""
        device = mean.device
        _check_tensor("means", mean, device, 3)
        _check_tensor("scales", scale, device, 3)
        _check_tensor("quats", quat, device, 4)
        _check_tensor("densities", density, device)
        _check_tensor("colors", features, device, 3)
        n = mean.shape[0]
        for name, t in (("scales", scale), ("quats", quat), ("colors", features), ("densities", density)):
            if t.shape[0] != n:
                raise RuntimeError(f"All inputs ({name}) must have the same 0 dimension")
        if features.dim() != 3:
            raise RuntimeError("Features must have 3 channels. (N, d, 3)")
        if density.numel() != n:
            raise RuntimeError("densities must hold one value per ellipsoid")
        self.device = device
        self.tensors = tuple(t.contiguous() for t in (mean, scale, quat, density, features))
        self.num_prims = n
        self.sh_coeffs = features.shape[1]
        self.dc_only = bool(dc_only)
        lib = N.load()
        nbytes = lib.ever_scene_workspace_bytes(n, self.sh_coeffs)
        self.workspace = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        self.c = N.EverScene()
        m, s, q, d, f = self.tensors
        with torch.cuda.device(device):
            build = lib.ever_scene_build_dc if self.dc_only else lib.ever_scene_build
            N.check(build(N.ptr(m), N.ptr(s), N.ptr(q), N.ptr(d), N.ptr(f), n, self.sh_coeffs,
                          N.ptr(self.workspace), int(self.workspace.numel()), ctypes.byref(self.c), _stream(device)))

    def rebuild(self):
        """Rebuilds the BVH and records in place from the (possibly updated) input tensors.

        The workspace and every device pointer of the scene stay the same, so launches
        recorded in a CUDA graph keep working across rebuilds.
        """
        m, s, q, d, f = self.tensors
        with torch.cuda.device(self.device):
            lib = N.load()
            build = lib.ever_scene_build_dc if self.dc_only else lib.ever_scene_build
            N.check(build(N.ptr(m), N.ptr(s), N.ptr(q), N.ptr(d), N.ptr(f), self.num_prims, self.sh_coeffs,
                          N.ptr(self.workspace), int(self.workspace.numel()), ctypes.byref(self.c),
                          _stream(self.device)))

    def refit(self, with_features=True):
        """Refits the BVH in place to the (updated) input tensors, keeping the last build's
        Morton order and tree topology: cheaper than rebuild() between small updates."""
        m, s, q, d, f = self.tensors
        with torch.cuda.device(self.device):
            N.check(N.load().ever_scene_refit(N.ptr(m), N.ptr(s), N.ptr(q), N.ptr(d),
                                              N.ptr(f) if with_features else None, N.ptr(self.workspace),
                                              int(self.workspace.numel()), ctypes.byref(self.c),
                                              _stream(self.device)))

    def set_features(self, features):
        _check_tensor("colors", features, self.device, 3)
        if features.shape[0] != self.num_prims or features.shape[1] != self.sh_coeffs:
            raise RuntimeError("All inputs (colors) must have the same 0 dimension")
        f = features.contiguous()
        self.tensors = self.tensors[:4] + (f,)
        with torch.cuda.device(self.device):
            N.check(N.load().ever_scene_set_features(ctypes.byref(self.c), N.ptr(f), _stream(self.device)))


@dataclass
class ForwardResult:
    out: torch.Tensor             # (R,5)
    states: torch.Tensor          # (R,16)
    last_dirac: torch.Tensor      # (R,4)
    iters: torch.Tensor           # (R,) int32
    event_log: Optional[torch.Tensor]   # (R, log_cap) int32 ray-major (row = launch slot), Morton numbering
    touch_count: Optional[torch.Tensor] # (N,) int32
    ray_stats: Optional[torch.Tensor]   # (R,2)
    status: torch.Tensor          # (1,) int32


def trace_args(tmin, tmax, max_iters, sh_degree, depth_hint=None):
    """sh_degree None: the reference's DC-only forward colour; d: SH of degree d along rayd.
    depth_hint: optional (R,) float32 device tensor, a guess per ray of the t at which it stops
    (the frustum phase's first stage covers up to a packet's largest guess)."""
    a = N.EverTraceArgs()
    a.tmin, a.tmax, a.max_iters = float(tmin), float(tmax), int(max_iters)
    a.sh_degree = -1 if sh_degree is None else int(sh_degree)
    a.depth_hint = N.ptr(depth_hint)
    return a


def forward(scene: Scene, rayo, rayd, tmin=0.0, tmax=1000.0, max_iters=500, sh_degree=None, log_events=True,
            touch_count=False, ray_stats=False, ray_order=None, tune: Tune | None = None,
            buffers: ForwardResult | None = None, regrouped: bool = True,
            workspace: torch.Tensor | None = None, depth_hint: torch.Tensor | None = None) -> ForwardResult:
    """regrouped: with warp packets (tune.traversal 0) and k-buffers of up to 16 events,
    re-pack the rays that need more gather rounds into full warps between passes
    (ever_trace_forward_regrouped; same results, faster). workspace: optional uint8 scratch
    of ever_trace_forward_workspace_bytes(R)."""
    device = scene.device
    _check_tensor("ray_origins", rayo, device, 3)
    _check_tensor("ray_directions", rayd, device, 3)
    rayo = rayo.contiguous()
    rayd = rayd.contiguous()
    R = rayo.numel() // 3
    if rayd.numel() // 3 != R:
        raise RuntimeError("ray_origins and ray_directions must hold the same number of rays")
    if ray_order is not None:
        _check_tensor("ray_order", ray_order, device, None, torch.int32)
    if buffers is None:
        f32 = dict(dtype=torch.float32, device=device)
        buffers = ForwardResult(
            out=torch.empty((R, 5), **f32), states=torch.empty((R, 16), **f32),
            last_dirac=torch.empty((R, 4), **f32), iters=torch.empty(R, dtype=torch.int32, device=device),
            event_log=(torch.empty((R, max(int(max_iters), 0)), dtype=torch.int32, device=device)
                       if log_events else None),
            touch_count=(torch.zeros(scene.num_prims, dtype=torch.int32, device=device) if touch_count else None),
            ray_stats=(torch.empty((R, 2), **f32) if ray_stats else None),
            status=torch.zeros(1, dtype=torch.int32, device=device))
    o = N.EverForwardOut()
    o.out, o.states, o.last_dirac, o.iters = (N.ptr(buffers.out), N.ptr(buffers.states), N.ptr(buffers.last_dirac),
                                              N.ptr(buffers.iters))
    o.event_log = N.ptr(buffers.event_log)
    o.log_cap = 0 if buffers.event_log is None else buffers.event_log.shape[1]
    o.touch_count = N.ptr(buffers.touch_count)
    o.ray_stats = N.ptr(buffers.ray_stats)
    o.status = N.ptr(buffers.status)
    if depth_hint is not None:
        _check_tensor("depth_hint", depth_hint, device)
        if depth_hint.numel() != R:
            raise RuntimeError("depth_hint must hold one value per ray")
        depth_hint = depth_hint.contiguous()
    args = trace_args(tmin, tmax, max_iters, sh_degree, depth_hint)
    tune = tune or Tune()
    lib = N.load()
    with torch.cuda.device(device):
        # the packed passes pay for buffers of up to 16 events; with 32, most rays finish in
        # the first round and the extra passes only add their overhead
        if regrouped and tune.traversal in (0, 2) and tune.kbuf <= 16 and R < (1 << 31):
            need = int(lib.ever_trace_forward_workspace_bytes(R))
            if workspace is None or workspace.numel() < need:
                workspace = torch.empty(max(need, 256), dtype=torch.uint8, device=device)
            N.check(lib.ever_trace_forward_regrouped(ctypes.byref(scene.c), N.ptr(rayo), N.ptr(rayd), R,
                                                     ctypes.byref(args), N.ptr(ray_order), ctypes.byref(tune.c()),
                                                     ctypes.byref(o), N.ptr(workspace), int(workspace.numel()),
                                                     _stream(device)))
        else:
            N.check(lib.ever_trace_forward(ctypes.byref(scene.c), N.ptr(rayo), N.ptr(rayd), R, ctypes.byref(args),
                                           N.ptr(ray_order), ctypes.byref(tune.c()), ctypes.byref(o),
                                           _stream(device)))
    return buffers


@dataclass
class Gradients:
    mean: torch.Tensor
    scale: torch.Tensor
    quat: torch.Tensor
    density: torch.Tensor
    features: torch.Tensor
    rayo: torch.Tensor
    rayd: torch.Tensor
    means2d: Optional[torch.Tensor]


def backward(scene: Scene, rayo, rayd, fwd: ForwardResult, grad_out, tmin=0.0, tmax=1000.0, max_iters=500,
             sh_degree=None, wcts=None, want_means2d=False, ray_order=None, tune: Tune | None = None,
             workspace: torch.Tensor | None = None, slot_order=None) -> Gradients:
    """slot_order: optional launch order over the forward's slots (backward_order())."""
    device = scene.device
    if fwd.event_log is None:
        raise RuntimeError("backward needs the forward's event log (log_events=True)")
    rayo = rayo.contiguous()
    rayd = rayd.contiguous()
    grad_out = grad_out.contiguous()
    R = rayo.numel() // 3
    n = scene.num_prims
    m, s, q, d, f = scene.tensors
    f32 = dict(dtype=torch.float32, device=device)
    g = Gradients(torch.empty((n, 3), **f32), torch.empty((n, 3), **f32), torch.empty((n, 4), **f32),
                  torch.empty(n, **f32), torch.empty(f.shape, **f32), torch.empty((R, 3), **f32),
                  torch.empty((R, 3), **f32), torch.zeros((n, 2), **f32) if want_means2d else None)
    lib = N.load()
    need = lib.ever_backward_workspace_bytes(n, scene.sh_coeffs)
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(max(int(need), 256), dtype=torch.uint8, device=device)
    wct = None
    num_wct = 0
    if wcts is not None and want_means2d:
        wct = wcts.detach().to(device=device, dtype=torch.float32).contiguous().reshape(-1, 4, 4)
        num_wct = wct.shape[0]
    o = N.EverBackwardOut()
    o.dmean, o.dscale, o.dquat, o.ddensity = N.ptr(g.mean), N.ptr(g.scale), N.ptr(g.quat), N.ptr(g.density)
    o.dfeatures, o.drayo, o.drayd, o.dmeans2d = N.ptr(g.features), N.ptr(g.rayo), N.ptr(g.rayd), N.ptr(g.means2d)
    args = trace_args(tmin, tmax, max_iters, sh_degree)
    common = (ctypes.byref(scene.c), N.ptr(rayo), N.ptr(rayd), R, ctypes.byref(args), N.ptr(grad_out),
              N.ptr(fwd.states), N.ptr(fwd.iters), N.ptr(fwd.event_log), fwd.event_log.shape[1], N.ptr(wct), num_wct,
              N.ptr(m), N.ptr(s), N.ptr(q), N.ptr(workspace), int(workspace.numel()), N.ptr(ray_order))
    with torch.cuda.device(device):
        if slot_order is None:
            N.check(lib.ever_trace_backward(*common, ctypes.byref((tune or Tune()).c()), ctypes.byref(o),
                                            _stream(device)))
        else:
            _check_tensor("slot_order", slot_order, device, None, torch.int32)
            N.check(lib.ever_trace_backward_ordered(*common, N.ptr(slot_order), ctypes.byref((tune or Tune()).c()),
                                                    ctypes.byref(o), _stream(device)))
    return g


def backward_order(fwd: ForwardResult, ray_order=None, shift: int = 1,
                   workspace: torch.Tensor | None = None) -> torch.Tensor:
    """Backward launch order over the forward's slots: rays that consumed more events first,
    grouped by iters >> shift, coherent slot order within a group."""
    R = fwd.iters.numel()
    device = fwd.iters.device
    order = torch.empty(R, dtype=torch.int32, device=device)
    lib = N.load()
    need = int(lib.ever_ray_order_workspace_bytes(R))
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(max(need, 256), dtype=torch.uint8, device=device)
    with torch.cuda.device(device):
        N.check(lib.ever_backward_slot_order(N.ptr(fwd.iters), N.ptr(ray_order), R, int(shift), N.ptr(workspace),
                                             int(workspace.numel()), N.ptr(order), _stream(device)))
    return order


def ray_order(rayo, rayd, workspace: torch.Tensor | None = None) -> torch.Tensor:
    """A coherent launch order (int32 permutation) for the packet traversal."""
    device = rayo.device
    _check_tensor("ray_origins", rayo, device, 3)
    _check_tensor("ray_directions", rayd, device, 3)
    rayo = rayo.contiguous()
    rayd = rayd.contiguous()
    R = rayo.numel() // 3
    order = torch.empty(R, dtype=torch.int32, device=device)
    lib = N.load()
    need = int(lib.ever_ray_order_workspace_bytes(R))
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(max(need, 256), dtype=torch.uint8, device=device)
    with torch.cuda.device(device):
        N.check(lib.ever_ray_order(N.ptr(rayo), N.ptr(rayd), R, N.ptr(workspace), int(workspace.numel()),
                                   N.ptr(order), _stream(device)))
    return order


def reference_tri_collection(scene: Scene, fwd: ForwardResult, max_iters: int, ray_order=None) -> torch.Tensor:
    """The reference's tri_collection: (R*max_iters,) int32, iteration-major, original ids."""
    R = fwd.iters.numel()
    log = fwd.event_log
    if log is None or R == 0 or max_iters <= 0:
        return torch.zeros(R * max(int(max_iters), 0), dtype=torch.int32, device=scene.device)
    tri = torch.empty(R * int(max_iters), dtype=torch.int32, device=scene.device)
    with torch.cuda.device(scene.device):
        N.check(N.load().ever_event_log_to_reference(ctypes.byref(scene.c), N.ptr(log),
                                                     0 if log is None else log.shape[1], N.ptr(fwd.iters), R,
                                                     N.ptr(ray_order), N.ptr(tri), int(max_iters),
                                                     _stream(scene.device)))
    return tri
