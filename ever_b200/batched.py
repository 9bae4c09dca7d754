"""Batched tracing: many views over several scenes in one persistent forward launch and
one persistent backward launch, optionally captured as a CUDA graph.

Every buffer is allocated once at construction. A step rebuilds each scene's BVH in
place from its (in-place updated) parameter tensors, orders every view's rays
coherently, traces all views forward, replays them backward and turns each scene's
accumulated gradients into parameter gradients. With graph=True the whole step is
recorded once and then replayed, so a step costs one graph launch on the host.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _native as N
from . import tracer as T


@dataclass
class SceneGrads:
    mean: torch.Tensor
    scale: torch.Tensor
    quat: torch.Tensor
    density: torch.Tensor
    features: torch.Tensor


class BatchedTracer:
    def __init__(self, scenes, views, tmin=0.0, tmax=1000.0, max_iters=500, tune: T.Tune | None = None,
                 sh_degree=None, graph=False, scheduler=None):
        """scenes: list of (mean, scale, quat, density, features) CUDA tensors (kept by
        reference: update them in place between steps). views: list of (scene_index, rayo,
        rayd); the rays are copied into one concatenated buffer (self.rayo / self.rayd).
        scheduler: optional (CostModel, thresholds): every step then predicts each ray's
        cost bin and orders each view's rays costliest bin first."""
        if not scenes or not views:
            raise RuntimeError("a batch needs at least one scene and one view")
        self.device = scenes[0][0].device
        dev = self.device
        self.tmin, self.tmax, self.max_iters = float(tmin), float(tmax), int(max_iters)
        self.tune = tune or T.Tune()
        self.sh_degree = sh_degree
        self.scenes = [T.Scene(*sc) for sc in scenes]
        lib = N.load()
        self.bwd_ws = []
        for sc in self.scenes:
            nbytes = int(lib.ever_backward_workspace_bytes(sc.num_prims, sc.sh_coeffs))
            self.bwd_ws.append(torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev))
        counts = [int(v[1].shape[0]) for v in views]
        self.view_scene = [int(v[0]) for v in views]
        self.R = sum(counts)
        self.rayo = torch.cat([v[1].to(dev, torch.float32) for v in views]).contiguous()
        self.rayd = torch.cat([v[2].to(dev, torch.float32) for v in views]).contiguous()
        vt = (N.EverBatchView * len(views))()
        off = 0
        for i, c in enumerate(counts):
            vt[i].scene, vt[i].ray_offset, vt[i].ray_count = self.view_scene[i], off, c
            off += c
        self.view_offsets = [vt[i].ray_offset for i in range(len(views))]
        self.view_counts = counts
        slots = ctypes.c_int64(0)
        nbytes = int(lib.ever_batch_workspace_bytes(len(self.scenes), vt, len(views), ctypes.byref(slots)))
        if nbytes == 0:
            raise RuntimeError("invalid batch (1..64 scenes and views)")
        self.num_slots = slots.value
        self.batch_ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        sc_arr = (N.EverScene * len(self.scenes))(*[s.c for s in self.scenes])
        ws_arr = (ctypes.c_void_p * len(self.scenes))(*[b.data_ptr() for b in self.bwd_ws])
        self.batch = N.EverBatch()
        torch.cuda.synchronize(dev)
        N.check(lib.ever_batch_setup(sc_arr, ws_arr, len(self.scenes), vt, len(views), self.R,
                                     N.ptr(self.batch_ws), nbytes, ctypes.byref(self.batch)))
        f32 = dict(dtype=torch.float32, device=dev)
        R = self.R
        self.out = torch.empty((R, 5), **f32)
        self.states = torch.empty((R, 16), **f32)
        self.last_dirac = torch.empty((R, 4), **f32)
        self.iters = torch.empty(R, dtype=torch.int32, device=dev)
        self.ray_stats = torch.empty((R, 2), **f32)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.event_log = torch.empty((self.num_slots, self.max_iters), dtype=torch.int32, device=dev)
        self.grad_out = torch.zeros((R, 5), **f32)
        self.drayo = torch.empty((R, 3), **f32)
        self.drayd = torch.empty((R, 3), **f32)
        self.grads = [SceneGrads(torch.empty((s.num_prims, 3), **f32), torch.empty((s.num_prims, 3), **f32),
                                 torch.empty((s.num_prims, 4), **f32), torch.empty(s.num_prims, **f32),
                                 torch.empty((s.num_prims, s.sh_coeffs, 3), **f32)) for s in self.scenes]
        self._fo = N.EverForwardOut()
        self._fo.out, self._fo.states, self._fo.last_dirac = N.ptr(self.out), N.ptr(self.states), N.ptr(self.last_dirac)
        self._fo.iters, self._fo.event_log, self._fo.log_cap = N.ptr(self.iters), N.ptr(self.event_log), self.max_iters
        self._fo.touch_count, self._fo.ray_stats, self._fo.status = None, N.ptr(self.ray_stats), N.ptr(self.status)
        self._args = T.trace_args(self.tmin, self.tmax, self.max_iters, sh_degree)
        self._bo = []
        for g in self.grads:
            bo = N.EverBackwardOut()
            bo.dmean, bo.dscale, bo.dquat, bo.ddensity = N.ptr(g.mean), N.ptr(g.scale), N.ptr(g.quat), N.ptr(g.density)
            bo.dfeatures, bo.drayo, bo.drayd, bo.dmeans2d = N.ptr(g.features), None, None, None
            self._bo.append(bo)
        self.scheduler = None
        self.graph = None
        if scheduler is not None:
            self.set_scheduler(*scheduler)
        if graph:
            self.capture()

    def set_scheduler(self, cost_model, thresholds):
        """Uses the cost model's bins for the launch order from the next step on (a captured
        graph is recorded again)."""
        self.scheduler = (cost_model, [float(t) for t in thresholds])
        self.pred = torch.empty((self.R, 2), dtype=torch.float32, device=self.device)
        self.bins = torch.empty(self.R, dtype=torch.uint8, device=self.device)
        if self.graph is not None:
            self.capture()

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def rebuild(self):
        for s in self.scenes:
            s.rebuild()

    def order(self):
        lib = N.load()
        if self.scheduler is None:
            N.check(lib.ever_batch_order(ctypes.byref(self.batch), N.ptr(self.rayo), N.ptr(self.rayd), self._stream()))
            return
        cm, thr = self.scheduler
        cm.predict(self.rayo, self.rayd, thr, out=self.pred, bins_out=self.bins)
        N.check(lib.ever_batch_order_binned(ctypes.byref(self.batch), N.ptr(self.rayo), N.ptr(self.rayd),
                                            N.ptr(self.bins), self._stream()))

    def forward(self):
        N.check(N.load().ever_trace_forward_batched(ctypes.byref(self.batch), N.ptr(self.rayo), N.ptr(self.rayd),
                                                    ctypes.byref(self._args), ctypes.byref(self.tune.c()),
                                                    ctypes.byref(self._fo), self._stream()))

    def backward(self):
        lib = N.load()
        N.check(lib.ever_trace_backward_batched(ctypes.byref(self.batch), N.ptr(self.rayo), N.ptr(self.rayd),
                                                ctypes.byref(self._args), N.ptr(self.grad_out), N.ptr(self.states),
                                                N.ptr(self.iters), N.ptr(self.event_log), self.max_iters,
                                                N.ptr(self.drayo), N.ptr(self.drayd), ctypes.byref(self.tune.c()),
                                                self._stream()))
        for s, ws, bo in zip(self.scenes, self.bwd_ws, self._bo):
            m, sc, q, _, _ = s.tensors
            N.check(lib.ever_scene_finalize_gradients(ctypes.byref(s.c), N.ptr(m), N.ptr(sc), N.ptr(q), N.ptr(ws),
                                                      int(ws.numel()), ctypes.byref(bo), self._stream()))

    def step_body(self, backward=True):
        with torch.cuda.device(self.device):
            self.rebuild()
            self.order()
            self.forward()
            if backward:
                self.backward()

    def capture(self):
        """Records one whole step (rebuild, order, forward, backward, finalize) in a CUDA graph."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            for _ in range(2):
                self.step_body()
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step_body()
        self.graph = g

    def step(self, grad_out=None, backward=True):
        """One step. grad_out (R,5) is copied into the static buffer first."""
        if grad_out is not None:
            self.grad_out.copy_(grad_out)
        if self.graph is not None and backward:
            self.graph.replay()
        else:
            self.step_body(backward)
        return self.out

    def view_slice(self, v):
        o = self.view_offsets[v]
        return slice(o, o + self.view_counts[v])
