"""Learned ray-cost scheduler.

A 39 -> 64 -> 64 -> 2 ReLU MLP (BF16 weights and activations, FP32 accumulation, run by the
library's hand-written tcgen05 kernels) predicts each ray's cost from the point of its
line closest to the scene centre: [log(1 + consumed events), depth offset / scale]. It is
trained on the tracer's own per-ray logs (forward ray_stats: consumed events and the t
of the last event). Two uses:
- cost bins: predicted log-costs are cut into four bins by thresholds taken from the
  training predictions; rays are ordered bin by bin (costliest first), each bin in the
  coherent direction order;
- depth hint: the predicted stopping depth bounds each packet's frustum walk
  (tracer.forward(depth_hint=...)); a ray that goes on continues in the gather rounds.
The trace's results depend on neither (each ray's arithmetic is the same in any order and
with any hint). Gate switches a use on only when the model beats a constant on held-out
rays (and, when measured, beats the coherent order alone); plan() gives the order and hint
for one trace, the coherent order and no hint being the fallback.

No counterpart in the reference, whose OptiX launch order is the ray index.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native as N

MLP_PARAMS = N.MLP_PARAMS
OFF_W1, OFF_W2, OFF_W3, OFF_B1, OFF_B2, OFF_B3 = 0, 4096, 8192, 9216, 9280, 9344


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform hidden layers, a small output layer, zero biases; padding zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_PARAMS, np.float32)
    w1 = np.zeros((64, 64), np.float32)
    w1[:, :39] = rng.uniform(-1, 1, (64, 39)) * math.sqrt(6.0 / 39)
    w2 = rng.uniform(-1, 1, (64, 64)) * math.sqrt(6.0 / 64)
    w3 = np.zeros((16, 64), np.float32)
    w3[:2] = rng.uniform(-1, 1, (2, 64)) * math.sqrt(3.0 / 64)
    p[OFF_W1:OFF_W2] = w1.ravel()
    p[OFF_W2:OFF_W3] = w2.ravel()
    p[OFF_W3:OFF_B1] = w3.ravel()
    return p


class CostModel:
    """The MLP's parameters, Adam state and device buffers, with the library calls."""

    def __init__(self, centre: Sequence[float] = (0.0, 0.0, 0.0), scale: float = 1.0, seed: int = 0,
                 device=None, params: Optional[np.ndarray] = None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.lib = N.load()
        dev = self.device
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        if p.shape != (MLP_PARAMS,):
            raise ValueError(f"params must have {MLP_PARAMS} entries")
        self.params = torch.tensor(p, device=dev)
        self.w1 = torch.empty(64 * 64, dtype=torch.bfloat16, device=dev)
        self.w2 = torch.empty(64 * 64, dtype=torch.bfloat16, device=dev)
        self.w3 = torch.empty(16 * 64, dtype=torch.bfloat16, device=dev)
        self.adam_m = torch.zeros(MLP_PARAMS, device=dev)
        self.adam_v = torch.zeros(MLP_PARAMS, device=dev)
        self.grads = torch.zeros(MLP_PARAMS, device=dev)
        self.loss = torch.zeros(1, device=dev)
        self.error = torch.zeros(1, dtype=torch.int32, device=dev)
        self.workspace = torch.empty(int(self.lib.ever_mlp_workspace_bytes()), dtype=torch.uint8, device=dev)
        self.step_count = 0
        self.centre = tuple(float(c) for c in centre)
        self.scale = float(scale)
        self._s = N.EverMlp()
        self._s.params, self._s.w1, self._s.w2, self._s.w3 = (t.data_ptr() for t in
                                                                (self.params, self.w1, self.w2, self.w3))
        self._s.centre = (ctypes.c_float * 3)(*self.centre)
        self._s.inv_scale = 1.0 / self.scale
        self.pack()

    # ------------------------------------------------------------------ library calls
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def pack(self):
        N.check(self.lib.ever_mlp_pack(ctypes.byref(self._s), self._stream()))

    def load(self, params: np.ndarray):
        self.params.copy_(torch.as_tensor(np.asarray(params, np.float32)))
        self.pack()

    def check(self):
        """Raises if a tensor-core wait timed out in an earlier call (synchronises)."""
        if int(self.error.item()) != 0:
            raise RuntimeError("ever_b200: tensor-core wait timed out in the cost model")

    def clear_error(self):
        self.error.zero_()

    def set_wait_clocks(self, clocks: int = 0):
        """Bound of each wait for the tensor cores in clocks (0: the default, about a second)."""
        self._s.wait_clocks = int(clocks)

    @staticmethod
    def _rays(rayo, rayd):
        for t in (rayo, rayd):
            if t.dtype != torch.float32 or not t.is_contiguous() or t.dim() != 2 or t.shape[1] != 3:
                raise ValueError("rays must be contiguous float32 (R, 3)")
        return rayo.shape[0]

    def predict(self, rayo=None, rayd=None, thresholds: Optional[Sequence[float]] = None, feat=None,
                out: Optional[torch.Tensor] = None, bins_out: Optional[torch.Tensor] = None):
        """(pred (R, 2), bins (R,) uint8 or None). feat: pre-encoded (R, 64) inputs."""
        R = feat.shape[0] if feat is not None else self._rays(rayo, rayd)
        pred = out if out is not None else torch.empty((R, 2), dtype=torch.float32, device=self.device)
        bins = None
        thr = None
        if thresholds is not None:
            bins = bins_out if bins_out is not None else torch.empty(R, dtype=torch.uint8, device=self.device)
            thr = (ctypes.c_float * 3)(*[float(t) for t in thresholds])
        N.check(self.lib.ever_mlp_predict(ctypes.byref(self._s), N.ptr(rayo if feat is None else None),
                                          N.ptr(rayd if feat is None else None), N.ptr(feat), R, N.ptr(pred),
                                          N.ptr(bins), thr, N.ptr(self.error), self._stream()))
        return pred, bins

    def gradients(self, rayo, rayd, target, sample_idx=None, feat=None, weights=(1.0, 1.0)):
        """Writes self.grads and self.loss for the samples (all rays, or ray sample_idx[s])."""
        n = int(sample_idx.shape[0]) if sample_idx is not None else (
            feat.shape[0] if feat is not None else self._rays(rayo, rayd))
        N.check(self.lib.ever_mlp_gradients(
            ctypes.byref(self._s), N.ptr(rayo if feat is None else None), N.ptr(rayd if feat is None else None),
            N.ptr(feat), N.ptr(sample_idx), n, N.ptr(target), float(weights[0]), float(weights[1]),
            N.ptr(self.grads), N.ptr(self.loss), N.ptr(self.workspace), self.workspace.numel(), N.ptr(self.error),
            self._stream()))
        return self.grads, self.loss

    def adam_step(self, lr=3e-3, betas=(0.9, 0.999), eps=1e-8):
        self.step_count += 1
        N.check(self.lib.ever_mlp_adam(ctypes.byref(self._s), N.ptr(self.grads), N.ptr(self.adam_m),
                                       N.ptr(self.adam_v), float(lr), float(betas[0]), float(betas[1]), float(eps),
                                       self.step_count, self._stream()))

    def fit(self, rayo, rayd, target, epochs=2, batch=65536, lr=3e-3, weights=(1.0, 0.25), seed=0,
            lr_final=0.1):
        """Minibatch Adam over shuffled rays; the learning rate decays by cosine to
        lr * lr_final. Returns the per-step losses (device tensor)."""
        R = self._rays(rayo, rayd)
        gen = torch.Generator(device=self.device).manual_seed(seed)
        steps_per_epoch = max(1, (R + batch - 1) // batch)
        total = epochs * steps_per_epoch
        losses = torch.empty(total, device=self.device)
        k = 0
        for _ in range(epochs):
            perm = torch.randperm(R, device=self.device, generator=gen).to(torch.int32)
            for b in range(steps_per_epoch):
                idx = perm[b * batch:(b + 1) * batch]
                self.gradients(rayo, rayd, target, sample_idx=idx, weights=weights)
                losses[k:k + 1].copy_(self.loss)
                f = lr_final + (1 - lr_final) * 0.5 * (1 + math.cos(math.pi * k / max(1, total - 1)))
                self.adam_step(lr * f)
                k += 1
        return losses


# ---------------------------------------------------------------------- helpers
def cost_targets(ray_stats: torch.Tensor, rayo: torch.Tensor, rayd: torch.Tensor, centre=(0.0, 0.0, 0.0),
                 scale: float = 1.0) -> torch.Tensor:
    """(R, 2) training targets from a forward's ray_stats (consumed events, t of the last
    event): log(1 + events) and the depth offset from the line's closest point / scale."""
    c = torch.tensor(centre, dtype=torch.float32, device=rayo.device)
    n = rayd.norm(dim=1).clamp_min(1e-30)
    s_c = -((rayo - c) * rayd).sum(1) / n
    t = torch.empty((rayo.shape[0], 2), dtype=torch.float32, device=rayo.device)
    t[:, 0] = torch.log1p(ray_stats[:, 0])
    t[:, 1] = (ray_stats[:, 1] * n - s_c) / scale
    return t


def depth_from_prediction(pred: torch.Tensor, rayo: torch.Tensor, rayd: torch.Tensor, centre=(0.0, 0.0, 0.0),
                          scale: float = 1.0, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """(R,) stopping t guessed by the model (the inverse of cost_targets' depth column): the
    depth hint the tracer's frustum phase takes (tracer.forward(depth_hint=...))."""
    c = torch.tensor(centre, dtype=torch.float32, device=rayo.device)
    n = rayd.norm(dim=1).clamp_min(1e-30)
    s_c = -((rayo - c) * rayd).sum(1) / n
    d = (pred[:, 1] * scale + s_c) / n
    if out is None:
        return d
    out.copy_(d)
    return out


def quantile_thresholds(pred_cost: torch.Tensor, qs=(0.25, 0.5, 0.75), max_samples=1 << 22):
    """Three thresholds at quantiles of predicted log-costs (from the training rays)."""
    x = pred_cost.flatten().float()
    if x.numel() > max_samples:
        x = x[torch.linspace(0, x.numel() - 1, max_samples, device=x.device).long()]
    return [float(v) for v in torch.quantile(x, torch.tensor(qs, device=x.device))]


def binned_order(rayo: torch.Tensor, rayd: torch.Tensor, bins: torch.Tensor,
                 workspace: Optional[torch.Tensor] = None, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Launch order: costlier bins first, each in the coherent direction order."""
    lib = N.load()
    R = rayo.shape[0]
    need = int(lib.ever_ray_order_workspace_bytes(R))
    ws = workspace if workspace is not None and workspace.numel() >= need else torch.empty(
        need, dtype=torch.uint8, device=rayo.device)
    order = out if out is not None else torch.empty(R, dtype=torch.int32, device=rayo.device)
    N.check(lib.ever_ray_order_binned(N.ptr(rayo), N.ptr(rayd), N.ptr(bins), R, N.ptr(ws), ws.numel(), N.ptr(order),
                                      ctypes.c_void_p(torch.cuda.current_stream(rayo.device).cuda_stream)))
    return order


# ---------------------------------------------------------------------- gating
def heldout_r2(cm: "CostModel", rayo: torch.Tensor, rayd: torch.Tensor, ray_stats: torch.Tensor,
               centre=(0.0, 0.0, 0.0), scale: float = 1.0) -> tuple[float, float]:
    """Coefficient of determination of the model's two outputs (log events, depth) on rays it
    was not trained on, against the tracer's logs for them."""
    pred, _ = cm.predict(rayo, rayd)
    t = cost_targets(ray_stats, rayo, rayd, centre, scale)
    r2 = []
    for c in range(2):
        var = float(t[:, c].var())
        r2.append(1.0 - float(((pred[:, c] - t[:, c]) ** 2).mean()) / var if var > 0 else float("-inf"))
    return r2[0], r2[1]


class Gate:
    """Which uses of the model are switched on. A use is on only when the model predicts its
    target better than a constant on held-out rays (R^2 > 0) and, where a measured speedup
    against the coherent order alone is given, that speedup is above 1. Otherwise the plain
    coherent order (and no depth hint) is what runs."""

    def __init__(self, r2_events: float, r2_depth: float, speedup_bins: Optional[float] = None,
                 speedup_depth: Optional[float] = None):
        self.bins = r2_events > 0.0 and (speedup_bins is None or speedup_bins > 1.0)
        self.depth = r2_depth > 0.0 and (speedup_depth is None or speedup_depth > 1.0)


def plan(cm: "CostModel", rayo: torch.Tensor, rayd: torch.Tensor, gate: Gate, thresholds=None,
         centre=(0.0, 0.0, 0.0), scale: float = 1.0, workspace: Optional[torch.Tensor] = None):
    """(ray_order, depth_hint) for one trace: cost bins only if the gate allows them (with
    thresholds), the depth hint only if it allows that; the coherent order otherwise."""
    from . import tracer as T
    hint = None
    if gate.bins and thresholds is not None:
        pred, bins = cm.predict(rayo, rayd, thresholds=thresholds)
        order = binned_order(rayo, rayd, bins, workspace)
    else:
        pred = None
        order = T.ray_order(rayo, rayd, workspace)
    if gate.depth:
        if pred is None:
            pred, _ = cm.predict(rayo, rayd)
        hint = depth_from_prediction(pred, rayo, rayd, centre, scale)
    return order, hint
