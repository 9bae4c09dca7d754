"""The reference's object API (`sp`: OptixContext, Primitives, GAS, Forward,
SavedForBackward; splinetracers/fast_ellipsoid_splinetracer/py_binding.cpp:94-282), as used
by renderers that keep a scene across frames (integration_utils/fast_renderer.py:52-117).

Differences from the reference, on purpose:
- the BVH lives in the GAS object and persists: `GAS.refit()` follows updated ellipsoid
  parameters without a rebuild (`ever_scene_refit`), `GAS.rebuild()` rebuilds in place;
  `Forward.update_model(prims)` only swaps the colours, as in the reference;
- no device context is needed, so OptixContext holds only the device;
- `saved.faces` is not produced (zeros): nothing in the reference reads it;
- `initial_touch_inds` / `initial_touch_count` list the ellipsoids that contain ray 0's
  start point rayo[0] + tmin * rayd[0] (the reference lists the candidates whose box lies
  within tmin of rayo[0], a superset); `initial_drgb` is each ray's own initial density
  and colour sum, as the tracer uses it.
"""
from __future__ import annotations

import torch

from . import tracer as T


class OptixContext:
    def __init__(self, device):
        self.device = torch.device(device)


def _check3(name, t, last):
    if t.dim() != 2 or t.shape[1] != last or t.dtype != torch.float32:
        raise RuntimeError(f"{name} must be a float32 tensor of shape (N, {last})")


class Primitives:
    """Borrowed references to the ellipsoid tensors (the caller keeps them alive)."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.tensors = None

    def add_primitives(self, means, scales, quats, half_attribs, densities, colors):
        _check3("means", means, 3)
        _check3("scales", scales, 3)
        _check3("quats", quats, 4)
        n = means.shape[0]
        for name, t in (("scales", scales), ("quats", quats), ("colors", colors), ("densities", densities)):
            if t.shape[0] != n:
                raise RuntimeError(f"All inputs ({name}) must have the same 0 dimension")
        if colors.dim() != 3 or colors.shape[2] != 3:
            raise RuntimeError("Features must have 3 channels. (N, d, 3)")
        self.tensors = [means.contiguous(), scales.contiguous(), quats.contiguous(),
                        densities.reshape(-1).contiguous(), colors.contiguous()]
        self.num_prims = n
        self.feature_size = colors.shape[1]

    def set_features(self, colors):
        if colors.dim() != 3 or colors.shape[0] != self.num_prims:
            raise RuntimeError("All inputs (colors) must have the same 0 dimension")
        self.tensors[4] = colors.contiguous()


class GAS:
    """The BVH over a Primitives object; persistent across frames."""

    def __init__(self, context, device, prims: Primitives, enable_anyhit=True, fast_build=False,
                 enable_rebuild=True):
        if prims.tensors is None:
            raise RuntimeError("Primitives has no ellipsoids (call add_primitives first)")
        self.prims = prims
        self.scene = T.Scene(*prims.tensors)

    def _sync(self, prims):
        if prims is not None:
            self.prims = prims
        self.scene.tensors = tuple(t.contiguous() for t in self.prims.tensors)

    def refit(self, prims: Primitives | None = None):
        """Follow updated means/scales/quats/densities/colours, keeping the tree topology."""
        self._sync(prims)
        self.scene.refit()

    def rebuild(self, prims: Primitives | None = None):
        self._sync(prims)
        self.scene.rebuild()


class SavedForBackward:
    def __init__(self, states, diracs, iters, touch_count, faces):
        self.states, self.diracs, self.iters, self.touch_count, self.faces = states, diracs, iters, touch_count, faces


def _rotate(v, q):
    """rotate_vector(v, q) of the tracer, q = (r, x, y, z), not normalised."""
    u = -q[:, 1:4]
    t = 2.0 * torch.linalg.cross(u, v)
    return v + q[:, 0:1] * t + torch.linalg.cross(u, t)


class Forward:
    def __init__(self, context, device, prims: Primitives, enable_backward=False):
        self.device = torch.device(device)
        self.prims = prims
        self.enable_backward = enable_backward
        self.num_prims = prims.num_prims
        self.sh_degree = int(prims.feature_size ** 0.5) - 1

    def update_model(self, prims: Primitives):
        self.prims = prims

    def trace_rays(self, gas: GAS, ray_origins, ray_directions, tmin, tmax, max_iters, max_prim_size=3.0):
        f = self.prims.tensors[4]
        if gas.scene.tensors[4] is not f:
            gas.scene.set_features(f)
        rayo = ray_origins.reshape(-1, 3).contiguous()
        rayd = ray_directions.reshape(-1, 3).contiguous()
        R = rayo.shape[0]
        with torch.no_grad():
            order = T.ray_order(rayo, rayd) if R > 0 else None
            fwd = T.forward(gas.scene, rayo, rayd, tmin, tmax, max_iters, None, log_events=True, touch_count=True,
                            ray_order=order)
            init = T.forward(gas.scene, rayo, rayd, tmin, tmax, 0, None, log_events=False, ray_order=order)
            tri = T.reference_tri_collection(gas.scene, fwd, max_iters, order)
            touch_inds, touch_count = self._initial_members(rayo, rayd, tmin)
        saved = SavedForBackward(fwd.states, fwd.last_dirac, fwd.iters, fwd.touch_count,
                                 torch.zeros(R, dtype=torch.int32, device=rayo.device))
        return dict(color=fwd.out[:, :4].contiguous(), saved=saved, tri_collection=tri,
                    initial_drgb=init.states[:, 8:12].contiguous(), initial_touch_inds=touch_inds,
                    initial_touch_count=touch_count)

    def _initial_members(self, rayo, rayd, tmin):
        m, s, q, _, _ = self.prims.tensors
        n = m.shape[0]
        inds = torch.zeros(n, dtype=torch.int32, device=m.device)
        count = torch.zeros(1, dtype=torch.int32, device=m.device)
        if rayo.shape[0] == 0 or n == 0:
            return inds, count
        x0 = (rayo[0] + float(tmin) * rayd[0]).reshape(1, 3)
        local = _rotate(x0 - m, q) / s
        inside = torch.nonzero((local * local).sum(1) < 1.0).reshape(-1).to(torch.int32)
        inds[:inside.numel()] = inside
        count[0] = inside.numel()
        return inds, count
