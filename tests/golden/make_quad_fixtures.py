"""Generates tests/golden/quad_*.npz by running the reference's own quadrature oracle.

Runs only where the reference tree is available: pass its root as the first argument
or in the EVER_REFERENCE environment variable. The GPU box and the test suite only read
the committed .npz files.

    python tests/golden/make_quad_fixtures.py <path to the N-Demir/ever tree>

The reference oracle (splinetracers/quad.py, jaxutil/quadrature.py,
jaxutil/safe_math.py, utils/math_util.py) is imported unmodified from the reference
tree. JAX is not installed here, so a minimal numpy-backed stand-in module named
`jax` is put on sys.path first: `jax.numpy` is numpy, `vmap` loops over the mapped
axis, `jit` is the identity and `custom_jvp`/`custom_vjp` keep the primal function
(only forward values are taken). `plyfile` (imported by utils/math_util.py for PLY
export, unused here) is stubbed. One function is replaced after import:
`quadrature.lossfun_distortion` builds a 65536 x 65536 matrix (34 GB in float64);
it is swapped for the equivalent O(n) sorted-prefix form. The reference's tests
compare only RGB and opacity (tests/compare_quadrature.py:57,65), which come
entirely from the reference's code.

Cases mirror tests/compare_quadrature.py (origin outside / origin inside, N in
{1,5,10,20,40}, density_multi in {0.01,0.1,1}) with a fixed seed instead of the
reference's unseeded draws.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import tempfile
import types

import numpy as np

REF = None  # the reference tree's root, set by main() from argv[1] or EVER_REFERENCE
OUT_DIR = os.path.dirname(os.path.abspath(__file__))

_JAX_STANDIN = r'''
import numpy as _np
import numpy as numpy
class _Config:
    def update(self, *a, **k):
        pass
config = _Config()
def jit(f=None, **kw):
    return f if f is not None else (lambda g: g)
def _index(tree, axes, i):
    if axes is None:
        return tree
    if isinstance(axes, dict):
        return {k: _index(tree[k], axes[k], i) for k in tree}
    return _np.take(tree, i, axis=axes)
def _size(tree, axes):
    if axes is None:
        return None
    if isinstance(axes, dict):
        for k in axes:
            s = _size(tree[k], axes[k])
            if s is not None:
                return s
        return None
    return _np.shape(tree)[axes]
def vmap(fn, in_axes=0):
    def wrapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            n = n or _size(a, ax)
        outs = [fn(*[_index(a, ax, i) for a, ax in zip(args, axes)]) for i in range(n)]
        if isinstance(outs[0], tuple):
            return tuple(_np.stack([o[k] for o in outs]) for k in range(len(outs[0])))
        return _np.stack(outs)
    return wrapped
class _Custom:
    def __init__(self, f, *a, **k):
        self.f = f
    def __call__(self, *a, **k):
        return self.f(*a, **k)
    def defjvp(self, *a, **k):
        return a[0] if a else None
    def defvjp(self, *a, **k):
        return None
def custom_jvp(f=None, **kw):
    return _Custom(f)
def custom_vjp(f=None, **kw):
    return _Custom(f)
'''


def _install_standins(tmp):
    pkg = os.path.join(tmp, "jax")
    os.makedirs(pkg)
    with open(os.path.join(pkg, "__init__.py"), "w") as f:
        f.write(_JAX_STANDIN)
    with open(os.path.join(pkg, "numpy.py"), "w") as f:
        f.write("from numpy import *\nimport numpy as _n\nlinalg = _n.linalg\npi = _n.pi\n")
    plyfile = types.ModuleType("plyfile")
    plyfile.PlyData = plyfile.PlyElement = object
    sys.modules["plyfile"] = plyfile
    sys.path.insert(0, tmp)


def _load_reference_quad():
    sys.path.insert(1, REF)
    spec = importlib.util.spec_from_file_location("ref_quad", os.path.join(REF, "splinetracers", "quad.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    from jaxutil import quadrature  # the reference's module, resolved from REF

    def lossfun_distortion_prefix(t, w):
        u = 0.5 * (t[1:] + t[:-1])
        W = np.concatenate([[0.0], np.cumsum(w)[:-1]])
        S = np.concatenate([[0.0], np.cumsum(w * u)[:-1]])
        return 2.0 * np.sum(w * (u * W - S)) + np.sum(w ** 2 * np.diff(t)) / 3.0

    quadrature.lossfun_distortion = lossfun_distortion_prefix
    return mod


def _cases(rng):
    """Inputs drawn as tests/compare_quadrature.py:35-102 draws them (seeded)."""
    for kind in ("outside", "inside"):
        for N in (1, 5, 10, 20, 40):
            for dm in (0.01, 0.1, 1.0):
                scale = 0.5 * rng.random((N, 3))
                if kind == "outside":
                    mean = rng.random((N, 3))
                    mean[:, 0] *= 0.5
                    mean[:, 1] *= 0.5
                    mean[:, 2] += 0.5
                    tmin = 0.0
                else:
                    mean = 1.2 * rng.random((N, 3)) - 0.2
                    mean[:, 0] *= 0.5
                    mean[:, 1] *= 0.5
                    tmin = float(rng.random() * 0.3)
                q = 2 * rng.random((N, 4)) - 1
                quat = q / np.sqrt(np.sum(q ** 2, -1, keepdims=True))
                density = dm * rng.random((N, 1))
                feats = rng.random((N, 1, 3))
                yield kind, N, dm, dict(mean=mean, scale=scale, quat=quat, density=density, features=feats,
                                        rayo=np.array([[0.0, 0.0, 0.0]]), rayd=np.array([[0.0, 0.0, 1.0]]),
                                        tmin=tmin)


def main():
    global REF
    import torch
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EVER_REFERENCE")
    if not REF or not os.path.isdir(os.path.join(REF, "splinetracers")):
        sys.exit("usage: make_quad_fixtures.py <reference tree root> (or set EVER_REFERENCE)")
    with tempfile.TemporaryDirectory() as tmp:
        _install_standins(tmp)
        quad = _load_reference_quad()
        rng = np.random.default_rng(20241203)
        records = []
        for kind, N, dm, c in _cases(rng):
            # inputs are float32 tensors in the reference tests; round them the same way
            f32 = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v) for k, v in c.items()}
            t = {k: (torch.from_numpy(v) if isinstance(v, np.ndarray) else v) for k, v in f32.items()}
            out, _ = quad.trace_rays(t["mean"], t["scale"], t["quat"], t["density"], t["features"],
                                     t["rayo"], t["rayd"], t["tmin"], 3, return_extras=True)
            records.append(dict(kind=kind, N=N, dm=dm, out=np.asarray(out, np.float64).reshape(-1), **f32))
            print(kind, N, dm, np.asarray(out).reshape(-1)[:4])
        arrays = {}
        for i, r in enumerate(records):
            for k, v in r.items():
                arrays[f"c{i}_{k}"] = np.asarray(v)
        arrays["count"] = np.asarray(len(records))
        np.savez_compressed(os.path.join(OUT_DIR, "quad_reference.npz"), **arrays)


if __name__ == "__main__":
    main()
