"""ctypes wrapper of the CPU oracle (oracle/ever_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py as the checker. The product package never imports it.

Inputs follow the reference API (splinetracers/fast_ellipsoid_splinetracer.py:222-256):
mean (N,3), scale (N,3), quat (N,4) as (r,x,y,z), density (N,) or (N,1), features
(N,K,3), rayo (R,3), rayd (R,3).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libever_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(_HERE, "ever_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i64, i32, f32, f64 = ctypes.c_int64, ctypes.c_int, ctypes.c_float, ctypes.c_double
        L.ora_trace_f32.argtypes = [i64, i32, i32, P, P, P, P, P, i64, P, P, f32, f32, i32,
                                    P, P, P, P, P, P, i32]
        L.ora_trace_f64.argtypes = [i64, i32, i32, P, P, P, P, P, i64, P, P, f64, f64, i32,
                                    P, P, P, P, P, P, i32]
        L.ora_backward_f64.argtypes = [i64, i32, i32, P, P, P, P, P, i64, P, P, f64, f64, i32,
                                       P, P, P, P, P, P, P, P, P, P, i32]
        L.ora_backward_f32_replay.argtypes = L.ora_backward_f64.argtypes
        L.ora_backward_f32_stored.argtypes = L.ora_backward_f64.argtypes
        L.ora_backward_f32_stored.restype = ctypes.c_int
        L.ora_intersect_f32.argtypes = [P, P, P, P, P, f32, P]
        for fn in (L.ora_trace_f32, L.ora_trace_f64, L.ora_backward_f64, L.ora_backward_f32_replay,
                   L.ora_intersect_f32):
            fn.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _threads(nthreads):
    return int(nthreads or os.cpu_count() or 1)


@dataclass
class Scene:
    mean: np.ndarray
    scale: np.ndarray
    quat: np.ndarray
    density: np.ndarray
    features: np.ndarray  # (N, K, 3)

    @property
    def N(self):
        return self.mean.shape[0]

    @property
    def K(self):
        return self.features.shape[1]

    def as_dtype(self, dt):
        c = lambda a: np.ascontiguousarray(np.asarray(a, dtype=dt))
        return Scene(c(self.mean).reshape(-1, 3), c(self.scale).reshape(-1, 3), c(self.quat).reshape(-1, 4),
                     c(self.density).reshape(-1), c(self.features).reshape(self.mean.shape[0], -1, 3))


def sh_degree_of(K: int) -> int:
    """sqrt(K) - 1, as py_binding.cpp:206 derives the degree from the feature size."""
    return int(np.sqrt(K)) - 1


def colour_degree(sh_degree) -> int:
    """The SH degree the colour is evaluated at. None is the reference's forward: the DC
    term of every ellipsoid whatever K (shaders.slang:72-75, get_sh(sh_feats, 0) and
    eval_sh_col0), i.e. degree 0. An int d evaluates SH of degree d along rayd."""
    return 0 if sh_degree is None else int(sh_degree)


@dataclass
class Trace:
    out: np.ndarray        # (R,5) RGB, opacity, distortion
    states: np.ndarray     # (R,16) final SplineState
    last_dirac: np.ndarray # (R,4)
    iters: np.ndarray      # (R,) int32
    events: np.ndarray | None  # (max_iters, R) int32 reference ids, -1 where unused
    depth: np.ndarray      # (R,) t of the last consumed event


def trace(scene: Scene, rayo, rayd, tmin=0.0, tmax=1000.0, max_iters=500, sh_degree=None,
          precision="f32", with_events=True, nthreads=None) -> Trace:
    dt = np.float32 if precision == "f32" else np.float64
    s = scene.as_dtype(dt)
    rayo = np.ascontiguousarray(np.asarray(rayo, dtype=dt).reshape(-1, 3))
    rayd = np.ascontiguousarray(np.asarray(rayd, dtype=dt).reshape(-1, 3))
    R = rayo.shape[0]
    deg = colour_degree(sh_degree)
    out = np.zeros((R, 5), dt)
    states = np.zeros((R, 16), dt)
    last_dirac = np.zeros((R, 4), dt)
    iters = np.zeros(R, np.int32)
    events = np.full((max(max_iters, 0), R), -1, np.int32) if with_events else None
    depth = np.zeros(R, dt)
    fn = lib().ora_trace_f32 if precision == "f32" else lib().ora_trace_f64
    rc = fn(s.N, s.K, deg, _ptr(s.mean), _ptr(s.scale), _ptr(s.quat), _ptr(s.density), _ptr(s.features),
            R, _ptr(rayo), _ptr(rayd), float(tmin), float(tmax), int(max_iters), _ptr(out), _ptr(states),
            _ptr(last_dirac), _ptr(iters), _ptr(events), _ptr(depth), _threads(nthreads))
    assert rc == 0
    return Trace(out, states, last_dirac, iters, events, depth)


@dataclass
class Grads:
    mean: np.ndarray
    scale: np.ndarray
    quat: np.ndarray
    density: np.ndarray
    features: np.ndarray
    rayo: np.ndarray
    rayd: np.ndarray


def backward(scene: Scene, rayo, rayd, tmin, tmax, max_iters, events, iters, dout,
             sh_degree=None, nthreads=None, mode="f64") -> Grads:
    """Gradients (unclipped) along the given event sequence.

    mode "f64": exact FP64 analytic gradients (states stored by a forward replay).
    mode "f32_replay": the reference's scheme in FP32 (final state undone event by event
    with inverse_update_dual), which is also what the CUDA backward computes.
    mode "f32_stored": FP32 with the forward's states stored instead of undone.
    """
    s = scene.as_dtype(np.float64)
    rayo = np.ascontiguousarray(np.asarray(rayo, np.float64).reshape(-1, 3))
    rayd = np.ascontiguousarray(np.asarray(rayd, np.float64).reshape(-1, 3))
    R = rayo.shape[0]
    deg = colour_degree(sh_degree)
    events = np.ascontiguousarray(events, np.int32)
    iters = np.ascontiguousarray(iters, np.int32)
    dout = np.ascontiguousarray(np.asarray(dout, np.float64).reshape(R, 5))
    g = Grads(np.zeros((s.N, 3)), np.zeros((s.N, 3)), np.zeros((s.N, 4)), np.zeros(s.N),
              np.zeros((s.N, s.K, 3)), np.zeros((R, 3)), np.zeros((R, 3)))
    fn = {"f64": lib().ora_backward_f64, "f32_replay": lib().ora_backward_f32_replay,
          "f32_stored": lib().ora_backward_f32_stored}[mode]
    rc = fn(s.N, s.K, deg, _ptr(s.mean), _ptr(s.scale), _ptr(s.quat), _ptr(s.density),
            _ptr(s.features), R, _ptr(rayo), _ptr(rayd), float(tmin), float(tmax),
            int(max_iters), _ptr(events), _ptr(iters), _ptr(dout), _ptr(g.mean),
            _ptr(g.scale), _ptr(g.quat), _ptr(g.density), _ptr(g.features),
            _ptr(g.rayo), _ptr(g.rayd), _threads(nthreads))
    assert rc == 0
    return g


def finite_difference(scene: Scene, rayo, rayd, tmin, tmax, max_iters, dout, eps=1e-6,
                      sh_degree=None, which=("mean", "scale", "quat", "density", "features", "rayo", "rayd")):
    """FP64 central differences of L = sum(dout * out) through the FP64 forward."""
    base = scene.as_dtype(np.float64)
    rayo = np.asarray(rayo, np.float64).reshape(-1, 3).copy()
    rayd = np.asarray(rayd, np.float64).reshape(-1, 3).copy()
    dout = np.asarray(dout, np.float64)

    def loss(sc, ro, rd):
        tr = trace(sc, ro, rd, tmin, tmax, max_iters, sh_degree, precision="f64", with_events=False,
                   nthreads=1)
        return float((tr.out * dout).sum())

    res = {}
    for name in which:
        if name in ("rayo", "rayd"):
            arr = rayo if name == "rayo" else rayd
        else:
            arr = getattr(base, name)
        g = np.zeros_like(arr)
        flat, gflat = arr.reshape(-1), g.reshape(-1)
        for i in range(flat.size):
            old = flat[i]
            flat[i] = old + eps
            lp = loss(base, rayo, rayd)
            flat[i] = old - eps
            lm = loss(base, rayo, rayd)
            flat[i] = old
            gflat[i] = (lp - lm) / (2 * eps)
        res[name] = g
    return res


def intersect_f32(mean, scale, quat, rayo, rayd, tmin=0.0):
    a = lambda x: np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1))
    t = np.zeros(2, np.float32)
    hit = lib().ora_intersect_f32(_ptr(a(mean)), _ptr(a(scale)), _ptr(a(quat)), _ptr(a(rayo)), _ptr(a(rayd)),
                                  float(tmin), _ptr(t))
    return (t[0], t[1]) if hit else None
