"""Parity at the benchmark configurations' own shapes.

- config 1: 100,000 uniform ellipsoids, SH3 features, one 800x800 view from a seeded point
  at radius 3, forward + backward through trace_rays. Events bit-exact and outputs to
  1e-5 against the oracle on a seeded 2,048-ray subset; the subset rays' gradients
  against the oracle's reverse replay and exact FP64; FP64 central differences
  (the method of the reference's tests/grad_check.py:134-204) for all five ellipsoid
  tensors on a seeded 1,000-ellipsoid sub-scene.
- config 2: 1,000,000 clustered ellipsoids, SH3, one 1920x1080 view (2,073,600 rays), through
  trace_rays at its defaults, so the forward runs the regrouped packed passes (the view
  holds more than four times the B200's resident lanes). Events bit-exact and outputs to
  1e-5 on a seeded 1,000-ray subset; the subset rays' gradients against the replay.
- The max error against the FP64 oracle, per output and per gradient, is computed and
  bounded; with EVER_REPORT_DIR set it is also written there as fp64_errors.json.
"""
import json
import os

import numpy as np
import pytest
import torch

from ever_b200 import synthetic as S
from ever_b200.fast_ellipsoid_splinetracer import trace_rays
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NAMES = ("mean", "scale", "quat", "density", "features")
RTOL, ATOL = 1e-5, 1e-6
DIST_RTOL, DIST_ATOL = 1e-4, 1e-5
# Gradient tolerances, each as (rel, floor): every entry must satisfy
# |got - ref| <= rel * |ref| + floor * max|ref| (elementwise with a floor); the reports
# give max|got - ref| / max|ref| and the largest elementwise relative error over the
# entries above 1e-3 of the max.
# vs the oracle's FP32 reverse replay (the same algorithm; expf/powf last bits only):
REPLAY = (1e-3, 1e-5)
# vs exact FP64: FP32 evaluation of dt/dparams ~ 1/sqrt(h) at grazing hits limits the
# largest entries to ~1e-3 of the max (the reference's FP32 backward shares this)
EXACT = (1e-2, 2e-3)
# ray gradients sum only the few events of one ray, so one grazing event dominates them:
# measured up to 1.2% of the ray-gradient max against FP64 on the config-1 view
EXACT_RAY = (3e-2, 1e-2)
# vs FP64 central differences: tests/grad_check.py's 1e-2, on entries above 1e-3 of the max
FD = (1e-2, 2e-3)


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _errs(got, ref, floor=1e-3):
    """(max |d| / max |ref|, max elementwise |d|/|ref| over |ref| > floor * max |ref|)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    m = np.abs(ref).max() if ref.size else 0.0
    if m == 0.0:
        return float(np.abs(got).max() if got.size else 0.0), 0.0
    d = np.abs(got - ref)
    big = np.abs(ref) > floor * m
    return float(d.max() / m), float((d[big] / np.abs(ref[big])).max()) if big.any() else 0.0


def _assert_close(name, got, ref, tol):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    m = np.abs(ref).max() if ref.size else 0.0
    bad = np.abs(got - ref) > tol[0] * np.abs(ref) + tol[1] * m
    assert not bad.any(), (name, int(bad.sum()), got[bad][:5], ref[bad][:5], m)


def _clip(k, v):
    return np.clip(v, -50, 50) if k == "density" else np.clip(v, -1e3, 1e3)


def _trace_full(sc, ro, rd, dout):
    dev = _dev()
    t = {k: torch.tensor(np.ascontiguousarray(getattr(sc, k), np.float32), device=dev, requires_grad=True)
         for k in NAMES}
    rayo = torch.tensor(ro, device=dev, requires_grad=True)
    rayd = torch.tensor(rd, device=dev, requires_grad=True)
    out, extras = trace_rays(t["mean"], t["scale"], t["quat"], t["density"], t["features"], rayo, rayd,
                             return_extras=True)
    assert int(extras["status"].item()) == 0
    res = {"out": out.detach().cpu().numpy(), "iters": extras["iters"].cpu().numpy(),
           "tri": extras["tri_collection"].reshape(-1, ro.shape[0])}
    (out * torch.tensor(dout, dtype=torch.float32, device=dev)).sum().backward()
    res["grads"] = {k: v.grad.cpu().double().numpy() for k, v in t.items()}
    res["grads"]["rayo"] = rayo.grad.cpu().double().numpy()
    res["grads"]["rayd"] = rayd.grad.cpu().double().numpy()
    return res


def _subset_parity(sc, ro, rd, dout, res, sub):
    """Events, outputs and per-ray gradients of the rays `sub` against the oracle."""
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), sc.features)
    ref = O.trace(s, ro[sub], rd[sub], 0.0, 1000.0, 500)
    iters = res["iters"][sub]
    np.testing.assert_array_equal(iters, ref.iters)
    n = max(int(iters.max()) if iters.size else 0, 1)
    tri_dev = res["tri"]
    tri = tri_dev[:n][:, torch.as_tensor(sub, device=tri_dev.device)].cpu().numpy()
    mask = np.arange(tri.shape[0])[:, None] < iters[None, :]
    np.testing.assert_array_equal(np.where(mask, tri, -1), np.where(mask, ref.events[:tri.shape[0]], -1))
    out = res["out"][sub]
    np.testing.assert_allclose(out[:, :4], ref.out[:, :4], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(out[:, 4], ref.out[:, 4], rtol=DIST_RTOL, atol=DIST_ATOL)
    report = {}
    rep = O.backward(s, ro[sub], rd[sub], 0.0, 1000.0, 500, ref.events, ref.iters, dout[sub], mode="f32_replay")
    f64 = O.backward(s, ro[sub], rd[sub], 0.0, 1000.0, 500, ref.events, ref.iters, dout[sub], mode="f64")
    for k in ("rayo", "rayd"):
        g = res["grads"][k][sub]
        _assert_close(k, g, _clip(k, getattr(rep, k)), REPLAY)
        _assert_close(k, g, _clip(k, getattr(f64, k)), EXACT_RAY)
        a, e = _errs(g, _clip(k, getattr(f64, k)))
        report[k] = {"max_rel_to_max": a, "max_elementwise_rel": e}
    ref64 = O.trace(s, ro[sub], rd[sub], 0.0, 1000.0, 500, precision="f64", with_events=False)
    for c, name in enumerate(("R", "G", "B", "opacity", "distortion")):
        d = np.abs(out[:, c].astype(np.float64) - ref64.out[:, c])
        report[name] = {"max_abs": float(d.max()),
                        "max_rel": float((d / np.maximum(np.abs(ref64.out[:, c]), 1e-6)).max())}
    return report


def _write_report(name, data):
    d = os.environ.get("EVER_REPORT_DIR")
    if not d:
        return
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, "fp64_errors.json")
    allr = json.load(open(path)) if os.path.exists(path) else {}
    allr[name] = data
    with open(path, "w") as f:
        json.dump(allr, f, indent=1, sort_keys=True)


def test_config1_mid_scene_subset_and_fd_sub_scene():
    sc, cams = S.workload_mid()
    assert sc.N == 100_000 and sc.features.shape[1] == 16 and (cams[0].width, cams[0].height) == (800, 800)
    ro, rd = S.look_at_rays(cams[0])
    rng = np.random.default_rng(101)
    dout = rng.normal(size=(ro.shape[0], 5))
    res = _trace_full(sc, ro, rd, dout)
    sub = np.sort(rng.choice(ro.shape[0], 2048, replace=False))
    report = {"outputs_and_ray_grads_2048_rays": _subset_parity(sc, ro, rd, dout, res, sub)}
    assert int(res["iters"].max()) > 20  # the view crosses the cloud: long event sequences

    # FP64 central differences on a seeded 1,000-ellipsoid sub-scene, 64x64 rays of the view
    keep = np.sort(rng.choice(sc.N, 1000, replace=False))
    ss = sc.subset(keep)
    cam = S.Camera(cams[0].eye, 64, 64, cams[0].fov_y_deg)
    sro, srd = S.look_at_rays(cam)
    sdout = rng.normal(size=(sro.shape[0], 5))
    sres = _trace_full(ss, sro, srd, sdout)
    s = O.Scene(ss.mean, ss.scale, ss.quat, ss.density.reshape(-1), ss.features)
    tr = O.trace(s, sro, srd, 0.0, 1000.0, 500)
    g64 = O.backward(s, sro, srd, 0.0, 1000.0, 500, tr.events, tr.iters, sdout, mode="f64")
    s64 = s.as_dtype(np.float64)
    ro64, rd64 = sro.astype(np.float64), srd.astype(np.float64)

    def loss(sc64):
        return float((O.trace(sc64, ro64, rd64, 0.0, 1000.0, 500, precision="f64", with_events=False).out
                      * sdout).sum())

    eps = 1e-7
    grads_report = {}
    for k in NAMES:
        g = sres["grads"][k].reshape(getattr(s64, k).shape)
        ref = getattr(g64, k).reshape(g.shape)
        _assert_close(k, g, _clip(k, ref), EXACT)
        a, e = _errs(g, _clip(k, ref))
        grads_report[k] = {"max_rel_to_max": a, "max_elementwise_rel": e}
        flat_ref = np.abs(ref).reshape(-1)
        cand = np.nonzero(flat_ref > 1e-3 * flat_ref.max())[0]
        pick = rng.choice(cand, min(24, cand.size), replace=False)
        if k == "features":  # coefficients k >= 1 are not in the forward: FD and gradient are 0
            hi = np.nonzero((np.arange(flat_ref.size) // 3) % 16 >= 1)[0]
            pick = np.concatenate([pick, rng.choice(hi, 4, replace=False)])
        arr = getattr(s64, k).reshape(-1)
        fd = np.zeros(pick.size)
        for n, i in enumerate(pick):
            old = arr[i]
            arr[i] = old + eps
            lp = loss(s64)
            arr[i] = old - eps
            lm = loss(s64)
            arr[i] = old
            fd[n] = (lp - lm) / (2 * eps)
        got = g.reshape(-1)[pick]
        bad = np.abs(got - fd) > FD[0] * np.abs(fd) + FD[1] * flat_ref.max()
        assert not bad.any(), (k, pick[bad], got[bad], fd[bad])
        grads_report[k]["fd_entries_checked"] = int(pick.size)
    for k in ("rayo", "rayd"):
        a, e = _errs(sres["grads"][k], _clip(k, getattr(g64, k)))
        grads_report[k] = {"max_rel_to_max": a, "max_elementwise_rel": e}
    report["gradients_1000_ellipsoid_sub_scene_64x64"] = grads_report
    _write_report("config1_100k_uniform_sh3_800x800", report)


def test_config2_scene_scale_subset_regrouped():
    sc, cams = S.workload_scene()
    assert sc.N == 1_000_000 and (cams[0].width, cams[0].height) == (1920, 1080)
    ro, rd = S.look_at_rays(cams[0])
    # more rays than four times the resident lanes (148 SMs x 20 warps x 32): trace_rays
    # runs the regrouped forward with both splits
    assert ro.shape[0] > 4 * 148 * 20 * 32
    rng = np.random.default_rng(202)
    dout = rng.normal(size=(ro.shape[0], 5))
    res = _trace_full(sc, ro, rd, dout)
    sub = np.sort(rng.choice(ro.shape[0], 1000, replace=False))
    report = _subset_parity(sc, ro, rd, dout, res, sub)
    assert float(res["iters"].mean()) > 10.0
    _write_report("config2_1M_clustered_sh3_1920x1080", {"outputs_and_ray_grads_1000_rays": report})
