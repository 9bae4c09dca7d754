"""The drop-in's default colour is the reference forward's: the DC term of every
ellipsoid whatever the SH size K (splinetracers/fast_ellipsoid_splinetracer/slang/
shaders.slang:72-75, get_sh(sh_feats, 0) + eval_sh_col0). Checked at K=16 through
trace_rays with default arguments against the oracle's DC mode: events bit-exact,
RGB/opacity to 1e-5 relative, feature gradients of the coefficients k >= 1 exactly
zero, the DC and geometry gradients to the replay tolerance. View-dependent SH is the
explicit opt-in sh_degree=d and is checked the same way."""
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
REPLAY_TOL = 1e-4  # max abs error / max |gradient| vs the oracle's FP32 reverse replay


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _run(sc, ro, rd, dout, **kw):
    dev = _dev()
    t = {k: torch.tensor(np.ascontiguousarray(getattr(sc, k), np.float32), device=dev, requires_grad=True)
         for k in NAMES}
    rayo = torch.tensor(ro, device=dev, requires_grad=True)
    rayd = torch.tensor(rd, device=dev, requires_grad=True)
    out, extras = trace_rays(t["mean"], t["scale"], t["quat"], t["density"], t["features"], rayo, rayd,
                             return_extras=True, **kw)
    (out * torch.tensor(dout, dtype=torch.float32, device=dev)).sum().backward()
    assert int(extras["status"].item()) == 0
    g = {k: v.grad.cpu().double().numpy() for k, v in t.items()}
    g["rayo"], g["rayd"] = rayo.grad.cpu().double().numpy(), rayd.grad.cpu().double().numpy()
    R = ro.shape[0]
    tri = extras["tri_collection"].cpu().numpy().reshape(-1, R)
    return out.detach().cpu().numpy(), extras["iters"].cpu().numpy(), tri, g


def _rel_err(a, b):
    return np.abs(a - b).max() / (np.abs(b).max() + 1e-12)


def _clip(k, v):
    return np.clip(v, -50, 50) if k == "density" else np.clip(v, -1e3, 1e3)


def _check(sc, ro, rd, dout, sh_degree):
    kw = {} if sh_degree is None else {"sh_degree": sh_degree}
    out, iters, tri, g = _run(sc, ro, rd, dout, **kw)
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), sc.features)
    ref = O.trace(s, ro, rd, 0.0, 1000.0, 500, sh_degree)
    np.testing.assert_array_equal(iters, ref.iters)
    mask = np.arange(tri.shape[0])[:, None] < iters[None, :]
    np.testing.assert_array_equal(np.where(mask, tri, -1), np.where(mask, ref.events, -1))
    np.testing.assert_allclose(out[:, :4], ref.out[:, :4], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(out[:, 4], ref.out[:, 4], rtol=DIST_RTOL, atol=DIST_ATOL)
    rep = O.backward(s, ro, rd, 0.0, 1000.0, 500, ref.events, ref.iters, dout, sh_degree=sh_degree,
                     mode="f32_replay")
    rep = {"mean": rep.mean, "scale": rep.scale, "quat": rep.quat, "density": rep.density.reshape(-1, 1),
           "features": rep.features, "rayo": rep.rayo, "rayd": rep.rayd}
    for k in rep:
        assert _rel_err(g[k], _clip(k, rep[k])) < REPLAY_TOL, (k, _rel_err(g[k], _clip(k, rep[k])))
    return out, g


def test_default_is_reference_dc_colour_at_k16():
    sc = S.uniform_scene(3000, 3, seed=31)
    assert sc.features.shape[1] == 16
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(3.0, 31), 40, 30, 60.0))
    dout = np.random.default_rng(31).normal(size=(ro.shape[0], 5))
    out, g = _check(sc, ro, rd, dout, None)
    # coefficients k >= 1 do not take part in the reference forward: their gradient is 0
    assert np.all(g["features"][:, 1:, :] == 0.0)
    assert np.abs(g["features"][:, 0, :]).max() > 0.0
    # the image is the K=1 trace of the DC coefficients, bit for bit
    dc = S.SceneArrays(sc.mean, sc.scale, sc.quat, sc.density, np.ascontiguousarray(sc.features[:, :1]))
    out1, _, _, _ = _run(dc, ro, rd, dout)
    assert np.array_equal(out, out1)
    # and it differs from view-dependent SH: the default is not sh_degree=3
    out3, _, _, _ = _run(sc, ro, rd, dout, sh_degree=3)
    assert np.abs(out3[:, :3] - out[:, :3]).max() > 1e-3


@pytest.mark.parametrize("sh_degree", [0, 1, 3])
def test_explicit_sh_degree_matches_oracle(sh_degree):
    sc = S.uniform_scene(2000, 3, seed=32 + sh_degree)
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(3.0, 32), 32, 24, 60.0))
    dout = np.random.default_rng(32).normal(size=(ro.shape[0], 5))
    _, g = _check(sc, ro, rd, dout, sh_degree)
    nb = (sh_degree + 1) ** 2
    assert np.all(g["features"][:, nb:, :] == 0.0)


def test_dc_colour_follows_set_features_and_refit():
    # the records carry the DC colour: a new feature tensor (sp.Primitives.set_features /
    # Forward.update_model) and a refit must move it with the features
    from ever_b200 import tracer as T
    dev = _dev()
    sc = S.uniform_scene(1500, 3, seed=34)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 24, 24, 50.0))
    t = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), device=dev)
    scene = T.Scene(t(sc.mean), t(sc.scale), t(sc.quat), t(sc.density.reshape(-1)), t(sc.features))
    f2 = np.random.default_rng(35).normal(0, 0.3, sc.features.shape).astype(np.float32)
    scene.set_features(t(f2))
    a = T.forward(scene, t(ro), t(rd))
    scene.refit()
    b = T.forward(scene, t(ro), t(rd))
    ref = O.trace(O.Scene(sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), f2), ro, rd)
    for f in (a, b):
        np.testing.assert_array_equal(f.iters.cpu().numpy(), ref.iters)
        np.testing.assert_allclose(f.out.cpu().numpy()[:, :4], ref.out[:, :4], rtol=RTOL, atol=ATOL)
