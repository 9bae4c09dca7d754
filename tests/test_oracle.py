"""CPU tests of the oracle itself: pinned to the reference's own quadrature oracle
(fixtures made by tests/golden/make_quad_fixtures.py from splinetracers/quad.py),
known answers, FP32/FP64 agreement, and the FP64 backward against central differences
(the method of tests/grad_check.py)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import quad_np as Q

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "quad_reference.npz")


def _cases():
    z = np.load(GOLDEN)
    for i in range(int(z["count"])):
        yield {k: z[f"c{i}_{k}"] for k in ("kind", "N", "dm", "out", "mean", "scale", "quat", "density",
                                              "features", "rayo", "rayd", "tmin")}


@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: f"{c['kind']}-N{int(c['N'])}-d{float(c['dm'])}")
def test_oracle_matches_reference_quadrature(case):
    # tests/compare_quadrature.py: tracer tmax=100, quadrature tmax=3, RGB+opacity at 1e-4
    sc = O.Scene(case["mean"], case["scale"], case["quat"], case["density"], case["features"])
    tr = O.trace(sc, case["rayo"], case["rayd"], float(case["tmin"]), 100.0, 500)
    np.testing.assert_allclose(tr.out[0, :4], case["out"][:4], atol=1e-4, rtol=1e-4)


@pytest.mark.parametrize("case", [c for c in _cases() if int(c["N"]) <= 10],
                         ids=lambda c: f"{c['kind']}-N{int(c['N'])}-d{float(c['dm'])}")
def test_quad_restatement_matches_reference(case):
    q = Q.trace_rays(case["mean"], case["scale"], case["quat"], case["density"], case["features"],
                     case["rayo"], case["rayd"], float(case["tmin"]), 3.0)
    np.testing.assert_allclose(q[0], case["out"], atol=1e-7, rtol=1e-6)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_known_answer_centre_chord(axis):
    # one ellipsoid hit through its centre along a principal axis: chord 2*s_axis,
    # alpha = 1 - exp(-sigma*L), colour = alpha * (SH_C0 f0 + 0.5), events {entry, exit}
    s = np.array([0.3, 0.45, 0.6])
    mean = np.zeros(3)
    mean[axis] = 2.0
    d = np.zeros(3)
    d[axis] = 1.0
    f0 = np.array([0.3, -0.1, 0.25])
    sc = O.Scene(mean[None], s[None], np.array([[1.0, 0, 0, 0]]), np.array([1.7]), f0[None, None])
    tr = O.trace(sc, [[0, 0, 0]], d[None], 0.0, 100.0, 500)
    L = 2 * s[axis]
    alpha = 1 - np.exp(-1.7 * L)
    c = 0.28209479177387814 * f0 + 0.5
    np.testing.assert_allclose(tr.out[0, :3], alpha * c, rtol=2e-6)
    np.testing.assert_allclose(tr.out[0, 3], alpha, rtol=2e-6)
    assert tr.iters[0] == 2
    assert list(tr.events[:2, 0]) == [1, 0]  # entry id 2p+1, exit id 2p
    t01 = O.intersect_f32(mean, s, [1.0, 0, 0, 0], [0, 0, 0], d)
    np.testing.assert_allclose(t01, [2.0 - s[axis], 2.0 + s[axis]], rtol=1e-6)


def test_rotated_known_answer():
    # 90 deg about z swaps the x/y scales of a ray along x
    s = np.array([0.2, 0.5, 0.3])
    h = np.sqrt(0.5)
    q = np.array([h, 0, 0, h])
    t01 = O.intersect_f32([3, 0, 0], s, q, [0, 0, 0], [1, 0, 0])
    np.testing.assert_allclose(t01, [2.5, 3.5], rtol=1e-6)


def test_f32_matches_f64():
    from ever_b200 import synthetic as S
    sc = S.uniform_scene(300, 3, seed=5)
    ro, rd = S.look_at_rays(S.Camera(np.array([0, 0, 3.0]), 16, 16, 60))
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density, sc.features)
    a = O.trace(s, ro, rd, 0.0, 1000.0, 500)
    b = O.trace(s, ro, rd, 0.0, 1000.0, 500, precision="f64")
    assert (a.iters == b.iters).mean() > 0.98
    same = a.iters == b.iters
    np.testing.assert_allclose(a.out[same, :4], b.out[same, :4], atol=2e-5, rtol=1e-4)


def test_termination_and_truncation():
    from ever_b200 import synthetic as S
    sc = S.uniform_scene(400, 0, seed=3)
    ro, rd = S.look_at_rays(S.Camera(np.array([0, 0, 3.0]), 8, 8, 40))
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density, sc.features)
    full = O.trace(s, ro, rd, 0.0, 1000.0, 500)
    # a ray stops once logT >= 5.54
    assert (full.states[:, 12] < 5.54).sum() + (full.states[:, 12] >= 5.54).sum() == 64
    cut = O.trace(s, ro, rd, 0.0, 1000.0, 5)
    assert cut.iters.max() <= 5
    # truncated rays consumed a prefix of the full event sequence
    for j in range(64):
        n = cut.iters[j]
        assert list(cut.events[:n, j]) == list(full.events[:n, j])


def test_round_boundary_tie_drop():
    # 20 copies of one ellipsoid: the reference's 16-slot round ends at the 16th event
    # and the next round starts strictly after its t, dropping the tied events there.
    N = 20
    sc = O.Scene(np.tile([[0, 0, 2.0]], (N, 1)), np.tile([[0.3, 0.3, 0.3]], (N, 1)),
                 np.tile([[1.0, 0, 0, 0]], (N, 1)), np.full(N, 0.01), np.full((N, 1, 3), 0.1))
    tr = O.trace(sc, [[0, 0, 0]], [[0, 0, 1]], 0.0, 100.0, 500)
    # 20 entries at one t: 16 consumed, 4 dropped; then the 20 exits: 16 consumed, 4 dropped
    assert tr.iters[0] == 32
    ids = tr.events[:32, 0]
    assert all(i % 2 == 1 for i in ids[:16]) and all(i % 2 == 0 for i in ids[16:])


def test_exit_beyond_tmax_only_in_entry_round():
    # ellipsoid crossing tmax: its exit (t1 > tmax) counts only if seen in the round of its entry
    sc = O.Scene(np.array([[0, 0, 2.0]]), np.array([[0.5, 0.5, 0.5]]), np.array([[1.0, 0, 0, 0]]),
                 np.array([1.0]), np.full((1, 1, 3), 0.1))
    tr = O.trace(sc, [[0, 0, 0]], [[0, 0, 1]], 0.0, 2.0, 500)
    assert tr.iters[0] == 2  # entry at 1.5 <= tmax, exit at 2.5 in the same round
    tr = O.trace(sc, [[0, 0, 0]], [[0, 0, 1]], 0.0, 1.4, 500)
    assert tr.iters[0] == 0  # entry beyond tmax: nothing reported


def _grad_case(seed, sh3=False, inside=False):
    rng = np.random.default_rng(seed)
    if not sh3:
        # tests/grad_check.py:134-170: one ellipsoid, quat (0,0,0,1), two rays
        mean = 2 * rng.random((1, 3)) - 1
        mean[0, :2] *= 0.2
        sc = O.Scene(mean, 0.5 * rng.random((1, 3)) + 0.05, np.array([[0, 0, 0, 1.0]]), 1.1 * rng.random(1) + 0.1,
                     rng.random((1, 1, 3)))
        ro = np.array([[0, 0, 0], [0, 0, 0.1]])
        rd = np.array([[0, 0, 1.0], [0, 0, 1.0]])
        return sc, ro, rd, rng.random() * 0.3
    N = 10
    off = [-0.2, -0.2, -0.3] if inside else [-0.2, -0.2, 0.5]
    sc = O.Scene(rng.random((N, 3)) * [0.4, 0.4, 1.0] + off, 0.3 * rng.random((N, 3)) + 0.05,
                 rng.normal(size=(N, 4)), 3 * rng.random(N), rng.normal(size=(N, 16, 3)) * 0.3)
    ro = np.zeros((4, 3))
    rd = np.array([[0, 0, 1.0], [0.05, 0, 1], [0, 0.05, 1], [0.03, 0.03, 1]])
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    return sc, ro, rd, 0.02


@pytest.mark.parametrize("seed,sh3,inside", [(0, False, False), (1, False, False), (2, True, False),
                                             (3, True, True)])
def test_fp64_backward_matches_central_differences(seed, sh3, inside):
    sc, ro, rd, tmin = _grad_case(seed, sh3, inside)
    R = ro.shape[0]
    dout = np.random.default_rng(seed + 100).normal(size=(R, 5))
    tr = O.trace(sc, ro, rd, tmin, 100.0, 500, precision="f64")
    g = O.backward(sc, ro, rd, tmin, 100.0, 500, tr.events, tr.iters, dout)
    fd = O.finite_difference(sc, ro, rd, tmin, 100.0, 500, dout, eps=1e-6)
    for k, v in fd.items():
        np.testing.assert_allclose(getattr(g, k), v, atol=1e-6 * (1 + np.abs(v).max()), rtol=1e-5, err_msg=k)


def test_fp32_replay_backward_close_to_fp64():
    # The reference's FP32 scheme (inverse_update_dual replay) vs exact FP64: the gap is
    # FP32 conditioning at grazing hits, not the inverse updates (stored states give the same).
    from ever_b200 import synthetic as S
    sc = S.uniform_scene(600, 3, seed=21)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 12, 12, 50.0))
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density, sc.features)
    dout = np.random.default_rng(0).normal(size=(ro.shape[0], 5))
    tr = O.trace(s, ro, rd, 0.0, 1000.0, 500)
    g64 = O.backward(s, ro, rd, 0.0, 1000.0, 500, tr.events, tr.iters, dout)
    rep = O.backward(s, ro, rd, 0.0, 1000.0, 500, tr.events, tr.iters, dout, mode="f32_replay")
    sto = O.backward(s, ro, rd, 0.0, 1000.0, 500, tr.events, tr.iters, dout, mode="f32_stored")
    for k in ("mean", "scale", "quat", "density", "features", "rayo", "rayd"):
        a, b, c = getattr(rep, k), getattr(g64, k), getattr(sto, k)
        m = np.abs(b).max() + 1e-12
        assert np.abs(a - b).max() / m < 5e-3, k
        assert np.abs(a - c).max() / m < 1e-4, k
