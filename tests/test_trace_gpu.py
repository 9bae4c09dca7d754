"""GPU parity of the CUDA tracer against the CPU oracle (forward: bit-exact event
sequences and counts, colour/opacity/distortion within 1e-5 relative) and against the
reference's own quadrature outputs (tests/compare_quadrature.py tolerance 1e-4)."""
import os

import numpy as np
import pytest
import torch

from ever_b200 import synthetic as S
from ever_b200 import tracer as T
from ever_b200.fast_ellipsoid_splinetracer import trace_rays
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "quad_reference.npz")
RTOL = 1e-5   # RGB / opacity vs the FP32 oracle (last-bit expf differences only)
ATOL = 1e-6
DIST_RTOL = 1e-4  # distortion: sums of powf-warped midpoints, libm vs CUDA powf last bits
DIST_ATOL = 1e-5


def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def _gpu_trace(sc, ro, rd, tmin=0.0, tmax=1000.0, max_iters=500, sh_degree=None, tune=None, ray_order=None):
    dev = _dev()
    t = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), device=dev)
    scene = T.Scene(t(sc.mean), t(sc.scale), t(sc.quat), t(np.asarray(sc.density).reshape(-1)), t(sc.features))
    fwd = T.forward(scene, t(ro), t(rd), tmin, tmax, max_iters, sh_degree, log_events=True, touch_count=True,
                    ray_stats=True, tune=tune, ray_order=ray_order)
    tri = T.reference_tri_collection(scene, fwd, max_iters, ray_order)
    torch.cuda.synchronize()
    return scene, fwd, tri.cpu().numpy().reshape(max(max_iters, 0), -1)


def _oracle(sc, ro, rd, tmin=0.0, tmax=1000.0, max_iters=500, sh_degree=None):
    s = O.Scene(sc.mean, sc.scale, sc.quat, np.asarray(sc.density).reshape(-1), sc.features)
    return O.trace(s, ro, rd, tmin, tmax, max_iters, sh_degree)


def _assert_parity(fwd, tri, ref, check_events=True):
    iters = fwd.iters.cpu().numpy()
    np.testing.assert_array_equal(iters, ref.iters)
    if check_events:
        mask = np.arange(tri.shape[0])[:, None] < iters[None, :]
        np.testing.assert_array_equal(np.where(mask, tri, -1), np.where(mask, ref.events, -1))
    out = fwd.out.cpu().numpy()
    np.testing.assert_allclose(out[:, :4], ref.out[:, :4], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(out[:, 4], ref.out[:, 4], rtol=DIST_RTOL, atol=DIST_ATOL)
    np.testing.assert_array_equal(fwd.ray_stats.cpu().numpy()[:, 0], ref.iters.astype(np.float32))
    np.testing.assert_array_equal(fwd.ray_stats.cpu().numpy()[:, 1], ref.depth)
    assert int(fwd.status.item()) == 0


def test_small_uniform_sh0():
    sc, cams = S.workload_small()
    ro, rd = S.look_at_rays(cams[0])
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd))


@pytest.mark.parametrize("sh_degree", [None, 3])
@pytest.mark.parametrize("traversal", [0, 1, 2])
@pytest.mark.parametrize("kbuf,block", [(8, 64), (16, 128), (32, 256)])
def test_sh3_scene_all_launch_shapes(kbuf, block, traversal, sh_degree):
    sc = S.uniform_scene(3000, 3, seed=7)
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(3.0, 7), 40, 30, 60.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd, sh_degree=sh_degree,
                             tune=T.Tune(kbuf=kbuf, block=block, traversal=traversal))
    _assert_parity(fwd, tri, _oracle(sc, ro, rd, sh_degree=sh_degree))


def test_clustered_scene_subset():
    sc = S.clustered_scene(20000, 3, seed=2, n_clusters=40)
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(4.0, 2), 48, 27, 50.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd))


@pytest.mark.parametrize("max_iters", [1, 5, 17, 40])
def test_max_iters_truncation(max_iters):
    sc = S.uniform_scene(800, 0, seed=3)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 16, 16, 50.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd, max_iters=max_iters)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd, max_iters=max_iters))


@pytest.mark.parametrize("tmin,tmax", [(0.3, 1000.0), (1.0, 3.2), (0.0, 2.5)])
def test_tmin_tmax(tmin, tmax):
    sc = S.uniform_scene(800, 1, seed=4)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 16, 16, 50.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd, tmin=tmin, tmax=tmax)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd, tmin=tmin, tmax=tmax))


def test_rays_starting_inside_ellipsoids():
    # camera inside the cloud: many rays start inside one or more ellipsoids
    sc = S.uniform_scene(1500, 3, seed=6)
    sc.scale *= 3.0
    ro, rd = S.look_at_rays(S.Camera(np.array([0.05, 0.1, 0.2]), 20, 20, 90.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    ref = _oracle(sc, ro, rd)
    _assert_parity(fwd, tri, ref)


def test_unnormalised_quats_and_directions():
    sc = S.uniform_scene(600, 2, seed=8)
    rng = np.random.default_rng(0)
    sc.quat = (sc.quat * rng.uniform(0.7, 1.4, (600, 1))).astype(np.float32)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 16, 16, 50.0))
    rd = (rd * rng.uniform(0.5, 2.0, (rd.shape[0], 1))).astype(np.float32)
    _, fwd, tri = _gpu_trace(sc, ro, rd, tmin=0.1)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd, tmin=0.1))


@pytest.mark.parametrize("traversal", [0, 2])
def test_long_row_of_ellipsoids_overflows_the_packet_lists(traversal):
    # 1,200 disjoint small ellipsoids in a row along the z axis and a packet of rays down the
    # row: the packet can meet more leaves than its shared-memory list holds, so the frustum
    # phase hands the whole packet to the gather rounds; the results stay exact. (Disjoint
    # and spaced, so no two events of a ray share a t: the oracle orders such ties by index,
    # the GPU by Morton position.)
    rng = np.random.default_rng(17)
    n = 1200
    mean = np.stack([rng.uniform(-2e-3, 2e-3, n), rng.uniform(-2e-3, 2e-3, n), 0.5 + 0.05 * np.arange(n)], 1)
    sc = S.SceneArrays(mean.astype(np.float32), np.full((n, 3), 0.02, np.float32),
                       S.uniform_scene(n, 0, seed=17).quat, np.full((n, 1), 0.01, np.float32),
                       rng.normal(0, 0.5, (n, 1, 3)).astype(np.float32))
    ro = np.zeros((64, 3), np.float32)
    ang = rng.uniform(-2e-4, 2e-4, (64, 2))
    rd = np.stack([ang[:, 0], ang[:, 1], np.ones(64)], 1).astype(np.float32)
    _, fwd, tri = _gpu_trace(sc, ro, rd, tune=T.Tune(traversal=traversal), max_iters=3000)
    ref = _oracle(sc, ro, rd, max_iters=3000)
    iters = fwd.iters.cpu().numpy()
    np.testing.assert_array_equal(iters, ref.iters)
    mask = np.arange(tri.shape[0])[:, None] < iters[None, :]
    np.testing.assert_array_equal(np.where(mask, tri, -1), np.where(mask, ref.events, -1))
    # 2,400 events per ray: the last-bit differences of CUDA's and libm's expf add up to
    # a few 1e-5 of the colour over so many updates (1e-5 holds for the usual ~20 events)
    np.testing.assert_allclose(fwd.out.cpu().numpy()[:, :4], ref.out[:, :4], rtol=2e-4, atol=1e-6)
    assert int(fwd.iters.max()) > 1000
    _, ref, tref = _gpu_trace(sc, ro, rd, tune=T.Tune(traversal=2), max_iters=3000)
    assert torch.equal(fwd.out, ref.out) and torch.equal(fwd.states, ref.states) and np.array_equal(tri, tref)


def test_nested_shells_overflow_the_pending_buffer_midway():
    # 24 nested ellipsoids: a ray meets 24 entries before the first exit, so its 16-event
    # buffer overflows after some of the entries have been integrated; the rounds then
    # continue the ray from its last integrated event. Exact against the oracle and equal
    # bit for bit to the rounds-only mode.
    rng = np.random.default_rng(23)
    n = 24
    r = np.linspace(0.1, 1.2, n)
    sc = S.SceneArrays(rng.normal(0, 0.01, (n, 3)).astype(np.float32),
                       (r[:, None] * rng.uniform(0.9, 1.1, (n, 3))).astype(np.float32),
                       S.uniform_scene(n, 0, seed=23).quat, rng.uniform(0.05, 0.2, (n, 1)).astype(np.float32),
                       rng.normal(0, 0.5, (n, 1, 3)).astype(np.float32))
    ro, rd = S.look_at_rays(S.Camera(np.array([0.2, -0.1, 3.0]), 16, 16, 20.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd))
    assert int(fwd.iters.max()) >= 30
    _, ref, tref = _gpu_trace(sc, ro, rd, tune=T.Tune(traversal=2))
    assert torch.equal(fwd.out, ref.out) and torch.equal(fwd.states, ref.states) and np.array_equal(tri, tref)


@pytest.mark.parametrize("kind", ["half", "true", "random", "zero"])
def test_depth_hint_changes_no_result(kind):
    # the hint only sets where a packet's first frustum stage ends: rays that go on continue
    # in later stages, so any hint, good or bad, gives the same bits
    dev = _dev()
    sc = S.clustered_scene(30_000, 0, seed=51, n_clusters=60)
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(4.0, 51), 64, 48, 50.0))
    scene, ref, tref = _gpu_trace(sc, ro, rd)
    depth = ref.ray_stats[:, 1].clone()
    hint = {"half": 0.5 * depth, "true": depth, "zero": torch.zeros_like(depth),
            "random": torch.rand(depth.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(5)) * 8}[kind]
    t = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), device=dev)
    got = T.forward(scene, t(ro), t(rd), log_events=True, ray_stats=True, depth_hint=hint.contiguous())
    tri = T.reference_tri_collection(scene, got, 500).cpu().numpy().reshape(500, -1)
    for k in ("out", "states", "iters", "last_dirac"):
        assert torch.equal(getattr(got, k), getattr(ref, k)), k
    assert np.array_equal(tri, tref)
    assert int(got.status.item()) == 0


def test_duplicate_ellipsoids_round_boundary():
    # 20 identical ellipsoids: ties at the reference's 16-event round boundary
    N = 20
    sc = S.SceneArrays(np.tile([[0, 0, 2.0]], (N, 1)).astype(np.float32), np.full((N, 3), 0.3, np.float32),
                       np.tile([[1.0, 0, 0, 0]], (N, 1)).astype(np.float32), np.full((N, 1), 0.01, np.float32),
                       np.full((N, 1, 3), 0.1, np.float32))
    ro = np.zeros((1, 3), np.float32)
    rd = np.array([[0, 0, 1.0]], np.float32)
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    ref = _oracle(sc, ro, rd)
    np.testing.assert_array_equal(fwd.iters.cpu().numpy(), ref.iters)
    assert ref.iters[0] == 32
    # tie order among identical ellipsoids is implementation-defined (the reference's is
    # OptiX traversal order): compare entry/exit pattern and colour
    assert np.array_equal(tri[:32, 0] % 2, ref.events[:32, 0] % 2)
    np.testing.assert_allclose(fwd.out.cpu().numpy()[:, :4], ref.out[:, :4], rtol=RTOL, atol=ATOL)


def test_empty_and_single():
    dev = _dev()
    sc = S.uniform_scene(1, 0, seed=1)
    sc.mean[:] = [[0, 0, 0]]
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 8, 8, 30.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    _assert_parity(fwd, tri, _oracle(sc, ro, rd))
    # no ellipsoids
    z = torch.zeros((0, 3), device=dev)
    out = trace_rays(z, z, torch.zeros((0, 4), device=dev), torch.zeros((0, 1), device=dev),
                     torch.zeros((0, 1, 3), device=dev), torch.tensor(ro, device=dev), torch.tensor(rd, device=dev))
    assert out.shape == (64, 5) and float(out.abs().sum()) == 0.0
    # no rays
    s = S.uniform_scene(10, 0, seed=1)
    t = lambda a: torch.tensor(a, device=dev)
    out = trace_rays(t(s.mean), t(s.scale), t(s.quat), t(s.density), t(s.features), torch.zeros((0, 3), device=dev),
                     torch.zeros((0, 3), device=dev))
    assert out.shape == (0, 5)


@pytest.mark.parametrize("kind", ["random", "coherent"])
def test_ray_order_permutation_is_transparent(kind):
    sc = S.uniform_scene(2000, 3, seed=9)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 32, 32, 50.0))
    _, a, ta = _gpu_trace(sc, ro, rd)
    if kind == "random":
        perm = torch.randperm(ro.shape[0], generator=torch.Generator().manual_seed(0)).to(torch.int32).cuda()
    else:
        perm = T.ray_order(torch.tensor(ro, device="cuda"), torch.tensor(rd, device="cuda"))
        assert torch.equal(torch.sort(perm.long()).values, torch.arange(ro.shape[0], device="cuda"))
    _, b, tb = _gpu_trace(sc, ro, rd, ray_order=perm)
    assert torch.equal(a.out, b.out) and torch.equal(a.iters, b.iters) and torch.equal(a.states, b.states)
    assert np.array_equal(ta, tb)


def test_deterministic():
    sc = S.uniform_scene(2000, 3, seed=10)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 32, 32, 50.0))
    _, a, ta = _gpu_trace(sc, ro, rd)
    _, b, tb = _gpu_trace(sc, ro, rd)
    assert torch.equal(a.out, b.out) and np.array_equal(ta, tb)


def test_touch_count_matches_events():
    sc = S.uniform_scene(1000, 0, seed=12)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.0, 0.0, 3.0]), 32, 32, 50.0))
    _, fwd, tri = _gpu_trace(sc, ro, rd)
    iters = fwd.iters.cpu().numpy()
    mask = np.arange(tri.shape[0])[:, None] < iters[None, :]
    expect = np.bincount((tri[mask] // 2), minlength=1000)
    np.testing.assert_array_equal(fwd.touch_count.cpu().numpy(), expect)


def _golden():
    z = np.load(GOLDEN)
    for i in range(int(z["count"])):
        yield {k: z[f"c{i}_{k}"] for k in ("kind", "N", "dm", "out", "mean", "scale", "quat", "density",
                                              "features", "rayo", "rayd", "tmin")}


@pytest.mark.parametrize("case", list(_golden()), ids=lambda c: f"{c['kind']}-N{int(c['N'])}-d{float(c['dm'])}")
def test_matches_reference_quadrature(case):
    # tests/compare_quadrature.py: RGB + opacity vs the quadrature oracle at atol = rtol = 1e-4
    dev = _dev()
    t = lambda k: torch.tensor(np.ascontiguousarray(case[k], np.float32), device=dev)
    out = trace_rays(t("mean"), t("scale"), t("quat"), t("density"), t("features"), t("rayo"), t("rayd"),
                     float(case["tmin"]), 100.0)
    np.testing.assert_allclose(out[:, :4].cpu().numpy().reshape(-1), case["out"][:4], atol=1e-4, rtol=1e-4)


def test_argument_errors():
    dev = _dev()
    s = S.uniform_scene(10, 0, seed=1)
    t = lambda a: torch.tensor(a, device=dev)
    with pytest.raises(RuntimeError, match="last dimension"):
        trace_rays(t(s.mean[:, :2].copy()), t(s.scale), t(s.quat), t(s.density), t(s.features),
                   torch.zeros((1, 3), device=dev), torch.zeros((1, 3), device=dev))
    with pytest.raises(RuntimeError, match="CUDA"):
        trace_rays(torch.tensor(s.mean), t(s.scale), t(s.quat), t(s.density), t(s.features),
                   torch.zeros((1, 3), device=dev), torch.zeros((1, 3), device=dev))
    with pytest.raises(RuntimeError, match="same 0 dimension"):
        trace_rays(t(s.mean), t(s.scale[:5].copy()), t(s.quat), t(s.density), t(s.features),
                   torch.zeros((1, 3), device=dev), torch.zeros((1, 3), device=dev))
