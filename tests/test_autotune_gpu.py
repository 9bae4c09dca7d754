"""The autotuner times its candidates on the caller's workload and rejects any whose launch
raised a status flag: a traversal stack shallower than the tree overflows
(EVER_STATUS_STACK_OVERFLOW) and must never be picked. trace_rays then runs the cached
pick for its workload."""
import numpy as np
import pytest
import torch

from ever_b200 import autotune as AT
from ever_b200 import synthetic as S
from ever_b200 import tracer as T
from ever_b200.fast_ellipsoid_splinetracer import trace_rays

pytestmark = pytest.mark.gpu


def test_autotuner_rejects_an_overflowing_stack_and_trace_rays_uses_the_pick(tmp_path, monkeypatch):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dev = torch.device("cuda:0")
    sc = S.clustered_scene(20_000, 0, seed=41, n_clusters=40)
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(4.0, 41), 64, 48, 50.0))
    t = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), device=dev)
    scene = T.Scene(t(sc.mean), t(sc.scale), t(sc.quat), t(sc.density.reshape(-1)), t(sc.features))
    rayo, rayd = t(ro), t(rd)
    order = T.ray_order(rayo, rayd)

    def run(c):
        f = T.forward(scene, rayo, rayd, ray_order=order if c.ordered else None, tune=c.tune())
        return int(f.status.item())

    # gather rounds only (traversal 2), so the walk uses the stack for every ray
    shallow, deep = AT.Candidate(16, 128, 2, True, 8), AT.Candidate(16, 128, 2, True, 64)
    cache = tmp_path / "tune.json"
    key = AT.workload_key(scene.num_prims, rayo.shape[0], scene.sh_coeffs, dev)
    best, timings = AT.autotune(run, key, [shallow, deep], cache_path=str(cache), force=True)
    assert timings[shallow.name()] == f"status {1}"  # EVER_STATUS_STACK_OVERFLOW
    assert best == deep and isinstance(timings[deep.name()], float)
    # trace_rays looks the pick up by its workload key and gives the same image as the defaults
    monkeypatch.setenv("EVER_B200_CACHE", str(tmp_path))
    (tmp_path / "autotune.json").write_text(cache.read_text())
    assert AT.cached_tune(scene.num_prims, rayo.shape[0], scene.sh_coeffs, dev) == deep
    args = [t(getattr(sc, k)) for k in ("mean", "scale", "quat", "density", "features")]
    got = trace_rays(*args, rayo, rayd)
    want = trace_rays(*args, rayo, rayd, tune=T.Tune())
    assert torch.equal(got, want)
