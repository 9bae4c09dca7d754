"""A scene built for the DC colour only (ever_scene_build_dc: records carry their DC colour,
no feature rows are copied) traces exactly as a full scene at the default colour, forward
and backward, and refuses traces that need SH of degree > 0."""
import numpy as np
import pytest
import torch

from ever_b200 import synthetic as S
from ever_b200 import tracer as T

pytestmark = pytest.mark.gpu


def test_dc_scene_matches_full_scene_and_refuses_higher_degrees():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dev = torch.device("cuda:0")
    sc = S.clustered_scene(30_000, 3, seed=12, n_clusters=30)
    ro, rd = S.look_at_rays(S.Camera(S.sphere_point(4.0, 12), 96, 64, 50.0))
    t = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), device=dev)
    args = (t(sc.mean), t(sc.scale), t(sc.quat), t(sc.density.reshape(-1)), t(sc.features))
    rayo, rayd = t(ro), t(rd)
    order = T.ray_order(rayo, rayd)
    gout = torch.randn((rayo.shape[0], 5), device=dev, generator=torch.Generator(device=dev).manual_seed(3))
    res = {}
    for dc in (False, True):
        scene = T.Scene(*args, dc_only=dc)
        f = T.forward(scene, rayo, rayd, ray_order=order)
        g = T.backward(scene, rayo, rayd, f, gout, ray_order=order, slot_order=T.backward_order(f, order, 0))
        res[dc] = (f, g)
        if dc:
            with pytest.raises(RuntimeError, match="ever_scene_build_dc"):
                T.forward(scene, rayo, rayd, sh_degree=1, ray_order=order)
    (fa, ga), (fb, gb) = res[False], res[True]
    assert int(fb.status.item()) == 0 and int(fb.iters.max()) > 5
    assert torch.equal(fa.out, fb.out) and torch.equal(fa.iters, fb.iters)
    # each row of the ray-major log is written up to its ray's event count only
    written = torch.arange(fa.event_log.shape[1], device=dev)[None, :] < fa.iters[order.long()][:, None]
    assert torch.equal(torch.where(written, fa.event_log, -1), torch.where(written, fb.event_log, -1))
    for x, y in zip((ga.mean, ga.scale, ga.quat, ga.density, ga.features, ga.rayo, ga.rayd),
                    (gb.mean, gb.scale, gb.quat, gb.density, gb.features, gb.rayo, gb.rayd)):
        assert float((x - y).abs().max()) <= 1e-5 * float(y.abs().max()) + 1e-12  # float atomics: order only
