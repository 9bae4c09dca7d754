"""A scene loaded from a binary PLY file (ever_ply_read, the reference's scene layout and
conversion, splinetracers/fast_ellipsoid_splinetracer/ply_file_loader.cc:166-293) traced on
the GPU: events bit-exact and colours to 1e-5 against the oracle run on the oracle's own
numpy conversion of the same file (oracle/ply_np.py)."""
import numpy as np
import pytest
import torch

from ever_b200 import ply
from ever_b200 import synthetic as S
from ever_b200.fast_ellipsoid_splinetracer import trace_rays
from oracle import oracle as O
from oracle import ply_np as P

pytestmark = pytest.mark.gpu


def test_traced_ply_scene_matches_oracle(tmp_path):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(5)
    n = 4000
    mean = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    sh = rng.normal(0, 0.5, (n, 48)).astype(np.float32)
    opacity = rng.normal(0, 2, n).astype(np.float32)
    scale = np.log(np.expm1(rng.uniform(0.02, 0.12, (n, 3)))).astype(np.float32)  # softplus^-1 of the scales
    rot = rng.normal(size=(n, 4)).astype(np.float32)
    path = tmp_path / "scene.ply"
    P.write_ply(path, mean, sh, opacity, scale, rot)
    got = ply.read_scene(path, device=dev)
    want = P.convert(mean, sh, opacity, scale, rot)
    ro, rd = S.look_at_rays(S.Camera(np.array([0.3, 0.2, 3.0]), 40, 30, 55.0))
    out, extras = trace_rays(got["mean"], got["scale"], got["quat"], got["density"], got["features"],
                             torch.tensor(ro, device=dev), torch.tensor(rd, device=dev), return_extras=True)
    torch.cuda.synchronize()
    # the oracle traces the loader's own arrays (the float conversions agree to a few ulps; see
    # tests/test_ply_cpu.py), and its numpy conversion is checked against them on the host
    s = O.Scene(*(got[k].cpu().numpy() for k in ("mean", "scale", "quat", "density", "features")))
    for k in ("mean", "scale", "quat", "features"):
        np.testing.assert_allclose(getattr(s, k), want[k], rtol=2e-6, atol=1e-7, err_msg=k)
    ref = O.trace(s, ro, rd)
    iters = extras["iters"].cpu().numpy()
    np.testing.assert_array_equal(iters, ref.iters)
    tri = extras["tri_collection"].cpu().numpy().reshape(-1, ro.shape[0])
    mask = np.arange(tri.shape[0])[:, None] < iters[None, :]
    np.testing.assert_array_equal(np.where(mask, tri, -1), np.where(mask, ref.events, -1))
    np.testing.assert_allclose(out.cpu().numpy()[:, :4], ref.out[:, :4], rtol=1e-5, atol=1e-6)
    assert iters.max() > 10
