"""The binary PLY scene loader (ever_ply_count / ever_ply_read, host code) against the
reference's conversion restated in numpy (oracle/ply_np.py). No GPU needed."""
import numpy as np
import pytest

from ever_b200 import ply
from oracle import ply_np as P


def _arrays(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(n, 3)).astype(np.float32), rng.normal(size=(n, 48)).astype(np.float32),
            rng.normal(size=n).astype(np.float32) * 3, rng.normal(size=(n, 3)).astype(np.float32) * 3 - 2,
            rng.normal(size=(n, 4)).astype(np.float32))


def test_loader_matches_reference_conversion(tmp_path):
    mean, sh, op, sc, rot = _arrays(1000, 0)
    sc[:5] = [[6.0, 7.0, 30.0]] * 5  # softplus linear branch and the 25 cap
    op[:3] = [40.0, -40.0, 0.0]
    path = tmp_path / "scene.ply"
    P.write_ply(path, mean, sh, op, sc, rot)
    got = ply.read_scene(path)
    want = P.convert(mean, sh, op, sc, rot)
    for k in ("mean", "scale", "quat", "features"):
        np.testing.assert_allclose(got[k].numpy(), want[k], rtol=2e-6, atol=1e-7, err_msg=k)
    # density goes through log(1 - 0.99 sigmoid(o)): a last-bit difference between the C
    # library's and numpy's float exp is amplified near alpha = 0.99
    np.testing.assert_allclose(got["density"].numpy(), want["density"], rtol=1e-5, atol=1e-7)


def test_loader_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.ply"
    p.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 1\nend_header\n")
    with pytest.raises(RuntimeError, match="binary_little_endian"):
        ply.read_scene(p)
    mean, sh, op, sc, rot = _arrays(4, 1)
    P.write_ply(p, mean, sh, op, sc, rot)
    data = p.read_bytes()
    p.write_bytes(data[:-8])
    with pytest.raises(RuntimeError, match="truncated"):
        ply.read_scene(p)
    p.write_bytes(data.replace(b"property float rot_3\n", b""))
    with pytest.raises(RuntimeError, match="62 float properties"):
        ply.read_scene(p)
    with pytest.raises(RuntimeError, match="cannot open"):
        ply.read_scene(tmp_path / "missing.ply")
