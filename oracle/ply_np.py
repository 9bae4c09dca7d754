"""PLY scene writer and the reference's conversion restated in numpy (test infrastructure
only: imported by tests/, never by the product path).

Layout and conversion follow splinetracers/fast_ellipsoid_splinetracer/ply_file_loader.cc:
166-193 and 196-293: per vertex 62 little-endian floats (mean, normal, 48 SH values,
opacity, scale, rotation); quaternion q/(q.q), scale min(softplus(s) + 3e-4, 25),
density max(0, -log(max(1 - 0.99 sigmoid(o), 1e-10))) / (2 min scale).
"""
from __future__ import annotations

import numpy as np

NAMES = (["x", "y", "z", "nx", "ny", "nz"] + [f"f_dc_{i}" for i in range(3)] + [f"f_rest_{i}" for i in range(45)] +
         ["opacity"] + [f"scale_{i}" for i in range(3)] + [f"rot_{i}" for i in range(4)])


def write_ply(path, mean, sh48, opacity, scale, rot, normal=None):
    n = mean.shape[0]
    normal = np.zeros((n, 3), np.float32) if normal is None else normal
    data = np.concatenate([mean, normal, sh48, opacity.reshape(n, 1), scale, rot], 1).astype("<f4")
    assert data.shape[1] == 62
    head = ["ply", "format binary_little_endian 1.0", f"element vertex {n}"]
    head += [f"property float {name}" for name in NAMES] + ["end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        f.write(data.tobytes())


def convert(mean, sh48, opacity, scale, rot):
    f32 = np.float32
    q = rot.astype(f32)
    ln = (q * q).sum(1, dtype=f32).astype(f32)
    quat = (q / ln[:, None]).astype(f32)
    s = scale.astype(f32)
    sp = np.where(s > 5, s, np.log(f32(1) + np.exp(s)).astype(f32))
    sc = np.minimum(sp.astype(np.float64) + 3e-4, 25.0).astype(f32)
    norm = (2 * sc).min(1)
    alpha = (0.99 * (f32(1) / (f32(1) + np.exp(-opacity.astype(f32))))).astype(f32)
    inv_op = np.maximum(0.0, -np.log(np.maximum((f32(1) - alpha).astype(np.float64), 1e-10))).astype(f32)
    dens = (inv_op / norm).astype(f32)
    return dict(mean=mean.astype(f32), scale=sc, quat=quat, density=dens.reshape(-1, 1),
                features=sh48.astype(f32).reshape(-1, 16, 3))
