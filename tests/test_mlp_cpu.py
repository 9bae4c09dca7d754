"""CPU checks of the ray-cost MLP oracle (oracle/mlp_np.py) and of the cost-model ABI's host
validation. No GPU calls."""
import ctypes

import numpy as np
import pytest

from ever_b200 import _native as N
from ever_b200 import scheduler as SCH
from oracle import mlp_np as M


def _problem(n=40, seed=0):
    rng = np.random.default_rng(seed)
    p = M.init_params(seed + 1).astype(np.float64)
    p[M.OFF_B1:] += rng.normal(0, 0.1, M.NPARAMS - M.OFF_B1)
    p[M.OFF_W3 + 2 * 64:M.OFF_B1] = 0.0
    ro = rng.normal(0, 2, (n, 3)).astype(np.float32)
    rd = rng.normal(0, 1, (n, 3)).astype(np.float32)
    feat = M.encode(ro, rd, inv_scale=0.5).astype(np.float64)
    t = rng.normal(0, 1, (n, 2))
    return p, feat, t


def test_oracle_backward_matches_central_differences():
    p, feat, t = _problem()
    g, _ = M.gradients(p, feat, t, 1.0, 0.25, rounding=False)
    idx = list(range(0, M.NPARAMS, 89)) + [M.OFF_B1 + 3, M.OFF_B2 + 5, M.OFF_B3, M.OFF_B3 + 1, M.OFF_W3 + 64 + 9]
    h = 1e-6
    for i in idx:
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        fd = (M.loss_of(a, feat, t, 1.0, 0.25, False) - M.loss_of(b, feat, t, 1.0, 0.25, False)) / (2 * h)
        assert abs(fd - g[i]) < 1e-7 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding_known_answers():
    x = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, 1 + 2 ** -7 + 2 ** -9, -2.5, 0.0], np.float32)
    want = np.array([1.0, 1.0, 1 + 2 ** -6, 1 + 2 ** -7, -2.5, 0.0], np.float32)
    np.testing.assert_array_equal(M.bf16(x), want)  # ties go to even
    import torch
    y = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * 10.0 ** np.arange(-5, 5).repeat(1000)
    np.testing.assert_array_equal(M.bf16(y), torch.from_numpy(y).to(torch.bfloat16).float().numpy())


def test_bf16_rounding_of_oracle_is_the_only_difference_from_fp64():
    p, feat, t = _problem(200, 3)
    g64, _ = M.gradients(p, feat, t, rounding=False)
    g16, _ = M.gradients(p.astype(np.float32), feat.astype(np.float32), t.astype(np.float32))
    rel = np.abs(g16 - g64).max() / np.abs(g64).max()
    assert 1e-4 < rel < 5e-2  # bf16 has 8 significant bits


def test_encoding_is_the_closest_point_of_the_line():
    rng = np.random.default_rng(5)
    ro = rng.normal(0, 3, (100, 3)).astype(np.float32)
    rd = rng.normal(0, 1, (100, 3)).astype(np.float32)
    c = np.array([0.5, -0.25, 1.0])
    f = M.encode(ro, rd, c, 0.5)
    p = f[:, :3] / 0.5 + c
    d = rd / np.linalg.norm(rd, axis=1, keepdims=True)
    # p - o is parallel to d and p - c is orthogonal to d
    assert np.abs(np.cross(p - ro, d)).max() < 1e-4
    assert np.abs(np.sum((p - c) * d, 1)).max() < 1e-4
    np.testing.assert_allclose(f[:, 3:6], np.sin(np.pi * f[:, :3]), atol=1e-6)
    np.testing.assert_allclose(f[:, 6:9], np.cos(np.pi * f[:, :3]), atol=1e-6)
    np.testing.assert_allclose(f[:, 36:39], np.cos(32 * np.pi * f[:, :3]), atol=1e-4)
    assert np.all(f[:, 39:] == 0)


def test_product_init_matches_the_layout():
    p = SCH.init_params(0)
    assert p.shape == (N.MLP_PARAMS,) == (M.NPARAMS,)
    w1 = p[M.OFF_W1:M.OFF_W2].reshape(64, 64)
    w3 = p[M.OFF_W3:M.OFF_B1].reshape(16, 64)
    assert np.all(w1[:, 39:] == 0) and np.all(w3[2:] == 0) and np.all(p[M.OFF_B1:] == 0)


def test_cost_model_abi_host_validation():
    lib = N.load()
    assert lib.ever_mlp_workspace_bytes() == 160 * (N.MLP_PARAMS + 1) * 4
    m = N.EverMlp()
    assert lib.ever_mlp_pack(ctypes.byref(m), None) == 1
    assert b"null" in lib.ever_last_error()
    assert lib.ever_mlp_predict(None, None, None, None, 10, None, None, None, None, None) == 1
    m.params = m.w1 = m.w2 = m.w3 = 16  # dummy non-null pointers: only host checks run below
    assert lib.ever_mlp_predict(ctypes.byref(m), None, None, None, 10, None, None, None, None, None) == 1
    assert lib.ever_mlp_predict(ctypes.byref(m), None, None, None, -1, None, None, None, None, None) == 1
    assert lib.ever_mlp_gradients(ctypes.byref(m), None, None, None, None, 0, None, 1.0, 1.0, None, None, None, 0,
                                  None, None) == 1
    assert b"num_samples" in lib.ever_last_error()
    assert lib.ever_mlp_gradients(ctypes.byref(m), 16, 16, None, None, 8, 16, 1.0, 1.0, 16, None, 16, 10, 16,
                                  None) == 3  # EVER_ERR_WORKSPACE
    assert lib.ever_mlp_adam(ctypes.byref(m), 16, 16, 16, 1e-3, 0.9, 0.999, 1e-8, 0, None) == 1
    assert b"step" in lib.ever_last_error()
    assert lib.ever_ray_order_binned(16, 16, None, 10, None, 0, 16, None) == 1
    assert lib.ever_batch_order_binned(None, None, None, None, None) == 1
