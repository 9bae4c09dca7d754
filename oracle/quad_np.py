"""FP64 numpy restatement of the reference's quadrature oracle.

TEST INFRASTRUCTURE ONLY (checker for tests/ and the CPU baseline of bench.py).

Restates, for the query_ellipsoid kernel (the only one the reference's tests use):
  splinetracers/quad.py:54-61      query_ellipsoid: point inside ||R^T (x-mean)/max(s,1e-8)|| < 1
  splinetracers/quad.py:64-65      SH2RGB (DC only; the oracle reads features as (N,3))
  splinetracers/quad.py:91-117     2^16+1 linspace samples on [tmin, tmax] along x = rayo + t*rayd
  jaxutil/quadrature.py:46-88      alpha-compositing weights, colour = sum w * clip(sum sigma c / sum sigma, 0)
  jaxutil/quadrature.py:30-43      distortion loss, here in its O(n) sorted prefix form
  jaxutil/safe_math.py:130-157     safe_div returns 0 where |d| < float32 tiny
  utils/math_util.py:79-100        jquatToMat3 (note the transpose)
JAX is not installed, so this is numpy. One ray per call, as quad.py reshapes rayo to (1,3).
"""
from __future__ import annotations

import numpy as np

TINY32 = np.float64(np.finfo(np.float32).tiny)
MAX32 = np.float64(np.finfo(np.float32).max)


def quat_to_mat3(q):
    """jquatToMat3 (utils/math_util.py:79-100): the listed 3x3 transposed."""
    r, x, y, z = q
    m = np.array([
        1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - r * z), 2.0 * (x * z + r * y),
        2.0 * (x * y + r * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - r * x),
        2.0 * (x * z - r * y), 2.0 * (y * z + r * x), 1.0 - 2.0 * (x * x + y * y),
    ]).reshape(3, 3)
    return m.T


def sh2rgb(f):
    return 0.28209479177387814 * f + 0.5


def _safe_div(n, d):
    r = np.clip(n / np.where(np.abs(d) < TINY32, TINY32, d), -MAX32, MAX32)
    return np.where(np.abs(d) < TINY32, 0.0, r)


def _log1mexp(x):
    # jaxutil/quadrature.py:46-49: safe_log(1 - exp(-x)) with x clipped into [tiny, max]
    v = 1.0 - np.exp(-x)
    return np.log(np.clip(v, TINY32, MAX32))


def distortion_prefix(tdist, w):
    """lossfun_distortion (jaxutil/quadrature.py:30-43) without the n x n matrix.

    sum_ij w_i w_j |u_i - u_j| = 2 sum_i w_i (u_i W_<i - S_<i) for ascending u, plus
    the intra term sum w_i^2 dt_i / 3.
    """
    u = 0.5 * (tdist[1:] + tdist[:-1])
    W = np.concatenate([[0.0], np.cumsum(w)[:-1]])
    S = np.concatenate([[0.0], np.cumsum(w * u)[:-1]])
    inter = 2.0 * np.sum(w * (u * W - S))
    intra = np.sum(w ** 2 * np.diff(tdist)) / 3.0
    return inter + intra


def trace_ray(mean, scale, quat, density, features, rayo, rayd, tmin=0.0, tmax=1000.0,
              num_quad=2 ** 16):
    """Returns (5,) = [R, G, B, alpha, distortion] for one ray."""
    mean = np.asarray(mean, np.float64).reshape(-1, 3)
    scale = np.asarray(scale, np.float64).reshape(-1, 3)
    quat = np.asarray(quat, np.float64).reshape(-1, 4)
    density = np.asarray(density, np.float64).reshape(-1)
    feats = sh2rgb(np.asarray(features, np.float64).reshape(mean.shape[0], -1, 3)[:, 0, :])
    rayo = np.asarray(rayo, np.float64).reshape(3)
    rayd = np.asarray(rayd, np.float64).reshape(3)
    tdist = np.linspace(tmin, tmax, num_quad + 1)
    t_avg = 0.5 * (tdist[1:] + tdist[:-1])
    t_delta = np.diff(tdist)
    xs = rayo[None, :] + t_avg[:, None] * rayd[None, :]
    tot_d = np.zeros_like(t_avg)
    tot_c = np.zeros((t_avg.size, 3))
    for p in range(mean.shape[0]):
        q = quat[p] / np.sqrt(np.sum(quat[p] ** 2))
        R = quat_to_mat3(q)
        sc = ((xs - mean[p][None]) @ R.T) / np.maximum(scale[p][None], 1e-8)
        inside = np.linalg.norm(sc, axis=-1) < 1
        tot_d += np.where(inside, density[p], 0.0)
        tot_c += np.where(inside[:, None], density[p] * feats[p][None], 0.0)
    avg_c = np.clip(_safe_div(tot_c, tot_d[:, None]), 0, None)
    dd = tot_d * t_delta
    log_trans = -np.concatenate([[0.0], np.cumsum(dd[:-1])])
    w = np.exp(_log1mexp(dd) + log_trans)
    rgb = (w[:, None] * avg_c).sum(0)
    alpha = w.sum()
    return np.array([rgb[0], rgb[1], rgb[2], alpha, distortion_prefix(tdist, w)])


def trace_rays(mean, scale, quat, density, features, rayo, rayd, tmin=0.0, tmax=1000.0,
               num_quad=2 ** 16, nthreads=1):
    """(R, 5) for R rays; nthreads > 1 traces rays on that many threads (numpy releases the
    GIL inside its array loops, which hold nearly all of the work)."""
    rayo = np.asarray(rayo, np.float64).reshape(-1, 3)
    rayd = np.asarray(rayd, np.float64).reshape(-1, 3)
    one = lambda i: trace_ray(mean, scale, quat, density, features, rayo[i], rayd[i], tmin, tmax, num_quad)
    if nthreads <= 1 or rayo.shape[0] <= 1:
        rows = [one(i) for i in range(rayo.shape[0])]
    else:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=int(nthreads)) as ex:
            rows = list(ex.map(one, range(rayo.shape[0])))
    return np.stack(rows) if rows else np.zeros((0, 5))
