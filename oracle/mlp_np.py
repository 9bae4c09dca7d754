"""CPU oracle of the ray-cost MLP (test infrastructure only: imported by tests/, smoke()
and bench.py's CPU baseline, never by the product path).

The network has no counterpart in the reference. Its specification is the GPU kernel's:
- input: 39 features of the point of the ray's line closest to the scene centre, zero-padded
  to 64 columns (the kernel reads 48; columns 39.. are zero), rounded to bf16;
- layers: z1 = A0 W1^T + bf16(b1), A1 = bf16(relu(z1)); z2 = A1 W2^T + bf16(b2),
  A2 = bf16(relu(z2)); y = A2 W3^T + b3 (outputs 0 and 1 of 16);
- weights are the bf16 roundings of the fp32 parameters. The hidden layers' biases enter the
  tensor-core products as bf16 weights against a constant-1 input column, so they are
  summed with the products (in fp64 here) before the one rounding to fp32; the output bias
  is added in fp32 after it;
- loss: mean over the batch of w0 (y0 - t0)^2 + w1 (y1 - t1)^2;
- backward: G3 = bf16(dL/dy); dA2 = G3 W3, masked by A2 > 0, G2 = bf16(.); dA1 = G2 W2,
  masked by A1 > 0, G1 = bf16(.). Weight gradients are G^T A from the bf16 operands; the
  hidden layers' bias gradients are batch sums of the same bf16 G1, G2 (the kernel forms
  them as G^T 1 on the tensor cores), the output bias gradient the sum of the fp32 dL/dy.
Parameter block layout (fp32): W1 [64x64], W2 [64x64], W3 [16x64], b1 [64], b2 [64], b3 [16].
"""
from __future__ import annotations

import numpy as np

OFF_W1, OFF_W2, OFF_W3, OFF_B1, OFF_B2, OFF_B3, NPARAMS = 0, 4096, 8192, 9216, 9280, 9344, 9360
IN, HID, OUT, FEAT = 64, 64, 16, 39


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(x.shape)


def unpack(params, dtype=np.float32):
    p = np.asarray(params, dtype=dtype)
    return dict(w1=p[OFF_W1:OFF_W2].reshape(HID, IN), w2=p[OFF_W2:OFF_W3].reshape(HID, HID),
                w3=p[OFF_W3:OFF_B1].reshape(OUT, HID), b1=p[OFF_B1:OFF_B2], b2=p[OFF_B2:OFF_B3], b3=p[OFF_B3:])


def pack(w1, w2, w3, b1, b2, b3):
    return np.concatenate([np.ravel(a).astype(np.float32) for a in (w1, w2, w3, b1, b2, b3)])


def encode(rayo, rayd, centre=(0.0, 0.0, 0.0), inv_scale=1.0):
    """(R, 64) float32 encoding, following the kernel's fp32 operation order."""
    f32 = np.float32
    o = np.asarray(rayo, f32) - np.asarray(centre, f32)
    d = np.asarray(rayd, f32)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        n = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        inv = np.where(n > 0, f32(1) / np.where(n > 0, n, f32(1)), f32(0)).astype(f32)
        dn = d * inv[:, None]
        od = (o[:, 0] * dn[:, 0] + o[:, 1] * dn[:, 1]) + o[:, 2] * dn[:, 2]
        x = (o - od[:, None] * dn) * f32(inv_scale)
    x = np.where(np.isfinite(x), x, f32(0)).astype(f32)
    cols = [x[:, i] for i in range(3)]
    for q in range(6):
        s = f32(1 << q)
        arg = (s * x).astype(np.float64)
        cols += [np.sin(np.pi * arg[:, i]).astype(f32) for i in range(3)]
        cols += [np.cos(np.pi * arg[:, i]).astype(f32) for i in range(3)]
    feat = np.zeros((x.shape[0], IN), f32)  # columns FEAT.. stay zero
    feat[:, :FEAT] = np.stack(cols, 1)
    return feat


def _ops(rounding):
    """(round, to_acc) for the kernel's precision (bf16 operands, fp32 sums) or plain fp64."""
    if rounding:
        return bf16, (lambda x: np.asarray(x, np.float64).astype(np.float32))
    ident = lambda x: np.asarray(x, np.float64)
    return ident, ident


def forward(params, feat, rounding=True):
    rnd, acc = _ops(rounding)
    P = unpack(params, np.float32 if rounding else np.float64)
    w1, w2, w3 = rnd(P["w1"]), rnd(P["w2"]), rnd(P["w3"])
    d = np.float64
    feat = np.array(feat, copy=True)
    feat[:, FEAT:] = 0  # the kernel reads the 39 features only
    a0 = rnd(feat)
    a1 = rnd(np.maximum(acc(a0.astype(d) @ w1.astype(d).T + rnd(P["b1"]).astype(d)), 0))
    a2 = rnd(np.maximum(acc(a1.astype(d) @ w2.astype(d).T + rnd(P["b2"]).astype(d)), 0))
    y = acc(a2.astype(d) @ w3.astype(d).T) + P["b3"]
    return dict(a0=a0, a1=a1, a2=a2, y=y[:, :2], w1=w1, w2=w2, w3=w3)


def predict(params, feat):
    return forward(params, feat)["y"]


def loss_of(params, feat, target, w0=1.0, w1=1.0, rounding=True):
    e = forward(params, feat, rounding)["y"].astype(np.float64) - np.asarray(target, np.float64)
    return float(np.mean(w0 * e[:, 0] ** 2 + w1 * e[:, 1] ** 2))


def gradients(params, feat, target, w0=1.0, w1=1.0, rounding=True):
    """(grads [NPARAMS] float64, loss) of the mean weighted squared error. rounding=False
    gives the plain fp64 gradient of the same network (for finite-difference checks)."""
    rnd, acc = _ops(rounding)
    ft = np.float32 if rounding else np.float64
    F = forward(params, feat, rounding)
    B = feat.shape[0]
    inv_b = ft(1.0) / ft(B)
    e = (F["y"] - np.asarray(target, ft)).astype(ft)
    g = np.zeros((B, OUT), ft)
    g[:, 0] = ((ft(2) * ft(w0)) * e[:, 0]) * inv_b
    g[:, 1] = ((ft(2) * ft(w1)) * e[:, 1]) * inv_b
    loss = float(np.sum(w0 * e[:, 0].astype(np.float64) ** 2 + w1 * e[:, 1].astype(np.float64) ** 2) / B)
    d = np.float64
    G3 = rnd(g)
    g2 = np.where(F["a2"] > 0, acc(G3.astype(d) @ F["w3"].astype(d)), ft(0))
    G2 = rnd(g2)
    g1 = np.where(F["a1"] > 0, acc(G2.astype(d) @ F["w2"].astype(d)), ft(0))
    G1 = rnd(g1)
    gw1 = G1.astype(d).T @ F["a0"].astype(d)
    gw2 = G2.astype(d).T @ F["a1"].astype(d)
    gw3 = G3.astype(d).T @ F["a2"].astype(d)
    grads = np.concatenate([gw1.ravel(), gw2.ravel(), gw3.ravel(), G1.astype(d).sum(0), G2.astype(d).sum(0),
                            g.astype(d).sum(0)])
    return grads, loss


def init_params(seed=0):
    """He-uniform hidden layers, small output layer, zero biases; padding stays zero."""
    rng = np.random.default_rng(seed)
    w1 = np.zeros((HID, IN), np.float32)
    w1[:, :FEAT] = rng.uniform(-1, 1, (HID, FEAT)) * np.sqrt(6.0 / FEAT)
    w2 = (rng.uniform(-1, 1, (HID, HID)) * np.sqrt(6.0 / HID)).astype(np.float32)
    w3 = np.zeros((OUT, HID), np.float32)
    w3[:2] = rng.uniform(-1, 1, (2, HID)) * np.sqrt(3.0 / HID)
    return pack(w1, w2, w3, np.zeros(HID), np.zeros(HID), np.zeros(OUT))
