"""CPU restatement of the learned-proposal network -- test infrastructure.

The network has no counterpart in the reference (AVISM has no learned part);
this module is the checker for the library's GPU kernels: forward pass,
loss, backward pass and Adam step of the 12 -> 64 -> 64 -> 64 -> 2 ReLU MLP
with BF16 weights and FP32 accumulation, in float64 so that the GPU's FP32
sums can be compared with a tolerance.

Parameter vector (float32, NPARAM entries), the layout the C-ABI uses:
    mu[12], sigma[12]                 input normalisation
    W1[64][12], b1[64]                rows = output unit
    W2[64][64], b2[64]
    W3[64][64], b3[64]
    W4[2][64],  b4[2]
    slack[2]                          output margins (radius factor, width offset)
Forward (as the GPU): a0 = bf16((x - mu) / sigma); a_l = bf16(relu(W_l a_{l-1}
+ b_l)) for l = 1..3 with W_l rounded to bf16; y = W4 a3 + b4.
Loss: sum_j m_j (y_j - t_j)^2 / max(1, sum m).  Backward treats the bf16
roundings as identity (straight-through).
"""
from __future__ import annotations

import numpy as np

NF, H, NO = 12, 64, 2
SHAPES = [("mu", (NF,)), ("sigma", (NF,)), ("W1", (H, NF)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
          ("W3", (H, H)), ("b3", (H,)), ("W4", (NO, H)), ("b4", (NO,)), ("slack", (2,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
# parameters the optimiser updates (normalisation and slack are fixed)
TRAINABLE = ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = p[o:o + n].reshape(shp)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float32).ravel() for name, _ in SHAPES]).astype(np.float32)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def init_params(seed: int, mu=None, sigma=None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = {"mu": np.zeros(NF) if mu is None else mu, "sigma": np.ones(NF) if sigma is None else sigma,
         "slack": np.array([1.0, 0.0])}
    for l, (fo, fi) in enumerate([(H, NF), (H, H), (H, H), (NO, H)], start=1):
        d[f"W{l}"] = rng.standard_normal((fo, fi)) * np.sqrt(2.0 / fi)
        d[f"b{l}"] = np.zeros(fo)
    return pack(d)


def forward(p: np.ndarray, x: np.ndarray, keep=False, rounding=True):
    """Network outputs (n, 2).  rounding=False drops the bf16 roundings (for
    finite-difference checks of the backward pass)."""
    P = unpack(np.asarray(p, np.float64 if not rounding else np.float32))
    rnd = bf16 if rounding else (lambda a: a)
    a = rnd(((x.astype(np.float32) - P["mu"]) / P["sigma"]).astype(np.float32 if rounding else np.float64))
    a = np.asarray(a, np.float64)
    acts, zs = [a], []
    for l in (1, 2, 3):
        z = a @ np.asarray(rnd(P[f"W{l}"]), np.float64).T + P[f"b{l}"]
        zs.append(z)
        a = np.asarray(rnd(np.maximum(z, 0.0).astype(np.float32 if rounding else np.float64)), np.float64)
        acts.append(a)
    y = a @ np.asarray(rnd(P["W4"]), np.float64).T + P["b4"]
    return (y, acts, zs) if keep else y


def loss_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray, m: np.ndarray, rounding=True):
    """Loss and gradient (NPARAM, float64; zero for the fixed entries)."""
    P = unpack(np.asarray(p, np.float64 if not rounding else np.float32))
    rnd = bf16 if rounding else (lambda a: a)
    y, acts, zs = forward(p, x, keep=True, rounding=rounding)
    den = max(1.0, float(m.sum()))
    r = (y - t) * m
    loss = float((r * (y - t)).sum() / den)
    dy = 2.0 * r / den
    g = {name: np.zeros(shp) for name, shp in SHAPES}
    g["W4"] = dy.T @ acts[3]
    g["b4"] = dy.sum(0)
    da = dy @ np.asarray(rnd(P["W4"]), np.float64)
    for l in (3, 2, 1):
        dz = da * (zs[l - 1] > 0)
        g[f"W{l}"] = dz.T @ acts[l - 1]
        g[f"b{l}"] = dz.sum(0)
        da = dz @ np.asarray(rnd(P[f"W{l}"]), np.float64)
    return loss, np.concatenate([np.asarray(g[name], np.float64).ravel() for name, _ in SHAPES])


def adam_step(p, g, mstate, vstate, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the trainable entries (float64 state)."""
    mask = np.zeros(NPARAM, bool)
    o = 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        mask[o:o + n] = name in TRAINABLE
        o += n
    mstate = np.where(mask, b1 * mstate + (1 - b1) * g, mstate)
    vstate = np.where(mask, b2 * vstate + (1 - b2) * g * g, vstate)
    mh = mstate / (1 - b1 ** step)
    vh = vstate / (1 - b2 ** step)
    p = np.where(mask, p - lr * mh / (np.sqrt(vh) + eps), p).astype(np.float32)
    return p, mstate, vstate
