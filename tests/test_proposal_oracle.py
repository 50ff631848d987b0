"""CPU checks of the learned-proposal oracle (oracle/mlp.py): its backward
pass against finite differences, the bf16 rounding, and the parameter layout
the C-ABI declares."""
import os
import re

import numpy as np

from oracle import mlp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_nparam_matches_header():
    text = open(os.path.join(ROOT, "include", "avism_gpu.h")).read()
    n = int(re.search(r"#define AVISM_PROPOSAL_NPARAM (\d+)", text).group(1))
    assert n == mlp.NPARAM == 9308


def test_bf16_rounding_nearest_even():
    a = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159, 65504.0, 1e-40], np.float32)
    r = mlp.bf16(a)
    # bf16 keeps 8 significant bits: results are representable and within half an ulp
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)
    normal = np.abs(a) >= np.finfo(np.float32).tiny
    ulp = 2.0 ** (np.floor(np.log2(np.abs(a[normal]))) - 7)
    assert np.all(np.abs(r[normal] - a[normal]) <= ulp / 2)
    assert r[1] == 1.0            # 1 + 2^-8 is the tie between 1 and 1 + 2^-7: to even
    assert r[2] == np.float32(1.0078125)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    ns = 64
    x = rng.standard_normal((ns, mlp.NF)).astype(np.float32)
    t = rng.standard_normal((ns, mlp.NO))
    m = (rng.random((ns, mlp.NO)) < 0.7).astype(np.float64)
    p = mlp.init_params(5).astype(np.float64)
    P = mlp.unpack(p)
    for l in (1, 2, 3):
        P[f"b{l}"][:] = 0.1          # keep units away from the ReLU kink
    loss, g = mlp.loss_grad(p, x, t, m, rounding=False)
    o = 0
    offs = {}
    for name, shp in mlp.SHAPES:
        offs[name] = o
        o += int(np.prod(shp))
    picks = [offs["W1"] + 5, offs["b1"] + 3, offs["W2"] + 700, offs["b3"] + 10, offs["W4"] + 65, offs["b4"] + 1]
    for i in picks:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.loss_grad(pp, x, t, m, rounding=False)[0] - mlp.loss_grad(pm, x, t, m, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd), (i, fd, g[i])


def test_adam_moves_only_trainable_entries():
    p = mlp.init_params(1)
    g = np.ones(mlp.NPARAM)
    q, _, _ = mlp.adam_step(p, g, np.zeros(mlp.NPARAM), np.zeros(mlp.NPARAM), 1, 1e-2)
    P, Q = mlp.unpack(p), mlp.unpack(q)
    for name in ("mu", "sigma", "slack"):
        assert np.array_equal(P[name], Q[name])
    for name in mlp.TRAINABLE:
        assert not np.array_equal(P[name], Q[name])
