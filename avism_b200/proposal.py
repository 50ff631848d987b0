"""Learned proposal of the kNN search radius and the cube half-width: training
data from the method itself, training on the GPU, the committed weights.

No counterpart in the reference (AVISM has no learned part).  The network and
its kernels live in csrc/proposal.cu; this module drives them through the C-ABI:

  * ``make_samples`` runs the exact path on a particle set and returns, per
    sample, the 12 bin features and targets: log(r_K / bw) of the K-th
    neighbour distance of a query (random points and random particles) in the
    bin, and log(1 + w) of the half-width w of every accepted cube, at the bin
    of its centre;
  * ``train`` fits the network on the GPU (Adam, the library's own forward and
    backward kernels) and sets the radius slack so that most queries need no
    second radius attempt;
  * ``load_weights`` returns the committed parameters (proposal_weights.npy),
    trained on the two training workloads below by ``python -m
    avism_b200.proposal``.

Training workloads: the 64^3 periodic mock (2^18 particles, L = 100, eight
underdense spheres) and the 256^3 lognormal field (2^24 particles, L = 250,
P(k) ~ k^-1.5, sigma_ln = 1), both seeded.
"""
from __future__ import annotations

import json
import os

import numpy as np

from ._abi import Params

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "proposal_weights.npy")
META = os.path.join(HERE, "proposal_weights.json")
NF = 12


def load_weights(path: str = WEIGHTS) -> np.ndarray:
    p = np.load(path).astype(np.float32)
    if p.shape != (9308,):
        raise ValueError(f"{path}: expected 9308 parameters, got {p.shape}")
    return p


def _bins(x, nb, box):
    b = np.floor((x.astype(np.float64) + box / 2) * (nb / box)).astype(np.int64)
    return np.clip(b, 0, nb - 1)


def make_samples(gpu, p: Params, parts: dict, n_query: int = 200_000, seed: int = 0):
    """(features, targets, masks) of one particle set; targets / masks are (n, 2)."""
    rng = np.random.default_rng(seed)
    K = p.kneighbours
    box = p.lado0
    feat, nb, bw = gpu.proposal_features(p, parts)
    x, y, z = (np.asarray(parts[k], np.float32) for k in ("x", "y", "z"))
    n = len(x)
    # queries: uniform random points (the cells) and random particles
    nu = n_query // 2
    qu = rng.uniform(-box / 2, box / 2, (nu, 3)).astype(np.float32)
    pi = rng.integers(0, n, n_query - nu)
    qp = np.stack([x[pi], y[pi], z[pi]], 1)
    q = np.concatenate([qu, qp])
    _, dist = gpu.knn_search(x, y, z, q[:, 0].copy(), q[:, 1].copy(), q[:, 2].copy(), K,
                             box if p.periodic else 0.0)
    rk = dist[:, K - 1].astype(np.float64)
    rows = _bins(q[:, 0], nb, box) + nb * (_bins(q[:, 1], nb, box) + nb * _bins(q[:, 2], nb, box))
    fa = feat[rows]
    ta = np.zeros((len(q), 2), np.float32)
    ma = np.zeros((len(q), 2), np.float32)
    ta[:, 0] = np.log(np.maximum(rk, 1e-6) / bw)
    ma[:, 0] = 1.0
    # half-widths of the accepted cubes, at the bin of their centre
    r = gpu.run_level(Params(**{**p.__dict__, "learned": 0}), parts)
    cb = r["cubes"]
    from .avism import grid_setup
    g, _ = grid_setup(p)
    w = (np.asarray(cb["final_x"]) - np.asarray(cb["inicio_x"])) // 2
    cpos = [g.rx1 + (np.asarray(cb[k], np.float64) - 1) * g.dx for k in ("icx", "icy", "icz")]
    if p.periodic:
        cpos = [(c + box / 2) % box - box / 2 for c in cpos]
    crow = _bins(cpos[0], nb, box) + nb * (_bins(cpos[1], nb, box) + nb * _bins(cpos[2], nb, box))
    fb = feat[crow]
    tb = np.zeros((len(w), 2), np.float32)
    mb = np.zeros((len(w), 2), np.float32)
    tb[:, 1] = np.log1p(w)
    mb[:, 1] = 1.0
    return (np.concatenate([fa, fb]).astype(np.float32), np.concatenate([ta, tb]), np.concatenate([ma, mb]), bw)


def training_sets(gpu, small: bool = False):
    """Samples of the two training workloads (``small``: the mock only)."""
    from . import synth
    sets = []
    mock = synth.to_reader_units(synth.mock_spheres(seed=1001))
    sets.append(make_samples(gpu, Params(nx=64, periodic=1, lado0=100.0), mock, seed=1))
    if not small:
        ln = synth.to_reader_units(synth.lognormal(n=2 ** 24, ng=256, box=250.0, index=-1.5, sigma_ln=1.0,
                                                   vrms=350.0, seed=1002))
        sets.append(make_samples(gpu, Params(nx=256, periodic=1, lado0=250.0), ln, n_query=600_000, seed=2))
    f = np.concatenate([s[0] for s in sets])
    t = np.concatenate([s[1] for s in sets])
    m = np.concatenate([s[2] for s in sets])
    return f, t, m


def train(gpu, f, t, m, steps: int = 4000, batch: int = 4096, lr: float = 2e-3, seed: int = 0,
          quantile: float = 0.97):
    """Train the network on the GPU; returns (params, info)."""
    mu = f.mean(0)
    sg = f.std(0) + 1e-3
    rng = np.random.default_rng(seed)
    p0 = np.zeros(9308, np.float32)
    o = 0
    shapes = [("mu", (NF,)), ("sigma", (NF,)), ("W1", (64, NF)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
              ("W3", (64, 64)), ("b3", (64,)), ("W4", (2, 64)), ("b4", (2,)), ("slack", (2,))]
    init = {"mu": mu, "sigma": sg, "slack": np.array([1.0, 0.0])}
    for name, shp in shapes:
        k = int(np.prod(shp))
        if name in init:
            v = init[name]
        elif name.startswith("W"):
            v = rng.standard_normal(shp) * np.sqrt(2.0 / shp[1])
        else:
            v = np.zeros(shp)
        p0[o:o + k] = np.asarray(v, np.float32).ravel()
        o += k
    p1, curve = gpu.proposal_train(f, t, m, p0, steps=steps, batch=batch, lr=lr, seed=seed)
    y = gpu.proposal_infer(f, p1)
    r0 = (t[:, 0] - y[:, 0])[m[:, 0] > 0]
    r1 = (t[:, 1] - y[:, 1])[m[:, 1] > 0]
    slack0 = float(np.exp(np.quantile(r0, quantile)))
    p1[-2] = slack0
    p1[-1] = 0.0
    info = {"samples": int(len(f)), "steps": steps, "batch": batch, "lr": lr, "final_loss": float(curve[-1]),
            "radius_log_residual_std": float(np.std(r0)), "radius_slack": slack0,
            "width_log_residual_std": float(np.std(r1)) if len(r1) else None, "quantile": quantile}
    return p1, info


def main():
    from .avism import AvismGPU
    with AvismGPU(0) as gpu:
        f, t, m = training_sets(gpu)
        p, info = train(gpu, f, t, m)
    np.save(WEIGHTS, p)
    with open(META, "w") as fh:
        json.dump(info, fh, indent=1)
    print(json.dumps(info))


if __name__ == "__main__":
    main()
