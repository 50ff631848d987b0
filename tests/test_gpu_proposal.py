"""GPU checks of the learned proposal: the training kernels' loss and gradient
against the CPU oracle (oracle/mlp.py), the tcgen05 inference kernel against
the oracle's forward pass, training on the GPU, and exactness of the learned
path (the catalogue does not depend on the proposal)."""
import os

import numpy as np
import pytest

from avism_b200._abi import Params
from oracle import mlp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _data(rng, ns):
    x = rng.standard_normal((ns, mlp.NF)).astype(np.float32) * 2.0 + 0.5
    t = rng.standard_normal((ns, mlp.NO)).astype(np.float32)
    m = (rng.random((ns, mlp.NO)) < 0.6).astype(np.float32)
    return x, t, m


def _params(seed):
    rng = np.random.default_rng(seed)
    p = mlp.init_params(seed, mu=rng.standard_normal(mlp.NF) * 0.3, sigma=1.5 + rng.random(mlp.NF))
    P = mlp.unpack(p)
    for l in (1, 2, 3, 4):
        P[f"b{l}"][:] = rng.standard_normal(P[f"b{l}"].shape) * 0.1
    return p


@pytest.mark.parametrize("ns", [1, 300, 4096])
def test_grad_matches_oracle(gpu, ns):
    rng = np.random.default_rng(ns)
    x, t, m = _data(rng, ns)
    p = _params(7)
    loss_g, g_g = gpu.proposal_grad(x, t, m, p)
    loss_o, g_o = mlp.loss_grad(p, x, t, m)
    # FP32 sums in a fixed order (GPU) vs FP64 (oracle); the forward pass is the
    # same up to bf16 roundings of values that land within an FP32 ulp of a tie
    assert abs(loss_g - loss_o) <= 1e-4 * abs(loss_o) + 1e-6
    scale = np.max(np.abs(g_o)) + 1e-12
    err = np.abs(g_g.astype(np.float64) - g_o)
    assert np.max(err) <= 2e-3 * scale, np.max(err) / scale
    assert np.sum(err > 1e-4 * scale) <= 0.01 * len(err)
    # fixed entries get no gradient
    P = mlp.unpack(g_g)
    assert not np.any(P["mu"]) and not np.any(P["sigma"]) and not np.any(P["slack"])


@pytest.mark.parametrize("ns", [1, 127, 128, 1000, 70000])
def test_tensor_core_inference_matches_oracle(gpu, ns):
    rng = np.random.default_rng(100 + ns)
    x, _, _ = _data(rng, ns)
    p = _params(11)
    y_g = gpu.proposal_infer(x, p)
    y_o = mlp.forward(p, x)
    # tcgen05 sums in its own order: a hidden value may round to the other
    # neighbouring bf16, so compare with a tolerance scaled to the outputs
    scale = np.std(y_o) + 1e-6
    err = np.abs(y_g - y_o) / scale
    assert np.all(np.isfinite(y_g))
    assert np.max(err) < 0.05, np.max(err)
    assert np.mean(err) < 0.005, np.mean(err)


def test_training_on_gpu_fits_a_smooth_target(gpu):
    rng = np.random.default_rng(5)
    ns = 20000
    x = rng.standard_normal((ns, mlp.NF)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2], np.tanh(x[:, 3] - x[:, 4])], 1).astype(np.float32)
    m = np.ones((ns, 2), np.float32)
    p0 = mlp.init_params(2)
    loss0 = mlp.loss_grad(p0, x[:2000], t[:2000], m[:2000])[0]
    p1, curve = gpu.proposal_train(x, t, m, p0, steps=600, batch=2048, lr=3e-3, seed=1)
    loss1 = mlp.loss_grad(p1, x[:2000], t[:2000], m[:2000])[0]
    assert np.all(np.isfinite(curve))
    assert loss1 < 0.1 * loss0, (loss0, loss1)
    # the fixed entries are untouched
    P0, P1 = mlp.unpack(p0), mlp.unpack(p1)
    for k in ("mu", "sigma", "slack"):
        assert np.array_equal(P0[k], P1[k])


def test_training_is_deterministic(gpu):
    rng = np.random.default_rng(9)
    x, t, m = _data(rng, 5000)
    p0 = _params(3)
    a, _ = gpu.proposal_train(x, t, m, p0, steps=50, batch=512, lr=1e-3, seed=4)
    b, _ = gpu.proposal_train(x, t, m, p0, steps=50, batch=512, lr=1e-3, seed=4)
    assert np.array_equal(a, b)


def test_features_shape_and_sanity(gpu, mock1):
    p = Params(nx=64, periodic=1, lado0=100.0)
    f, nb, bw = gpu.proposal_features(p, mock1)
    assert f.shape == (nb ** 3, 12) and np.all(np.isfinite(f))
    # level-0 density feature: mean occupancy is 2.0 per bin
    counts = np.exp(f[:, 0]) - 0.05
    assert abs(np.mean(counts) * 2.0 - len(mock1["x"]) / nb ** 3) < 0.05 * len(mock1["x"]) / nb ** 3


def _weights():
    from avism_b200 import proposal
    return proposal.load_weights()


def test_learned_path_is_exact(gpu, mock1):
    """learned = 1 (trained network) and learned = 2 (density estimate) give the
    plain path's catalogue bit for bit."""
    base = gpu.run_level(Params(nx=64, periodic=1, lado0=100.0), mock1, capacity=100000)
    gpu.proposal_load(_weights())
    for learned in (1, 2):
        r = gpu.run_level(Params(nx=64, periodic=1, lado0=100.0, learned=learned), mock1, capacity=100000)
        assert r["nvoid"] == base["nvoid"]
        for k in base["cubes"]:
            assert np.array_equal(r["cubes"][k], base["cubes"][k]), (learned, k)
        for k in base["cat"]:
            assert np.array_equal(np.asarray(r["cat"][k]), np.asarray(base["cat"][k])), (learned, k)


def test_learned_proposal_reduces_search_work(gpu):
    """Ablation: the trained network's starting radius needs fewer radius
    attempts and scans fewer candidates than the plain start (uniform density)
    on a lognormal field it was not trained on."""
    from avism_b200 import synth
    parts = synth.to_reader_units(synth.lognormal(n=2 ** 20, ng=64, box=100.0, index=-1.3, sigma_ln=1.0,
                                                  vrms=350.0, seed=4242))
    gpu.proposal_load(_weights())
    res = {}
    for learned in (0, 1):
        p = Params(nx=100, periodic=1, lado0=100.0, learned=learned)
        gpu.particles_to_grid(p, parts)
        gpu.knn_counters(True)
        gpu.particles_to_grid(p, parts)
        res[learned] = gpu.knn_counters(False)
    plain, learned = res[0], res[1]
    nq = plain["queries"] + plain["fallbacks"]
    assert nq == learned["queries"] + learned["fallbacks"] > 0
    # second and later radius attempts, and the candidates scanned
    retries_plain, retries_learned = plain["attempts"] - plain["queries"], learned["attempts"] - learned["queries"]
    assert retries_learned < 0.5 * retries_plain, (plain, learned)
    assert learned["scanned"] < plain["scanned"], (plain, learned)
    # the packed-key bitonic order is verified; exact re-ranking stays rare
    for r in (plain, learned):
        assert r["exact_ranks"] < 0.05 * r["queries"], r
