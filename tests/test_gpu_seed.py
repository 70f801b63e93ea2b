"""Learned congestion seed on the GPU (tcgen05 implicit-GEMM convolutions)
against the CPU oracle of the same network (oracle/seed_oracle.c).

Tolerances: the GPU rounds to BF16 at the points the oracle does and
accumulates in f32 (TMEM) where the oracle uses f64, so an activation or
gradient can round to the neighbouring BF16 value; the loss must agree to
1e-3 relative and every layer's weight and bias gradient to 3e-2 relative
(L2 norm of the difference over the norm of the oracle's gradient)."""
import numpy as np
import pytest

import instantgr_b200 as ig
from oracle_py import seed_grad, seed_slices

pytestmark = pytest.mark.gpu


def _tiles(T, S, seed):
    r = np.random.default_rng(seed)
    x = r.normal(0, 1, (T, S, S, 16)).astype(np.float32)
    x[..., 14:] = 0
    t = np.abs(r.normal(0, 1, (T, S, S, 16))).astype(np.float32)
    t[..., 10:] = 0
    return x, t


@pytest.mark.parametrize("S,halo,T", [(48, 8, 2), (64, 16, 1)])
def test_seed_gradients_match_cpu_oracle(S, halo, T):
    m = ig.Seed(3)
    m.set_tile(S, halo)
    p = m.params()
    x, t = _tiles(T, S, 5)
    loss_g, g_g = m.grad(x, t)
    loss_o, g_o = seed_grad(x, t, p, halo, rounded=True)
    assert abs(loss_g - loss_o) <= 1e-3 * loss_o, (loss_g, loss_o)
    for i, (ws, bs) in enumerate(seed_slices()):
        for sl, what in ((ws, "weights"), (bs, "bias")):
            a, b = g_g[sl], g_o[sl]
            err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
            assert err <= 3e-2, f"layer {i} {what}: relative error {err:.3g}"
    m.close()


def test_seed_training_learns_a_smooth_demand_map():
    """A target that is a fixed function of the features is learned: the mean
    squared error falls well below that of the untrained network and of the
    best constant prediction."""
    r = np.random.default_rng(7)
    m = ig.Seed(11)
    m.set_tile(64, 8)
    maps = []
    for _ in range(4):
        X = Y = 96
        f = np.zeros((X, Y, 16), np.float32)
        # smooth random fields as features
        for c in range(14):
            g = r.normal(0, 1, (X // 8 + 2, Y // 8 + 2))
            f[..., c] = np.kron(g, np.ones((8, 8)))[:X, :Y] * 0.5
        tg = np.zeros((X, Y, 16), np.float32)
        for l in range(1, 10):
            tg[..., l] = np.maximum(0, 0.6 * f[..., 1] + 0.4 * f[..., 2] - 0.3 * f[..., 4 + l]) + 0.2
        maps.append(m.add_map(f, tg))
        maps_np = tg
    before = np.mean([m.evaluate(i)["mse"] for i in maps])
    curve = m.train(300, tiles=4, lr=2e-3, seed=1)
    after = np.mean([m.evaluate(i)["mse"] for i in maps])
    const = float(np.var(maps_np[..., :10]))
    assert np.all(np.isfinite(curve))
    assert after < 0.2 * before, (before, after)
    assert after < 0.5 * const, (const, after)
    m.close()
