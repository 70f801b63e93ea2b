"""CPU oracle of the learned congestion seed (oracle/seed_oracle.c), pinned by
finite differences: the network has no counterpart in InstantGR, so its
gradients are checked against the derivative of its own exact (f64, no BF16
rounding) loss."""
import numpy as np

from oracle_py import seed_grad, seed_slices


def _case(S=8, halo=2, T=1, seed=0):
    r = np.random.default_rng(seed)
    x = r.normal(0, 1, (T, S, S, 16)).astype(np.float32)
    x[..., 14:] = 0
    t = r.normal(0, 1, (T, S, S, 16)).astype(np.float32)
    p = []
    for (ci, co), (ws, bs) in zip([(16, 32), (32, 64), (64, 64), (64, 64), (64, 32), (32, 16)], seed_slices()):
        p.append(r.normal(0, np.sqrt(2.0 / (9 * ci)), ws.stop - ws.start))
        p.append(r.normal(0, 0.1, bs.stop - bs.start))
    return x, t, np.concatenate(p).astype(np.float32), halo


def test_seed_oracle_gradient_matches_finite_differences():
    x, t, p, halo = _case()
    loss, g = seed_grad(x, t, p, halo, rounded=False)
    assert loss > 0
    r = np.random.default_rng(1)
    h = 1e-4  # small against the distance of most pre-activations from the ReLU kink
    checked = 0
    for ws, bs in seed_slices():
        for sl in (ws, bs):
            for i in r.choice(np.arange(sl.start, sl.stop), 4, replace=False):
                q = p.copy()
                q[i] += h
                lp, _ = seed_grad(x, t, q, halo, rounded=False)
                q[i] -= 2 * h
                lm, _ = seed_grad(x, t, q, halo, rounded=False)
                fd = (lp - lm) / (2 * h)
                assert abs(fd - g[i]) <= 1e-2 * max(1e-3, abs(fd)) + 1e-6, (i, fd, g[i])
                checked += 1
    assert checked == 48


def test_seed_oracle_rounding_is_close_to_exact():
    x, t, p, halo = _case(S=12, halo=2, seed=3)
    l0, g0 = seed_grad(x, t, p, halo, rounded=False)
    l1, g1 = seed_grad(x, t, p, halo, rounded=True)
    assert abs(l1 - l0) <= 2e-2 * l0
    assert np.linalg.norm(g1 - g0) <= 5e-2 * np.linalg.norm(g0)
