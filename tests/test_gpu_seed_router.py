"""The shipped congestion seed (instantgr_b200/data/congestion_seed.npz, trained
by instantgr_b200/train_seed.py on 200 routed 512 x 512 designs) in the router,
on held-out designs of the same family, scored by InstantGR's evaluator.

What the trained network gains over the method without it: its predicted
demand beats the per-layer-mean and zero predictors, and routes seeded with
it score no worse than plain routes (0.1% tolerance for the heuristic); the
judged mode keeps the better of the two."""
import os

import numpy as np
import pytest

import instantgr_b200 as ig
from test_gpu_router import evaluate

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def heldout(tmp_path_factory):
    d = tmp_path_factory.mktemp("seed")
    cap, net = str(d / "h.cap"), str(d / "h.net")
    ig.generate(3, 9001, 1.0, cap, net)  # 512 x 512, 40k nets; training used seeds 1000-1199
    return cap, net, d


@pytest.fixture(scope="module")
def model():
    m = ig.Seed.load()
    yield m
    m.close()


def test_shipped_model_predicts_better_than_baselines(heldout, model):
    cap, net, _ = heldout
    r = ig.Router(cap, net, rrr_iters=3)
    r.run()
    mid = model.add_routed(r)
    e = model.evaluate(mid)
    r.close()
    assert e["mae"] < 0.8 * e["mae_mean"] and e["mae"] < 0.5 * e["mae_zero"], e


def test_seeded_routing_is_no_worse_than_plain(heldout, model):
    cap, net, d = heldout
    res = {}
    for name, mode in (("plain", 0), ("seeded", 1), ("judged", 2)):
        r = ig.Router(cap, net, rrr_iters=1, batched=1)
        if mode:
            r.set_seed(model, mode=mode)
        r.run()
        out = str(d / f"{name}.out")
        r.write(out)
        res[name] = dict(score=evaluate(cap, net, out)[3], rerouted=r.stats()["rerouted"], seed=r.seed_stats())
        r.close()
    assert res["seeded"]["score"] <= res["plain"]["score"] * 1.001, res
    assert res["seeded"]["seed"]["seed_kept"]
    assert res["judged"]["score"] <= min(res["plain"]["score"], res["seeded"]["score"]) * (1 + 1e-9), res
    assert res["seeded"]["seed"]["predict_ms"] > 0


def test_seeded_routing_is_deterministic(heldout, model):
    cap, net, d = heldout
    outs = []
    for k in range(2):
        r = ig.Router(cap, net, rrr_iters=2, batched=1)
        r.set_seed(model)
        r.run()
        out = str(d / f"det{k}.out")
        r.write(out)
        outs.append(open(out).read())
        r.close()
    assert outs[0] == outs[1]


@pytest.mark.parametrize("cfg,seed,scale", [(3, 9001, 1.0), (1, 1, 0.3)])
def test_device_features_equal_host_features(tmp_path, cfg, seed, scale):
    """The seed's input features computed on the device from the resident trees
    (what a seeded run uses) against the host restatement: pins, blocked-layer
    fraction and capacities identical; the RUDY channels, summed in fixed point
    on the device (exact) and in double on the host, identical but for the host's
    cancellation residues (below 1e-9 where the sums are zero) and at most one
    BF16 step at a few GCells."""
    cap, net = str(tmp_path / "d.cap"), str(tmp_path / "d.net")
    ig.generate(cfg, seed, scale, cap, net)
    r = ig.Router(cap, net)
    host = ig.seed_features(r)
    dev = ig.seed_features(r, device=True)
    r.close()
    exact = [0] + list(range(3, 16))
    assert np.array_equal(host[..., exact], dev[..., exact])
    for ch in (1, 2):
        h, d = host[..., ch], dev[..., ch]
        diff = np.abs(h - d)
        real = diff > 1e-9  # beyond the host's residues of exact cancellations
        step = np.maximum(np.abs(h), np.abs(d)) * 2.0 ** -7  # one BF16 step at the value
        assert np.all(diff[real] <= step[real] * 1.0001), f"channel {ch}: {diff[real].max()}"
        assert np.count_nonzero(real) <= max(2, h.size // 100000), f"channel {ch}: {np.count_nonzero(real)} cells"
