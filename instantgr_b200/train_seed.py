"""Trains the learned congestion seed on demand maps of the plain router.

    python -m instantgr_b200.train_seed [--designs 200] [--steps 2000] [--out instantgr_b200/data/congestion_seed.npz]

Training data: seeded synthetic 512 x 512, 40k-net designs (`igr_generate`
configuration 3: the pin-count mixture, bounding boxes and hotspots of the
800k-net configuration), each routed by the plain router (phase 1 and
rip-up-and-reroute); features and the routed demand of every design are kept
in device memory.  Held-out designs (other seeds) measure the mean absolute
error of the predicted demand against two baselines: predicting zero and
predicting the mean demand of each layer.  The parameters and the report are
written to `--out` (numpy .npz).
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

import instantgr_b200 as ig

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "congestion_seed.npz")


def routed_maps(seeds, workdir, rrr_iters, seed_model=None):
    """Generates, routes and adds each design to the model's training maps; yields (seed, map id, router stats)."""
    for s in seeds:
        cap, net = os.path.join(workdir, f"d{s}.cap"), os.path.join(workdir, f"d{s}.net")
        ig.generate(3, s, 1.0, cap, net)
        r = ig.Router(cap, net, rrr_iters=rrr_iters)
        r.run()
        mid = seed_model.add_routed(r) if seed_model is not None else -1
        st = r.stats()
        r.close()
        os.remove(cap)
        os.remove(net)
        yield s, mid, st


def map_errors(model: ig.Seed, mids):
    """MSE and MAE of the model and the MAE of the zero and per-layer-mean baselines
    (demand in units of 8 tracks), averaged over maps."""
    e = [model.evaluate(m) for m in mids]
    return {k: float(np.mean([x[k] for x in e])) for k in e[0]}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--designs", type=int, default=200)
    ap.add_argument("--heldout", type=int, default=8)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--tiles", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--rrr-iters", type=int, default=3)
    ap.add_argument("--init-seed", type=int, default=1)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--workdir", default=None)
    args = ap.parse_args(argv)
    t0 = time.time()
    model = ig.Seed(args.init_seed)
    work = args.workdir or tempfile.mkdtemp(prefix="igr_seed_")
    os.makedirs(work, exist_ok=True)
    train_ids, held_ids = [], []
    for _, mid, _ in routed_maps(range(1000, 1000 + args.designs), work, args.rrr_iters, model):
        train_ids.append(mid)
    for _, mid, _ in routed_maps(range(5000, 5000 + args.heldout), work, args.rrr_iters, model):
        held_ids.append(mid)
    t_data = time.time() - t0
    before = map_errors(model, held_ids)
    # training draws tiles from the training maps only: they come first in the pool
    curve = []
    t1 = time.time()
    schedule = [(args.lr, args.steps // 2), (args.lr / 3, args.steps // 4), (args.lr / 10, args.steps - 3 * (args.steps // 4))]
    held = set(held_ids)
    assert all(m < min(held) for m in train_ids)
    for i, (lr, n) in enumerate(schedule):
        curve += list(model.train(n, args.tiles, lr, seed=10 + i, maps=len(train_ids)))
    t_train = time.time() - t1
    after = map_errors(model, held_ids)
    train_err = map_errors(model, train_ids[:8])
    report = dict(designs=args.designs, heldout=args.heldout, steps=args.steps, tiles=args.tiles, lr=args.lr,
                  rrr_iters=args.rrr_iters, data_seconds=round(t_data, 1), train_seconds=round(t_train, 1),
                  heldout_before=before, heldout_after=after, train_after=train_err,
                  loss_first=float(np.mean(curve[:20])), loss_last=float(np.mean(curve[-20:])))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez(args.out, params=model.params(), report=json.dumps(report))
    print(json.dumps(report), flush=True)
    model.close()


if __name__ == "__main__":
    main()
