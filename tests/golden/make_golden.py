"""Generates the golden fixtures of tests/golden/ from InstantGR itself.

The reference kernels run through oracle/_ref/ref_harness (built by
`make -C oracle ref` from the unmodified reference sources; needs a GPU), the
reference reader and pin selection through oracle/_ref/ref_front (CPU), and
the whole reference router through oracle/_ref/instantgr_ref scored by
oracle/_ref/evaluator.  Inputs come from tests/cases.py with fixed seeds.

    python tests/golden/make_golden.py --out <dir> [--cpu-only]

Every fixture is an .npz holding the inputs and the reference's outputs.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)
import cases  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

COST_CASES = [
    dict(seed=1, X=40, Y=30, dir0=0),
    dict(seed=2, X=520, Y=12, dir0=1, unit_wire=0.3, unit_via=1.5),
    dict(seed=3, X=33, Y=600, dir0=0, edge_len=7, unit_via=3.5),
]
PATTERN_CASES = [dict(seed=11, X=40, Y=30, dir0=0, n=80), dict(seed=12, X=64, Y=50, dir0=1, n=120, uw=0.3)]
DAG_CASES = [dict(seed=21, X=48, Y=40, dir0=0, n=50), dict(seed=22, X=60, Y=60, dir0=1, n=60)]


def harness(mode: str, arrays, dtypes, tmp: str):
    fin, fout = os.path.join(tmp, mode + ".in"), os.path.join(tmp, mode + ".out")
    cases.write_harness_input(fin, arrays)
    subprocess.run([os.path.join(REF, "ref_harness"), mode, fin, fout], check=True, stdout=subprocess.DEVNULL)
    return cases.read_harness_output(fout, dtypes)


def ref_cost(g, tmp):
    return harness("cost", cases.grid_arrays(g), [np.float32, np.float32, np.float64], tmp)


def make_cost(out, tmp):
    for i, c in enumerate(COST_CASES):
        g = cases.grid_case(c["seed"], X=c["X"], Y=c["Y"], dir0=c["dir0"], unit_wire=c.get("unit_wire", 1.0),
                            unit_via=c.get("unit_via", 2.0), edge_len=c.get("edge_len", 1))
        w, v, p = ref_cost(g, tmp)
        np.savez_compressed(os.path.join(out, f"cost_{i}.npz"), **_grid(g), wcost=w, vcost=v, presum=p)


def _grid(g):
    return {k: np.asarray(v) for k, v in g.items()}


def make_pattern(out, tmp):
    for i, c in enumerate(PATTERN_CASES):
        g = cases.grid_case(c["seed"], X=c["X"], Y=c["Y"], dir0=c["dir0"], unit_wire=c.get("uw", 1.0))
        _, vc, ps = ref_cost(g, tmp)
        tb = cases.tree_batch(g, c["seed"] + 1, n=c["n"])
        stamp = 5
        arrs = cases.grid_arrays(g) + [vc, ps, np.array([stamp], np.int32), tb["node_off"], tb["nodes"], tb["par"],
                                      tb["pins"]]
        pre, routes, dem, st = harness("pattern", arrs, [np.int32, np.int32, np.float32, np.int32], tmp)
        np.savez_compressed(os.path.join(out, f"pattern_{i}.npz"), **_grid(g), vcost=vc, presum=ps, stamp=stamp,
                            **{k: v for k, v in tb.items()}, ref_pre=pre, ref_routes=routes, ref_demand=dem,
                            ref_stamps=st)
        # rip-up marking and congestion view on the committed state
        g2 = dict(g)
        g2["demand"] = dem
        of, xs, ys = harness("ripup", cases.grid_arrays(g2) + [tb["pins"], routes], [np.int32, np.float32,
                                                                                     np.float32], tmp)
        np.savez_compressed(os.path.join(out, f"ripup_{i}.npz"), **_grid(g2), pins=tb["pins"], routes=routes,
                            route_off=tb["route_off"], ref_of=of, ref_xsum=xs, ref_ysum=ys)


def make_dag(out, tmp):
    for i, c in enumerate(DAG_CASES):
        g = cases.grid_case(c["seed"], X=c["X"], Y=c["Y"], dir0=c["dir0"])
        _, vc, ps = ref_cost(g, tmp)
        d = cases.dag_batch(g, c["seed"] + 1, n=c["n"])
        stamp = 9
        arrs = cases.grid_arrays(g) + [vc, ps, np.array([stamp], np.int32), d["node_off"], d["nodes"], d["depth"],
                                      d["par_off"], d["par"], d["child_slot"], d["child_num"], d["pins"]]
        pre, routes, dem, st = harness("dag", arrs, [np.int32, np.int32, np.float32, np.int32], tmp)
        np.savez_compressed(os.path.join(out, f"dag_{i}.npz"), **_grid(g), vcost=vc, presum=ps, stamp=stamp,
                            **{k: v for k, v in d.items()}, ref_pre=pre, ref_routes=routes, ref_demand=dem,
                            ref_stamps=st)


def make_dagbuild(out, tmp):
    g = cases.grid_case(31, X=90, Y=80, dir0=0, load=2.0)
    rng = np.random.default_rng(31)
    tb = cases.tree_batch(g, 32, n=120, kmax=9)
    # congestion view of a loaded grid (exclusive prefix sums of max overflow)
    cap = g["cap"].reshape(g["L"], g["X"], g["Y"])
    dem = g["demand"].reshape(g["L"], g["X"], g["Y"]) * 2
    ov = np.maximum(dem - cap, 0).max(axis=0).astype(np.float32)
    xs = np.zeros_like(ov)
    ys = np.zeros_like(ov)
    xs[1:, :] = np.cumsum(ov[:-1, :], axis=0)
    ys[:, 1:] = np.cumsum(ov[:, :-1], axis=1)
    tree_off, pos, adj_off, adj = [0], [], [0], []
    for k in range(len(tb["node_off"]) - 1):
        a, b = tb["node_off"][k], tb["node_off"][k + 1]
        par = tb["par"][a:b]
        nb = [[] for _ in range(b - a)]
        for v in range(1, b - a):
            nb[v].append(int(par[v]))
            nb[int(par[v])].append(v)
        for v in range(b - a):
            rng.shuffle(nb[v])
            adj += nb[v]
            adj_off.append(len(adj))
        pos += tb["nodes"][a:b].tolist()
        tree_off.append(len(pos))
    arrs = [np.array([g["X"], g["Y"], 0], np.int32), xs.reshape(-1), ys.reshape(-1), np.array(tree_off, np.int32),
            np.array(pos, np.int32), np.array(adj_off, np.int32), np.array(adj, np.int32)]
    (res,) = harness("dagbuild", arrs, [np.int32], tmp)
    np.savez_compressed(os.path.join(out, "dagbuild.npz"), X=g["X"], Y=g["Y"], mode=0, xsum=xs.reshape(-1),
                        ysum=ys.reshape(-1), tree_off=np.array(tree_off, np.int32), pos=np.array(pos, np.int32),
                        adj_off=np.array(adj_off, np.int32), adj=np.array(adj, np.int32), ref=res)


def make_front(out, tmp):
    import instantgr_b200 as ig
    cap, net = os.path.join(out, "front.cap"), os.path.join(out, "front.net")
    ig.generate_custom(64, 64, 400, seed=5, cap_mode=0, block_frac=0.05, pin_mode=0, hifanout_frac=0.02,
                       bbox_median=8, bbox_sigma=1.0, cap=cap, net=net)
    subprocess.run([os.path.join(REF, "ref_front"), cap, net, os.path.join(out, "front_pins.txt")], check=True,
                   stdout=subprocess.DEVNULL)


def make_e2e(out, tmp):
    """Reference router on a small design: evaluator score and wall time."""
    import instantgr_b200 as ig
    res = {}
    for name, X, Y, n, seed in (("e2e_small", 96, 96, 3000, 41), ("e2e_mid", 256, 256, 20000, 42)):
        cap, net, guide = (os.path.join(tmp, name + s) for s in (".cap", ".net", ".out"))
        ig.generate_custom(X, Y, n, seed=seed, cap_mode=0, block_frac=0.05, pin_mode=0, bbox_median=8,
                           bbox_sigma=1.0, cap=cap, net=net)
        t0 = time.time()
        p = subprocess.run([os.path.join(REF, "instantgr_ref"), "-cap", cap, "-net", net, "-out", guide], cwd=tmp,
                           capture_output=True, text=True)
        wall = time.time() - t0
        if p.returncode != 0:
            res[name] = dict(error=p.stderr[-2000:])
            continue
        ev = subprocess.run([os.path.join(REF, "evaluator"), cap, net, guide], capture_output=True, text=True)
        stat = [l for l in ev.stdout.splitlines() if l.startswith("FOR_STAT")]
        res[name] = dict(X=X, Y=Y, nets=n, seed=seed, wall_s=wall, for_stat=stat[0] if stat else None,
                         stdout_tail=p.stdout[-1500:])
    with open(os.path.join(out, "e2e_reference.json"), "w") as f:
        json.dump(res, f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--cpu-only", action="store_true")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    steps = [("front", make_front)]
    if not a.cpu_only:
        steps += [("cost", make_cost), ("pattern", make_pattern), ("dag", make_dag), ("dagbuild", make_dagbuild),
                  ("e2e", make_e2e)]
    with tempfile.TemporaryDirectory() as tmp:
        for name, fn in steps:
            if a.only and name not in a.only.split(","):
                continue
            t0 = time.time()
            fn(a.out, tmp)
            print(f"{name}: {time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    main()
