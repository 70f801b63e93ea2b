"""Detour DAGs built on the device (igr_build_dags) against the reference's
golden DAGs and against the host builder (igr_build_dag, itself pinned to the
same golden vectors) on seeded trees and congestion views: bit-exact records.
The router-level test routes with the device DAGs and with the host DAGs and
compares the written guides byte for byte."""
import os

import numpy as np
import pytest

import instantgr_b200 as ig
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_device_dags_match_reference_golden():
    f = np.load(os.path.join(GOLDEN, "dagbuild.npz"))
    X, Y, mode = int(f["X"]), int(f["Y"]), int(f["mode"])
    recs, off = ig.build_dags(X, Y, mode, f["tree_off"], f["pos"], f["adj_off"], f["adj"], f["xsum"], f["ysum"])
    assert np.array_equal(recs, f["ref"])
    assert off[-1] == f["ref"].size


def _trees(rng, X, Y, n, max_pins):
    """Seeded Steiner trees in the router's layout: pins on layers 0..8 first,
    Steiner nodes on layer 9, adjacency appended per edge in edge order."""
    tree_off, pos, adj_off, adj = [0], [], [0], []
    for _ in range(n):
        k = int(rng.integers(2, max_pins + 1))
        span = int(rng.choice([8, 40, 200, 600]))
        x0, y0 = int(rng.integers(0, X)), int(rng.integers(0, Y))
        xs = np.clip(x0 + rng.integers(-span, span + 1, k), 0, X - 1)
        ys = np.clip(y0 + rng.integers(-span, span + 1, k), 0, Y - 1)
        nx, ny, ed = ig.steiner(xs, ys)
        m = len(nx)
        if m < 2:
            continue
        npins = len({(int(a), int(b)) for a, b in zip(xs, ys)})
        lay = [int(rng.integers(0, 9)) if v < npins else 9 for v in range(m)]
        nb = [[] for _ in range(m)]
        for a, b in ed:
            nb[a].append(int(b))
            nb[b].append(int(a))
        for v in range(m):
            pos.append(lay[v] * X * Y + int(nx[v]) * Y + int(ny[v]))
            adj.extend(nb[v])
            adj_off.append(len(adj))
        tree_off.append(len(pos))
    return (np.array(tree_off, np.int32), np.array(pos, np.int32), np.array(adj_off, np.int32),
            np.array(adj, np.int32))


def _view(rng, X, Y, density):
    """Prefix sums of a sparse non-negative overflow map along x and along y."""
    ofx = np.where(rng.random((X, Y)) < density, rng.random((X, Y)) * 3, 0).astype(np.float32)
    ofy = np.where(rng.random((X, Y)) < density, rng.random((X, Y)) * 3, 0).astype(np.float32)
    xsum = np.cumsum(ofx, axis=0, dtype=np.float32)
    ysum = np.cumsum(ofy, axis=1, dtype=np.float32)
    return xsum.ravel(), ysum.ravel()


@pytest.mark.parametrize("mode,seed,max_pins,density", [(0, 1, 6, 0.05), (1, 2, 12, 0.2), (2, 3, 12, 0.5),
                                                         (2, 4, 40, 0.3)])
def test_device_dags_match_host_builder(mode, seed, max_pins, density):
    """Modes 0..2, sparse to dense congestion; up to 40 pins per tree, which
    sends the largest trees to the larger work-area classes."""
    rng = np.random.default_rng(seed)
    X, Y = 700, 500
    tree_off, pos, adj_off, adj = _trees(rng, X, Y, 300, max_pins)
    xsum, ysum = _view(rng, X, Y, density)
    recs, off = ig.build_dags(X, Y, mode, tree_off, pos, adj_off, adj, xsum, ysum)
    assert off.size == tree_off.size
    for k in range(tree_off.size - 1):
        a, b = int(tree_off[k]), int(tree_off[k + 1])
        want = ig.build_dag(X, Y, mode, pos[a:b], adj_off[a:b + 1] - adj_off[a], adj[adj_off[a]:adj_off[b]], xsum,
                            ysum)
        assert np.array_equal(recs[off[k]:off[k + 1]], want), f"tree {k}"


def test_device_dags_reject_bad_trees():
    X, Y = 50, 50
    xs, ys = np.zeros(X * Y, np.float32), np.zeros(X * Y, np.float32)
    with pytest.raises(ig.IgrError):  # one node
        ig.build_dags(X, Y, 2, [0, 1], [5], [0, 0], np.zeros(0, np.int32), xs, ys)
    with pytest.raises(ig.IgrError):  # neighbour outside the tree
        ig.build_dags(X, Y, 2, [0, 2], [5, 7], [0, 1, 2], [1, 2], xs, ys)


@pytest.mark.parametrize("cfg", [0])
def test_router_with_device_dags_matches_host_dags(tmp_path, cfg):
    """The rip-up passes with DAGs, conflict points and batch arrays made on the
    device give the guides of the host-built path, byte for byte."""
    cap, net = str(tmp_path / "d.cap"), str(tmp_path / "d.net")
    ig.generate(cfg, 3, 1.0, cap, net)
    outs, stats = [], []
    for host in (1, 0):
        out = str(tmp_path / f"g{host}.out")
        r = ig.Router(cap, net, rrr_iters=3, host_dags=host)
        r.run()
        r.write(out)
        st = r.stats()
        stats.append((st["wirelength"], st["via_cost"], st["overflow_cost"]))
        assert st["dag_host_ms"] > 0  # detour DAGs were built
        r.close()
        outs.append(open(out, "rb").read())
    assert stats[0] == stats[1]
    assert outs[0] == outs[1]
