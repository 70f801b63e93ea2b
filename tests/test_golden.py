"""The CPU oracle and the host passes against golden vectors produced by
InstantGR itself (tests/golden/make_golden.py: the reference's kernels through
oracle/ref_harness.cu on a B200).  These pin the oracle before it is trusted as
the checker of the CUDA kernels."""
import numpy as np
import pytest

import instantgr_b200 as ig
from conftest import golden
from oracle_py import Oracle

RTOL = 1e-5


def grid_of(f):
    keys = ["L", "X", "Y", "DIR", "xlen", "ylen", "unit_wire", "unit_via", "short", "cap", "demand"]
    g = {k: f[k] for k in keys}
    for k in ("L", "X", "Y", "DIR"):
        g[k] = int(g[k])
    for k in ("unit_wire", "unit_via"):
        g[k] = float(g[k])
    return g


@pytest.mark.parametrize("i", range(3))
def test_oracle_cost_refresh_matches_reference(i):
    f = golden(f"cost_{i}.npz")
    g = grid_of(f)
    w, v, p = Oracle(g).cost_refresh(g["demand"])
    np.testing.assert_allclose(w, f["wcost"], rtol=RTOL, atol=0)
    np.testing.assert_allclose(v, f["vcost"], rtol=RTOL, atol=0)
    np.testing.assert_allclose(p, f["presum"], rtol=RTOL, atol=1e-9)


@pytest.mark.parametrize("i", range(2))
def test_oracle_pattern_route_matches_reference(i):
    f = golden(f"pattern_{i}.npz")
    g = grid_of(f)
    o = Oracle(g)
    stamp = int(f["stamp"])
    total = int(f["ref_routes"].size)
    routes = np.zeros(total, np.int32)
    pre = np.zeros(o.N, np.int32)
    st = np.zeros(o.N, np.int32)
    assert o.pattern_route(f["vcost"], f["presum"], f["node_off"], f["nodes"], f["par"], f["route_off"],
                           f["route_cap"], routes, pre, st, stamp) == 0
    assert np.array_equal(pre, f["ref_pre"]), "difference array after the DP"
    for k in range(len(f["route_off"])):
        a = int(f["route_off"][k])
        m = int(f["ref_routes"][a])
        assert np.array_equal(routes[a:a + m], f["ref_routes"][a:a + m]), f"net {k}"
    dem = g["demand"].copy()
    o.commit_wires(pre, dem, st, stamp)
    o.commit_vias(f["route_off"], routes, dem, st, stamp, 1)
    assert np.array_equal(dem, f["ref_demand"])
    assert np.array_equal(st, f["ref_stamps"])


@pytest.mark.parametrize("i", range(2))
def test_oracle_ripup_and_view_match_reference(i):
    f = golden(f"ripup_{i}.npz")
    g = grid_of(f)
    o = Oracle(g)
    is_of = o.mark_overflow(g["demand"], f["route_off"], f["routes"], 0, 10)
    assert np.nonzero(is_of)[0].tolist() == f["ref_of"].tolist()
    xs, ys = o.congestion_view(g["demand"])
    check_view_against_racy_reference(g, xs, ys, f["ref_xsum"], f["ref_ysum"])


def per_cell_from_prefix(pre, X, Y, axis):
    """Cell values behind an exclusive prefix sum along `axis` (the last cell is not recoverable)."""
    a = pre.reshape(X, Y)
    return np.diff(a, axis=axis)


def check_view_against_racy_reference(g, xs, ys, rx, ry):
    """extract_congestionView takes the maximum over layers with a plain
    read-max-write per layer thread (src/graph.hpp:552-554), so concurrent layers
    can lose updates: the reference's per-cell maxima are at most the true
    maxima, and equal wherever a single layer overflows."""
    X, Y, L = g["X"], g["Y"], g["L"]
    cap = g["cap"].reshape(L, X, Y)
    dem = g["demand"].reshape(L, X, Y)
    over = dem > cap
    single = over.sum(axis=0) <= 1
    for mine, ref, axis in ((xs, rx, 0), (ys, ry, 1)):
        m = per_cell_from_prefix(mine, X, Y, axis)
        r = per_cell_from_prefix(ref, X, Y, axis)
        assert (r <= m).all(), "reference maxima cannot exceed the exact maxima"
        sl = single[:-1, :] if axis == 0 else single[:, :-1]
        assert np.array_equal(r[sl], m[sl]), "cells with one overflowing layer must agree"
    assert (rx <= xs).all() and (ry <= ys).all()


def _route_sets(routes, off, n):
    out = []
    for k in range(n):
        a = int(off[k])
        m = int(routes[a])
        pairs = routes[a + 1:a + m].reshape(-1, 2)
        out.append(sorted(map(tuple, np.sort(pairs, axis=1).tolist())))
    return out


@pytest.mark.parametrize("i", range(2))
def test_oracle_dag_route_matches_reference(i):
    f = golden(f"dag_{i}.npz")
    g = grid_of(f)
    o = Oracle(g)
    stamp = int(f["stamp"])
    d = {k: f[k] for k in ("node_off", "nodes", "depth", "par_off", "par", "child_slot", "child_num")}
    total = int(f["ref_routes"].size)
    routes = np.zeros(total, np.int32)
    pre = np.zeros(o.N, np.int32)
    st = np.zeros(o.N, np.int32)
    assert o.dag_route(f["vcost"], f["presum"], d, f["route_off"], f["route_cap"], routes, pre, st, stamp) == 0
    assert np.array_equal(pre, f["ref_pre"])
    n = len(f["route_off"])
    # the reference appends segments with atomicAdd: compare per net as sets
    assert _route_sets(routes, f["route_off"], n) == _route_sets(f["ref_routes"], f["route_off"], n)
    dem = g["demand"].copy()
    o.commit_wires(pre, dem, st, stamp)
    o.commit_vias(f["route_off"], routes, dem, st, stamp, 1)
    assert np.array_equal(dem, f["ref_demand"])
    assert np.array_equal(st, f["ref_stamps"])


def test_dag_builder_matches_reference():
    """Host detour-DAG construction (net::generate_detours_reconstruct) vs the reference."""
    f = golden("dagbuild.npz")
    X, Y, mode = int(f["X"]), int(f["Y"]), int(f["mode"])
    ref = f["ref"]
    p = 0
    toff, adj_off = f["tree_off"], f["adj_off"]
    for k in range(len(toff) - 1):
        a, b = int(toff[k]), int(toff[k + 1])
        m = int(ref[p])
        E = int(ref[p + 1 + 4 * m])
        npt = int(ref[p + 2 + 4 * m + 2 * E])
        rec = ref[p:p + 3 + 4 * m + 2 * E + npt]
        p += rec.size
        ao = adj_off[a:b + 1] - adj_off[a]
        adj = f["adj"][adj_off[a]:adj_off[b]]
        mine = ig.build_dag(X, Y, mode, f["pos"][a:b], ao, adj, f["xsum"], f["ysum"])
        assert np.array_equal(mine, rec), f"net {k}"
    assert p == ref.size
