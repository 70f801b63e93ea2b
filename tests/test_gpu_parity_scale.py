"""Parity with InstantGR at the benchmark sizes.

The golden fixtures cover small grids; here the reference itself runs on the
configured designs, on the GPU box, through the tools built from its own
sources under oracle/_ref:
  * ref_cpu `trees`: the reference's reader, pin selection, net split and
    Steiner trees (db::read, build_cuda_database, construct_rsmt) against the
    routing nets and DFS trees of this router, net for net;
  * ref_harness: the reference's cost kernels, tree DP and commits on a whole
    phase-1 batch of the 840x1140, 130k-net design (split high-fanout nets and
    nets of more than 16 tree nodes included), and its detour-DAG builder, DAG
    DP and commits on a reroute batch of the 1600x1600, 800k-net design (the
    nets phase 1 leaves overflowing, their old routes ripped up first).
Given the same demand the cost maps must be bit-identical, and given the
reference's cost map every difference array, route, demand and stamp must be
bit-identical (phase-2 routes as sets per net: the reference emits segments in
atomic order).  The end-to-end evaluator total on the 130k-net design must be
within 0.5% of the reference router's, both ways.
"""
import math
import os
import subprocess

import numpy as np
import pytest

import instantgr_b200 as ig
import cases
from conftest import ROOT
from test_golden import _route_sets

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref")
GEN = os.path.join(ROOT, "instantgr_b200", "bin", "igr_generate")
EVALUATOR = os.path.join(REF, "evaluator")


def _design(tmp, cfg, scale=1.0, seed=1):
    cap, net = os.path.join(tmp, f"c{cfg}_{scale:g}.cap"), os.path.join(tmp, f"c{cfg}_{scale:g}.net")
    if not os.path.exists(net):
        subprocess.run([GEN, "--config", str(cfg), "--seed", str(seed), "--scale", str(scale), "--cap", cap,
                        "--net", net], check=True)
    return cap, net


@pytest.fixture(scope="module")
def work(tmp_path_factory):
    return str(tmp_path_factory.mktemp("scale"))


def _harness(mode, arrays, dtypes, tmp):
    fin, fout = os.path.join(tmp, mode + ".in"), os.path.join(tmp, mode + ".out")
    cases.write_harness_input(fin, arrays)
    subprocess.run([os.path.join(REF, "ref_harness"), mode, fin, fout], check=True, stdout=subprocess.DEVNULL,
                   timeout=900)
    out = cases.read_harness_output(fout, dtypes)
    os.remove(fin)
    os.remove(fout)
    return out


def _ctx(g):
    c = ig.Ctx(g["L"], g["X"], g["Y"], g["DIR"], g["xlen"], g["ylen"], g["unit_wire"], g["unit_via"], g["short"],
               g["cap"])
    c.set_demand(g["demand"])
    return c


def _read_ref_trees(path):
    a = np.fromfile(path, dtype=np.int32)
    n = int(a[0])
    p = 1
    out = []
    for _ in range(n):
        orig, npins = int(a[p]), int(a[p + 1])
        p += 2 + npins
        m = int(a[p])
        nodes = a[p + 1:p + 1 + m]
        par = a[p + 1 + m:p + 1 + 2 * m]
        p += 1 + 2 * m
        out.append((orig, nodes, par))
    return out


def _plan_trees(plan):
    """routing-net id -> (nodes, par) of this router's last run."""
    ids, noff = plan["net_ids"], plan["node_off"]
    trees = {}
    for k, r in enumerate(ids.tolist()):
        a, b = int(noff[k]), int(noff[k + 1])
        trees[r] = (plan["nodes"][a:b], plan["par"][a:b])
    return trees


@pytest.mark.parametrize("cfg,scale", [(1, 0.1), (2, 0.05)])
def test_routing_nets_and_trees_match_reference(work, cfg, scale):
    """Every routing net of the design (the split of nets with more than 12
    pins included) with the same tree in the same DFS preorder as the
    reference's, on the design families with 65-500- and 2-1000-pin nets."""
    cap, net = _design(work, cfg, scale)
    out = os.path.join(work, "trees.bin")
    subprocess.run([os.path.join(REF, "ref_cpu"), cap, net, "trees", out], check=True, stdout=subprocess.DEVNULL,
                   timeout=900)
    ref = _read_ref_trees(out)
    r = ig.Router(cap, net, rrr_iters=0)
    r.run()
    _, R = r.sizes()
    mine = _plan_trees(r.plan())
    r.close()
    assert R == len(ref)
    bad = [k for k in range(R) if not (np.array_equal(mine[k][0], ref[k][1]) and np.array_equal(mine[k][1], ref[k][2]))]
    assert not bad, f"{len(bad)} of {R} trees differ, first {bad[:5]}"


def test_phase1_batch_bit_exact_at_full_size(work):
    """A whole phase-1 batch of the 840x1140, 130k-net design on the routed
    demand: cost map, tree DP, difference array, routes, demand, stamps."""
    cap, net = _design(work, 1)
    r = ig.Router(cap, net, rrr_iters=0)
    r.run()
    plan, g = r.plan(), r.grid()
    g["demand"] = r.demand()
    r.close()
    boff, noff = plan["batch_off"], plan["node_off"]
    sizes = np.diff(noff)
    big = [int(np.count_nonzero(sizes[boff[b]:boff[b + 1]] > 16)) for b in range(len(boff) - 1)]
    b = int(np.argmax(big))
    assert big[b] > 0
    a, e = int(boff[b]), int(boff[b + 1])
    node_off = (noff[a:e + 1] - noff[a]).astype(np.int32)
    nodes = plan["nodes"][noff[a]:noff[e]].copy()
    par = plan["par"][noff[a]:noff[e]].copy()
    pins = np.array([max(1, math.ceil(c / 12)) for c in plan["route_cap"][a:e]], np.int32)
    route_cap = (12 * pins).astype(np.int32)
    route_off = np.concatenate([[0], np.cumsum(route_cap)[:-1]]).astype(np.int64)
    # the reference's cost map on this demand, and this build's
    _, vc, ps = _harness("cost", cases.grid_arrays(g), [np.float32, np.float32, np.float64], work)
    c = _ctx(g)
    c.cost_refresh()
    v2, p2 = c.costs()
    assert np.array_equal(v2, vc), f"vcost: {np.count_nonzero(v2 != vc)} cells differ"
    assert np.array_equal(p2, ps), f"presum: {np.count_nonzero(p2 != ps)} cells differ"
    stamp = 7
    ref_pre, ref_routes, ref_dem, ref_st = _harness(
        "pattern", cases.grid_arrays(g) + [vc, ps, np.array([stamp], np.int32), node_off, nodes, par, pins],
        [np.int32, np.int32, np.float32, np.int32], work)
    c.set_costs(vc, ps)
    routes = np.zeros(ref_routes.size, np.int32)
    c.pattern_route(node_off, nodes, par, route_off, route_cap, routes, stamp)
    assert np.array_equal(c.pre(), ref_pre)
    for k in range(e - a):
        o = int(route_off[k])
        m = int(ref_routes[o])
        assert np.array_equal(routes[o:o + m], ref_routes[o:o + m]), f"net {k} of batch {b}"
    c.commit_wires(stamp)
    c.commit_vias(route_off, routes, stamp, 1)
    assert np.array_equal(c.demand(), ref_dem)
    assert np.array_equal(c.stamps(), ref_st)
    c.close()


def test_reroute_batch_bit_exact_at_full_size(work):
    """The nets that phase 1 leaves overflowing on the 1600x1600, 800k-net
    design (InstantGR's rip-up rule), their old routes ripped up, their detour
    DAGs built by the reference's builder from the congestion view, and one
    batch of them through the reference's DAG DP and this build's."""
    cap, net = _design(work, 2)
    r = ig.Router(cap, net, rrr_iters=0)
    r.run()
    plan, g = r.plan(), r.grid()
    g["demand"] = r.demand()
    _, R = r.sizes()
    recs = [r.route(k) for k in range(R)]
    r.close()
    lens = np.array([x.size for x in recs], np.int64)
    off = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
    routes = np.concatenate(recs).astype(np.int32)
    c = _ctx(g)
    is_of = c.mark_overflow(off, routes, 0, 10)
    of = np.nonzero(is_of)[0]
    assert of.size > 1000
    xs, ys = c.congestion_view()
    # the overflowing nets' trees (adjacency from the DFS parents)
    trees = _plan_trees(plan)
    sel = of[:4000]
    tree_off, pos, adj_off, adj = [0], [], [0], []
    for k in sel.tolist():
        nd, pa = trees[k]
        m = nd.size
        nb = [[] for _ in range(m)]
        for v in range(1, m):
            nb[v].append(int(pa[v]))
            nb[int(pa[v])].append(v)
        for v in range(m):
            adj += nb[v]
            adj_off.append(len(adj))
        pos += nd.tolist()
        tree_off.append(len(pos))
    X, Y = g["X"], g["Y"]
    (rec,) = _harness("dagbuild", [np.array([X, Y, 0], np.int32), xs, ys, np.array(tree_off, np.int32),
                                   np.array(pos, np.int32), np.array(adj_off, np.int32), np.array(adj, np.int32)],
                      [np.int32], work)
    # nets whose DAG has a node of more than 10 child slots keep their route (the
    # reference packs the slot as a decimal digit)
    d0 = cases.dag_records_batch(rec)
    keep = [k for k in range(sel.size)
            if int(d0["child_num"][d0["node_off"][k]:d0["node_off"][k + 1]].max(initial=0)) <= 10]
    d = cases.dag_records_batch(rec, nets=set(keep))
    n = len(d["node_off"]) - 1
    pins = np.array([max(1, math.ceil((8 * m + 1) / 100)) for m in np.diff(d["node_off"])], np.int32)
    route_cap = (100 * pins).astype(np.int32)
    route_off = np.concatenate([[0], np.cumsum(route_cap)[:-1]]).astype(np.int64)
    # rip-up of their phase-1 routes (commit_wire_demand / commit_via_demand with K = -1)
    old = off[sel[keep]]
    c.ripup_wires(old, routes, 1, -1)
    c.commit_vias(old, routes, 1, -1)
    g["demand"] = c.demand()
    c.close()
    _, vc, ps = _harness("cost", cases.grid_arrays(g), [np.float32, np.float32, np.float64], work)
    c = _ctx(g)
    c.cost_refresh()
    v2, p2 = c.costs()
    assert np.array_equal(v2, vc) and np.array_equal(p2, ps)
    stamp = 3
    ref_pre, ref_routes, ref_dem, ref_st = _harness(
        "dag", cases.grid_arrays(g) + [vc, ps, np.array([stamp], np.int32), d["node_off"], d["nodes"], d["depth"],
                                       d["par_off"], d["par"], d["child_slot"], d["child_num"], pins],
        [np.int32, np.int32, np.float32, np.int32], work)
    c.set_costs(vc, ps)
    mine = np.zeros(ref_routes.size, np.int32)
    c.dag_route(d["node_off"], d["nodes"], d["depth"], d["par_off"], d["par"], d["child_slot"], d["child_num"],
                route_off, route_cap, mine, stamp)
    assert np.array_equal(c.pre(), ref_pre)
    assert _route_sets(mine, route_off, n) == _route_sets(ref_routes, route_off, n)
    c.commit_wires(stamp)
    c.commit_vias(route_off, mine, stamp, 1)
    assert np.array_equal(c.demand(), ref_dem)
    assert np.array_equal(c.stamps(), ref_st)
    c.close()


def _for_stat(cap, net, out):
    p = subprocess.run([EVALUATOR, cap, net, out], capture_output=True, text=True, timeout=900)
    stat = [line for line in p.stdout.splitlines() if line.startswith("FOR_STAT")]
    assert stat, p.stdout[-2000:]
    return float(stat[0].split()[4])


def test_score_within_half_percent_of_reference_router_at_130k_nets(work):
    """The whole flow on the 840x1140, 130k-net design, one rip-up pass as
    InstantGR's main.cpp: evaluator totals of this router and of the
    reference's sm_100a build (oracle/_ref/instantgr_ref) within 0.5% either way."""
    cap, net = _design(work, 1)
    mine_out, ref_out = os.path.join(work, "mine.guide"), os.path.join(work, "ref.guide")
    ig.route_files(cap, net, mine_out, rrr_iters=1)
    subprocess.run([os.path.join(REF, "instantgr_ref"), "-cap", cap, "-net", net, "-out", ref_out], check=True,
                   stdout=subprocess.DEVNULL, timeout=900)
    mine, theirs = _for_stat(cap, net, mine_out), _for_stat(cap, net, ref_out)
    assert abs(mine - theirs) <= 0.005 * theirs, (mine, theirs)


def _conflict_points(nodes, par, Y, XY):
    """2-D conflict points of one tree (net::construct_rsmt, src/database_cuda.hpp:
    746-820): its nodes, and per edge its end points or its two bend corners."""
    pts = set(int(v) % XY for v in nodes)
    for i in range(1, len(nodes)):
        a, b = int(nodes[i]) % XY, int(nodes[int(par[i])]) % XY
        xa, ya, xb, yb = a // Y, a % Y, b // Y, b % Y
        if xa != xb and ya != yb:
            pts.add(xa * Y + yb)
            pts.add(xb * Y + ya)
    return pts


def _reference_phase1_batches(cap, net, runs):
    """Phase-1 batch counts of the reference router (its colouring is
    nondeterministic: database_cuda.hpp:437), from its log."""
    counts = []
    for _ in range(runs):
        p = subprocess.run([os.path.join(REF, "instantgr_ref"), "-cap", cap, "-net", net, "-out", os.devnull],
                           capture_output=True, text=True, timeout=900)
        gen = [line.split() for line in p.stdout.splitlines() if line.strip().startswith("Generation")]
        assert gen, p.stdout[-1500:]
        counts.append(int(gen[0][2]))
    return counts


def test_phase1_colouring_properties_and_batch_count_at_130k_nets(work):
    """The deterministic colouring on the 840x1140, 130k-net design: no two nets
    of a batch share a conflict point, every net is in exactly one batch, and the
    number of batches lies within the range of the reference's (racy) colouring
    over three runs of the reference router, widened by 10%."""
    cap, net = _design(work, 1)
    r = ig.Router(cap, net, rrr_iters=0)
    r.run()
    plan = r.plan()
    nb = int(r.stats()["batches1"])
    _, R = r.sizes()
    g = r.grid()
    r.close()
    Y, XY = g["Y"], g["X"] * g["Y"]
    boff, noff = plan["batch_off"], plan["node_off"]
    assert len(boff) - 1 == nb and int(boff[-1]) == R
    assert sorted(plan["net_ids"].tolist()) == list(range(R))
    for b in range(nb):
        seen = set()
        for k in range(int(boff[b]), int(boff[b + 1])):
            a, e = int(noff[k]), int(noff[k + 1])
            pts = _conflict_points(plan["nodes"][a:e], plan["par"][a:e], Y, XY)
            assert not (pts & seen), f"batch {b}: nets share a conflict point"
            seen |= pts
    ref = _reference_phase1_batches(cap, net, 3)
    lo, hi = min(ref), max(ref)
    assert 0.9 * lo <= nb <= 1.1 * hi, (nb, ref)


@pytest.mark.parametrize("X,Y,dir0", [(5000, 8, 0), (8, 5000, 1), (15360, 4, 0)])
def test_long_track_costs_bit_exact_vs_reference(work, X, Y, dir0):
    """Tracks longer than 4096 GCells (up to the reference's 15,360): the cost
    model and the f64 Sklansky prefix sums bit-identical to the reference's
    kernels on the same demand."""
    g = cases.grid_case(61, X=X, Y=Y, dir0=dir0)
    _, vc, ps = _harness("cost", cases.grid_arrays(g), [np.float32, np.float32, np.float64], work)
    c = _ctx(g)
    c.cost_refresh()
    v2, p2 = c.costs()
    c.close()
    assert np.array_equal(v2, vc), f"vcost: {np.count_nonzero(v2 != vc)} cells differ"
    assert np.array_equal(p2, ps), f"presum: {np.count_nonzero(p2 != ps)} cells differ"


def test_grid_with_5000_gcell_tracks_routes(work):
    """A 5000x1000 design (horizontal tracks of 5000 GCells, beyond the fused
    batch commit's 4096, so phase 1 commits with the separate launches):
    routed with a rip-up pass, records well formed, and the device
    evaluation's wire length equal to the router's own count."""
    X, Y = 5000, 1000
    cap, net = os.path.join(work, "g5k.cap"), os.path.join(work, "g5k.net")
    ig.generate_custom(X, Y, 40000, seed=77, cap_mode=1, block_frac=0.0, pin_mode=1, bbox_median=10,
                       bbox_sigma=1.2, hotspots=4, hotspot_frac=0.4, cap=cap, net=net)
    r = ig.Router(cap, net, rrr_iters=1)
    r.run()
    ev = r.evaluate()
    st = r.stats()
    _, R = r.sizes()
    XY = X * Y
    for k in range(0, R, max(1, R // 2000)):
        rec = r.route(k)
        assert rec[0] == len(rec) and rec[0] % 2 == 1
        a, b = rec[1::2], rec[2::2]
        via = a // XY != b // XY
        assert np.all(~via | ((a % XY) == (b % XY)))
    r.close()
    assert np.isfinite(ev["total"]) and ev["total"] > 0
    assert abs(ev["wirelength"] - st["wirelength"]) <= 1e-6 * st["wirelength"]
