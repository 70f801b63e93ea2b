"""CUDA kernels (through the C ABI) against the CPU oracle on seeded inputs.

Tolerances: cost tables within 1e-5 relative (the reference's __expf against
the oracle's exp); every integer, route, stamp and demand result bit-exact
(demand values are half units, exact in float).  The DP and commit kernels get
the GPU's own cost map handed to the oracle, so their comparison is exact.
"""
import numpy as np
import pytest

import instantgr_b200 as ig
import cases
from oracle_py import Oracle, color as orc_color

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def ctx_for(g):
    c = ig.Ctx(g["L"], g["X"], g["Y"], g["DIR"], g["xlen"], g["ylen"], g["unit_wire"], g["unit_via"], g["short"],
               g["cap"])
    c.set_demand(g["demand"])
    return c


GRIDS = [
    dict(seed=1, X=40, Y=30, dir0=0),
    dict(seed=2, X=300, Y=17, dir0=1, unit_wire=0.3),
    dict(seed=3, X=23, Y=1100, dir0=0, edge_len=3, unit_via=1.5),
    dict(seed=4, X=257, Y=513, dir0=1),
]


@pytest.mark.parametrize("gp", GRIDS)
def test_cost_refresh_matches_oracle(gp):
    gp = dict(gp)
    g = cases.grid_case(gp.pop("seed"), **gp)
    c = ctx_for(g)
    c.cost_refresh()
    v, p = c.costs()
    _, ov, op = Oracle(g).cost_refresh(g["demand"])
    np.testing.assert_allclose(v, ov, rtol=RTOL, atol=0)
    np.testing.assert_allclose(p, op, rtol=RTOL, atol=1e-9)


def test_dirty_refresh_equals_full_refresh():
    g = cases.grid_case(5, X=120, Y=90, dir0=0)
    c = ctx_for(g)
    c.cost_refresh()
    # change demand on a few cells through a via commit, then refresh only dirty tracks
    XY = g["X"] * g["Y"]
    routes = np.array([3, 2 * XY + 10 * g["Y"] + 20, 6 * XY + 10 * g["Y"] + 20], np.int32)
    c.commit_vias(np.array([0], np.int64), routes, stamp=1, K=1)
    c.cost_refresh(only_dirty=True)
    v1, p1 = c.costs()
    c.cost_refresh(only_dirty=False)
    v2, p2 = c.costs()
    assert np.array_equal(v1, v2) and np.array_equal(p1, p2)


def _pattern_case(seed, X, Y, dir0, n, kmax=8, uw=1.0):
    g = cases.grid_case(seed, X=X, Y=Y, dir0=dir0, unit_wire=uw)
    tb = cases.tree_batch(g, seed + 1, n=n, kmax=kmax)
    return g, tb


@pytest.mark.parametrize("seed,X,Y,dir0,n,kmax", [(11, 40, 30, 0, 80, 8), (12, 64, 50, 1, 200, 8),
                                                  (13, 120, 100, 0, 150, 24)])
def test_pattern_route_and_commit_match_oracle(seed, X, Y, dir0, n, kmax):
    g, tb = _pattern_case(seed, X, Y, dir0, n, kmax)
    c = ctx_for(g)
    c.cost_refresh()
    vc, ps = c.costs()
    total = int(tb["route_off"][-1] + tb["route_cap"][-1])
    stamp = 7
    r_gpu = np.zeros(total, np.int32)
    c.pattern_route(tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], tb["route_cap"], r_gpu, stamp)
    pre_gpu = c.pre()
    o = Oracle(g)
    r_orc = np.zeros(total, np.int32)
    pre = np.zeros(o.N, np.int32)
    st = np.zeros(o.N, np.int32)
    assert o.pattern_route(vc, ps, tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], tb["route_cap"], r_orc,
                           pre, st, stamp) == 0
    for k in range(n):
        a = int(tb["route_off"][k])
        m = int(r_orc[a])
        assert np.array_equal(r_gpu[a:a + m], r_orc[a:a + m]), f"net {k}"
    assert np.array_equal(pre_gpu, pre)
    # wire commit then via commit
    c.commit_wires(stamp)
    dem = g["demand"].copy()
    wl = o.commit_wires(pre, dem, st, stamp)
    assert np.array_equal(c.stamps(), st)
    o.commit_vias(tb["route_off"], r_orc, dem, st, stamp, 1)
    c.commit_vias(tb["route_off"], r_gpu, stamp, 1)
    assert np.array_equal(c.demand(), dem)
    assert np.array_equal(c.pre(), np.zeros_like(pre))
    wl_gpu, vias_gpu, _ = c.score()
    assert wl_gpu == wl


def test_pattern_route_reports_a_record_too_short():
    """A route record that cannot hold a net's segments: the oracle stops there
    (status -1) and the kernel reports IGR_ERR_CAPACITY."""
    g, tb = _pattern_case(14, 40, 30, 0, 60, 8)
    cap = tb["route_cap"].copy()
    k = int(np.argmax(np.diff(tb["node_off"])))  # the net with the most nodes
    cap[k] = 3
    c = ctx_for(g)
    c.cost_refresh()
    vc, ps = c.costs()
    total = int(tb["route_off"][-1] + tb["route_cap"][-1])
    with pytest.raises(ig.IgrError) as e:
        c.pattern_route(tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], cap, np.zeros(total, np.int32), 7)
    assert e.value.code == -5
    c.close()
    o = Oracle(g)
    z = np.zeros(o.N, np.int32)
    assert o.pattern_route(vc, ps, tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], cap,
                           np.zeros(total, np.int32), z, z.copy(), 7) == -1


def test_ripup_and_overflow_marking_match_oracle():
    g, tb = _pattern_case(21, 60, 50, 0, 250, 8)
    c = ctx_for(g)
    c.cost_refresh()
    vc, ps = c.costs()
    total = int(tb["route_off"][-1] + tb["route_cap"][-1])
    r = np.zeros(total, np.int32)
    c.pattern_route(tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], tb["route_cap"], r, 3)
    c.commit_wires(3)
    c.commit_vias(tb["route_off"], r, 3, 1)
    dem = c.demand()
    o = Oracle(g)
    for thr, me in ((0, 10), (0, 0), (-2, 3)):
        assert np.array_equal(c.mark_overflow(tb["route_off"], r, thr, me),
                              o.mark_overflow(dem, tb["route_off"], r, thr, me))
    xs, ys = c.congestion_view()
    oxs, oys = o.congestion_view(dem)
    assert np.array_equal(xs, oxs) and np.array_equal(ys, oys)
    # rip-up of half of the nets: wires (K=-1) then vias with the same stamp
    st = c.stamps()
    d2 = dem.copy()
    half = tb["route_off"][::2].copy()
    o.ripup_wires(half, r, d2, st, 4, -1)
    o.commit_vias(half, r, d2, st, 4, -1)
    c.ripup_wires(half, r, 4, -1)
    c.commit_vias(half, r, 4, -1)
    assert np.array_equal(c.demand(), d2)
    assert np.array_equal(c.stamps(), st)
    _, _, of = c.score()
    np.testing.assert_allclose(of, o.overflow_cost(d2), rtol=RTOL)


@pytest.mark.parametrize("keep_map", [1, 0])
@pytest.mark.parametrize("seed,n", [(31, 300), (32, 1500), (33, 6000)])
def test_coloring_matches_oracle(seed, n, keep_map):
    """Both forms of the colouring: the round-0 claim map kept up to date across
    batches (the default of igr_color_batches), and cleared and re-claimed for
    every batch (the router's form below 2M nets)."""
    X, Y = 64, 48
    args = cases.color_case(seed, X, Y, n)
    g = cases.grid_case(1, X=X, Y=Y)
    c = ctx_for(g)
    ig.set_test_hook(ig.HOOK_COLOR_KEEP_MAP, keep_map)
    try:
        b_gpu, nb_gpu = c.color_batches(*args, sparsity=3)
    finally:
        ig.set_test_hook(ig.HOOK_RESET)
    b_orc, nb_orc = orc_color(X, Y, *args, sparsity=3)
    assert nb_gpu == nb_orc
    assert np.array_equal(b_gpu, b_orc)
    # no two nets of a batch share a conflict point
    pt_off, pts = args[0], args[1]
    for b in range(nb_gpu):
        cells = [p for k in np.nonzero(b_gpu == b)[0] for p in pts[pt_off[k]:pt_off[k + 1]]]
        assert len(cells) == len(set(cells))


def _dag_vs_oracle(g, d, stamp=11):
    """GPU DAG DP, backtrace and demand against the oracle; returns the nets compared."""
    n = len(d["node_off"]) - 1
    c = ctx_for(g)
    c.cost_refresh()
    vc, ps = c.costs()
    total = int(d["route_off"][-1] + d["route_cap"][-1])
    r_gpu = np.zeros(total, np.int32)
    c.dag_route(d["node_off"], d["nodes"], d["depth"], d["par_off"], d["par"], d["child_slot"], d["child_num"],
                d["route_off"], d["route_cap"], r_gpu, stamp)
    pre_gpu = c.pre()
    c.close()
    o = Oracle(g)
    r_orc = np.zeros(total, np.int32)
    pre = np.zeros(o.N, np.int32)
    st = np.zeros(o.N, np.int32)
    assert o.dag_route(vc, ps, d, d["route_off"], d["route_cap"], r_orc, pre, st, stamp) == 0
    for k in range(n):
        a = int(d["route_off"][k])
        m = int(r_orc[a])
        assert np.array_equal(r_gpu[a:a + m], r_orc[a:a + m]), f"net {k}"
    assert np.array_equal(pre_gpu, pre)
    return n


@pytest.mark.parametrize("seed,dir0,load", [(43, 0, 1.0), (44, 1, 2.5)])
def test_dag_route_on_detour_builder_dags(seed, dir0, load):
    """The DAGs of the detour builder (golden records of the reference builder:
    mirrored trunks, Z-shape alternatives, split long edges; nodes with up to 36
    parents and 5 child slots, depth up to 13) through the DAG DP, against the
    oracle on two cost maps."""
    from conftest import golden
    f = golden("dagbuild.npz")
    X, Y = int(f["X"]), int(f["Y"])
    g = cases.grid_case(seed, X=X, Y=Y, dir0=dir0, load=load)
    d = cases.dag_records_batch(f["ref"])
    assert int(np.max(np.diff(d["par_off"]))) >= 30
    assert _dag_vs_oracle(g, d) == len(f["tree_off"]) - 1


@pytest.mark.parametrize("seed,X,Y,dir0,n", [(41, 48, 40, 0, 50), (42, 70, 60, 1, 120)])
def test_dag_route_matches_oracle(seed, X, Y, dir0, n):
    g = cases.grid_case(seed, X=X, Y=Y, dir0=dir0)
    d = cases.dag_batch(g, seed + 1, n=n)
    c = ctx_for(g)
    c.cost_refresh()
    vc, ps = c.costs()
    total = int(d["route_off"][-1] + d["route_cap"][-1])
    r_gpu = np.zeros(total, np.int32)
    stamp = 11
    c.dag_route(d["node_off"], d["nodes"], d["depth"], d["par_off"], d["par"], d["child_slot"], d["child_num"],
                d["route_off"], d["route_cap"], r_gpu, stamp)
    pre_gpu = c.pre()
    o = Oracle(g)
    r_orc = np.zeros(total, np.int32)
    pre = np.zeros(o.N, np.int32)
    st = np.zeros(o.N, np.int32)
    assert o.dag_route(vc, ps, d, d["route_off"], d["route_cap"], r_orc, pre, st, stamp) == 0
    for k in range(n):
        a = int(d["route_off"][k])
        m = int(r_orc[a])
        assert m > 1, f"net {k} produced no route"
        assert np.array_equal(r_gpu[a:a + m], r_orc[a:a + m]), f"net {k}"
    assert np.array_equal(pre_gpu, pre)


@pytest.mark.parametrize("split,stage", [(2, 1024), (4096, 1024), (4096, 0), (4096, 40), (2, 40), (4096, 100)])
def test_dag_route_split_by_size_matches_oracle(split, stage):
    """A batch of DAGs of 3 to about 110 nodes through the DAG DP with the
    split for batches of many nets on (the DAGs of at most 64 nodes in 2-warp
    CTAs beside the larger ones on a second stream, which the router uses for
    batches of 4096 nets or more) and off (then the DAGs of more than 96 nodes
    run beside the others with more shared memory), and with every DAG, none,
    or those of at most 40 or 100 nodes staged in shared memory, against the
    oracle."""
    g = cases.grid_case(45, X=90, Y=80, dir0=0)
    d = cases.dag_batch(g, 46, n=120, kmax=40)
    sizes = np.diff(d["node_off"])
    assert (sizes <= 40).sum() > 0 and (sizes > 64).sum() > 0
    ig.set_test_hook(ig.HOOK_DAG_SPLIT_NETS, split)
    ig.set_test_hook(ig.HOOK_DAG_STAGE_NODES, stage)
    try:
        assert _dag_vs_oracle(g, d) == 120
    finally:
        ig.set_test_hook(ig.HOOK_RESET)


def test_state_dump_and_load_round_trip(tmp_path):
    """igr_dump_state / igr_load_state: a second context loaded from the file of
    the first holds the same demand, costs, stamps and difference array (taken
    after a tree-DP batch, before its commit), and commits and refreshes to the
    same grid; a file of another grid size, a short file and a missing file are
    refused."""
    g, tb = _pattern_case(31, 64, 50, 1, 120, 8)
    c = ctx_for(g)
    c.cost_refresh()
    total = int(tb["route_off"][-1] + tb["route_cap"][-1])
    r = np.zeros(total, np.int32)
    c.pattern_route(tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], tb["route_cap"], r, 5)
    path = str(tmp_path / "state.bin")
    c.dump_state(path)
    d = ig.Ctx(g["L"], g["X"], g["Y"], g["DIR"], g["xlen"], g["ylen"], g["unit_wire"], g["unit_via"], g["short"],
               g["cap"])
    d.load_state(path)
    for get in ("demand", "stamps", "pre"):
        assert np.array_equal(getattr(c, get)(), getattr(d, get)()), get
    (v1, p1), (v2, p2) = c.costs(), d.costs()
    assert np.array_equal(v1, v2) and np.array_equal(p1, p2)
    for x in (c, d):
        x.commit_wires(5)
        x.commit_vias(tb["route_off"], r, 5, 1)
        x.cost_refresh(only_dirty=True)
    assert np.array_equal(c.demand(), d.demand())
    (v1, p1), (v2, p2) = c.costs(), d.costs()
    assert np.array_equal(v1, v2) and np.array_equal(p1, p2)
    other = cases.grid_case(32, X=40, Y=30, dir0=1)
    e = ctx_for(other)
    with pytest.raises(ig.IgrError) as err:
        e.load_state(path)
    assert err.value.code == -1
    short = str(tmp_path / "short.bin")
    with open(path, "rb") as f, open(short, "wb") as o:
        o.write(f.read(1000))
    with pytest.raises(ig.IgrError) as err:
        d.load_state(short)
    assert err.value.code == -3
    with pytest.raises(ig.IgrError) as err:
        d.load_state(str(tmp_path / "missing.bin"))
    assert err.value.code == -2
    for x in (c, d, e):
        x.close()
