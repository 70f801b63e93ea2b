"""CUDA kernels (through the C ABI) against golden vectors produced by
InstantGR's own kernels on the same inputs (tests/golden/make_golden.py).

Cost tables are compared bit for bit: the fused kernel evaluates the same
expressions with the same __expf intrinsic and keeps the Sklansky association
of the reference's prefix sum.  Routes, difference array, demand and stamps
are compared exactly."""
import numpy as np
import pytest

import instantgr_b200 as ig
from conftest import golden
from test_golden import grid_of, _route_sets, check_view_against_racy_reference

pytestmark = pytest.mark.gpu


def ctx_for(g):
    c = ig.Ctx(g["L"], g["X"], g["Y"], g["DIR"], g["xlen"], g["ylen"], g["unit_wire"], g["unit_via"], g["short"],
               g["cap"])
    c.set_demand(g["demand"])
    return c


@pytest.mark.parametrize("i", range(3))
def test_cost_refresh_bit_exact_vs_reference(i):
    f = golden(f"cost_{i}.npz")
    g = grid_of(f)
    c = ctx_for(g)
    c.cost_refresh()
    v, p = c.costs()
    assert np.array_equal(v, f["vcost"]), f"vcost: {np.count_nonzero(v != f['vcost'])} cells differ"
    assert np.array_equal(p, f["presum"]), f"presum: {np.count_nonzero(p != f['presum'])} cells differ"


@pytest.mark.parametrize("i", range(2))
def test_pattern_route_bit_exact_vs_reference(i):
    f = golden(f"pattern_{i}.npz")
    g = grid_of(f)
    c = ctx_for(g)
    c.set_costs(f["vcost"], f["presum"])
    stamp = int(f["stamp"])
    routes = np.zeros(int(f["ref_routes"].size), np.int32)
    c.pattern_route(f["node_off"], f["nodes"], f["par"], f["route_off"], f["route_cap"], routes, stamp)
    assert np.array_equal(c.pre(), f["ref_pre"])
    for k in range(len(f["route_off"])):
        a = int(f["route_off"][k])
        m = int(f["ref_routes"][a])
        assert np.array_equal(routes[a:a + m], f["ref_routes"][a:a + m]), f"net {k}"
    c.commit_wires(stamp)
    c.commit_vias(f["route_off"], routes, stamp, 1)
    assert np.array_equal(c.demand(), f["ref_demand"])
    assert np.array_equal(c.stamps(), f["ref_stamps"])


@pytest.mark.parametrize("i", range(2))
def test_ripup_marking_vs_reference(i):
    f = golden(f"ripup_{i}.npz")
    g = grid_of(f)
    c = ctx_for(g)
    is_of = c.mark_overflow(f["route_off"], f["routes"], 0, 10)
    assert np.nonzero(is_of)[0].tolist() == f["ref_of"].tolist()
    xs, ys = c.congestion_view()
    check_view_against_racy_reference(g, xs, ys, f["ref_xsum"], f["ref_ysum"])


@pytest.mark.parametrize("i", range(2))
def test_dag_route_vs_reference(i):
    f = golden(f"dag_{i}.npz")
    g = grid_of(f)
    c = ctx_for(g)
    c.set_costs(f["vcost"], f["presum"])
    stamp = int(f["stamp"])
    routes = np.zeros(int(f["ref_routes"].size), np.int32)
    c.dag_route(f["node_off"], f["nodes"], f["depth"], f["par_off"], f["par"], f["child_slot"], f["child_num"],
                f["route_off"], f["route_cap"], routes, stamp)
    assert np.array_equal(c.pre(), f["ref_pre"])
    n = len(f["route_off"])
    assert _route_sets(routes, f["route_off"], n) == _route_sets(f["ref_routes"], f["route_off"], n)
    c.commit_wires(stamp)
    c.commit_vias(f["route_off"], routes, stamp, 1)
    assert np.array_equal(c.demand(), f["ref_demand"])
    assert np.array_equal(c.stamps(), f["ref_stamps"])
