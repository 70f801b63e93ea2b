"""igr_pattern_route_static against igr_pattern_route, through the C ABI.

igr_pattern_route_static is the phase-1 tree DP for callers that cannot let a
library allocate device memory: hosts whose pool allocator owns the whole GPU,
loops where a cudaMalloc could synchronise the device and stall other streams,
and processes that must fix their memory footprint before they start.  Its
scratch (the layer tables of nets with more than 16 tree nodes, per-net
offsets and the work counter) is one fixed array in the library's device
image; inputs and outputs are the caller's device arrays.

Both entry points run the same DP kernel on the same cost map, so routes,
difference array, demand and stamps must be bit-identical.  Two batches are
routed back to back so that the second call starts with the first call's
leftover scratch.  The file sorts last so that a run which stops at the first
failure has run every other test before it.
"""
import numpy as np
import pytest

import instantgr_b200 as ig
import cases

pytestmark = pytest.mark.gpu


def _ctx(g):
    c = ig.Ctx(g["L"], g["X"], g["Y"], g["DIR"], g["xlen"], g["ylen"], g["unit_wire"], g["unit_via"], g["short"],
               g["cap"])
    c.set_demand(g["demand"])
    return c


def _route_static(c, tb, stamp, total):
    import torch
    dev = {k: torch.from_numpy(np.ascontiguousarray(tb[k])).cuda()
           for k in ("node_off", "nodes", "par", "route_off", "route_cap")}
    routes = torch.zeros(total, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    c.pattern_route_static(len(tb["route_off"]), dev["node_off"].data_ptr(), int(tb["node_off"][-1]),
                           dev["nodes"].data_ptr(), dev["par"].data_ptr(), dev["route_off"].data_ptr(),
                           dev["route_cap"].data_ptr(), routes.data_ptr(), total, stamp)
    return routes.cpu().numpy()


def test_static_scratch_tree_dp_matches_allocating_entry_on_two_calls():
    g = cases.grid_case(51, X=120, Y=100)
    batches = [cases.tree_batch(g, 52, n=150, kmax=24), cases.tree_batch(g, 53, n=220, kmax=30)]
    for tb in batches:
        assert (np.diff(tb["node_off"]) > 16).any(), "the batch must put some nets in scratch"
    ca, cb = _ctx(g), _ctx(g)
    for call, tb in enumerate(batches):
        stamp = 11 + call
        ca.cost_refresh()
        cb.cost_refresh()
        total = int(tb["route_off"][-1] + tb["route_cap"][-1])
        r_a = np.zeros(total, np.int32)
        ca.pattern_route(tb["node_off"], tb["nodes"], tb["par"], tb["route_off"], tb["route_cap"], r_a, stamp)
        r_b = _route_static(cb, tb, stamp, total)
        assert np.array_equal(r_a, r_b), f"call {call}: route records differ"
        assert np.array_equal(ca.pre(), cb.pre()), f"call {call}: difference arrays differ"
        for c, r in ((ca, r_a), (cb, r_b)):
            c.commit_wires(stamp)
            c.commit_vias(tb["route_off"], r, stamp, 1)
        assert np.array_equal(ca.demand(), cb.demand())
        assert np.array_equal(ca.stamps(), cb.stamps())
    ca.close()
    cb.close()


def test_static_scratch_rejects_oversized_batches():
    import torch
    g = cases.grid_case(54, X=64, Y=48)
    c = _ctx(g)
    dummy = torch.zeros(16, dtype=torch.int64, device="cuda")
    p = dummy.data_ptr()
    with pytest.raises(ig.IgrError) as e:
        c.pattern_route_static(ig.STATIC_MAX_NETS + 1, p, 0, p, p, p, p, p, 0, 1)
    assert e.value.code == ig.IGR_ERR_CAPACITY and "nets per call" in str(e.value)
    # 2000 chains of 80 nodes: 160k nodes in scratch need about 80 MB (> 64 MiB)
    n, k = 2000, 80
    xy = g["X"] * g["Y"]
    node_off = np.arange(n + 1, dtype=np.int32) * k
    nodes = (np.arange(n * k, dtype=np.int64) % xy).astype(np.int32)
    par = np.tile(np.arange(-1, k - 1, dtype=np.int32), n)
    cap = np.full(n, 8 * k + 1, np.int32)
    off = (np.arange(n, dtype=np.int64) * int(cap[0]))
    tb = dict(node_off=node_off, nodes=nodes, par=par, route_off=off, route_cap=cap)
    total = n * int(cap[0])
    with pytest.raises(ig.IgrError) as e:
        _route_static(c, tb, 1, total)
    assert e.value.code == ig.IGR_ERR_CAPACITY and "static scratch holds" in str(e.value)
    # the context and the array stay usable after a rejection
    small = cases.tree_batch(g, 55, n=40, kmax=20)
    tot = int(small["route_off"][-1] + small["route_cap"][-1])
    r = _route_static(c, small, 2, tot)
    assert (r[small["route_off"]] > 0).all()
    c.close()
