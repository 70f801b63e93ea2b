"""End-to-end routing through the C ABI and the command line, scored by the
reference's own evaluator (run/evaluator.cpp built into oracle/_ref)."""
import json
import os
import subprocess

import numpy as np
import pytest

import instantgr_b200 as ig
from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

EVALUATOR = os.path.join(ROOT, "oracle", "_ref", "evaluator")


def evaluate(cap, net, out):
    p = subprocess.run([EVALUATOR, cap, net, out], capture_output=True, text=True, timeout=600)
    stat = [l for l in p.stdout.splitlines() if l.startswith("FOR_STAT")]
    # the evaluator returns 1 after a complete evaluation and exits 0 after printing
    # the name of a disconnected net (run/evaluator.cpp:267-276, :509-513)
    assert stat, p.stdout[-2000:] + p.stderr[-2000:]
    opens = [l for l in p.stdout.splitlines() if l.startswith("Number of open nets")]
    assert opens and opens[0].split(":")[1].strip() == "0"
    return [float(v) for v in stat[0].split()[1:]]


@pytest.fixture(scope="module")
def small_design(tmp_path_factory):
    d = tmp_path_factory.mktemp("design")
    cap, net = str(d / "s.cap"), str(d / "s.net")
    ig.generate_custom(96, 96, 3000, seed=41, cap_mode=0, block_frac=0.05, pin_mode=0, bbox_median=8,
                       bbox_sigma=1.0, cap=cap, net=net)
    return cap, net, d


def test_route_files_produces_connected_guides(small_design):
    cap, net, d = small_design
    out = str(d / "s.out")
    ig.route_files(cap, net, out)
    wl, via, of, tot = evaluate(cap, net, out)
    assert tot == wl + via + of or abs(tot - (wl + via + of)) <= 2


@pytest.mark.parametrize("rrr", [0, 3])
def test_device_evaluation_matches_the_evaluator(small_design, rrr):
    """igr_router_evaluate against the reference evaluator run on the written
    guides: wire length and via costs exactly, overflow and total to the
    evaluator's printed integers (sums of exp terms in another order)."""
    cap, net, d = small_design
    r = ig.Router(cap, net, rrr_iters=rrr)
    r.run()
    out = str(d / f"eval{rrr}.out")
    r.write(out)
    mine = r.evaluate()
    r.close()
    wl, via, of, tot = evaluate(cap, net, out)
    assert round(mine["wirelength"]) == wl and round(mine["via"]) == via, (mine, wl, via)
    assert abs(mine["overflow"] - of) <= 1 and abs(mine["total"] - tot) <= 1, (mine, of, tot)


def test_device_evaluation_on_a_rerouted_design(tmp_path):
    """The 256x256, 20k-net configuration with rip-up and reroute passes."""
    cap, net, out = str(tmp_path / "c0.cap"), str(tmp_path / "c0.net"), str(tmp_path / "c0.out")
    ig.generate(0, 3, 1.0, cap, net)
    r = ig.Router(cap, net, rrr_iters=3)
    r.run()
    r.write(out)
    mine = r.evaluate()
    r.close()
    wl, via, of, tot = evaluate(cap, net, out)
    assert round(mine["wirelength"]) == wl and round(mine["via"]) == via, (mine, wl, via)
    assert abs(mine["overflow"] - of) <= 1 and abs(mine["total"] - tot) <= 1, (mine, of, tot)


def test_cli_matches_library(small_design):
    cap, net, d = small_design
    out1, out2 = str(d / "a.out"), str(d / "b.out")
    ig.route_files(cap, net, out1)
    p = subprocess.run([ig.ROUTE_BIN, "-cap", cap, "-net", net, "-out", out2], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    assert open(out1).read() == open(out2).read(), "routing must be deterministic"


def test_batched_form_matches_plain_form(small_design):
    """Size classes, autotuned launch shapes and the CUDA graph change no result."""
    cap, net, d = small_design
    outs = []
    for batched in (0, 1, 1):  # the second batched run replays the cached graph
        out = str(d / f"batched{batched}_{len(outs)}.out")
        r = ig.Router(cap, net, rrr_iters=2, batched=batched)
        r.run()
        if batched:
            r.run()
        r.write(out)
        outs.append(open(out).read())
        r.close()
    assert outs[0] == outs[1] == outs[2]


def test_fused_batch_commit_matches_split_commit(small_design):
    """The fused per-track commit + cost refresh of phase 1 gives the demand,
    routes and statistics of separate cost-refresh, wire-commit and via-commit
    launches (phase 1 only, where the fusion applies)."""
    cap, net, d = small_design
    res = []
    for split in (1, 0):
        r = ig.Router(cap, net, rrr_iters=0, batched=1, split_commit=split)
        r.run()
        out = str(d / f"split{split}.out")
        r.write(out)
        s = r.stats()
        res.append((r.demand(), open(out).read(), s["wirelength"], s["via_cost"], s["overflow_cost"]))
        r.close()
    assert np.array_equal(res[0][0], res[1][0]), "demand differs"
    assert res[0][1] == res[1][1], "route guides differ"
    assert res[0][2:] == res[1][2:]


def test_router_stats_and_gpu_score(small_design):
    cap, net, d = small_design
    r = ig.Router(cap, net, rrr_iters=1)
    r.run()
    s = r.stats()
    assert s["routing_nets"] > 0 and s["batches1"] > 0
    out = str(d / "c.out")
    r.write(out)
    wl, via, of, tot = evaluate(cap, net, out)
    # the in-run estimate counts wires per edge and vias per layer like the evaluator
    assert abs(s["wirelength"] - wl) <= 1e-6 * max(1, wl)
    r.close()


def test_more_iterations_do_not_worsen_score(small_design):
    cap, net, d = small_design
    scores = []
    for it in (1, 3):
        out = str(d / f"it{it}.out")
        ig.route_files(cap, net, out, rrr_iters=it)
        scores.append(evaluate(cap, net, out)[3])
    assert scores[1] <= scores[0] * 1.005


def test_score_close_to_reference_router(tmp_path):
    """Same design as the reference run recorded in tests/golden/e2e_reference.json:
    evaluator total within 0.5%."""
    path = os.path.join(GOLDEN, "e2e_reference.json")
    if not os.path.exists(path):
        pytest.fail("e2e_reference.json missing (tests/golden/make_golden.py)")
    ref = json.load(open(path))
    for name, rec in ref.items():
        if "for_stat" not in rec or not rec["for_stat"]:
            continue
        cap, net, out = (str(tmp_path / (name + s)) for s in (".cap", ".net", ".out"))
        ig.generate_custom(rec["X"], rec["Y"], rec["nets"], seed=rec["seed"], cap_mode=0, block_frac=0.05,
                           pin_mode=0, bbox_median=8, bbox_sigma=1.0, cap=cap, net=net)
        ig.route_files(cap, net, out)
        mine = evaluate(cap, net, out)[3]
        theirs = float(rec["for_stat"].split()[4])
        assert mine <= theirs * 1.005, (name, mine, theirs)


def test_route_records_after_rerouting(tmp_path):
    """Records read back one net at a time after rip-up passes on the 256x256,
    20k-net configuration (the records are packed on the device before the
    copy): every record well formed, wires straight, vias on one GCell, and
    the same records from a second router."""
    cap, net = str(tmp_path / "c0.cap"), str(tmp_path / "c0.net")
    ig.generate(0, 3, 1.0, cap, net)
    X = Y = 256
    recs = []
    for _ in range(2):
        r = ig.Router(cap, net, rrr_iters=3)
        r.run()
        _, rn = r.sizes()
        recs.append([r.route(k) for k in range(rn)])
        assert r.stats()["dag_host_ms"] > 0  # rip-up passes rerouted nets
        r.close()
    assert all(np.array_equal(a, b) for a, b in zip(*recs))
    XY = X * Y
    for rec in recs[0]:
        assert rec[0] == len(rec) and rec[0] % 2 == 1
        a, b = rec[1::2], rec[2::2]
        xa, ya, xb, yb = a % XY // Y, a % Y, b % XY // Y, b % Y
        via = a // XY != b // XY
        assert np.all(~via | ((xa == xb) & (ya == yb)))
        assert np.all(via | (xa == xb) | (ya == yb))


@pytest.mark.parametrize("hook,values", [("HOOK_SHAPE_DEDUPE", (0, 1)), ("HOOK_COLOR_KEEP_MIN_NETS", (2000000, 1)),
                                         ("HOOK_DAG_STAGE_NODES", (0, 1024))])
def test_colouring_variants_give_the_same_routing(tmp_path, hook, values):
    """Conflict points and claims kept once per net or with every repetition,
    the round-0 claim map cleared per batch or kept up to date, and the DAG DP
    with its DAGs in global or in shared memory: the same phase-1 batches, and
    the same demand after three rip-up passes (whose colourings use the same
    variants).  The order of the nets inside a batch comes from an atomic
    scatter and does not matter (they share no state)."""
    cap, net = str(tmp_path / "d.cap"), str(tmp_path / "d.net")
    ig.generate(1, 5, 0.2, cap, net)
    res = []
    for v in values:
        ig.set_test_hook(getattr(ig, hook), v)
        try:
            r = ig.Router(cap, net, rrr_iters=3)
            r.run()
            p = r.plan()
            res.append((p["batch_off"], p["net_ids"], r.demand(), r.stats()["color_rounds"]))
            r.close()
        finally:
            ig.set_test_hook(ig.HOOK_RESET)
    (b0, i0, d0, c0), (b1, i1, d1, c1) = res
    assert np.array_equal(b0, b1)
    for b in range(len(b0) - 1):
        assert np.array_equal(np.sort(i0[b0[b]:b0[b + 1]]), np.sort(i1[b1[b]:b1[b + 1]])), f"batch {b}"
    assert np.array_equal(d0, d1)
    assert c0 == c1
