"""Host-side checks that need no GPU: the C ABI library, the .cap/.net reader
and pin selection against the reference's own front end, the Steiner
provider, the generator."""
import os
import re

import numpy as np
import pytest

import instantgr_b200 as ig
from conftest import GOLDEN, ROOT


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "instantgr_b200.h")).read()
    declared = set(re.findall(r"\b(igr_[a-z_0-9]+)\s*\(", hdr))
    L = ig.lib()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert declared == set(ig.EXPORTS)


def _load_front(path=os.path.join(GOLDEN, "front_pins.txt")):
    """Per net: pins in the reference's order, stacked-pin vias as pairs in order."""
    rows = []
    for line in open(path):
        a, b = line.rstrip("\n").split("|")
        ex = [int(v) for v in b.split()]
        rows.append(([int(v) for v in a.split()], list(zip(ex[0::2], ex[1::2]))))
    return rows


def _pin_mismatches(cap, net, ref):
    r = ig.Router(cap, net)
    dn, _ = r.sizes()
    assert dn == len(ref)
    bad = []
    for n in range(dn):
        pins, extra = r.pins(n)
        if (pins.tolist(), [tuple(e) for e in extra.tolist()]) != ref[n]:
            bad.append(n)
    r.close()
    return bad


def test_reader_and_pin_selection_match_reference():
    """db::read + net::init (src/database.hpp:38-415) vs the reference binary's
    output: the same pins in the same order (the iteration order of net::init's
    robin_hood sets, which also decides ties in the > 4-pin greedy) for every net."""
    ref = _load_front()
    bad = _pin_mismatches(os.path.join(GOLDEN, "front.cap"), os.path.join(GOLDEN, "front.net"), ref)
    assert not bad, f"nets {bad[:10]} differ from the reference"


REF_FRONT = os.path.join(ROOT, "oracle", "_ref", "ref_front")
GEN = os.path.join(ROOT, "instantgr_b200", "bin", "igr_generate")


@pytest.mark.skipif(not os.path.exists(REF_FRONT), reason="reference front end not built (oracle/_ref)")
@pytest.mark.parametrize("cfg,seed,scale", [(0, 3, 0.5), (1, 1, 0.05), (2, 1, 0.02)])
def test_pin_selection_matches_reference_on_generated_designs(tmp_path, cfg, seed, scale):
    """The same check live, through the reference's front end, on designs with
    high-fanout nets (65-500 pins) and the 2-1000-pin mixture."""
    import subprocess
    cap, net, out = (str(tmp_path / f) for f in ("d.cap", "d.net", "pins.txt"))
    subprocess.run([GEN, "--config", str(cfg), "--seed", str(seed), "--scale", str(scale), "--cap", cap, "--net", net],
                   check=True)
    subprocess.run([REF_FRONT, cap, net, out], check=True, capture_output=True)
    bad = _pin_mismatches(cap, net, _load_front(out))
    assert not bad, f"nets {bad[:10]} differ from the reference"


ROBIN_CHECK = os.path.join(ROOT, "oracle", "_ref", "robin_check")


@pytest.mark.skipif(not os.path.exists(ROBIN_CHECK), reason="robin_hood order check not built (oracle/_ref)")
def test_robin_hood_iteration_order_restatement():
    """instantgr_b200/csrc/robin_order.hpp against the reference's vendored
    robin_hood tables on seeded insertion sequences (growth, clear(), long
    probe runs that halve the info increment)."""
    import subprocess
    p = subprocess.run([ROBIN_CHECK], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and " 0 mismatches" in p.stdout, p.stdout[-500:]


def test_reader_rejects_malformed_files(tmp_path):
    cap = tmp_path / "bad.cap"
    cap.write_text("9 4 4\n1 2\n")
    net = tmp_path / "bad.net"
    net.write_text("n0\n(\n[(1, 0, 0)]\n)\n")
    with pytest.raises(ig.IgrError) as e:
        ig.Router(str(cap), str(net))
    assert e.value.code in (-3,)
    with pytest.raises(ig.IgrError) as e:
        ig.Router(str(tmp_path / "missing.cap"), str(net))
    assert e.value.code == -2


def _tree_ok(px, py, edges, pts):
    n = len(px)
    assert len(edges) == n - 1
    parent = list(range(n))

    def f(v):
        while parent[v] != v:
            v = parent[v]
        return v
    for a, b in edges:
        ra, rb = f(a), f(b)
        assert ra != rb, "cycle"
        parent[ra] = rb
    nodes = set(zip(px.tolist(), py.tolist()))
    assert set(pts) <= nodes
    return sum(abs(int(px[a]) - int(px[b])) + abs(int(py[a]) - int(py[b])) for a, b in edges)


def _mst_len(pts):
    n = len(pts)
    d = [1 << 60] * n
    d[0] = 0
    used = [False] * n
    tot = 0
    for _ in range(n):
        v = min((i for i in range(n) if not used[i]), key=lambda i: d[i])
        used[v] = True
        tot += d[v]
        for i in range(n):
            if not used[i]:
                d[i] = min(d[i], abs(pts[i][0] - pts[v][0]) + abs(pts[i][1] - pts[v][1]))
    return tot


@pytest.mark.parametrize("seed", range(6))
def test_steiner_provider_is_a_short_tree(seed):
    r = np.random.default_rng(seed)
    for k in (2, 3, 4, 7, 12, 40, 150):
        pts = sorted({(int(a), int(b)) for a, b in r.integers(0, 60, size=(k, 2))})
        x = np.array([p[0] for p in pts]); y = np.array([p[1] for p in pts])
        px, py, ed = ig.steiner(x, y)
        wl = _tree_ok(px, py, ed.tolist(), pts)
        assert wl <= _mst_len(pts)
        deg = np.bincount(ed.reshape(-1), minlength=len(px))
        assert (deg[len(pts):] >= 3).all(), "Steiner points have degree >= 3"
        # independent of input order
        perm = r.permutation(len(pts))
        qx, qy, qe = ig.steiner(x[perm], y[perm])
        assert (qx == px).all() and (qy == py).all() and (qe == ed).all()


def test_steiner_degree_three_is_flute_closed_form():
    # FLUTE's d=3 tree joins the three points at the median point (src/flute.hpp:1411-1434)
    px, py, ed = ig.steiner([0, 10, 4], [7, 3, 0])
    assert (4, 3) in set(zip(px.tolist(), py.tolist()))
    assert len(ed) == 3


def test_generator_is_deterministic(tmp_path):
    a = [str(tmp_path / f) for f in ("a.cap", "a.net")]
    b = [str(tmp_path / f) for f in ("b.cap", "b.net")]
    ig.generate(0, 7, 0.05, *a)
    ig.generate(0, 7, 0.05, *b)
    assert open(a[0], "rb").read() == open(b[0], "rb").read()
    assert open(a[1], "rb").read() == open(b[1], "rb").read()
    ig.generate(0, 8, 0.05, *b)
    assert open(a[1], "rb").read() != open(b[1], "rb").read()


def _scan_cap(text: str):
    """Sequential restatement of the .cap scanner (src/database.hpp:247-330):
    integers and reals are runs starting at a digit (reals also take dots),
    anything else between them is skipped; names run to the next blank."""
    p = 0
    n = len(text)

    def num(real):
        nonlocal p
        while p < n and not text[p].isdigit():
            p += 1
        if p >= n:
            raise ValueError("end of input")
        ans, scale = 0.0, 0.0
        while p < n and (text[p].isdigit() or (real and text[p] == ".")):
            if text[p] == ".":
                scale = 1.0
            else:
                scale *= 10
                ans = ans * 10 + int(text[p])
            p += 1
        return (ans if scale == 0 else ans / scale) if real else int(ans)

    def token():
        nonlocal p
        while p < n and text[p] in " \n":
            p += 1
        b = p
        while p < n and text[p] not in " \n":
            p += 1
        return text[b:p]

    L, X, Y = num(False), num(False), num(False)
    for _ in range(2 + L):
        num(True)
    for _ in range(X - 1 + Y - 1):
        num(False)
    cap = np.zeros((L, X, Y), np.float32)
    for lay in range(L):
        if token() != f"metal{lay + 1}":
            raise ValueError("layer name")
        num(False)
        num(True)
        for y in range(Y):
            for x in range(X):
                cap[lay, x, y] = np.float32(num(True))
    return cap


def _cap_text(r, X, Y, style):
    vals = r.integers(0, 40, size=(10, Y, X)) / r.choice([1, 2, 4, 8], size=(10, Y, X))
    out = [f"10 {X} {Y}\n1 4\n" + " ".join("0.5" for _ in range(10)) + "\n"]
    out.append(" ".join(str(int(v)) for v in r.integers(1, 4, X - 1)) + "\n")
    out.append(" ".join(str(int(v)) for v in r.integers(1, 4, Y - 1)) + "\n")
    for lay in range(10):
        out.append(f"metal{lay + 1} {lay % 2} 1.5\n")
        rows = []
        for y in range(Y):
            items = [f"{v:g}" if v != int(v) else str(int(v)) for v in vals[lay, y]]
            if style == 1:
                items = [("." + i[2:]) if i.startswith("0.") else i for i in items]  # ".5" reads as 5
                rows.append("  ".join(items) + " ")
            elif style == 2:
                rows.append(",\t".join(items))
            else:
                rows.append(" ".join(items))
        out.append((" " if style == 1 else "\n").join(rows) + "\n")
    return "".join(out)


@pytest.mark.parametrize("style", [0, 1, 2])
def test_capacity_reader_matches_the_sequential_scanner(tmp_path, style):
    """The capacity values are parsed in pieces on several threads; the result is
    the sequential scanner's for any spacing, separators and number forms."""
    r = np.random.default_rng(11 + style)
    X, Y = 97, 131
    text = _cap_text(r, X, Y, style)
    cap, net = tmp_path / "t.cap", tmp_path / "t.net"
    cap.write_text(text)
    net.write_text("n0\n(\n[(1, 0, 0)]\n[(1, 3, 4)]\n)\n")
    ref = _scan_cap(text)
    g = ig.Router(str(cap), str(net)).grid()
    assert np.array_equal(g["cap"].reshape(9, X, Y), ref[1:])


def test_capacity_reader_rejects_junk_before_a_layer_name(tmp_path):
    r = np.random.default_rng(5)
    text = _cap_text(r, 40, 30, 0).replace("\nmetal4 ", "\nx metal4 ", 1)
    cap, net = tmp_path / "t.cap", tmp_path / "t.net"
    cap.write_text(text)
    net.write_text("n0\n(\n[(1, 0, 0)]\n[(1, 3, 4)]\n)\n")
    with pytest.raises(ig.IgrError) as e:
        ig.Router(str(cap), str(net))
    assert e.value.code == -3


def test_router_refuses_to_write_or_evaluate_before_routing(tmp_path):
    """Writing guides or scoring needs a routed result; both fail with IGR_ERR_STATE
    (no GPU is needed to open a design or to get these errors)."""
    cap, net = str(tmp_path / "t.cap"), str(tmp_path / "t.net")
    ig.generate_custom(32, 32, 50, seed=3, cap_mode=0, block_frac=0.0, cap=cap, net=net)
    r = ig.Router(cap, net)
    with pytest.raises(ig.IgrError) as e:
        r.evaluate()
    assert e.value.code == -7
    with pytest.raises(ig.IgrError) as e:
        r.write(str(tmp_path / "t.out"))
    assert e.value.code == -7
    r.close()


@pytest.mark.parametrize("key,bad,good", [("HOOK_DAG_STAGE_NODES", (-1, 4097), (0, 4096)),
                                          ("HOOK_DAG_SPLIT_NETS", (0, -5), (1, 4096)),
                                          ("HOOK_WAIT_NS", (-1,), (0, 2_000_000_000))])
def test_test_hooks_check_their_ranges(key, bad, good):
    """Test hooks take values in their documented ranges and refuse others with
    IGR_ERR_INVALID, leaving the setting unchanged (no GPU is involved)."""
    try:
        for v in bad:
            with pytest.raises(ig.IgrError) as e:
                ig.set_test_hook(getattr(ig, key), v)
            assert e.value.code == ig.IGR_ERR_INVALID
        for v in good:
            ig.set_test_hook(getattr(ig, key), v)
    finally:
        ig.set_test_hook(ig.HOOK_RESET)
