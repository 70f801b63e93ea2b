"""Seeded inputs for the parity tests and the golden fixtures.

Grids of routing layers with integer capacities and half-unit demands, trees
in DFS preorder (the phase-1 DP input, src/Lshape_route.hpp:191-208) and
detour-style DAGs (corner alternatives for bent edges, split long edges;
the phase-2 DP input, src/Lshape_route_detour.hpp:911-1016).
"""
from __future__ import annotations

import numpy as np


def grid_case(seed: int, X: int = 40, Y: int = 30, L: int = 9, dir0: int = 0, unit_wire: float = 1.0,
              unit_via: float = 2.0, edge_len: int = 1, load: float = 1.0) -> dict:
    r = np.random.default_rng(seed)
    cap = r.integers(0, 9, size=(L, X, Y)).astype(np.float32)
    cap[r.random((L, X, Y)) < 0.05] = 0.0
    dem = (r.integers(0, 2 * 10, size=(L, X, Y)) * 0.5 * load).astype(np.float32)
    dem[r.random((L, X, Y)) < 0.4] = 0.0
    xlen = (r.integers(1, 3, size=X - 1) * edge_len).astype(np.int32)
    ylen = (r.integers(1, 3, size=Y - 1) * edge_len).astype(np.int32)
    short = np.round(r.uniform(0.5, 2.0, size=L), 3).astype(np.float64)
    return dict(L=L, X=X, Y=Y, DIR=dir0, xlen=xlen, ylen=ylen, unit_wire=unit_wire, unit_via=unit_via,
                short=short, cap=cap.reshape(-1), demand=dem.reshape(-1))


def _tree(r, g, k, steiner_p=0.4):
    X, Y = g["X"], g["Y"]
    w = int(min(X, r.integers(3, 24)))
    h = int(min(Y, r.integers(3, 24)))
    x0 = int(r.integers(0, X - w + 1))
    y0 = int(r.integers(0, Y - h + 1))
    seen = set()
    pts = []
    while len(pts) < k and len(seen) < w * h:
        p = (x0 + int(r.integers(0, w)), y0 + int(r.integers(0, h)))
        if p in seen:
            continue
        seen.add(p)
        pts.append(p)
    layers = [int(r.integers(0, 3)) for _ in pts]
    nodes = [(p[0], p[1], l) for p, l in zip(pts, layers)]
    edges = []
    for i in range(1, len(pts)):
        j = int(r.integers(0, i))
        px, py, _ = nodes[j]
        cx, cy, _ = nodes[i]
        if px != cx and py != cy and r.random() < steiner_p and (cx, py) not in seen:
            seen.add((cx, py))
            nodes.append((cx, py, 9))
            s = len(nodes) - 1
            edges += [(i, s), (s, j)]
        else:
            edges.append((i, j))
    # adjacency, then DFS preorder from node 0
    n = len(nodes)
    adj = [[] for _ in range(n)]
    for a, b in edges:
        adj[a].append(b)
        adj[b].append(a)
    order, opar = [], []
    idx = {}
    stack = [(0, -1)]
    while stack:
        v, p = stack.pop()
        idx[v] = len(order)
        order.append(v)
        opar.append(idx[p] if p >= 0 else -1)
        for e in reversed(adj[v]):
            if e != p:
                stack.append((e, v))
    XY = X * Y
    pos = [nodes[v][2] * XY + nodes[v][0] * Y + nodes[v][1] for v in order]
    return pos, opar, len(pts)


def tree_batch(g: dict, seed: int, n: int = 60, kmax: int = 8) -> dict:
    r = np.random.default_rng(seed)
    node_off, nodes, par, pins = [0], [], [], []
    for _ in range(n):
        k = int(r.integers(2, kmax + 1))
        pos, p, npins = _tree(r, g, k)
        nodes += pos
        par += p
        node_off.append(len(nodes))
        pins.append(npins)
    node_off = np.array(node_off, np.int32)
    cnt = np.diff(node_off)
    # route records: the reference's 12 ints per pin, raised so that no record can overflow
    slots = np.maximum(np.array(pins), (8 * cnt + 1 + 11) // 12).astype(np.int32)
    return dict(node_off=node_off, nodes=np.array(nodes, np.int32), par=np.array(par, np.int32),
                pins=slots, route_cap=(slots * 12).astype(np.int32),
                route_off=np.concatenate([[0], np.cumsum(slots * 12)[:-1]]).astype(np.int64))


def dag_from_tree(g: dict, r, pos, par, split_long=6):
    """Detour-style DAG of one preorder tree: bent edges get both corners as
    alternatives, long straight edges an optional midpoint."""
    X, Y = g["X"], g["Y"]
    XY = X * Y
    dn = [int(v) for v in pos]  # DAG nodes: tree nodes first
    parents = [[] for _ in dn]   # (parent, slot)
    slot_of = {}
    for i in range(1, len(pos)):
        p = par[i]
        s = slot_of.get(p, 0)
        slot_of[p] = s + 1
        px, py = pos[p] // Y % X, pos[p] % Y
        cx, cy = pos[i] // Y % X, pos[i] % Y
        if px != cx and py != cy:
            for mx, my in ((px, cy), (cx, py)):
                dn.append(9 * XY + mx * Y + my)
                parents.append([(p, s)])
                parents[i].append((len(dn) - 1, 0))
        elif abs(px - cx) + abs(py - cy) >= split_long and r.random() < 0.5:
            mx, my = (px + cx) // 2, (py + cy) // 2
            dn.append(9 * XY + mx * Y + my)
            parents.append([(p, s)])
            parents[i].append((len(dn) - 1, 0))
        else:
            parents[i].append((p, s))
    m = len(dn)
    child_num = [0] * m
    for v in range(m):
        for p, s in parents[v]:
            child_num[p] = max(child_num[p], s + 1)
    # depth = longest path from the root
    depth = [0] * m
    children = [[] for _ in range(m)]
    for v in range(m):
        for p, _ in parents[v]:
            children[p].append(v)
    indeg = [len(parents[v]) for v in range(m)]
    q = [v for v in range(m) if indeg[v] == 0]
    while q:
        v = q.pop()
        for c in children[v]:
            depth[c] = max(depth[c], depth[v] + 1)
            indeg[c] -= 1
            if indeg[c] == 0:
                q.append(c)
    return dn, parents, child_num, depth


def dag_batch(g: dict, seed: int, n: int = 40, kmax: int = 6) -> dict:
    r = np.random.default_rng(seed)
    tb = tree_batch(g, seed + 1000, n=n, kmax=kmax)
    node_off, nodes, depth, par_off, par, slot, child_num, pins = [0], [], [], [0], [], [], [], []
    for k in range(n):
        a, b = tb["node_off"][k], tb["node_off"][k + 1]
        pos = tb["nodes"][a:b].tolist()
        pp = tb["par"][a:b].tolist()
        dn, parents, cn, dep = dag_from_tree(g, r, pos, pp)
        base = len(nodes)
        nodes += dn
        depth += dep
        child_num += cn
        for v in range(len(dn)):
            for p, s in parents[v]:
                par.append(base + p)
                slot.append(s)
            par_off.append(len(par))
        node_off.append(len(nodes))
        pins.append(max(1, (8 * len(dn) + 1 + 99) // 100))
    pins = np.array(pins, np.int32)
    return dict(node_off=np.array(node_off, np.int32), nodes=np.array(nodes, np.int32),
                depth=np.array(depth, np.int32), par_off=np.array(par_off, np.int32),
                par=np.array(par, np.int32), child_slot=np.array(slot, np.int32),
                child_num=np.array(child_num, np.int32), pins=pins, route_cap=(pins * 100).astype(np.int32),
                route_off=np.concatenate([[0], np.cumsum(pins * 100)[:-1]]).astype(np.int64))


def color_case(seed: int, X: int = 64, Y: int = 48, n: int = 300):
    """Conflict shapes of n nets: points (2-D cells) and tree segments."""
    r = np.random.default_rng(seed)
    pt_off, pts, h_off, hs, v_off, vs = [0], [], [0], [], [0], []
    for _ in range(n):
        k = int(r.integers(2, 6))
        x0, y0 = int(r.integers(0, X - 8)), int(r.integers(0, Y - 8))
        p = sorted({(x0 + int(r.integers(0, 8)), y0 + int(r.integers(0, 8))) for _ in range(k)})
        for (x, y) in p:
            pts.append(x * Y + y)
        for (xa, ya), (xb, yb) in zip(p[:-1], p[1:]):
            hs += [min(xa, xb) * Y + ya, max(xa, xb) * Y + ya]
            vs += [xb * Y + min(ya, yb), xb * Y + max(ya, yb)]
        pt_off.append(len(pts))
        h_off.append(len(hs) // 2)
        v_off.append(len(vs) // 2)
    a = lambda v: np.array(v, np.int32)  # noqa: E731
    return a(pt_off), a(pts), a(h_off), a(hs), a(v_off), a(vs)


def write_harness_input(path: str, arrays) -> None:
    """Length-prefixed little-endian arrays, the input format of oracle/ref_harness.cu."""
    with open(path, "wb") as f:
        for a in arrays:
            a = np.ascontiguousarray(a)
            f.write(np.int64(a.size).tobytes())
            f.write(a.tobytes())


def read_harness_output(path: str, dtypes) -> list:
    out = []
    with open(path, "rb") as f:
        for dt in dtypes:
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            out.append(np.frombuffer(f.read(n * np.dtype(dt).itemsize), dt).copy())
    return out


def grid_arrays(g: dict):
    return [np.array([g["L"], g["X"], g["Y"], g["DIR"]], np.int32),
            np.array([g["unit_wire"], g["unit_via"]], np.float64), np.asarray(g["short"], np.float64),
            np.asarray(g["xlen"], np.int32), np.asarray(g["ylen"], np.int32), np.asarray(g["cap"], np.float32),
            np.asarray(g["demand"], np.float32)]


def dag_records_batch(ref, nets=None) -> dict:
    """Batch in the layout of dag_batch from flat detour-DAG records
    [m, nodes, par_num, child_num, depth, E, par, child_idx, npoints, points]
    (the output of igr_build_dag), nets in record order."""
    node_off, nodes, depth, par_off, par, slot, child_num = [0], [], [], [0], [], [], []
    p = 0
    k = 0
    while p < ref.size:
        m = int(ref[p])
        nd = ref[p + 1:p + 1 + m]
        pn = ref[p + 1 + m:p + 1 + 2 * m]
        cn = ref[p + 1 + 2 * m:p + 1 + 3 * m]
        dep = ref[p + 1 + 3 * m:p + 1 + 4 * m]
        E = int(ref[p + 1 + 4 * m])
        pr = ref[p + 2 + 4 * m:p + 2 + 4 * m + E]
        ci = ref[p + 2 + 4 * m + E:p + 2 + 4 * m + 2 * E]
        npt = int(ref[p + 2 + 4 * m + 2 * E])
        p += 3 + 4 * m + 2 * E + npt
        if nets is not None and k not in nets:
            k += 1
            continue
        k += 1
        base = len(nodes)
        nodes += nd.tolist()
        depth += dep.tolist()
        child_num += cn.tolist()
        q = 0
        for v in range(m):
            for _ in range(int(pn[v])):
                par.append(base + int(pr[q]))
                slot.append(int(ci[q]))
                q += 1
            par_off.append(len(par))
        node_off.append(len(nodes))
    node_off = np.array(node_off, np.int32)
    cap = (8 * np.diff(node_off) + 1).astype(np.int32)
    return dict(node_off=node_off, nodes=np.array(nodes, np.int32), depth=np.array(depth, np.int32),
                par_off=np.array(par_off, np.int32), par=np.array(par, np.int32),
                child_slot=np.array(slot, np.int32), child_num=np.array(child_num, np.int32), route_cap=cap,
                route_off=np.concatenate([[0], np.cumsum(cap)[:-1]]).astype(np.int64))
