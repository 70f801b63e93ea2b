"""ctypes binding of the CPU oracle (oracle/liboracle.so) — TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class Grid(C.Structure):
    _fields_ = [("L", C.c_int), ("X", C.c_int), ("Y", C.c_int), ("DIR", C.c_int),
                ("xlen", C.POINTER(C.c_int)), ("ylen", C.POINTER(C.c_int)),
                ("unit_wire", C.c_double), ("unit_via", C.c_double),
                ("short_cost", C.POINTER(C.c_double)), ("cap", C.POINTER(C.c_float))]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(HERE, f) for f in ("oracle.c", "seed_oracle.c")]
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(f) for f in srcs):
            build()
        L = C.CDLL(LIB)
        gp = C.POINTER(Grid)
        L.orc_cost_refresh.argtypes = [gp, _f32p, _f32p, _f32p, _f64p]
        L.orc_pattern_route.argtypes = [gp, _f32p, _f64p, C.c_int, _i32p, _i32p, _i32p, _i64p, _i32p, _i32p, _i32p,
                                        _i32p, C.c_int]
        L.orc_commit_wires.argtypes = [gp, _i32p, _f32p, _i32p, C.c_int]
        L.orc_commit_wires.restype = C.c_int64
        L.orc_commit_vias.argtypes = [gp, C.c_int, _i64p, _i32p, _f32p, _i32p, C.c_int, C.c_int]
        L.orc_commit_vias.restype = C.c_int64
        L.orc_ripup_wires.argtypes = [gp, C.c_int, _i64p, _i32p, _f32p, _i32p, C.c_int, C.c_int]
        L.orc_ripup_wires.restype = C.c_int64
        L.orc_mark_overflow.argtypes = [gp, _f32p, C.c_int, _i64p, _i32p, C.c_int, C.c_int, _u8p]
        L.orc_congestion_view.argtypes = [gp, _f32p, _f32p, _f32p]
        L.orc_overflow_cost.argtypes = [gp, _f32p]
        L.orc_overflow_cost.restype = C.c_double
        L.orc_color.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, C.c_int, _i32p]
        L.orc_dag_route.argtypes = [gp, _f32p, _f64p, C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p,
                                    _i64p, _i32p, _i32p, _i32p, _i32p, C.c_int]
        L.orc_seed_params.restype = C.c_int
        L.orc_seed_grad.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p, C.c_int]
        L.orc_seed_grad.restype = C.c_double
        _lib = L
    return _lib


def seed_grad(x, target, params, halo, rounded=True):
    """Loss and parameter gradient of the congestion-seed network (seed_oracle.c),
    tiles [T][S][S][16]; `rounded` rounds to BF16 where the GPU stores BF16."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    p = np.ascontiguousarray(params, dtype=np.float32)
    g = np.zeros(lib().orc_seed_params(), np.float32)
    loss = lib().orc_seed_grad(x.shape[0], x.shape[1], halo, x.reshape(-1), t.reshape(-1), p, g, 1 if rounded else 0)
    return loss, g


SEED_LAYERS = [(16, 32), (32, 64), (64, 64), (64, 64), (64, 32), (32, 16)]  # (cin, cout) of the six convolutions


def seed_slices():
    """(weight slice, bias slice) of each layer in the flat parameter vector."""
    out, o = [], 0
    for ci, co in SEED_LAYERS:
        nw = co * 9 * ci
        out.append((slice(o, o + nw), slice(o + nw, o + nw + co)))
        o += nw + co
    return out


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Oracle:
    """Grid-bound oracle calls; `g` is a case dict (tests/cases.py)."""

    def __init__(self, g: dict):
        self.g = g
        self._keep = [_i32(g["xlen"]), _i32(g["ylen"]), np.ascontiguousarray(g["short"], dtype=np.float64),
                      np.ascontiguousarray(g["cap"], dtype=np.float32).reshape(-1)]
        self.s = Grid(g["L"], g["X"], g["Y"], g["DIR"], self._keep[0].ctypes.data_as(C.POINTER(C.c_int)),
                      self._keep[1].ctypes.data_as(C.POINTER(C.c_int)), g["unit_wire"], g["unit_via"],
                      self._keep[2].ctypes.data_as(C.POINTER(C.c_double)),
                      self._keep[3].ctypes.data_as(C.POINTER(C.c_float)))
        self.N = g["L"] * g["X"] * g["Y"]

    def cost_refresh(self, demand):
        w = np.zeros(self.N, np.float32)
        v = np.zeros(self.N, np.float32)
        p = np.zeros(self.N, np.float64)
        lib().orc_cost_refresh(C.byref(self.s), np.ascontiguousarray(demand, np.float32).reshape(-1), w, v, p)
        return w, v, p

    def pattern_route(self, vcost, presum, node_off, nodes, par, route_off, route_cap, routes, pre, stamps, stamp):
        rc = lib().orc_pattern_route(C.byref(self.s), vcost, presum, len(route_off), _i32(node_off), _i32(nodes),
                                     _i32(par), np.ascontiguousarray(route_off, np.int64), _i32(route_cap), routes,
                                     pre, stamps, stamp)
        return rc

    def commit_wires(self, pre, demand, stamps, stamp):
        return lib().orc_commit_wires(C.byref(self.s), pre, demand, stamps, stamp)

    def commit_vias(self, route_off, routes, demand, stamps, stamp, K=1):
        return lib().orc_commit_vias(C.byref(self.s), len(route_off), np.ascontiguousarray(route_off, np.int64),
                                     _i32(routes), demand, stamps, stamp, K)

    def ripup_wires(self, route_off, routes, demand, stamps, stamp, K=-1):
        return lib().orc_ripup_wires(C.byref(self.s), len(route_off), np.ascontiguousarray(route_off, np.int64),
                                     _i32(routes), demand, stamps, stamp, K)

    def mark_overflow(self, demand, route_off, routes, threshold=0, min_edges=10):
        o = np.zeros(len(route_off), np.uint8)
        lib().orc_mark_overflow(C.byref(self.s), np.ascontiguousarray(demand, np.float32).reshape(-1),
                                len(route_off), np.ascontiguousarray(route_off, np.int64), _i32(routes), threshold,
                                min_edges, o)
        return o

    def congestion_view(self, demand):
        xy = self.g["X"] * self.g["Y"]
        xs = np.zeros(xy, np.float32)
        ys = np.zeros(xy, np.float32)
        lib().orc_congestion_view(C.byref(self.s), np.ascontiguousarray(demand, np.float32).reshape(-1), xs, ys)
        return xs, ys

    def overflow_cost(self, demand):
        return lib().orc_overflow_cost(C.byref(self.s), np.ascontiguousarray(demand, np.float32).reshape(-1))

    def dag_route(self, vcost, presum, d, route_off, route_cap, routes, pre, stamps, stamp):
        return lib().orc_dag_route(C.byref(self.s), vcost, presum, len(route_off), _i32(d["node_off"]),
                                   _i32(d["nodes"]), _i32(d["depth"]), _i32(d["par_off"]), _i32(d["par"]),
                                   _i32(d["child_slot"]), _i32(d["child_num"]),
                                   np.ascontiguousarray(route_off, np.int64), _i32(route_cap), routes, pre, stamps,
                                   stamp)


def color(X, Y, pt_off, pts, h_off, hseg, v_off, vseg, sparsity=15):
    n = len(pt_off) - 1
    out = np.zeros(max(n, 1), np.int32)
    nb = lib().orc_color(X, Y, n, _i32(pt_off), _i32(pts), _i32(h_off), _i32(hseg), _i32(v_off), _i32(vseg),
                         sparsity, out)
    return out[:n], nb
