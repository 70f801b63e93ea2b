"""instantgr_b200: B200-native GPU global router, a drop-in for InstantGR's hot path.

Python access to the C ABI of include/instantgr_b200.h (libigr_b200.so, built
in-tree by instantgr_b200/build.py).  The native library is required: there
is no CPU fallback, and importing an operator without it raises.

Two levels, as in the C ABI:
  * Router / route_files: the `-cap/-net/-out` flow of InstantGR.
  * Ctx: the device operators of the hot path (cost refresh, tree DP, commit,
    rip-up marking, congestion view, colouring, DAG DP) on one grid.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libigr_b200.so")
ROUTE_BIN = os.path.join(_HERE, "bin", "igr_route")

IGR_OK = 0
IGR_ERR_INVALID, IGR_ERR_CAPACITY, IGR_ERR_STATE = -1, -5, -7
ERRORS = {-1: "INVALID", -2: "IO", -3: "FORMAT", -4: "CUDA", -5: "CAPACITY", -6: "TIMEOUT", -7: "STATE"}

_lib: Optional[C.CDLL] = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")

# every symbol of include/instantgr_b200.h
EXPORTS = [
    "igr_default_options", "igr_route_files", "igr_router_open", "igr_router_run", "igr_router_write",
    "igr_router_evaluate",
    "igr_router_stats", "igr_router_kstats", "igr_router_sizes", "igr_router_route", "igr_router_pins",
    "igr_router_demand", "igr_router_close", "igr_router_plan", "igr_router_grid", "igr_set_device",
    "igr_generate", "igr_generate_custom", "igr_create", "igr_destroy", "igr_last_error", "igr_set_demand",
    "igr_get_demand", "igr_get_stamp", "igr_get_pre", "igr_cost_refresh", "igr_get_costs", "igr_set_costs", "igr_dump_state", "igr_load_state",
    "igr_pattern_route", "igr_pattern_route_static", "igr_commit_wires", "igr_commit_vias", "igr_ripup_wires",
    "igr_mark_overflow",
    "igr_congestion_view", "igr_score", "igr_color_batches", "igr_dag_route", "igr_build_dag", "igr_build_dags",
    "igr_steiner",
    "igr_seed_create", "igr_seed_destroy", "igr_seed_last_error", "igr_seed_set_tile", "igr_seed_params",
    "igr_seed_set_params", "igr_seed_features", "igr_seed_features_device", "igr_seed_add_map", "igr_seed_add_routed", "igr_seed_train",
    "igr_seed_eval", "igr_seed_predict", "igr_seed_time_forward", "igr_seed_grad", "igr_router_set_seed", "igr_router_seed_stats",
    "igr_test_hook",
]


class Options(C.Structure):
    _fields_ = [("rrr_iters", C.c_int), ("threads", C.c_int), ("mode", C.c_int), ("verbose", C.c_int),
                ("batched", C.c_int), ("profile", C.c_int), ("split_commit", C.c_int),
                ("host_dags", C.c_int), ("reserved", C.c_int * 5)]


class GridDesc(C.Structure):
    _fields_ = [("L", C.c_int32), ("X", C.c_int32), ("Y", C.c_int32), ("dir0", C.c_int32),
                ("x_edge_len", C.POINTER(C.c_int32)), ("y_edge_len", C.POINTER(C.c_int32)),
                ("unit_wire", C.c_double), ("unit_via", C.c_double), ("short_cost", C.POINTER(C.c_double)),
                ("capacity", C.POINTER(C.c_float))]


class IgrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"igr error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Loads libigr_b200.so; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"native library missing: {LIB_PATH} (run python instantgr_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.igr_last_error.restype = C.c_char_p
    L.igr_last_error.argtypes = [vp]
    L.igr_default_options.argtypes = [C.POINTER(Options)]
    L.igr_route_files.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(Options)]
    L.igr_router_open.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(Options), C.POINTER(vp)]
    L.igr_router_run.argtypes = [vp]
    L.igr_router_write.argtypes = [vp, C.c_char_p]
    L.igr_router_evaluate.argtypes = [vp, C.c_void_p, C.c_void_p]
    L.igr_router_stats.argtypes = [vp, _f64p, C.c_int]
    L.igr_router_kstats.argtypes = [vp, _f64p, C.c_int]
    L.igr_router_plan.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.igr_router_grid.argtypes = [vp, vp, vp, vp, vp, vp]
    L.igr_set_device.argtypes = [C.c_int]
    L.igr_router_sizes.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.igr_router_route.argtypes = [vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int)]
    L.igr_router_demand.argtypes = [vp, _f32p]
    L.igr_router_pins.argtypes = [vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int)]
    L.igr_router_close.argtypes = [vp]
    L.igr_router_close.restype = None
    L.igr_generate.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_char_p, C.c_char_p]
    L.igr_generate_custom.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_double, C.c_int,
                                      C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, C.c_char_p,
                                      C.c_char_p]
    L.igr_create.argtypes = [C.POINTER(GridDesc), C.POINTER(vp)]
    L.igr_destroy.argtypes = [vp]
    L.igr_set_demand.argtypes = [vp, _f32p]
    L.igr_get_demand.argtypes = [vp, _f32p]
    L.igr_get_stamp.argtypes = [vp, _i32p]
    L.igr_get_pre.argtypes = [vp, _i32p]
    L.igr_cost_refresh.argtypes = [vp, C.c_int]
    L.igr_get_costs.argtypes = [vp, _f32p, _f64p]
    L.igr_set_costs.argtypes = [vp, _f32p, _f64p]
    L.igr_dump_state.argtypes = [vp, C.c_char_p]
    L.igr_load_state.argtypes = [vp, C.c_char_p]
    L.igr_pattern_route.argtypes = [vp, C.c_int, _i32p, _i32p, _i32p, _i64p, _i32p, _i32p, C.c_int32]
    L.igr_pattern_route_static.argtypes = [vp, C.c_int, vp, C.c_int64, vp, vp, vp, vp, vp, C.c_int64, C.c_int32]
    L.igr_commit_wires.argtypes = [vp, C.c_int32]
    L.igr_commit_vias.argtypes = [vp, C.c_int, _i64p, _i32p, C.c_int32, C.c_int32]
    L.igr_ripup_wires.argtypes = [vp, C.c_int, _i64p, _i32p, C.c_int32, C.c_int32]
    L.igr_mark_overflow.argtypes = [vp, C.c_int, _i64p, _i32p, C.c_int32, C.c_int32, _u8p]
    L.igr_congestion_view.argtypes = [vp, _f32p, _f32p]
    L.igr_score.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.igr_color_batches.argtypes = [vp, C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, C.c_int32, _i32p,
                                    C.POINTER(C.c_int32)]
    L.igr_dag_route.argtypes = [vp, C.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i64p, _i32p,
                                _i32p, C.c_int32]
    L.igr_build_dag.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _i32p, _f32p, _f32p, _i32p,
                                C.c_int64, C.POINTER(C.c_int64)]
    L.igr_build_dags.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _i32p, _i32p, _f32p, _f32p,
                                 vp, C.c_int64, _i64p, C.POINTER(C.c_int64)]
    L.igr_steiner.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i32p, C.c_int, C.POINTER(C.c_int), _i32p,
                              C.c_int, C.POINTER(C.c_int)]
    L.igr_router_set_seed.argtypes = [vp, vp, C.c_double, C.c_int, C.c_int, C.c_int]
    L.igr_router_seed_stats.argtypes = [vp, _f64p, C.c_int]
    L.igr_seed_create.argtypes = [C.c_uint64, C.POINTER(vp)]
    L.igr_seed_destroy.argtypes = [vp]
    L.igr_seed_last_error.restype = C.c_char_p
    L.igr_seed_last_error.argtypes = [vp]
    L.igr_seed_set_tile.argtypes = [vp, C.c_int, C.c_int]
    L.igr_seed_params.argtypes = [vp, vp, C.c_int64, C.POINTER(C.c_int64)]
    L.igr_seed_set_params.argtypes = [vp, _f32p, C.c_int64]
    L.igr_seed_features.argtypes = [vp, _f32p]
    L.igr_seed_features_device.argtypes = [vp, _f32p]
    L.igr_seed_add_map.argtypes = [vp, C.c_int, C.c_int, _f32p, _f32p, C.POINTER(C.c_int32)]
    L.igr_seed_add_routed.argtypes = [vp, vp, C.POINTER(C.c_int32)]
    L.igr_seed_train.argtypes = [vp, C.c_int, C.c_int, C.c_float, C.c_uint64, C.c_int, vp]
    L.igr_seed_eval.argtypes = [vp, C.c_int, _f64p, C.c_int]
    L.igr_seed_predict.argtypes = [vp, C.c_int, C.c_int, _f32p, _f32p]
    L.igr_seed_time_forward.argtypes = [vp, C.c_int, C.c_int, _f64p, _f64p]
    L.igr_seed_grad.argtypes = [vp, C.c_int, _f32p, _f32p, C.POINTER(C.c_double), vp]
    L.igr_test_hook.argtypes = [C.c_int, C.c_int64]
    _lib = L
    return L


def _check(rc: int, ctx=None) -> None:
    if rc != IGR_OK:
        msg = lib().igr_last_error(ctx).decode(errors="replace")
        raise IgrError(rc, msg)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


(HOOK_RESET, HOOK_WAIT_NS, HOOK_BARRIER_PHANTOM, HOOK_MBAR_PROBE, HOOK_COLOR_KEEP_MAP, HOOK_DAG_SPLIT_NETS,
 HOOK_COLOR_KEEP_MIN_NETS, HOOK_SHAPE_DEDUPE, HOOK_DAG_STAGE_NODES) = range(9)


def set_test_hook(key: int, value: int = 0) -> None:
    """Process-wide test hook (igr_test_hook); HOOK_RESET restores every default."""
    _check(lib().igr_test_hook(key, value))


def set_device(device: int) -> None:
    """CUDA device of the calling thread for the library's calls."""
    _check(lib().igr_set_device(device))


def default_options(**kw) -> Options:
    o = Options()
    lib().igr_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def route_files(cap: str, net: str, out: str, **kw) -> None:
    """`InstantGR -cap <cap> -net <net> -out <out>` (src/main.cpp:91-102)."""
    o = default_options(**kw)
    _check(lib().igr_route_files(cap.encode(), net.encode(), out.encode(), C.byref(o)))


def generate(cfg: int, seed: int, scale: float, cap: str, net: str) -> None:
    _check(lib().igr_generate(cfg, seed, scale, cap.encode(), net.encode()))


def generate_custom(X, Y, nets, seed=1, cap_mode=0, block_frac=0.05, pin_mode=0, hifanout_frac=0.0,
                    bbox_median=8.0, bbox_sigma=1.0, hotspots=0, hotspot_frac=0.0, cap="d.cap", net="d.net"):
    _check(lib().igr_generate_custom(X, Y, nets, seed, cap_mode, block_frac, pin_mode, hifanout_frac, bbox_median,
                                     bbox_sigma, hotspots, hotspot_frac, cap.encode(), net.encode()))


# limits of igr_pattern_route_static (IGR_STATIC_SCRATCH_BYTES, IGR_STATIC_MAX_NETS)
STATIC_SCRATCH_BYTES = 64 << 20
STATIC_MAX_NETS = 1 << 20
SEED_CONVS = 6  # convolutions of the learned seed (IGR_SEED_CONVS)

KERNEL_CLASSES = ["cost_refresh", "pattern_dp", "wire_commit", "via_commit", "dag_dp", "coloring", "ripup",
                  "phase1_graph", "commit_refresh"]

STATS = ["routing_nets", "rerouted", "wirelength", "via_cost", "overflow_cost", "route_s", "batches1", "p1_ms",
         "rrr_ms", "dag_host_ms", "launches", "design_nets", "color_rounds", "h2d_bytes", "d2h_bytes",
         "setup_h2d_bytes"]


class Router:
    """Stage-by-stage router over one design (igr_router_*)."""

    def __init__(self, cap: str, net: str, **kw):
        self.h = C.c_void_p()
        o = default_options(**kw)
        _check(lib().igr_router_open(cap.encode(), net.encode(), C.byref(o), C.byref(self.h)))

    def run(self) -> None:
        _check(lib().igr_router_run(self.h))

    def write(self, out: str) -> None:
        _check(lib().igr_router_write(self.h, out.encode()))

    def evaluate(self) -> dict:
        """Scores the last run on the device with the ISPD2024 evaluator's rules
        (the FOR_STAT values before rounding, and the overflow loss per layer)."""
        out = np.zeros(4, np.float64)
        layers = np.zeros(9, np.float64)
        _check(lib().igr_router_evaluate(self.h, out.ctypes.data_as(C.c_void_p), layers.ctypes.data_as(C.c_void_p)))
        return dict(wirelength=float(out[0]), via=float(out[1]), overflow=float(out[2]), total=float(out[3]),
                    layer_loss=layers)

    def stats(self) -> dict:
        v = np.zeros(len(STATS), dtype=np.float64)
        _check(lib().igr_router_stats(self.h, v, len(STATS)))
        return dict(zip(STATS, v.tolist()))

    def kstats(self) -> dict:
        v = np.zeros(3 * len(KERNEL_CLASSES), dtype=np.float64)
        _check(lib().igr_router_kstats(self.h, v, len(v)))
        return {k: dict(launches=int(v[3 * i]), ms=float(v[3 * i + 1]), bytes=float(v[3 * i + 2]))
                for i, k in enumerate(KERNEL_CLASSES)}

    def plan(self) -> dict:
        """Phase-1 routing order, batches and trees of the last run."""
        s = np.zeros(3, dtype=np.int64)
        L = lib()
        nul = None
        _check(L.igr_router_plan(self.h, s.ctypes.data_as(C.c_void_p), nul, nul, nul, nul, nul, nul))
        n, b, m = (int(v) for v in s)
        ids, boff = np.zeros(n, np.int32), np.zeros(b + 1, np.int32)
        noff, nodes, par, cap = np.zeros(n + 1, np.int32), np.zeros(m, np.int32), np.zeros(m, np.int32), \
            np.zeros(n, np.int32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _check(L.igr_router_plan(self.h, p(s), p(ids), p(boff), p(noff), p(nodes), p(par), p(cap)))
        return dict(net_ids=ids, batch_off=boff, node_off=noff, nodes=nodes, par=par, route_cap=cap)

    def grid(self) -> dict:
        """Grid of the design as a case dict (tests/cases.py layout)."""
        hdr = np.zeros(4, np.int32)
        L = lib()
        _check(L.igr_router_grid(self.h, hdr.ctypes.data_as(C.c_void_p), None, None, None, None))
        Lr, X, Y, d0 = (int(v) for v in hdr)
        costs = np.zeros(2 + Lr, np.float64)
        xl, yl = np.zeros(X - 1, np.int32), np.zeros(Y - 1, np.int32)
        cap = np.zeros(Lr * X * Y, np.float32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _check(L.igr_router_grid(self.h, p(hdr), p(costs), p(xl), p(yl), p(cap)))
        return dict(L=Lr, X=X, Y=Y, DIR=d0, xlen=xl, ylen=yl, unit_wire=float(costs[0]), unit_via=float(costs[1]),
                    short=costs[2:].copy(), cap=cap, demand=np.zeros_like(cap))

    def demand(self) -> np.ndarray:
        """Device demand of the routing layers after the last run, [l][x][y]."""
        hdr = np.zeros(4, np.int32)
        _check(lib().igr_router_grid(self.h, hdr.ctypes.data_as(C.c_void_p), None, None, None, None))
        out = np.zeros(int(hdr[0]) * int(hdr[1]) * int(hdr[2]), np.float32)
        _check(lib().igr_router_demand(self.h, out))
        return out

    def set_seed(self, model, alpha: float = 1.0, mode: int = 1, kind: int = 1, levels: int = 4) -> None:
        """Attach a learned congestion seed (igr_router_set_seed); mode 0 detaches."""
        self._seed = model
        _check(lib().igr_router_set_seed(self.h, model.h if model is not None else None, alpha, mode, kind, levels),
               self.h)

    def seed_stats(self) -> dict:
        v = np.zeros(4, np.float64)
        _check(lib().igr_router_seed_stats(self.h, v, 4))
        return dict(seed_kept=bool(v[0]), seeded_score=v[1], plain_score=v[2], predict_ms=v[3])

    def sizes(self):
        a, b = C.c_int64(), C.c_int64()
        _check(lib().igr_router_sizes(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def route(self, net: int) -> np.ndarray:
        n = C.c_int()
        _check(lib().igr_router_route(self.h, net, None, 0, C.byref(n)))
        out = np.zeros(n.value, dtype=np.int32)
        _check(lib().igr_router_route(self.h, net, out.ctypes.data_as(C.c_void_p), n.value, C.byref(n)))
        return out

    def pins(self, net: int):
        """(pins, extra vias) chosen for design net `net`."""
        n = C.c_int()
        _check(lib().igr_router_pins(self.h, net, None, 0, C.byref(n)))
        out = np.zeros(n.value, dtype=np.int32)
        _check(lib().igr_router_pins(self.h, net, out.ctypes.data_as(C.c_void_p), n.value, C.byref(n)))
        k = int(out[0])
        pins = out[1:1 + k]
        e = int(out[1 + k])
        extra = out[2 + k:2 + k + 2 * e].reshape(-1, 2)
        return pins, extra

    def close(self) -> None:
        if self.h:
            lib().igr_router_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ctx:
    """Device state of one grid and the hot-path operators on it (igr_create ...)."""

    def __init__(self, L, X, Y, dir0, xlen, ylen, unit_wire, unit_via, short_cost, cap):
        self._keep = [_i32(xlen), _i32(ylen), np.ascontiguousarray(short_cost, dtype=np.float64),
                      np.ascontiguousarray(cap, dtype=np.float32).reshape(-1)]
        d = GridDesc(L, X, Y, dir0, self._keep[0].ctypes.data_as(C.POINTER(C.c_int32)),
                     self._keep[1].ctypes.data_as(C.POINTER(C.c_int32)), unit_wire, unit_via,
                     self._keep[2].ctypes.data_as(C.POINTER(C.c_double)),
                     self._keep[3].ctypes.data_as(C.POINTER(C.c_float)))
        self.L, self.X, self.Y, self.N = L, X, Y, L * X * Y
        self.h = C.c_void_p()
        _check(lib().igr_create(C.byref(d), C.byref(self.h)))

    def _c(self, rc):
        _check(rc, self.h)

    def close(self):
        if self.h:
            lib().igr_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_demand(self, dem):
        self._c(lib().igr_set_demand(self.h, np.ascontiguousarray(dem, dtype=np.float32).reshape(-1)))

    def demand(self):
        o = np.zeros(self.N, dtype=np.float32)
        self._c(lib().igr_get_demand(self.h, o))
        return o

    def stamps(self):
        o = np.zeros(self.N, dtype=np.int32)
        self._c(lib().igr_get_stamp(self.h, o))
        return o

    def pre(self):
        o = np.zeros(self.N, dtype=np.int32)
        self._c(lib().igr_get_pre(self.h, o))
        return o

    def cost_refresh(self, only_dirty=False):
        self._c(lib().igr_cost_refresh(self.h, 1 if only_dirty else 0))

    def costs(self):
        v = np.zeros(self.N, dtype=np.float32)
        p = np.zeros(self.N, dtype=np.float64)
        self._c(lib().igr_get_costs(self.h, v, p))
        return v, p

    def dump_state(self, path: str):
        """Demand, costs, stamps and difference array to a file (igr_dump_state)."""
        self._c(lib().igr_dump_state(self.h, str(path).encode()))

    def load_state(self, path: str):
        """Grid state from a file of igr_dump_state (same grid size)."""
        self._c(lib().igr_load_state(self.h, str(path).encode()))

    def set_costs(self, vcost, presum):
        self._c(lib().igr_set_costs(self.h, np.ascontiguousarray(vcost, dtype=np.float32).reshape(-1),
                                    np.ascontiguousarray(presum, dtype=np.float64).reshape(-1)))

    def pattern_route(self, node_off, nodes, par, route_off, route_cap, routes, stamp):
        self._c(lib().igr_pattern_route(self.h, len(route_off), _i32(node_off), _i32(nodes), _i32(par),
                                        _i64(route_off), _i32(route_cap), routes, stamp))
        return routes

    def pattern_route_static(self, n, node_off, total_nodes, nodes, par, route_off, route_cap, routes,
                             routes_len, stamp):
        """Tree DP over caller-owned DEVICE arrays (integer device addresses),
        with its scratch in the library's fixed device array: no allocation
        (igr_pattern_route_static)."""
        self._c(lib().igr_pattern_route_static(self.h, n, node_off, total_nodes, nodes, par, route_off, route_cap,
                                               routes, routes_len, stamp))

    def commit_wires(self, stamp):
        self._c(lib().igr_commit_wires(self.h, stamp))

    def commit_vias(self, route_off, routes, stamp, K=1):
        self._c(lib().igr_commit_vias(self.h, len(route_off), _i64(route_off), _i32(routes), stamp, K))

    def ripup_wires(self, route_off, routes, stamp, K=-1):
        self._c(lib().igr_ripup_wires(self.h, len(route_off), _i64(route_off), _i32(routes), stamp, K))

    def mark_overflow(self, route_off, routes, threshold=0, min_edges=10):
        o = np.zeros(len(route_off), dtype=np.uint8)
        self._c(lib().igr_mark_overflow(self.h, len(route_off), _i64(route_off), _i32(routes), threshold,
                                        min_edges, o))
        return o

    def congestion_view(self):
        xs = np.zeros(self.X * self.Y, dtype=np.float32)
        ys = np.zeros(self.X * self.Y, dtype=np.float32)
        self._c(lib().igr_congestion_view(self.h, xs, ys))
        return xs, ys

    def score(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self._c(lib().igr_score(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def color_batches(self, pt_off, pts, h_off, hseg, v_off, vseg, sparsity=15):
        n = len(pt_off) - 1
        out = np.zeros(max(n, 1), dtype=np.int32)
        nb = C.c_int32()
        self._c(lib().igr_color_batches(self.h, n, _i32(pt_off), _i32(pts), _i32(h_off), _i32(hseg),
                                        _i32(v_off), _i32(vseg), sparsity, out, C.byref(nb)))
        return out[:n], nb.value

    def dag_route(self, node_off, nodes, depth, par_off, par, child_slot, child_num, route_off, route_cap, routes,
                  stamp):
        self._c(lib().igr_dag_route(self.h, len(route_off), _i32(node_off), _i32(nodes), _i32(depth),
                                    _i32(par_off), _i32(par), _i32(child_slot), _i32(child_num), _i64(route_off),
                                    _i32(route_cap), routes, stamp))
        return routes


def build_dags(X, Y, mode, tree_off, pos, adj_off, adj, xsum, ysum):
    """Detour DAGs of many trees built on the device (igr_build_dags); returns the
    records of build_dag end to end and their offsets [n+1]."""
    tree_off, pos, adj_off, adj = _i32(tree_off), _i32(pos), _i32(adj_off), _i32(adj)
    xs = np.ascontiguousarray(xsum, dtype=np.float32)
    ys = np.ascontiguousarray(ysum, dtype=np.float32)
    n = len(tree_off) - 1
    rec_off = np.zeros(n + 1, dtype=np.int64)
    total = C.c_int64()
    _check(lib().igr_build_dags(X, Y, mode, n, tree_off, pos, adj_off, adj, xs, ys, None, 0, rec_off,
                                C.byref(total)))
    out = np.zeros(max(total.value, 1), dtype=np.int32)
    _check(lib().igr_build_dags(X, Y, mode, n, tree_off, pos, adj_off, adj, xs, ys,
                                out.ctypes.data_as(C.c_void_p), total.value, rec_off, C.byref(total)))
    return out[: total.value], rec_off


def build_dag(X, Y, mode, pos, adj_off, adj, xsum, ysum):
    """Detour DAG of one tree (host, net::generate_detours_reconstruct); returns the
    flat record [m, nodes, par_num, child_num, depth, E, par, child_idx, npoints, points]."""
    pos, adj_off, adj = _i32(pos), _i32(adj_off), _i32(adj)
    xs = np.ascontiguousarray(xsum, dtype=np.float32)
    ys = np.ascontiguousarray(ysum, dtype=np.float32)
    n = C.c_int64()
    cap = 1 << 16
    while True:
        out = np.zeros(cap, dtype=np.int32)
        _check(lib().igr_build_dag(X, Y, mode, len(pos), pos, adj_off, adj, xs, ys, out, cap, C.byref(n)))
        if n.value <= cap:
            return out[: n.value]
        cap = n.value


def steiner(x, y):
    """Steiner provider: returns (node x, node y, edges [m,2], npins)."""
    x, y = _i32(x), _i32(y)
    n = len(x)
    cap = 2 * n + 2
    nx = np.zeros(cap, dtype=np.int32)
    ny = np.zeros(cap, dtype=np.int32)
    ed = np.zeros(2 * cap, dtype=np.int32)
    nn, ne = C.c_int(), C.c_int()
    _check(lib().igr_steiner(n, x, y, nx, ny, cap, C.byref(nn), ed, cap, C.byref(ne)))
    return nx[: nn.value], ny[: nn.value], ed[: 2 * ne.value].reshape(-1, 2)


SEED_MODEL_PATH = os.path.join(_HERE, "data", "congestion_seed.npz")


class Seed:
    """Learned congestion seed (igr_seed_*): BF16 convolutional demand predictor
    trained and run on the tcgen05 tensor cores."""

    @classmethod
    def load(cls, path: str = SEED_MODEL_PATH) -> "Seed":
        """The model of a parameter file written by train_seed (default: the shipped model)."""
        return cls(1, params=np.load(path)["params"])

    def __init__(self, init_seed: int = 1, params=None):
        self.h = C.c_void_p()
        self._c(lib().igr_seed_create(init_seed, C.byref(self.h)))
        if params is not None:
            self.set_params(params)

    def _c(self, rc):
        if rc != IGR_OK:
            raise IgrError(rc, lib().igr_seed_last_error(self.h).decode(errors="replace"))

    def close(self):
        if self.h:
            lib().igr_seed_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tile(self, size: int, halo: int):
        self._c(lib().igr_seed_set_tile(self.h, size, halo))

    def params(self) -> np.ndarray:
        n = C.c_int64()
        self._c(lib().igr_seed_params(self.h, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._c(lib().igr_seed_params(self.h, out.ctypes.data_as(C.c_void_p), n.value, C.byref(n)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._c(lib().igr_seed_set_params(self.h, p, p.size))

    def add_map(self, features, target) -> int:
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        X, Y = f.shape[0], f.shape[1]
        i = C.c_int32()
        self._c(lib().igr_seed_add_map(self.h, X, Y, f.reshape(-1), t.reshape(-1), C.byref(i)))
        return i.value

    def add_routed(self, router: "Router") -> int:
        i = C.c_int32()
        self._c(lib().igr_seed_add_routed(self.h, router.h, C.byref(i)))
        return i.value

    def train(self, steps: int, tiles: int = 8, lr: float = 1e-3, seed: int = 1, maps: int = 0) -> np.ndarray:
        """Adam steps on random tiles of stored maps 0..maps-1 (0: all); per-step MSE."""
        c = np.zeros(max(steps, 1), np.float64)
        self._c(lib().igr_seed_train(self.h, steps, tiles, lr, seed, maps, c.ctypes.data_as(C.c_void_p)))
        return c[:steps]

    def evaluate(self, map_id: int) -> dict:
        """Errors of a stored map's prediction and of the zero / per-layer-mean baselines."""
        v = np.zeros(4, np.float64)
        self._c(lib().igr_seed_eval(self.h, map_id, v, 4))
        return dict(mse=v[0], mae=v[1], mae_zero=v[2], mae_mean=v[3])

    def predict(self, features) -> np.ndarray:
        f = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros_like(f)
        self._c(lib().igr_seed_predict(self.h, f.shape[0], f.shape[1], f.reshape(-1), out.reshape(-1)))
        return out

    def time_forward(self, tiles: int = 16, reps: int = 5) -> dict:
        """Device time of the forward convolutions (tcgen05 implicit GEMMs) over
        `tiles` tiles: per convolution ms per pass and FLOPs per pass, and the
        whole pass's TFLOP/s (igr_seed_time_forward)."""
        ms = np.zeros(SEED_CONVS, np.float64)
        fl = np.zeros(SEED_CONVS, np.float64)
        self._c(lib().igr_seed_time_forward(self.h, tiles, reps, ms, fl))
        return dict(layer_ms=ms.tolist(), layer_flops=fl.tolist(),
                    tflops=float(fl.sum() / (ms.sum() * 1e-3) / 1e12) if ms.sum() > 0 else 0.0)

    def grad(self, x, target):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        g = np.zeros(self.params().size, np.float32)
        loss = C.c_double()
        self._c(lib().igr_seed_grad(self.h, x.shape[0], x.reshape(-1), t.reshape(-1), C.byref(loss),
                                    g.ctypes.data_as(C.c_void_p)))
        return loss.value, g


def seed_features(router: "Router", device: bool = False) -> np.ndarray:
    """Input features of an opened router's design, [X][Y][16], on the host
    threads or (device=True) on the GPU as a seeded run computes them."""
    hdr = np.zeros(4, np.int32)
    _check(lib().igr_router_grid(router.h, hdr.ctypes.data_as(C.c_void_p), None, None, None, None))
    out = np.zeros((int(hdr[1]), int(hdr[2]), 16), np.float32)
    fn = lib().igr_seed_features_device if device else lib().igr_seed_features
    _check(fn(router.h, out.reshape(-1)), router.h)
    return out
