#!/usr/bin/env python
"""Benchmark of the GPU global-routing hot path, on InstantGR's metric: route
wall time and nets/s at equal evaluator score, plain form against the batched
form with the learned congestion seed.

One step = one complete route of the design with the design read and its trees
built (inputs resident): colouring, phase 1 (per batch: cost refresh, tree DP,
commit) and `--rrr-iters` rip-up-and-reroute passes (overflow marking, detour
DAGs, colouring, per batch: rip-up, cost refresh, DAG DP, commit).
Default workload: 10 layers, 1600x1600 GCells, 800,000 nets (pin-count mixture,
6 hotspots), 3 RRR passes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` = design nets per second of the plain drop-in form (K CUDA-event-timed
steps); the batched form and the batched form with the learned seed are timed
beside it, each with its evaluator total.  `e2e` = the same
metric through the public API with host files every step (open: read, pins,
trees, device set-up; route; write the guides).  `reference_gpu` = the
reference's own sm_100a build (oracle/_ref/instantgr_ref) and this project's
command line on the same design, wall time and evaluator totals.

N > 1 runs N independent replicas (the router does not shard), one per GPU;
`value` is the nets of all replicas over the slowest replica's time.

`--impl reference` times the reference's CPU implementation of the path
(oracle/_ref/ref_cpu: the reference's own host code, and the oracle for the
stages it runs only as CUDA kernels) on the host cores, on a window of the same
design: the nets whose access points all lie in a centred window covering
`--ref-window` of each side.  It loads none of this project's router code.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
GEN_BIN = os.path.join(ROOT, "instantgr_b200", "bin", "igr_generate")
ROUTE_BIN = os.path.join(ROOT, "instantgr_b200", "bin", "igr_route")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

CONFIGS = {
    0: dict(name="256x256x10, 20k nets", X=256, Y=256, nets=20000),
    1: dict(name="840x1140x10, 130k nets, 1% 65-500-pin nets", X=840, Y=1140, nets=130000),
    2: dict(name="1600x1600x10, 800k nets, pin mixture 70/20/9.5/0.5%, 6 hotspots", X=1600, Y=1600, nets=800000),
    4: dict(name="3000x3000x10, 10M nets, 4 clusters", X=3000, Y=3000, nets=10000000),
}
METRIC = "route throughput (design nets/s): plain vs batched+learned at equal evaluator score"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--rrr-iters", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--ref-window", type=float, default=0.5,
                    help="side of the reference arm's centred window, as a fraction of the grid's sides")
    ap.add_argument("--workdir", default=os.environ.get("IGR_BENCH_DIR", "/tmp/igr_bench"))
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference sm_100a build's run")
    ap.add_argument("--route-only", action="store_true",
                    help="route --warmup + --steps times and print the router statistics (profiling runs)")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "learned"],
                    help="router form of --route-only")
    ap.add_argument("--window", action="store_true",
                    help="--route-only on the centred window of the design that the reference arm routes "
                         "(--ref-window): a smaller case of the same density, for profiling captures")
    ap.add_argument("--micro", choices=["refresh", "seed"],
                    help="kernel cases for profiling: cost refresh on a seeded 1600x1600x9 grid (every track "
                         "dirty, none, a sixth, every track), or the learned seed's forward convolutions")
    ap.add_argument("--tiles", type=int, default=16, help="tiles of --micro seed")
    return ap.parse_args()


def workload(args) -> dict:
    cfg = CONFIGS[args.config]
    return dict(workload=f"global routing, {cfg['name']}, {args.rrr_iters} RRR passes", headline_form="plain",
                config_index=args.config,
                scale=args.scale, rrr_iters=args.rrr_iters, seed=args.seed,
                l2="per-step state exceeds L2 (inputs larger than L2)")


def design_files(args, window=None) -> tuple[str, str]:
    """The seeded design (or a window of it), written by the stand-alone generator."""
    os.makedirs(args.workdir, exist_ok=True)
    tag = "" if window is None else "_w%d_%d_%d_%d" % tuple(window)
    base = os.path.join(args.workdir, f"c{args.config}_s{args.seed}_x{args.scale:g}{tag}")
    cap, net = base + ".cap", base + ".net"
    if not (os.path.exists(cap) and os.path.exists(net)):
        tmpc, tmpn = cap + f".{os.getpid()}", net + f".{os.getpid()}"
        cmd = [GEN_BIN, "--config", str(args.config), "--seed", str(args.seed), "--scale", str(args.scale),
               "--cap", tmpc, "--net", tmpn]
        if window is not None:
            cmd += ["--window"] + [str(v) for v in window]
        subprocess.run(cmd, check=True)
        os.replace(tmpc, cap)
        os.replace(tmpn, net)
    return cap, net


def ref_window(args) -> list[int]:
    """Centred window of the reference arm's sample: [x0, y0, w, h]."""
    cfg = CONFIGS[args.config]
    w = max(2, int(round(cfg["X"] * args.ref_window)))
    h = max(2, int(round(cfg["Y"] * args.ref_window)))
    return [(cfg["X"] - w) // 2, (cfg["Y"] - h) // 2, w, h]


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def stop(self) -> dict:
        if not self.p:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(self.rows))


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return dict(hbm_gbs=d.get("hbm_gbs", 6650.0), bf16_tflops=d.get("bf16_tflops", 1590.0), src="of measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, src="of fallback")


def max_over_ranks(ms: float, dist=None, device: str = "cpu") -> float:
    """The slowest rank's time: every rank takes part in one MAX all-reduce (the
    same collective step on every rank); `dist` None means a single rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(nets_per_replica: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job nets/s of `world` independent replicas that each routed `steps`
    times, over the slowest replica's time."""
    return nets_per_replica * steps * world / (max_ms / 1e3)


def host_threads() -> int:
    """Host threads the CPU baselines use (all cores unless OMP_NUM_THREADS says otherwise)."""
    v = os.environ.get("OMP_NUM_THREADS", "")
    return int(v) if v.isdigit() and int(v) > 0 else (os.cpu_count() or 1)


def profile_traffic() -> dict:
    """Per-launch DRAM traffic of the profiled kernels (ncu dram__bytes_read.sum +
    dram__bytes_write.sum) from the committed summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def run_ref_cpu(cap: str, net: str, steps: int, warmup: int, rrr: int, threads: int, timeout: float = 1500) -> dict:
    """The reference route on the host cores (oracle/_ref/ref_cpu); its setup
    record and per-step records."""
    exe = os.path.join(REF_DIR, "ref_cpu")
    if not os.path.exists(exe):
        raise RuntimeError(f"{exe} missing (built by `make -C oracle ref` where the reference tree is present)")
    p = subprocess.run([exe, cap, net, str(steps), str(warmup), str(rrr), str(threads)], capture_output=True,
                       text=True, timeout=timeout)
    recs = [json.loads(line[7:]) for line in p.stdout.splitlines() if line.startswith("REFCPU ")]
    if p.returncode != 0 or not recs:
        raise RuntimeError(f"ref_cpu failed (rc {p.returncode}): {p.stderr[-400:]}")
    setup = recs[0]
    timed = [r for r in recs[1:] if r.get("timed")]
    if len(timed) != steps:
        raise RuntimeError(f"ref_cpu printed {len(timed)} timed steps of {steps}")
    return dict(setup=setup, steps=timed)


def evaluator_total(cap: str, net: str, out: str) -> dict:
    """The reference evaluator's FOR_STAT (run/evaluator.cpp) of a guide file."""
    p = subprocess.run([os.path.join(REF_DIR, "evaluator"), cap, net, out], capture_output=True, text=True,
                       timeout=900)
    for line in p.stdout.splitlines():
        if line.startswith("FOR_STAT"):
            wl, via, of, tot = (float(v) for v in line.split()[1:5])
            return dict(wirelength=wl, via=via, overflow=of, total=tot)
    return dict(error=f"no FOR_STAT (rc {p.returncode})")


def reference_gpu(cap: str, net: str, workdir: str, rrr_iters: int) -> dict:
    """CLI wall time of the reference's own sm_100a build and of this project's
    command line on the same design, and the reference evaluator's totals of both
    guide files.  The reference does one rip-up pass (src/main.cpp:45-68)."""
    exe = os.path.join(REF_DIR, "instantgr_ref")
    if not os.path.exists(exe):
        return dict(unavailable=f"{exe} missing")
    res = {}
    outs = {}
    for name, cmd in (("reference", [exe, "-cap", cap, "-net", net, "-out"]),
                      ("this_build", [ROUTE_BIN, "-cap", cap, "-net", net, "--rrr-iters", "1", "-out"])):
        out = os.path.join(workdir, f"guides_{name}.out")
        t0 = time.perf_counter()
        p = subprocess.run(cmd + [out], capture_output=True, text=True, timeout=900)
        dt = time.perf_counter() - t0
        outs[name] = out
        res[name] = dict(cli_wall_s=round(dt, 3), rc=p.returncode)
    evs = {}
    th = [threading.Thread(target=lambda k: evs.__setitem__(k, evaluator_total(cap, net, outs[k])), args=(k,))
          for k in outs]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for k in outs:
        res[k]["evaluator"] = evs.get(k)
    if res["reference"]["rc"] == 0 and res["this_build"]["rc"] == 0:
        res["cli_speedup"] = round(res["reference"]["cli_wall_s"] / res["this_build"]["cli_wall_s"], 3)
        a, b = evs.get("this_build", {}).get("total"), evs.get("reference", {}).get("total")
        if a and b:
            res["score_delta_pct"] = round(100.0 * (a - b) / b, 5)
    res["note"] = "both with one rip-up-and-reroute pass, as the reference's main.cpp; wall clock of the process"
    return res


def route_only(args):
    import instantgr_b200 as ig
    cap, net = design_files(args, ref_window(args) if args.window else None)
    r = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=1, verbose=1,
                  batched=0 if args.form == "plain" else 1)
    m = None
    if args.form == "learned":
        m = ig.Seed.load()
        r.set_seed(m, alpha=1.0, mode=1, kind=1, levels=4)
    for _ in range(args.warmup + args.steps):
        r.run()
    print(json.dumps(dict(form=args.form, stats=r.stats(), kernels=r.kstats(), evaluator=r.evaluate()["total"])),
          flush=True)
    r.close()
    if m is not None:
        m.close()


KERNEL_NAMES = {
    "cost_refresh": "cost_refresh_kernel (wire/via cost and f64 Sklansky prefix sums of the dirty tracks, reroute passes)",
    "commit_refresh": "commit_refresh_kernel (phase-1 batch commit fused with the cost refresh of the dirty tracks)",
    "coloring": "coloring_kernel (persistent cooperative batch colouring)",
    "pattern_dp": "pattern_route_kernel (tree DP per net, phase 1)",
    "dag_dp": "dag_edge_cost + dag_net_kernel (detour-DAG DP and backtrace per net, reroute passes)",
    "ripup": "rip-up: overflow marking, congestion view, wire/via rip-up",
}


def micro(args):
    """Kernel cases for profiling (CUDA events or ncu), one JSON line.

    refresh: a 1600x1600x9 grid with seeded capacity (0..8, 5% zero) and demand
    (half units): cost refresh with every track dirty, then with none, then
    after via commits that dirty about a sixth of the tracks (twice), then two
    full refreshes.  seed: two forward passes of the shipped seed network over
    --tiles tiles (the first untimed), per convolution."""
    import instantgr_b200 as ig
    if args.micro == "seed":
        m = ig.Seed.load()
        r = m.time_forward(tiles=args.tiles, reps=2)
        m.close()
        print(json.dumps(dict(micro="seed", tiles=args.tiles, **r)), flush=True)
        return r
    X = Y = 1600
    L = 9
    rng = np.random.default_rng(7)
    cap = rng.integers(0, 9, size=(L, X, Y)).astype(np.float32)
    cap[rng.random((L, X, Y)) < 0.05] = 0.0
    dem = (rng.integers(0, 20, size=(L, X, Y)) * 0.5).astype(np.float32)
    dem[rng.random((L, X, Y)) < 0.4] = 0.0
    xlen = rng.integers(1, 3, size=X - 1).astype(np.int32)
    ylen = rng.integers(1, 3, size=Y - 1).astype(np.int32)
    short = np.round(rng.uniform(0.5, 2.0, size=L), 3)
    c = ig.Ctx(L, X, Y, 0, xlen, ylen, 1.0, 2.0, short, cap.reshape(-1))
    c.set_demand(dem.reshape(-1))
    nv = 300  # vias from layer 0 to layer 8 at random GCells: 8 tracks dirty each
    xs, ys = rng.integers(0, X, nv), rng.integers(0, Y, nv)
    routes = np.zeros(3 * nv, np.int32)
    routes[0::3] = 3
    routes[1::3] = xs * Y + ys
    routes[2::3] = 8 * X * Y + xs * Y + ys
    off = np.arange(nv, dtype=np.int64) * 3

    def wall_us(f):
        t0 = time.perf_counter()
        f()
        return round((time.perf_counter() - t0) * 1e6, 1)

    res = dict(micro="refresh", grid=[L, X, Y], cells=L * X * Y)
    res["all_dirty_us"] = wall_us(lambda: c.cost_refresh(True))
    res["none_dirty_us"] = wall_us(lambda: c.cost_refresh(True))
    res["partial_us"] = []
    for k in range(2):
        c.commit_vias(off, routes, stamp=10 + k, K=1)
        res["partial_us"].append(wall_us(lambda: c.cost_refresh(True)))
        c.commit_vias(off, routes, stamp=20 + k, K=-1)
        c.cost_refresh(True)
    res["full_us"] = [wall_us(lambda: c.cost_refresh(False)) for _ in range(2)]
    res["note"] = "host wall time of each call, including its launch and synchronisation"
    c.close()
    print(json.dumps(res), flush=True)
    return res


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    wl = workload(args)
    if args.route_only:
        return route_only(args)
    if args.micro:
        return micro(args)
    if args.impl == "reference":
        return bench_reference(args, rank, world, wl)

    import torch
    import instantgr_b200 as ig
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    ig.set_device(local)
    cap, net = design_files(args) if rank == 0 or world == 1 else (None, None)
    if dist:
        dist.barrier()
        cap, net = design_files(args)

    model = ig.Seed.load()
    # the timed routers run without per-launch events (they cost about 3% of a
    # route); the per-kernel classes come from profiled twins run outside the
    # timed region on the same design
    rp = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=0, batched=0)  # plain drop-in form
    rb = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=0, batched=1)  # batched form
    rl = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=0, batched=1)  # batched + learned seed
    rl.set_seed(model, alpha=1.0, mode=1, kind=1, levels=4)
    design_nets, routing_nets = rp.sizes()
    for _ in range(max(args.warmup, 0)):
        rl.run()
        rb.run()
        rp.run()

    def sync_all():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
            torch.cuda.synchronize()

    def timed(router, fn):
        """K steps bracketed by barrier + synchronize; device time (CUDA events) max over ranks."""
        sync_all()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launches = 0
        for _ in range(args.steps):
            fn()
            if router is not None:
                launches += int(router.stats()["launches"])
        e1.record()
        sync_all()
        return max_over_ranks(e0.elapsed_time(e1), dist, "cuda"), launches

    clk = Clocks(local)
    clk.start()
    ms_l, launches_l = timed(rl, rl.run)
    ms_b, launches_b = timed(rb, rb.run)
    ms_p, launches_p = timed(rp, rp.run)
    clocks = clk.stop()

    def kernel_classes(batched, seeded):
        """Per-kernel-class device time (CUDA events around every launch) of one
        route of a profiled twin, after one untimed route."""
        r = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=1, batched=batched)
        if seeded:
            r.set_seed(model, alpha=1.0, mode=1, kind=1, levels=4)
        r.run()
        r.run()
        ks = r.kstats()
        r.close()
        return ks

    ks_p = kernel_classes(0, False) if rank == 0 else {}
    ks_l = kernel_classes(1, True) if rank == 0 else {}
    ev_l, ev_b, ev_p = rl.evaluate(), rb.evaluate(), rp.evaluate()
    sl, sb, sp = rl.stats(), rb.stats(), rp.stats()

    # e2e: the whole `-cap/-net/-out` flow through the public API with host files
    # (read, pins, trees, upload, route, download, write guides), plain form
    # Every step writes a new guide file, as one `-cap/-net/-out` run does (a
    # step that overwrote the previous step's file would also pay for dropping
    # its pages while they are written back); the files go after the timing.
    out = os.path.join(args.workdir, f"guides_r{rank}.out")
    e2e_bytes = []
    e2e_files = []

    def e2e_step():
        path = f"{out}.{len(e2e_files)}"
        e2e_files.append(path)
        r = ig.Router(cap, net, rrr_iters=args.rrr_iters, batched=0)
        r.run()
        r.write(path)
        st = r.stats()
        e2e_bytes.append((st["setup_h2d_bytes"] + st["h2d_bytes"], st["d2h_bytes"]))
        r.close()

    for path in [out] + [f"{out}.{k}" for k in range(args.steps)]:
        if os.path.exists(path):
            os.remove(path)
    ms_e2e, _ = timed(None, e2e_step)
    for path in e2e_files:
        if os.path.exists(path):
            os.remove(path)

    result = None
    if rank == 0:
        value = replica_throughput(design_nets, args.steps, world, ms_p)
        h2d, d2h = e2e_bytes[-1]
        pk = measured_peaks()
        tr = profile_traffic()

        def roof_of(ks, k):
            v = ks[k]
            ach = v["bytes"] / (v["ms"] / 1e3) / 1e9 if v["ms"] else 0.0
            n = max(v["launches"], 1)
            traffic = tr.get(f"{k}_bytes_per_launch")
            if traffic is None and f"{k}_bytes_per_cell" in tr:
                # measured DRAM bytes per refreshed cell x the cells of an average
                # launch (20 algorithmic bytes per refreshed cell)
                traffic = round(tr[f"{k}_bytes_per_cell"] * v["bytes"] / n / 20.0)
            return dict(kernel=KERNEL_NAMES.get(k, k), bound="hbm", achieved=round(ach, 1), peak=pk["hbm_gbs"],
                        unit="GB/s", frac=round(ach / pk["hbm_gbs"], 4), peak_src=pk["src"],
                        traffic=traffic,
                        algorithmic_bytes_per_launch=round(v["bytes"] / n, 1),
                        avg_launch_us=round(1e3 * v["ms"] / n, 3))

        # every class is timed per launch in the plain form; the roofline object is
        # the HBM-bound class with the largest share (the phase-1 fused commit and
        # refresh, or the reroute passes' refresh), every class with its time and
        # bound beside it
        hbm = [k for k in ("commit_refresh", "cost_refresh") if ks_p.get(k, {}).get("ms")]
        dom = max(hbm, key=lambda k: ks_p[k]["ms"]) if hbm else "cost_refresh"
        roof = roof_of(ks_p, dom)
        roof["dominant_kernel"] = dom
        roof["classes"] = {k: roof_of(ks_p, k) for k in ks_p if ks_p[k]["bytes"] > 0}
        roof["kernel_ms_per_step_plain"] = {k: round(v["ms"], 3) for k, v in ks_p.items()}
        roof["kernel_ms_per_step_batched_learned"] = {k: round(v["ms"], 3) for k, v in ks_l.items()}
        roof["kernel_classes_from"] = "one route of a profiled twin (CUDA events around every launch), untimed"

        # the tensor-core kernel: the learned seed's forward convolutions
        # (umma_gemm_kernel) over 16 tiles of 288 x 288 GCells, CUDA events
        try:
            tf = model.time_forward(tiles=16, reps=5)
            roof["tensor_core"] = dict(
                kernel="umma_gemm_kernel (tcgen05.mma kind::f16, BF16 operands, f32 accumulators in TMEM; "
                       "the seed network's six 3x3 convolutions as implicit GEMMs, 16 tiles of 288x288)",
                bound="tensor", unit="TFLOP/s", achieved=round(tf["tflops"], 2), peak=pk["bf16_tflops"],
                frac=round(tf["tflops"] / pk["bf16_tflops"], 4), peak_src=pk["src"] + " (cuBLAS bf16 burst)",
                layer_ms=[round(v, 4) for v in tf["layer_ms"]],
                layer_tflops=[round(f / (m * 1e-3) / 1e12, 2) if m > 0 else 0.0
                              for f, m in zip(tf["layer_flops"], tf["layer_ms"])],
                gflop_per_pass=round(sum(tf["layer_flops"]) / 1e9, 2))
        except Exception as ex:  # reported, never required
            roof["tensor_core"] = dict(unavailable=f"failed: {ex}")
        roof["latency_bound_classes"] = {
            "coloring": "grid barriers and dependent L2 accesses; DRAM nearly idle (profiles/coloring_kernel_c1.md)",
            "pattern_dp": "issue/latency bound tree DP (profiles/pattern_route_kernel_c1_largest_batch.md)",
            "dag_dp": "bound by the dependent levels of the largest DAGs (profiles/dag_net_kernel_c2.md)",
        }
        cpu = None
        rgpu = None
        if world == 1:
            try:
                win = ref_window(args)
                wc, wn = design_files(args, win)
                r = run_ref_cpu(wc, wn, 1, 0, args.rrr_iters, host_threads())
                s0 = r["steps"][0]
                cpu = dict(value=round(r["setup"]["design_nets"] / s0["seconds"], 2), unit="nets/s",
                           cores=r["setup"]["threads"], kind="reference",
                           sample=cpu_sample_text(args, win, r))
            except Exception as ex:  # the CPU baseline is reported, never required
                cpu = dict(value=None, unit="nets/s", cores=host_threads(), kind="reference", sample=f"failed: {ex}")
            if not args.no_reference_gpu:
                try:
                    rgpu = reference_gpu(cap, net, args.workdir, args.rrr_iters)
                except Exception as ex:
                    rgpu = dict(unavailable=f"failed: {ex}")

        def form(ms, launches, ev, st):
            return dict(value=round(replica_throughput(design_nets, args.steps, world, ms), 2),
                        ms_per_step=round(ms / args.steps, 3), gpu_launches=launches,
                        evaluator_total=round(ev["total"], 1), rerouted_last_pass=int(st["rerouted"]),
                        phase1_ms=round(st["p1_ms"], 3), rrr_ms=round(st["rrr_ms"], 3))

        plain = form(ms_p, launches_p, ev_p, sp)
        result = dict(metric=METRIC, value=round(value, 2), unit="nets/s",
                      n_gpus=world, steps=args.steps, warmup=args.warmup, ms_per_step=round(ms_p / args.steps, 3),
                      higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32/f64 costs, i32 demand",
                      data="synthetic (seeded generator, ISPD2024 format)", config=wl,
                      parallelism="replicas" if world > 1 else "single GPU",
                      e2e=dict(value=round(replica_throughput(design_nets, args.steps, world, ms_e2e), 2),
                               unit="nets/s", h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(d2h)),
                      roofline=roof, cpu_baseline=cpu, clocks=clocks, gpu_launches=launches_p,
                      forms=dict(
                          batched_learned=form(ms_l, launches_l, ev_l, sl),
                          batched=form(ms_b, launches_b, ev_b, sb),
                          plain=plain),
                      plain_over_batched_learned_time=round(ms_p / ms_l, 3),
                      score_batched_learned_vs_plain_pct=round(100.0 * (ev_l["total"] - ev_p["total"])
                                                               / ev_p["total"], 5),
                      reference_gpu=rgpu,
                      detail=dict(design_nets=design_nets, routing_nets=routing_nets,
                                  batches1=sp["batches1"], rerouted_last=sp["rerouted"], host_cores=os.cpu_count(),
                                  e2e_ms_per_step=round(ms_e2e / args.steps, 3)))
        print(json.dumps(result), flush=True)
    rl.close()
    rb.close()
    rp.close()
    model.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def cpu_sample_text(args, win, r) -> str:
    st = r["setup"]
    s = r["steps"]
    secs = [x["seconds"] for x in s]
    return (f"oracle/_ref/ref_cpu: the reference's host code (reader, pin selection, net split, Steiner trees, "
            f"host colouring generate_batches_rsmt, detour-DAG builder on {st['threads']} threads) and the oracle's "
            f"restatement of its kernels (OpenMP, {st['threads']} threads), one complete route with "
            f"{args.rrr_iters} RRR passes of the {win[2]}x{win[3]} window at ({win[0]}, {win[1]}) of the same design: "
            f"{st['design_nets']} design nets, {st['routing_nets']} routing nets; rerouted per pass "
            f"{s[0]['rerouted']}; {len(s)} step(s) of {statistics.mean(secs):.2f} s")


def bench_reference(args, rank, world, wl):
    """The reference's CPU implementation of the path on the host cores (rank 0 only)."""
    if rank != 0:
        return None
    win = ref_window(args)
    cap, net = design_files(args, win)
    try:
        r = run_ref_cpu(cap, net, args.steps, max(args.warmup, 0), args.rrr_iters, host_threads())
    except Exception as ex:
        res = dict(impl="reference", unavailable=f"reference CPU route failed: {ex}")
        print(json.dumps(res), flush=True)
        return res
    secs = [s["seconds"] for s in r["steps"]]
    ms = 1e3 * sum(secs) / len(secs)
    nets = r["setup"]["design_nets"]
    v = nets / (ms / 1e3)
    cpu = dict(value=round(v, 2), unit="nets/s", cores=r["setup"]["threads"], kind="reference",
               sample=cpu_sample_text(args, win, r))
    res = dict(impl="reference", metric=METRIC, value=round(v, 2), unit="nets/s", n_gpus=world, steps=args.steps,
               warmup=args.warmup, ms_per_step=round(ms, 3), higher_is_better=True, scaling="weak",
               vs_baseline=None, dtype="f32/f64 costs, i32 demand", data="synthetic (seeded generator, ISPD2024 format)",
               config=wl, cpu_baseline=cpu,
               e2e=dict(value=round(v, 2), unit="nets/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0),
               detail=dict(window=win, design_nets=nets, routing_nets=r["setup"]["routing_nets"],
                           read_s=r["setup"]["read_s"], nets_trees_s=r["setup"]["nets_trees_s"],
                           batches1=r["steps"][0]["batches1"], rerouted=r["steps"][0]["rerouted"],
                           step_seconds=[round(x, 3) for x in secs]))
    print(json.dumps(res), flush=True)
    return res


if __name__ == "__main__":
    main()
