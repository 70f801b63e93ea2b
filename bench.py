#!/usr/bin/env python
"""Benchmark of the GPU global-routing hot path (InstantGR's metric: route
wall time and nets/s at equal evaluator score).

One step = one complete route of the synthetic design with the design already
read and its trees built (inputs resident): phase 1 (colouring, per-batch
cost refresh, tree DP, commit) and `--rrr-iters` rip-up-and-reroute passes.
Default workload: 10 layers, 840x1140 GCells, 130,000 nets, 3 RRR passes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the router does not shard), one per GPU;
`value` is the nets of all replicas over the slowest replica's time.
`--impl reference` times the CPU restatement of the same hot path (the
oracle: cost refresh, tree DP and commit per batch, phase 1 only) on the host
cores, on a bounded sample of the same plan.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    0: dict(name="256x256x10, 20k nets", X=256, Y=256, nets=20000),
    1: dict(name="840x1140x10, 130k nets, 1% 65-500-pin nets, 3 RRR passes", X=840, Y=1140, nets=130000),
    2: dict(name="1600x1600x10, 800k nets, pin mixture, 6 hotspots", X=1600, Y=1600, nets=800000),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--rrr-iters", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--workdir", default=os.environ.get("IGR_BENCH_DIR", "/tmp/igr_bench"))
    ap.add_argument("--cpu-batches", type=int, default=0, help="batches in the CPU sample (0 = auto)")
    ap.add_argument("--route-only", action="store_true",
                    help="route --warmup + --steps times and print the router statistics (profiling runs)")
    return ap.parse_args()


def route_only(args):
    import instantgr_b200 as ig
    cap, net = design_files(args)
    r = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=1)
    for _ in range(args.warmup + args.steps):
        r.run()
    print(json.dumps(dict(stats=r.stats(), kernels=r.kstats())), flush=True)
    r.close()


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


def design_files(args) -> tuple[str, str]:
    os.makedirs(args.workdir, exist_ok=True)
    base = os.path.join(args.workdir, f"c{args.config}_s{args.seed}_x{args.scale:g}")
    cap, net = base + ".cap", base + ".net"
    if not (os.path.exists(cap) and os.path.exists(net)):
        import instantgr_b200 as ig
        tmpc, tmpn = cap + f".{os.getpid()}", net + f".{os.getpid()}"
        ig.generate(args.config, args.seed, args.scale, tmpc, tmpn)
        os.replace(tmpc, cap)
        os.replace(tmpn, net)
    return cap, net


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return dict(hbm_gbs=d.get("hbm_gbs", 6650.0), src="of measured")
    return dict(hbm_gbs=6650.0, src="of fallback")


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


def omp_threads() -> int:
    """Host threads the OpenMP-parallel oracle uses (all cores unless OMP_NUM_THREADS says otherwise)."""
    v = os.environ.get("OMP_NUM_THREADS", "")
    return int(v) if v.isdigit() and int(v) > 0 else (os.cpu_count() or 1)


def profile_traffic() -> dict:
    """Per-launch DRAM traffic of the profiled kernels (ncu dram__bytes_read.sum +
    dram__bytes_write.sum) from the committed summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def cpu_sample(router, grid, plan, max_batches: int, budget_s: float = 20.0):
    """CPU restatement (oracle) of the phase-1 hot path on the first batches of the
    same plan: per batch a full cost refresh, the tree DP and the commits."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import Oracle
    o = Oracle(grid)
    N = o.N
    dem = np.zeros(N, np.float32)
    pre = np.zeros(N, np.int32)
    st = np.zeros(N, np.int32)
    w = np.zeros(N, np.float32)
    boff = plan["batch_off"]
    nb = len(boff) - 1
    cap = plan["route_cap"].astype(np.int64)
    roff = np.concatenate([[0], np.cumsum(cap)[:-1]]).astype(np.int64)
    routes = np.zeros(int(cap.sum()) + 1, np.int32)
    t0 = time.perf_counter()
    nets = 0
    b = 0
    while b < nb and (max_batches == 0 or b < max_batches):
        a, e = int(boff[b]), int(boff[b + 1])
        _, vc, ps = o.cost_refresh(dem)
        n0, n1 = int(plan["node_off"][a]), int(plan["node_off"][e])
        o.pattern_route(vc, ps, plan["node_off"][a:e + 1] - n0, plan["nodes"][n0:n1], plan["par"][n0:n1],
                        roff[a:e], plan["route_cap"][a:e], routes, pre, st, b + 1)
        o.commit_wires(pre, dem, st, b + 1)
        o.commit_vias(roff[a:e], routes, dem, st, b + 1, 1)
        nets += e - a
        b += 1
        if max_batches == 0 and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return nets / dt, dict(batches=b, of_batches=nb, nets=nets, seconds=dt)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = CONFIGS[args.config]
    workload = dict(workload=f"global routing, {cfg['name']}", config_index=args.config, scale=args.scale,
                    rrr_iters=args.rrr_iters, seed=args.seed, l2="per-step state exceeds L2 (inputs larger than L2)")
    if args.route_only:
        return route_only(args)
    if args.impl == "reference":
        return bench_reference(args, rank, world, workload)

    import torch
    import numpy as np
    import instantgr_b200 as ig
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    ig.set_device(local)
    cap, net = design_files(args) if rank == 0 or world == 1 else (None, None)
    if dist:
        dist.barrier()
        cap, net = design_files(args)

    rb = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=1, batched=1)  # batched form (headline)
    rp = ig.Router(cap, net, rrr_iters=args.rrr_iters, profile=1, batched=0)  # plain drop-in form
    design_nets, routing_nets = rb.sizes()
    for _ in range(max(args.warmup, 0)):
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
        launches, ks = 0, {}
        for _ in range(args.steps):
            fn()
            if router is not None:
                launches += int(router.stats()["launches"])
                for k, v in router.kstats().items():
                    t = ks.setdefault(k, dict(launches=0, ms=0.0, bytes=0.0))
                    for f in t:
                        t[f] += v[f]
        e1.record()
        sync_all()
        return max_over_ranks(e0.elapsed_time(e1), dist, "cuda"), launches, ks

    clk = Clocks(local)
    clk.start()
    ms_b, launches_b, ks_b = timed(rb, rb.run)
    ms_p, launches_p, ks_p = timed(rp, rp.run)
    clocks = clk.stop()
    sb, sp = rb.stats(), rp.stats()
    same = all(sb[k] == sp[k] for k in ("wirelength", "via_cost", "overflow_cost"))

    # e2e: the whole `-cap/-net/-out` flow through the public API with host files
    # (read, upload, route, download, write guides), batched form
    out = os.path.join(args.workdir, f"guides_r{rank}.out")
    e2e_bytes = []

    def e2e_step():
        r = ig.Router(cap, net, rrr_iters=args.rrr_iters, batched=1)
        r.run()
        r.write(out)
        st = r.stats()
        e2e_bytes.append((st["setup_h2d_bytes"] + st["h2d_bytes"], st["d2h_bytes"]))
        r.close()

    ms_e2e, _, _ = timed(None, e2e_step)

    result = None
    if rank == 0:
        value = replica_throughput(design_nets, args.steps, world, ms_b)
        value_plain = replica_throughput(design_nets, args.steps, world, ms_p)
        e2e_value = replica_throughput(design_nets, args.steps, world, ms_e2e)
        plan = rp.plan()
        h2d, d2h = e2e_bytes[-1]
        # roofline of the dominant kernel class of the plain form (every class is
        # timed per launch there) and, beside it, of every class with byte counts
        pk = measured_peaks()
        tr = profile_traffic()

        def roof_of(k):
            v = ks_p[k]
            ach = v["bytes"] / (v["ms"] / 1e3) / 1e9 if v["ms"] else 0.0
            n = max(v["launches"], 1)
            return dict(kernel=KERNEL_NAMES.get(k, k), bound="hbm", achieved=round(ach, 1), peak=pk["hbm_gbs"],
                        unit="GB/s", frac=round(ach / pk["hbm_gbs"], 4), peak_src=pk["src"],
                        traffic=tr.get(f"{k}_bytes_per_launch"),
                        algorithmic_bytes_per_launch=round(v["bytes"] / n, 1),
                        avg_launch_us=round(1e3 * v["ms"] / n, 3))

        dom = max((k for k in ks_p if ks_p[k]["bytes"] > 0), key=lambda k: ks_p[k]["ms"])
        roof = roof_of(dom)
        roof["dominant_kernel"] = dom
        roof["classes"] = {k: roof_of(k) for k in ks_p if ks_p[k]["bytes"] > 0}
        roof["kernel_ms_per_step_plain"] = {k: round(v["ms"] / args.steps, 3) for k, v in ks_p.items()}
        roof["kernel_ms_per_step_batched"] = {k: round(v["ms"] / args.steps, 3) for k, v in ks_b.items()}
        cpu = None
        if world == 1:
            try:
                g = rp.grid()
                v, info = cpu_sample(rp, g, plan, args.cpu_batches)
                cpu = dict(value=round(v, 2), unit="nets/s", cores=omp_threads(), kind="port",
                           sample=f"oracle phase-1 (cost refresh + tree DP + commit) on the first "
                                  f"{info['batches']} of {info['of_batches']} batches ({info['nets']} nets, "
                                  f"{info['seconds']:.1f} s)")
            except Exception as ex:  # the CPU baseline is reported, never required
                cpu = dict(value=None, unit="nets/s", cores=omp_threads(), kind="port", sample=f"failed: {ex}")
        result = dict(metric="route throughput (nets/s), batched RRR router", value=round(value, 2), unit="nets/s",
                      n_gpus=world, steps=args.steps, warmup=args.warmup, ms_per_step=round(ms_b / args.steps, 3),
                      higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32/f64 costs, i32 demand",
                      data="synthetic (seeded generator, ISPD2024 format)", config=workload,
                      parallelism="replicas" if world > 1 else "single GPU",
                      e2e=dict(value=round(e2e_value, 2), unit="nets/s", h2d_bytes_per_step=int(h2d),
                               d2h_bytes_per_step=int(d2h)),
                      roofline=roof, cpu_baseline=cpu, clocks=clocks, gpu_launches=launches_b,
                      plain=dict(value=round(value_plain, 2), ms_per_step=round(ms_p / args.steps, 3),
                                 gpu_launches=launches_p, same_result_as_batched=same),
                      detail=dict(design_nets=design_nets, routing_nets=routing_nets,
                                  wirelength=sb["wirelength"], via_cost=sb["via_cost"],
                                  overflow_cost=sb["overflow_cost"], batches1=sb["batches1"],
                                  rerouted_last=sb["rerouted"], p1_ms=sb["p1_ms"], rrr_ms=sb["rrr_ms"],
                                  dag_host_ms=sb["dag_host_ms"], route_s=sb["route_s"],
                                  host_cores=os.cpu_count()))
        print(json.dumps(result), flush=True)
    rb.close()
    rp.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


KERNEL_NAMES = {
    "cost_refresh": "commit_refresh / cost_refresh (fused batch commit, wire/via cost, f64 Sklansky prefix sums)",
    "coloring": "coloring_kernel (persistent cooperative batch colouring)",
    "pattern_dp": "pattern_route_kernel (tree DP per net, phase 1)",
}


def bench_reference(args, rank, world, workload):
    """CPU restatement of the hot path (oracle port) on the host cores, rank 0 only."""
    if rank != 0:
        return None
    import instantgr_b200 as ig
    cap, net = design_files(args)
    r = ig.Router(cap, net, rrr_iters=0)
    r.run()  # plan (batches and trees) of the same design
    g = r.grid()
    plan = r.plan()
    design_nets, _ = r.sizes()
    vals, infos = [], []
    nb = args.cpu_batches  # 0: every batch of phase 1, within the time budget
    for i in range(args.warmup + args.steps):
        v, info = cpu_sample(r, g, plan, nb)
        if i >= args.warmup:
            vals.append(v)
            infos.append(info)
    v = statistics.median(vals)
    sample = (f"oracle phase-1 (cost refresh + tree DP + commit) on the first {infos[0]['batches']} of "
              f"{infos[0]['of_batches']} batches ({infos[0]['nets']} nets) per step")
    res = dict(impl="reference", metric="route throughput (nets/s), plain RRR router", value=round(v, 2),
               unit="nets/s", n_gpus=world, steps=args.steps, warmup=args.warmup,
               ms_per_step=round(1e3 * infos[0]["nets"] / v, 3), higher_is_better=True, scaling="weak",
               vs_baseline=None, dtype="f32/f64 costs, i32 demand", data="synthetic (seeded generator)",
               config=workload,
               cpu_baseline=dict(value=round(v, 2), unit="nets/s", cores=omp_threads(), kind="port", sample=sample),
               e2e=dict(value=round(v, 2), unit="nets/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(res), flush=True)
    r.close()
    return res


if __name__ == "__main__":
    main()
