#!/usr/bin/env python3
"""Benchmark of the D-core engine on one node.

Default workload: full D-core decomposition of a seeded directed R-MAT graph,
scale 22 (4,194,304 vertices), edge factor 16, (a, b, c) = (.57, .19, .19),
self-loops and duplicates removed, labels permuted (65,245,102 edges with
seed 1).  One step = one decomposition of the device-resident graph: kmax of
every vertex and every row lmax[k][v], k = 0..kmax, written densely to HBM
(the reference's dcore() output, main.cu:197-262).

  value  edges/s = (edges of all ranks) / (max over ranks of the device time
         per step), CUDA events on the engine's stream
  e2e    the same metric through the C ABI with host buffers: pinned host
         edges -> dc_graph_create (upload + device CSR/CSC build) ->
         dc_decompose -> dc_get_kmaxes + dc_get_lmax_rows (dense rows to
         pinned host memory), wall clock with both sides synchronized

--impl reference times the CPU oracle port of the same decomposition on the
host cores (the reference has no CPU implementation of the path).

Multi-GPU (torchrun): every rank decomposes its own seeded graph of the same
size (weak scaling, replicas; no data-path collective).
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "d-core-cuda_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOADS = {
    "decomp-rmat22": dict(gen="rmat", scale=22, ef=16, seed=1,
                          desc="R-MAT scale 22, edge factor 16, a=.57 b=.19 c=.19, dedup, permuted"),
    "decomp-rmat20": dict(gen="rmat", scale=20, ef=16, seed=1,
                          desc="R-MAT scale 20, edge factor 16, a=.57 b=.19 c=.19, dedup, permuted"),
    "decomp-er10k": dict(gen="er", n=10_000, m=100_000, seed=1, desc="directed G(n=10000, m=100000)"),
    # maintenance: R-MAT graph + stream of 50% inserts of absent edges and 50%
    # deletes of present edges, valid in sequence, in several batch sizes
    "maint-rmat24": dict(gen="rmat", scale=24, ef=16, seed=1, ops=1_000_000, maint=True,
                         sizes=[(1, 20), (100, 20), (10_000, 20), (1_000_000, 1)],
                         desc="R-MAT scale 24, edge factor 16 + 1e6-op update stream (50% insert / 50% delete)"),
    "maint-rmat22": dict(gen="rmat", scale=22, ef=16, seed=1, ops=1_000_000, maint=True,
                         sizes=[(1, 20), (100, 20), (10_000, 20), (1_000_000, 1)],
                         desc="R-MAT scale 22, edge factor 16 + 1e6-op update stream (50% insert / 50% delete)"),
}
METRIC_MAINT = "updates/s batched D-core maintenance"
METRIC = "edges/s full D-core decomposition"


def make_graph(dc, w, rank):
    seed = w["seed"] + rank
    if w["gen"] == "rmat":
        V, s, d = dc.gen_rmat(w["scale"], w["ef"], seed)
    else:
        s, d = dc.gen_er(w["n"], w["m"], seed)
        V = w["n"]
    return V, s, d


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_traffic(kernel, workload):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload, {}).get(kernel)


def cpu_baseline(w, V, s, d, budget_s=20.0):
    """Oracle port on the host cores: kmax pass plus a stratified sample of
    rows, extrapolated to the full decomposition."""
    from oracle import oracle
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    K, kmaxes = oracle.kmax(V, s, d)
    t_kmax = time.perf_counter() - t0
    # probe one row to size the sample
    t0 = time.perf_counter()
    oracle.row(V, s, d, kmaxes, 0)
    t_row0 = time.perf_counter() - t0
    rows_total = K + 1
    want = max(min(rows_total, 2 * threads), int(budget_s * threads / max(t_row0, 1e-3)))
    want = max(1, min(rows_total, want))
    stride = max(1, rows_total // want)
    n, row_secs = oracle.rows_sample(V, s, d, kmaxes, K, stride, threads)
    # all rows run in parallel over `threads` threads: estimated wall time is
    # the kmax pass plus the extrapolated row-seconds spread over the threads
    t_est = t_kmax + row_secs * rows_total / n / threads
    return {"value": len(s) / t_est, "unit": "edges/s", "cores": threads, "kind": "port",
            "sample": f"kmax pass + {n} of {rows_total} rows (every {stride}th row), bucket-queue peel per row "
                      f"on {threads} threads; all-row time extrapolated from summed row seconds "
                      f"({t_est:.1f} s estimated)"}


def run_reference(args, w, rank, world):
    if rank != 0:
        return
    import dcore_b200 as dc
    V, s, d = make_graph(dc, w, 0)
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(w, V, s, d, budget_s=args.cpu_seconds)
        if i >= args.warmup:
            vals.append(b["value"])
            base = b
    value = float(np.mean(vals))
    metric, unit = METRIC, "edges/s"
    if w.get("maint"):
        # the CPU path maintains by recomputing (the reference's own check,
        # checkDCore): one batch of 10,000 updates costs one decomposition
        metric, unit = METRIC_MAINT, "updates/s"
        value = 10_000 * value / len(s)
        base = dict(base, unit=unit, sample=base["sample"] + "; one recomputation per batch of 10,000 updates")
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * len(s) / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload, "graph": w["desc"], "V": V, "E": int(len(s))},
            "cpu_baseline": dict(base, value=value),
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_maintenance(args, w, rank, world, local):
    """Update stream in batches of several sizes; every batch leaves the
    decomposition equal to a full recomputation of the updated graph."""
    import torch
    import dcore_b200 as dc
    torch.cuda.set_device(local)
    V, s, d = make_graph(dc, w, rank)
    u, v, dl = dc.gen_updates(V, s, d, w["ops"], 0.5, w["seed"] + 1000 + rank)
    g = dc.Graph.from_edges(V, s, d, device=local, gap_min=2, gap_div=16)
    g.decompose(dc.METHOD_INCREMENTAL)
    sampler = ClockSampler(local)
    launches0 = dc.launch_count()
    sampler.start()
    pos = 0
    per_size = {}
    for bs, nb in w["sizes"]:
        nb = min(nb, (len(u) - pos) // bs)
        if nb <= 0:
            continue
        lat = []
        methods = []
        for _ in range(nb):
            st = g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], args.maint_method)
            lat.append(st["total_ms"])
            methods.append(st["method"])
            pos += bs
        lat = np.array(lat)
        per_size[str(bs)] = {"batches": nb, "updates_per_s": bs * nb / (lat.sum() / 1000.0),
                             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                             "methods": {"local": methods.count(1), "repeel": methods.count(2)}}
    clocks = sampler.stop()
    launches = dc.launch_count() - launches0
    head = per_size.get("10000") or per_size[max(per_size, key=lambda k: int(k))]
    line = {"metric": METRIC_MAINT, "value": head["updates_per_s"], "unit": "updates/s", "n_gpus": world,
            "steps": sum(x["batches"] for x in per_size.values()), "warmup": 1,
            "ms_per_step": head["p50_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": args.workload, "graph": w["desc"], "V": V, "E": int(len(s)),
                       "headline": "batches of 10,000 updates", "per_batch_size": per_size,
                       "exactness": "each batch leaves kmaxes and rows equal to a full recomputation",
                       "method": {0: "scheduler", 1: "local", 2: "re-peel"}[args.maint_method]},
            "gpu_launches": int(launches), "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.free()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="decomp-rmat22")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--maint-method", type=int, default=0, help="0 scheduler, 1 local, 2 re-peel")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w, rank, world)
        return
    if w.get("maint"):
        run_maintenance(args, w, rank, world, local)
        return

    import torch
    import dcore_b200 as dc
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    V, s, d = make_graph(dc, w, rank)
    E = int(len(s))
    g = dc.Graph.from_edges(V, s, d, device=local)
    stream = torch.cuda.ExternalStream(g.stream())

    def step():
        g.decompose(dc.METHOD_INCREMENTAL)
        g.materialize_rows()  # dense rows (kmax+1) x V in HBM

    for _ in range(args.warmup):
        g.release_rows()
        step()
    infos = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = dc.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(args.steps):
        g.release_rows()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        infos.append(g.decomp_info())
    launches = dc.launch_count() - launches0
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    total_ms = float(np.sum(times))
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    ms_per_step = max_ms / args.steps
    value = world * E / (ms_per_step / 1000.0)
    K = infos[-1]["kmax"]

    # ---- roofline of the dominant kernel (engine counters, CUDA events)
    peak, peak_kind = peaks()
    inf = infos[-1]
    peel_ms = float(np.mean([i["kmax_ms"] for i in infos]))
    rows_ms = float(np.mean([i["rows_ms"] for i in infos]))
    kernels = {
        # fused kmax + row-0 peel: per pass 12 B per edge (id + two-sided
        # degree update) + 16 B per vertex, two passes
        "k_peel2": {"ms": peel_ms, "bytes": 2 * (12.0 * E + 16.0 * V)},
        # row-to-row refinement: 8 B per adjacency entry read (id + neighbour
        # value) + 16 B per evaluation (value, two counters, queue state)
        "k_trans2": {"ms": rows_ms, "bytes": 8.0 * inf.get("entries", 0) + 16.0 * inf["evals"]},
    }
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    ach = kernels[dom]["bytes"] / (kernels[dom]["ms"] / 1000.0) / 1e9
    roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind, "traffic": kernel_traffic(dom, args.workload),
            "kernels": {k: {"ms": v["ms"], "alg_bytes": v["bytes"],
                            "achieved_gbs": v["bytes"] / (v["ms"] / 1000.0) / 1e9 if v["ms"] else None}
                        for k, v in kernels.items()}}

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if args.e2e_steps > 0:
        hs = dc.pinned_array(E, np.uint32)
        hd = dc.pinned_array(E, np.uint32)
        hs[:] = s
        hd[:] = d
        hk = dc.pinned_array(V, np.int32)
        hrows = dc.pinned_array((K + 1) * V, np.int32).reshape(K + 1, V)
        et = []
        for i in range(args.e2e_steps + 1):
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g2 = dc.Graph.from_edges(V, hs, hd, device=local)
            k2, _ = g2.decompose(dc.METHOD_INCREMENTAL)
            g2.kmaxes(out=hk)
            g2.rows(0, k2 + 1, out=hrows[:k2 + 1])
            g2.free()
            torch.cuda.synchronize()
            if i > 0:  # first call is a warm-up
                et.append(time.perf_counter() - t0)
        te = torch.tensor([float(np.mean(et))], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": world * E / float(te.item()), "unit": "edges/s", "h2d_bytes_per_step": 8 * E,
               "d2h_bytes_per_step": 4 * V * (K + 2), "timing": "wall clock, synchronized, mean of steps"}
        if np.any(hrows[0] != g.rows(0, 1)[0]):
            raise RuntimeError("e2e rows differ from the device-resident run")

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, V, s, d, budget_s=args.cpu_seconds)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": args.workload, "graph": w["desc"], "V": V, "E": E, "kmax": K,
                           "lmax": inf["lmax"], "method": "incremental rows", "output": "dense rows in HBM",
                           "l2": "inputs larger than L2 (graph %.0f MB, rows %.0f MB)" % (
                               8.0 * E / 2**20, 4.0 * (K + 1) * V / 2**20),
                           "parallelism": f"replicas x{world}"},
                "phases_ms": {"peel": peel_ms, "rows": rows_ms,
                              "other": ms_per_step - peel_ms - rows_ms},
                "gpu_launches": int(launches), "roofline": roof, "e2e": e2e, "cpu_baseline": cpu,
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    g.free()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
