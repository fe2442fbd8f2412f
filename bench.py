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
    "decomp-rmat19": dict(gen="rmat", scale=19, ef=16, seed=1,
                          desc="R-MAT scale 19, edge factor 16, a=.57 b=.19 c=.19, dedup, permuted"),
    "decomp-er10k": dict(gen="er", n=10_000, m=100_000, seed=1, desc="directed G(n=10000, m=100000)"),
    # maintenance: R-MAT graph + stream of 50% inserts of absent edges and 50%
    # deletes of present edges, valid in sequence, in several batch sizes
    # (20 batches of 1, 100 and 10,000 updates, then one of 1,000,000)
    "maint-rmat24": dict(gen="rmat", scale=24, ef=16, seed=1, ops=1_202_020, maint=True,
                         sizes=[(1, 20), (100, 20), (10_000, 20), (1_000_000, 1)],
                         desc="R-MAT scale 24, edge factor 16 + 1e6-op update stream (50% insert / 50% delete)"),
    "maint-rmat22": dict(gen="rmat", scale=22, ef=16, seed=1, ops=1_202_020, maint=True,
                         sizes=[(1, 20), (100, 20), (10_000, 20), (1_000_000, 1)],
                         desc="R-MAT scale 22, edge factor 16 + 1e6-op update stream (50% insert / 50% delete)"),
    # serving loop: 64 device-resident graphs, open-loop Poisson arrivals
    "serve-64": dict(serve=True, n_graphs=64, scales=(16, 22), efs=(8, 32), seed=1, budget_gb=150.0,
                     rate=25.0, requests=500, sat_rate=2000.0, sat_requests=4000, max_request=10_000,
                     insert_frac=0.6, workers=4,
                     desc="64 R-MAT graphs, scale U{16..22}, edge factor U{8..32}; Poisson arrivals of requests "
                          "of log-uniform 1..1e4 updates (60% insert / 40% delete) on uniformly chosen graphs; "
                          "150 GB HBM admission budget; continuous batching"),
    # learned scheduler against the rule of thumb on R-MAT 23
    "sched-rmat23": dict(sched=True, scale=23, ef=16, seed=1, train_scales=(20, 21, 22, 23), train_batches=40,
                         train_max=65_536, train_hot_frac=0.25, eval_batches=60, eval_max=1_000_000, hot_frac=0.1,
                         desc="R-MAT scale 23, edge factor 16; batches of log-uniform 1..1e6 updates "
                              "(50% insert / 50% delete), 10% of batches on the top-1% out-degree vertices"),
}
METRIC_SERVE = "updates/s serving loop"
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


def parse_tuning(text):
    """--tuning "peel_bps,rows_bps,chunk[,cut1,...]" -> set_tuning arguments
    (cuts in per mille of kmax, at most seven)."""
    f = [int(x) for x in text.split(",") if x.strip()]
    if len(f) < 3 or len(f) > 10:
        raise ValueError("--tuning wants peel_bps,rows_bps,chunk and up to seven cuts")
    return f[0], f[1], f[2], f[3:]


def kernel_traffic(kernel, workload):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload, {}).get(kernel)


def reference_gpu(V, s, d, g):
    """The reference's own GPU dcore() on the same graph (oracle/_ref), timed
    around the call as the reference times it (host clock, its allocation,
    uploads, per-row degree resets and per-row result copies included), and
    its result compared with the engine's."""
    from oracle import ref_gpu
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/ref_dcore not built (reference sources absent at build time)"}
    if V >= ref_gpu.MAX_V:
        return {"unavailable": f"V = {V} >= 1,000,000: the reference's unchecked per-block peel buffers "
                               "(1,000,000 entries, src/cuda_utils.cuh:10-13) can overflow; not run"}
    kmax, lmax, kmaxes, rows, ms = ref_gpu.dcore(V, s, d)
    same = (kmax == g.decomp_info()["kmax"] and np.array_equal(kmaxes, g.kmaxes())
            and np.array_equal(rows, g.rows()))
    return {"ms": ms, "edges_per_s": len(s) / (ms / 1000.0), "same_result": bool(same),
            "timing": "host clock around dcore(), as main.cu:249-254 reports it"}


def make_graph_oracle(w, rank):
    """The same seeded graph as make_graph, built by the oracle's restatement
    of the generators (the reference arm never loads the engine library)."""
    from oracle import oracle
    seed = w["seed"] + rank
    if w["gen"] == "rmat":
        return oracle.gen_rmat(w["scale"], w["ef"], seed)
    s, d = oracle.gen_er(w["n"], w["m"], seed)
    return w["n"], s, d


def decomp_config(args, w, V, E, kmax, lmax, world):
    """The config of a decomposition line; both arms print exactly this."""
    return {"workload": args.workload, "graph": w["desc"], "V": int(V), "E": int(E), "kmax": int(kmax),
            "lmax": int(lmax), "output": "kmax per vertex and dense rows lmax[k][v], k = 0..kmax",
            "l2": "inputs larger than L2 (graph %.0f MB, rows %.0f MB)" % (8.0 * E / 2**20,
                                                                         4.0 * (kmax + 1) * V / 2**20),
            "parallelism": f"replicas x{world}"}


def peel_bytes(V, s, d, kmaxes):
    """Algorithmic bytes of the fused peel (kmax and row 0), as a per-row peel
    moves them (the reference's passes, main.cu:27-195): the kmax pass
    B_K = 12 E + 16 V (out-adjacency ids, in-degree read-modify-write;
    offsets, degree init, result and state per vertex) and row 0
    B_0 = 8 D_0 + 16 I_0 + 24 V (D_0 = all list entries, I_0 = E)."""
    E = float(len(s))
    return (12.0 * E + 16.0 * V) + (8.0 * 2 * E + 16.0 * E + 24.0 * V)


def refinement_bytes(V, s, d, kmaxes, rows):
    """Algorithmic bytes of rows 1..kmax derived row to row, from the oracle's
    result: every value that changes from row k-1 to row k is evaluated once,
    reading its lists' prefixes inside C_k = {kmax >= k} (4 B id + 4 B
    neighbour value per entry), its old value and its new value (4 + 4 B),
    and recording the change (v, k, l: 12 B); every vertex leaving C_k is
    marked (4 B).  Unchanged values cost nothing: this is the floor of a
    refinement that evaluates each change exactly once.  Returns (bytes,
    changes, entries)."""
    K = rows.shape[0] - 1
    cv, ck = [], []
    for k0 in range(1, K + 1, 16):
        k1 = min(K + 1, k0 + 16)
        ks = np.arange(k0, k1)
        m = (rows[k0:k1] != rows[k0 - 1:k1 - 1]) & (kmaxes[None, :] >= ks[:, None])
        kk, vv = np.nonzero(m)
        cv.append(vv.astype(np.int64))
        ck.append(ks[kk].astype(np.int64))
    cv = np.concatenate(cv) if cv else np.zeros(0, np.int64)
    ck = np.concatenate(ck) if ck else np.zeros(0, np.int64)
    W = K + 2
    entries = 0
    for a, b in ((s, d), (d, s)):  # out-lists, then in-lists
        keys = np.sort(a.astype(np.int64) * W + (K + 1 - kmaxes[b].astype(np.int64)))
        hi = np.searchsorted(keys, cv * W + (K + 1 - ck), side="right")
        lo = np.searchsorted(keys, cv * W, side="left")
        entries += int((hi - lo).sum())
        del keys
    leaving = int(V - np.count_nonzero(kmaxes == K))
    return 8.0 * entries + 20.0 * len(cv) + 4.0 * leaving, int(len(cv)), entries


def oracle_decomposition(V, s, d, rows=None):
    """The oracle's full decomposition on all host threads, timed from its
    built CSR/CSC to the last row (no sampling, no extrapolation)."""
    from oracle import oracle
    K, L, kmaxes, out, secs, nt = oracle.dcore_timed(V, s, d, 0, rows)
    return {"kmax": K, "lmax": L, "kmaxes": kmaxes, "rows": out, "seconds": secs, "threads": nt}


def host_cpu():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_from(res, E, what):
    return {"value": E / res["seconds"], "unit": "edges/s", "cores": res["threads"], "kind": "port",
            "sample": f"{what}: one full decomposition (kmax pass + all {res['kmax'] + 1} rows, bucket-queue "
                      f"peel per row, rows in parallel) on {res['threads']} threads of {host_cpu()}, "
                      f"{res['seconds']:.2f} s, timed from the built CSR/CSC; no sampling"}


def check_parity(g, res, chunk=32):
    """The engine's decomposition against the oracle's: kmax, lmax, every
    kmax value and every dense row (checkDCore's criterion, main.cu:276-293).
    Raises on any difference."""
    info = g.decomp_info()
    K = res["kmax"]
    if (info["kmax"], info["lmax"]) != (K, res["lmax"]):
        raise RuntimeError(f"parity: kmax/lmax {info['kmax']}/{info['lmax']} != oracle {K}/{res['lmax']}")
    if not np.array_equal(g.kmaxes(), res["kmaxes"]):
        raise RuntimeError("parity: kmax values differ from the oracle")
    for k0 in range(0, K + 1, chunk):
        n = min(chunk, K + 1 - k0)
        if not np.array_equal(g.rows(k0, n), res["rows"][k0:k0 + n]):
            raise RuntimeError(f"parity: rows {k0}..{k0 + n - 1} differ from the oracle")
    return {"vs": "oracle (CPU restatement, oracle/dcore_oracle.c)", "exact": True, "kmax": K,
            "rows_checked": K + 1, "values_checked": int((K + 1) * len(res["kmaxes"]) + len(res["kmaxes"]))}


def check_against_oracle(g, V, s, d, chunk=32):
    """kmax, lmax, every kmax value and every row of the engine's current
    decomposition against the oracle's decomposition of the edge list
    (s, d), computed a chunk of rows at a time so that large graphs fit in
    host memory (checkDCore's criterion, main.cu:276-293).  Raises on any
    difference."""
    from oracle import oracle
    t0 = time.perf_counter()
    og = oracle.BuiltGraph(V, s, d)
    K, okmaxes = og.kmax()
    info = g.decomp_info()
    if info["kmax"] != K:
        raise RuntimeError(f"parity: kmax {info['kmax']} != oracle {K}")
    if not np.array_equal(g.kmaxes(), okmaxes):
        raise RuntimeError("parity: kmax values differ from the oracle")
    lmax = 0
    buf = None
    for k0 in range(0, K + 1, chunk):
        k1 = min(K + 1, k0 + chunk)
        want = og.rows(okmaxes, k0, k1, out=buf)
        buf = want.base if want.base is not None else want
        lmax = max(lmax, int(want.max()) if want.size else 0)
        if not np.array_equal(g.rows(k0, k1 - k0), want):
            raise RuntimeError(f"parity: rows {k0}..{k1 - 1} differ from the oracle")
    og.close()
    if info["lmax"] != lmax:
        raise RuntimeError(f"parity: lmax {info['lmax']} != oracle {lmax}")
    return {"vs": "oracle (CPU restatement, oracle/dcore_oracle.c)", "exact": True, "kmax": K,
            "rows_checked": K + 1, "values_checked": int((K + 2) * V), "oracle_s": time.perf_counter() - t0}


def run_reference(args, w, rank, world):
    """The reference arm: the oracle's CPU restatement of the reference's
    decomposition (the reference has no CPU implementation of the path) on
    all host threads, one full decomposition per step.  Rank 0 only; nothing
    of the engine is loaded."""
    if rank != 0:
        return
    if w.get("serve") or w.get("sched") or w.get("maint"):
        run_reference_recompute(args, w)
        return
    V, s, d = make_graph_oracle(w, 0)
    E = int(len(s))
    rows = None
    secs, res = [], None
    for i in range(args.warmup + args.steps):
        res = oracle_decomposition(V, s, d, rows)
        rows = res["rows"].base if res["rows"].base is not None else res["rows"]
        if i >= args.warmup:
            secs.append(res["seconds"])
    ms = 1000.0 * float(np.mean(secs))
    value = E / (ms / 1000.0)
    line = {"metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic", "impl": "reference",
            "config": decomp_config(args, w, V, E, res["kmax"], res["lmax"], world),
            "cpu_baseline": dict(cpu_baseline_from(res, E, "each step"), value=value),
            "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_seconds": secs}
    print(json.dumps(line), flush=True)


def run_reference_recompute(args, w):
    """CPU path for the maintenance, scheduler and serving workloads: the
    reference keeps a decomposition current by recomputing it (checkDCore,
    main.cu:264-293), so every batch costs one full decomposition of its
    graph on the host cores.  Each step times one full oracle decomposition
    of the workload's graph (for serving: the graph of median size)."""
    from oracle import oracle
    if w.get("serve"):
        scales, efs, phases = serve_plan(w, 0, args.requests, args.rate)
        _, gid, size, _ = phases[1]
        nominal = (2.0 ** scales) * efs
        mid = int(np.argsort(nominal)[len(nominal) // 2])
        V, s, d = oracle.gen_rmat(int(scales[mid]), int(efs[mid]), w["seed"] * 1000 + mid)
        what = f"graph {mid} of the mix (scale {scales[mid]}, edge factor {efs[mid]})"
    else:
        V, s, d = oracle.gen_rmat(w["scale"], w["ef"], w["seed"])
        what = w["desc"].split(";")[0]
    E = int(len(s))
    rows, secs, res = None, [], None
    for i in range(args.warmup + args.steps):
        res = oracle_decomposition(V, s, d, rows)
        rows = res["rows"].base if res["rows"].base is not None else res["rows"]
        if i >= args.warmup:
            secs.append(res["seconds"])
    rate = E / float(np.mean(secs))  # edges/s of one recomputation
    if w.get("serve"):
        dedup = E / nominal[mid]
        seconds = float(np.sum(nominal[gid] * dedup / rate))  # one recomputation per request
        value = float(size.sum()) / seconds
        metric = METRIC_SERVE
        note = "every request costs one recomputation of its graph at the measured edges/s"
        config = {"workload": args.workload, "graphs": w["desc"], "requests": int(len(gid))}
    elif w.get("sched"):
        ev_sizes = _log_uniform(np.random.default_rng(w["seed"] + 77), w["eval_batches"], w["eval_max"])
        value = float(ev_sizes.mean()) * rate / E
        metric = METRIC_MAINT
        note = "every batch costs one recomputation of the graph"
        config = {"workload": args.workload, "graph": w["desc"], "V": V, "E": E}
    else:
        value = 10_000 * rate / E
        metric = METRIC_MAINT
        note = "one recomputation per batch of 10,000 updates"
        config = {"workload": args.workload, "graph": w["desc"], "V": V, "E": E}
    base = cpu_baseline_from(res, E, what)
    line = {"metric": metric, "value": value, "unit": "updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(secs)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic", "impl": "reference",
            "config": config, "cpu_baseline": dict(base, value=value, unit="updates/s",
                                                   sample=base["sample"] + "; " + note),
            "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    g.set_row_repair(args.row_repair)
    if args.tuning:
        g.set_tuning(*parse_tuning(args.tuning))
        tune_src = "given (--tuning)"
    elif args.autotune:
        g.autotune()  # launch shapes and row cuts of the recomputations, chosen on the initial graph
        tune_src = "autotuner (dc_autotune) on the initial graph, before the timed batches"
    else:
        tune_src = "defaults"
    tuning = g.tuning()
    g.decompose(dc.METHOD_INCREMENTAL)
    # the memory pool holds as much again as the graph uses, so a store
    # rebuild inside a timed batch maps no new pages (a warm serving process)
    reserve = int(g.device_bytes())
    dc.reserve_device_memory(local, reserve)
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
        local_rows = 0
        local_ins = 0
        captured = 0
        detail = []
        for _ in range(nb):
            st = g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], args.maint_method)
            lat.append(st["total_ms"])
            methods.append(st["method"])
            local_rows += st["rows_local"] & 1
            local_ins += (st["rows_local"] >> 1) & 1
            # per batch: ms (apply, kmax/row-0 update, rows), rows recomputed
            # or repaired, method, store rebuilt
            detail.append([round(st["total_ms"], 2), round(st["apply_ms"], 2), round(st["core_ms"], 2),
                           round(st["rows_ms"], 2), st["rows_recomputed"], st["rows_local"], st["method"],
                           st["rebuilt"], round(st["del_repair_ms"], 2), round(st["ins_repair_ms"], 2),
                           st["ins_scanned"], st["captured"]])
            captured += st["captured"]
            pos += bs
        lat = np.array(lat)
        per_size[str(bs)] = {"batches": nb, "updates_per_s": bs * nb / (lat.sum() / 1000.0),
                             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                             "methods": {"local": methods.count(1), "repeel": methods.count(2)},
                             "rows_repaired_in_place": {"deletions": local_rows, "insertions": local_ins},
                             "captured_graph_batches": captured,
                             "batch_detail": {"fields": ["total_ms", "apply_ms", "core_ms", "rows_ms",
                                                         "rows_recomputed", "rows_repaired", "method", "rebuilt",
                                                         "del_repair_ms", "ins_repair_ms", "ins_scanned",
                                                         "captured"],
                                              "batches": detail}}
    clocks = sampler.stop()
    launches = dc.launch_count() - launches0
    parity = None
    if rank == 0 and not args.no_oracle:
        # the maintained decomposition after the whole stream against the
        # oracle's decomposition of the final edge set
        fs, fd = _final_edges(s, d, u[:pos], v[:pos], dl[:pos])
        parity = check_against_oracle(g, V, fs, fd)
        parity["after"] = f"{pos} updates in {sum(x['batches'] for x in per_size.values())} batches"
    head = per_size.get("10000") or per_size[max(per_size, key=lambda k: int(k))]
    line = {"metric": METRIC_MAINT, "value": head["updates_per_s"], "unit": "updates/s", "n_gpus": world,
            "steps": sum(x["batches"] for x in per_size.values()), "warmup": 1,
            "ms_per_step": head["p50_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": args.workload, "graph": w["desc"], "V": V, "E": int(len(s)),
                       "headline": "batches of 10,000 updates", "per_batch_size": per_size,
                       "method": {0: "scheduler", 1: "local", 2: "re-peel"}[args.maint_method],
                       "row_repair": bool(args.row_repair), "tuning": dict(tuning, source=tune_src),
                       "memory_pool_reserved_gb": round(reserve / 1e9, 2)},
            "gpu_launches": int(launches), "parity": parity, "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.free()


def _final_edges(s, d, u, v, dl):
    """Edge list after a valid update stream (multiplicities 0/1)."""
    keys = np.concatenate([(s.astype(np.uint64) << 32) | d, (u.astype(np.uint64) << 32) | v])
    w = np.concatenate([np.ones(len(s), np.int64), np.where(dl == 1, -1, 1).astype(np.int64)])
    uk, inv = np.unique(keys, return_inverse=True)
    cnt = np.zeros(len(uk), np.int64)
    np.add.at(cnt, inv, w)
    fk = uk[cnt > 0]
    return (fk >> 32).astype(np.uint32), (fk & 0xFFFFFFFF).astype(np.uint32)


def _log_uniform(rng, n, hi):
    return np.minimum(hi, np.exp(rng.uniform(0, np.log(hi), n)).astype(np.int64) + 1)


def serve_plan(w, rank, requests=None, rate=None):
    """Graph sizes and the two request phases: (arrival times, graph, size)
    at the latency rate, then at the saturation rate."""
    rng = np.random.default_rng(w["seed"] * 7919 + rank)
    n = w["n_graphs"]
    scales = rng.integers(w["scales"][0], w["scales"][1] + 1, n)
    efs = rng.integers(w["efs"][0], w["efs"][1] + 1, n)
    phases = []
    for R, lam in ((requests or w["requests"], rate or w["rate"]), (w["sat_requests"], w["sat_rate"])):
        t_arr = np.cumsum(rng.exponential(1.0 / lam, R))
        gid = rng.integers(0, n, R)
        size = _log_uniform(rng, R, w["max_request"])
        phases.append((t_arr, gid, size, lam))
    return scales, efs, phases


def _serve_phase(dc, srv, graphs, ids, pos, t_arr, gid, size, local):
    info0 = srv.info()
    launches0 = dc.launch_count()
    sampler = ClockSampler(local)
    sampler.start()
    t0 = time.perf_counter()
    for r in range(len(t_arr)):
        delay = t0 + t_arr[r] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        g, k, p = int(gid[r]), int(size[r]), int(pos[gid[r]])
        _, _, _, u, v, dl = graphs[g]
        srv.submit(ids[g], u[p:p + k], v[p:p + k], dl[p:p + k])
        pos[g] = p + k
    srv.drain()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    comp = srv.completions()
    info = srv.info()
    if (comp["status"] != 0).any():
        raise RuntimeError(f"{int((comp['status'] != 0).sum())} requests failed")
    lat = comp["latency_ms"]
    nb = int(info["batches"] - info0["batches"])
    return {"requests": int(len(t_arr)), "updates": int(size.sum()), "wall_s": wall,
            "updates_per_s": float(size.sum()) / wall, "offered_updates_per_s": float(size.sum()) / float(t_arr[-1]),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                           "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "batches": nb, "mean_requests_per_batch": len(t_arr) / max(1, nb),
            "gpu_launches": int(dc.launch_count() - launches0), "clocks": clocks}


def run_serve(args, w, rank, world, local):
    """Serving loop over many device-resident graphs.  Requests arrive
    open-loop at Poisson times in two phases: below capacity (latency:
    submission to the end of the batch holding the request, p50/p99) and at
    saturation (throughput: updates of all requests / (last completion - first
    submission)).  A sample of graphs is checked afterwards against a fresh
    decomposition of its final edge set."""
    from concurrent.futures import ThreadPoolExecutor
    import torch
    import dcore_b200 as dc
    torch.cuda.set_device(local)
    scales, efs, phases = serve_plan(w, rank, args.requests, args.rate)
    n = w["n_graphs"]
    need = sum(np.bincount(gid, weights=size, minlength=n) for _, gid, size, _ in phases).astype(np.int64)

    def gen(i):
        V, s, d = dc.gen_rmat(int(scales[i]), int(efs[i]), w["seed"] * 1000 + 17 * rank + i)
        u, v, dl = dc.gen_updates(V, s, d, int(need[i]), w["insert_frac"], w["seed"] * 1000 + 500 + i)
        return V, s, d, u, v, dl

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        graphs = list(ex.map(gen, range(n)))
    t_gen = time.perf_counter() - t0
    E_tot = int(sum(len(g[1]) for g in graphs))
    workers = args.workers or w["workers"]
    srv = dc.Server(int(w["budget_gb"] * 1e9), max_concurrent=workers, method=args.maint_method, device=local)
    ids = [srv.add_graph(g[0], g[1], g[2]) for g in graphs]
    t0 = time.perf_counter()
    for i in ids:  # admit and decompose every graph before the timed phases
        srv.result(i, graphs[i][0], rows=False)
    t_admit = time.perf_counter() - t0
    pos = np.zeros(n, np.int64)
    lat_phase = _serve_phase(dc, srv, graphs, ids, pos, *phases[0][:3], local)
    sat_phase = _serve_phase(dc, srv, graphs, ids, pos, *phases[1][:3], local)
    info = srv.info()
    # exactness on a sample: the three smallest graphs and the largest one of
    # scale <= 19 (dense rows of the largest graphs run to tens of GB)
    order = np.argsort([len(g[1]) for g in graphs])
    mid = [int(i) for i in order if scales[i] <= 19][-1:]
    checked = []
    from oracle import oracle
    for i in list(order[:3]) + mid:
        V, s, d, u, v, dl = graphs[i]
        km, rows = srv.result(ids[i], V)
        fs, fd = _final_edges(s, d, u[:pos[i]], v[:pos[i]], dl[:pos[i]])
        okm, olm, okmaxes, orows = oracle.dcore(V, fs, fd)
        if not (np.array_equal(okmaxes, km) and np.array_equal(orows, rows)):
            raise RuntimeError(f"graph {i}: served result differs from the oracle's decomposition")
        checked.append(int(i))
    srv.free()
    value = sat_phase["updates_per_s"]
    clocks = sat_phase.pop("clocks")
    lat_clocks = lat_phase.pop("clocks")
    line = {"metric": METRIC_SERVE, "value": value, "unit": "updates/s", "n_gpus": world,
            "steps": sat_phase["requests"], "warmup": 0, "ms_per_step": lat_phase["latency_ms"]["p50"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": args.workload, "graphs": w["desc"], "n_graphs": n, "E_total": E_tot,
                       "scales": scales.tolist(), "edge_factors": efs.tolist(), "workers": workers,
                       "budget_gb": w["budget_gb"], "method": {0: "scheduler", 1: "local", 2: "re-peel"}[
                           args.maint_method],
                       "gen_s": t_gen, "admit_s": t_admit,
                       "step": "one request (submission to completion)",
                       "value": "updates/s of the saturation phase; ms_per_step = p50 latency below capacity"},
            "latency_phase": dict(lat_phase, offered_req_s=phases[0][3], clocks=lat_clocks),
            "saturation_phase": dict(sat_phase, offered_req_s=phases[1][3]),
            "hbm": {"peak_charged_gb": info["peak_bytes"] / 1e9, "measured_resident_gb": info["measured_bytes"] / 1e9,
                    "resident": info["resident"], "evictions": info["evictions"]},
            "e2e": {"value": value, "unit": "updates/s",
                    "h2d_bytes_per_step": float(9 * sat_phase["updates"] / sat_phase["requests"]),
                    "d2h_bytes_per_step": 0,
                    "timing": "wall clock through dc_server_submit/drain with host request buffers"},
            "gpu_launches": sat_phase["gpu_launches"],
            "parity": {"vs": "oracle (CPU restatement, oracle/dcore_oracle.c)", "exact": True,
                       "graphs_checked": checked, "what": "kmax values and every dense row after all requests"},
            "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_row_sharded(args, w, rank, world, local, dist):
    """Row sharding of ONE decomposition (strong scaling): every rank holds the
    same graph, computes kmax and row 0, derives the same row ranges from
    dc_row_weights and computes its range straight from row 0, writing its
    dense rows into its own HBM (no exchange).  With --emulate-ranks N on one
    GPU the N ranges run one after another on the device, each rank's time
    being the shared kmax/row-0/weights time plus its own range; ranks never
    wait on one another, so the maximum is what N GPUs would take."""
    import torch
    import dcore_b200 as dc
    import dcore_dist
    nranks = args.emulate_ranks if args.emulate_ranks > 1 else world
    V, s, d = make_graph(dc, w, 0)  # the same graph on every rank
    E = int(len(s))
    g = dc.Graph.from_edges(V, s, d, device=local)
    stream = torch.cuda.ExternalStream(g.stream())
    bufs = {}

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        return e

    def step(ranks):
        e0 = ev()
        g.decompose_rows(0, 0)  # kmax + row 0, recomputed
        wts = g.row_weights()
        e1 = ev()
        shards = dcore_dist.row_shards(wts, nranks)
        per = {}
        for r in ranks:
            a0, b0 = shards[r]
            t0 = ev()
            if a0 <= b0:
                g.decompose_rows(a0, b0)
                n = b0 - a0 + 1
                if r not in bufs or bufs[r].numel() < n * V:
                    bufs[r] = torch.empty(n * V, dtype=torch.int32, device=f"cuda:{local}")
                g.rows_to_device(a0, n, bufs[r].data_ptr())
            t1 = ev()
            per[r] = (t0, t1)
        t_end = ev()
        t_end.synchronize()
        shared = e0.elapsed_time(e1)
        return shared, {r: a.elapsed_time(b) for r, (a, b) in per.items()}, shards

    ranks = list(range(nranks)) if args.emulate_ranks > 1 else [rank]
    for _ in range(args.warmup):
        step(ranks)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = dc.launch_count()
    step_ms, shared_ms, range_ms = [], [], {r: [] for r in ranks}
    for _ in range(args.steps):
        sh, per, shards = step(ranks)
        shared_ms.append(sh)
        for r in ranks:
            range_ms[r].append(per[r])
        step_ms.append(sh + max(per.values()))
    launches = dc.launch_count() - launches0
    clocks = sampler.stop()
    mine = float(np.mean(step_ms))
    ms = dcore_dist.max_over_ranks(mine, dist, device=f"cuda:{local}")
    if rank == 0:
        line = {"metric": METRIC, "value": E / (ms / 1000.0), "unit": "edges/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": {"workload": args.workload, "graph": w["desc"], "V": V, "E": E,
                           "parallelism": f"row shards x{nranks}" + (" (emulated on one GPU)"
                                                                     if args.emulate_ranks > 1 else ""),
                           "output": "dense rows of each range in its rank's HBM",
                           "shards": [list(map(int, x)) for x in shards]},
                "per_rank_ms": {"kmax_row0_weights": float(np.mean(shared_ms)),
                                "ranges": {str(r): float(np.mean(v)) for r, v in range_ms.items()}},
                "gpu_launches": int(launches), "clocks": clocks}
        print(json.dumps(line), flush=True)
    g.free()


def _stream_times(dc, g, u, v, dl, sizes, method):
    """Per batch: device ms, method, rows repaired in place (bit 0
    deletions, bit 1 insertions)."""
    pos, ms, methods, local, phases = 0, [], [], [], []
    for bs in sizes:
        st = g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], method)
        ms.append(st["total_ms"])
        methods.append(st["method"])
        local.append(st["rows_local"])
        phases.append([round(st["apply_ms"], 2), round(st["core_ms"], 2), round(st["rows_ms"], 2), st["rebuilt"],
                       st["captured"]])
        pos += bs
    _stream_times.phases = phases
    return np.array(ms), np.array(methods), np.array(local)


def _hot_stream(dc, V, s, d, sizes, hot_frac, rng, seed):
    od = np.bincount(s, minlength=V)
    hot = np.argsort(-od, kind="stable")[:max(1, V // 100)].astype(np.uint32)
    hot_batch = rng.uniform(size=len(sizes)) < hot_frac
    op_hot = np.repeat(hot_batch.astype(np.uint8), sizes)
    u, v, dl = dc.gen_updates_hot(V, s, d, int(np.sum(sizes)), 0.5, seed, hot, op_hot)
    return u, v, dl, hot_batch


def run_sched(args, w, rank, world, local):
    """Learned scheduler against the rule of thumb.  Training: fresh R-MAT
    graphs, log-uniform batch streams (10% hot) applied to two copies, one
    per path -- incremental (local kmax / row-0 update, rows repaired in
    place wherever the batch fits) and full (fused re-peel, rows
    recomputed) -- logging features and device times; the network learns
    log(time) of each path.  Evaluation: a fresh R-MAT 23 graph and stream
    applied to two copies, one with the network attached, one with the rule
    of thumb (method by batch size, rows by the default row mode); both must
    end equal to the oracle's decomposition of the final edge set."""
    import torch
    import dcore_b200 as dc
    torch.cuda.set_device(local)
    rng = np.random.default_rng(w["seed"] + 31 * rank)
    # ---- training log: fresh graphs of several sizes (the graph-size
    # features must vary), each stream applied to one copy per method
    Xs, Ts = [], []
    t0 = time.perf_counter()
    for j, scale in enumerate(w["train_scales"]):
        V, s, d = dc.gen_rmat(scale, w["ef"], w["seed"] + 100 + 10 * j + rank)
        tr_sizes = _log_uniform(rng, w["train_batches"], w["train_max"])
        u, v, dl, _ = _hot_stream(dc, V, s, d, tr_sizes, w["train_hot_frac"], rng, w["seed"] + 200 + j)
        logs = []
        for method, mode in ((dc.MAINT_LOCAL, 3), (dc.MAINT_REPEEL, 0)):
            with dc.Graph.from_edges(V, s, d, device=local, gap_min=2, gap_div=16) as g:
                g.set_row_repair(mode)
                g.decompose()
                g.maint_log(True)
                _stream_times(dc, g, u, v, dl, tr_sizes, method)
                logs.append(g.maint_log())
        (X, _, ta), (_, _, tb) = logs
        Xs.append(X)
        Ts.append(np.log(np.stack([ta[:, 0], tb[:, 0]], 1).clip(1e-3)))
    X = np.concatenate(Xs).astype(np.float32)
    T = np.concatenate(Ts).astype(np.float32)
    sched = dc.Scheduler(seed=w["seed"])
    sched.set_norm(X.mean(0), 1.0 / (X.std(0) + 1e-3))
    loss = sched.train(X, T, np.ones_like(T, np.uint8), epochs=800, lr=3e-3)
    t_train = time.perf_counter() - t0
    # ---- evaluation stream on R-MAT 23
    V, s, d = dc.gen_rmat(w["scale"], w["ef"], w["seed"] + rank)
    ev_sizes = _log_uniform(np.random.default_rng(w["seed"] + 77), w["eval_batches"], w["eval_max"])
    u, v, dl, hot_batch = _hot_stream(dc, V, s, d, ev_sizes, w["hot_frac"], rng, w["seed"] + 300)
    res = {}
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = dc.launch_count()
    # the two policies take the batches in turn on their own copies (each
    # batch timed on the wall clock around dc_maintain, which returns after
    # the batch): both see the same device state -- memory pool growth, L2 --
    # so neither pays a one-time cost the other skips
    graphs = {}
    for name, sch in (("learned", sched), ("rule", None)):
        g = dc.Graph.from_edges(V, s, d, device=local, gap_min=2, gap_div=16)
        g.decompose()  # default row mode: the rule's rows; the network sets the path per batch
        g.set_scheduler(sch)
        graphs[name] = g
        res[name] = {"wall": [], "ms": [], "methods": [], "rows_local": [], "phases": [], "graph": g}
    # the memory pool holds as much again as both copies use (store rebuilds
    # inside timed batches map no new pages, as in a warm serving process)
    dc.reserve_device_memory(local, int(sum(g.device_bytes() for g in graphs.values())))
    torch.cuda.synchronize()
    pos = 0
    for i, bs in enumerate(ev_sizes):
        order = ("learned", "rule") if i % 2 == 0 else ("rule", "learned")
        for name in order:
            t0 = time.perf_counter()
            st = graphs[name].maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], dc.MAINT_AUTO)
            r = res[name]
            r["wall"].append(time.perf_counter() - t0)
            r["ms"].append(st["total_ms"])
            r["methods"].append(st["method"])
            r["rows_local"].append(st["rows_local"])
            r["phases"].append([round(st["apply_ms"], 2), round(st["core_ms"], 2), round(st["rows_ms"], 2),
                                st["rebuilt"], st["captured"]])
        pos += bs
    for name, r in res.items():
        for k in ("ms", "methods", "rows_local"):
            r[k] = np.array(r[k])
        r["wall_s"] = float(np.sum(r["wall"]))
        r["device_ms"] = float(r["ms"].sum())
    launches = dc.launch_count() - launches0
    clocks = sampler.stop()
    fs, fd = _final_edges(s, d, u, v, dl)
    parity = {}
    for name in res:
        if not args.no_oracle:
            parity[name] = check_against_oracle(res[name]["graph"], V, fs, fd)
        res[name]["graph"].free()
    L, Rr = res["learned"], res["rule"]
    updates = int(ev_sizes.sum())
    value = updates / L["wall_s"]
    diff = (L["methods"] != Rr["methods"]) | (L["rows_local"] != Rr["rows_local"])
    line = {"metric": METRIC_MAINT, "value": value, "unit": "updates/s", "n_gpus": world,
            "steps": int(len(ev_sizes)), "warmup": 1, "ms_per_step": float(np.median(L["ms"])),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": args.workload, "graph": w["desc"], "V": V, "E": int(len(s)),
                       "updates": updates, "hot_batches": int(hot_batch.sum()),
                       "train": {"graphs": f"R-MAT scales {list(w['train_scales'])}, edge factor {w['ef']}, "
                                           "fresh seeds",
                                 "batches": int(w["train_batches"]) * len(w["train_scales"]),
                                 "max_batch": w["train_max"], "hot_fraction": w["train_hot_frac"],
                                 "paths": "incremental (local, row mode 3) and full (re-peel, row mode 0), "
                                          "one copy of the graph each",
                                 "final_loss": float(loss), "seconds": t_train}},
            "parity": parity or None,
            "scheduler": {"learned_wall_s": L["wall_s"], "rule_wall_s": Rr["wall_s"],
                          "gain_wall": Rr["wall_s"] / L["wall_s"],
                          "learned_device_ms": L["device_ms"], "rule_device_ms": Rr["device_ms"],
                          "gain_device": Rr["device_ms"] / L["device_ms"],
                          "batches_decided_differently": int(diff.sum()),
                          "ms_on_differing_batches": {"learned": float(L["ms"][diff].sum()),
                                                      "rule": float(Rr["ms"][diff].sum())},
                          "learned_methods": {"local": int((L["methods"] == 1).sum()),
                                              "repeel": int((L["methods"] == 2).sum())},
                          "rule_methods": {"local": int((Rr["methods"] == 1).sum()),
                                           "repeel": int((Rr["methods"] == 2).sum())},
                          "batch_detail": {"fields": ["updates", "hot", "learned_ms", "learned_method",
                                                      "learned_rows_in_place", "rule_ms", "rule_method",
                                                      "rule_rows_in_place", "learned [apply, core, rows ms, rebuilt, "
                                                      "captured]", "rule [same]"],
                                           "batches": [[int(ev_sizes[i]), int(hot_batch[i]),
                                                        round(float(L["ms"][i]), 2), int(L["methods"][i]),
                                                        int(L["rows_local"][i]), round(float(Rr["ms"][i]), 2),
                                                        int(Rr["methods"][i]), int(Rr["rows_local"][i]),
                                                        L["phases"][i], Rr["phases"][i]]
                                                       for i in range(len(ev_sizes))]}},
            "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": float(9 * updates / len(ev_sizes)),
                    "d2h_bytes_per_step": 0, "timing": "wall clock of dc_maintain calls with host batches"},
            "gpu_launches": int(launches), "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_decomposition(args, w, rank, world, local, dist):
    """Full decompositions of a freshly loaded graph.  The graph's edge list
    stays resident in HBM; before each step (untimed) a new handle builds the
    CSR/CSC from it, so every timed step is a first decomposition of that
    graph: the fused peel, the neighbour-kmax reordering of the lists, rows
    1..kmax, the skyline and the dense rows written to HBM.  Afterwards the
    result is checked against the oracle's full decomposition, whose timing
    is the CPU baseline."""
    import torch
    import dcore_b200 as dc
    V, s, d = make_graph(dc, w, rank)
    E = int(len(s))
    dev = torch.device("cuda", local)
    d_src = torch.from_numpy(s.view(np.int32)).to(dev)
    d_dst = torch.from_numpy(d.view(np.int32)).to(dev)
    g0 = dc.Graph.from_edges(V, s, d, device=local)
    if args.tuning:
        g0.set_tuning(*parse_tuning(args.tuning))
        tuning, tune_src = g0.tuning(), "given (--tuning)"
    elif args.autotune:
        tuning, _ = g0.autotune()
        tune_src = "autotuner (dc_autotune) on the graph, before the timed steps"
    else:
        tuning, tune_src = g0.tuning(), "defaults"
    g0.free()

    def fresh(cuts=True):
        h = dc.Graph.from_device_edges(V, E, d_src.data_ptr(), d_dst.data_ptr(), device=local)
        h.set_tuning(tuning["peel_blocks_per_sm"], tuning["rows_blocks_per_sm"], tuning["peel_chunk"],
                     tuning["rows_split_permille"] if cuts else [])
        h.synchronize()
        return h

    def timed_step(h):
        """(ms, engine launches) of one decomposition + dense rows on h."""
        st = torch.cuda.ExternalStream(h.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        n0 = dc.launch_count()
        e0.record(st)
        h.decompose(dc.METHOD_INCREMENTAL)
        h.materialize_rows()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1), dc.launch_count() - n0

    for _ in range(args.warmup):
        h = fresh()
        timed_step(h)
        h.free()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    times, infos, launches = [], [], 0
    g = None
    for i in range(args.steps):
        if g is not None:
            g.free()
        g = fresh()
        ms, n = timed_step(g)
        times.append(ms)
        launches += n
        infos.append(g.decomp_info())
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    t = torch.tensor([float(np.sum(times))], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps
    value = world * E / (ms_per_step / 1000.0)
    inf = infos[-1]
    K = inf["kmax"]

    # ---- the same step with rows 1..kmax in one persistent launch (no cuts)
    single = None
    if any(tuning["rows_split_permille"]):
        st_ms = []
        for i in range(4):
            h = fresh(cuts=False)
            ms, _ = timed_step(h)
            if i:
                st_ms.append((ms, h.decomp_info()["rows_ms"]))
            h.free()
        sm = float(np.mean([x for x, _ in st_ms]))
        single = {"ms_per_step": sm, "value": E / (sm / 1000.0), "rows_ms": float(np.mean([r for _, r in st_ms])),
                  "steps": len(st_ms), "note": "same step and launch shapes, rows 1..kmax in one persistent "
                                               "k_trans2 launch"}

    # ---- end to end through the C ABI with host buffers
    e2e, hrows = None, None
    if args.e2e_steps > 0:
        hs = dc.pinned_array(E, np.uint32)
        hd = dc.pinned_array(E, np.uint32)
        hs[:] = s
        hd[:] = d
        hk = dc.pinned_array(V, np.int32)
        hrows = dc.pinned_array((K + 1) * V, np.int32).reshape(K + 1, V)
        et, ph = [], []
        for i in range(args.e2e_steps + 1):
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g2 = dc.Graph.from_edges(V, hs, hd, device=local)
            g2.set_tuning(tuning["peel_blocks_per_sm"], tuning["rows_blocks_per_sm"], tuning["peel_chunk"],
                          tuning["rows_split_permille"])
            t1 = time.perf_counter()
            k2, _ = g2.decompose(dc.METHOD_INCREMENTAL)
            t2 = time.perf_counter()
            g2.kmaxes(out=hk)
            g2.rows(0, k2 + 1, out=hrows[:k2 + 1])
            t3 = time.perf_counter()
            g2.free()
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            if i > 0:  # first call is a warm-up
                et.append(t4 - t0)
                ph.append([t1 - t0, t2 - t1, t3 - t2, t4 - t3])
        te = torch.tensor([float(np.mean(et))], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": world * E / float(te.item()), "unit": "edges/s", "h2d_bytes_per_step": 8 * E,
               "d2h_bytes_per_step": 4 * V * (K + 2), "timing": "wall clock, synchronized, mean of steps",
               "steps": len(et),
               "phases_ms": dict(zip(["create_and_upload", "decompose", "download", "free"],
                                     (1000.0 * np.mean(ph, 0)).round(3).tolist()))}

    # ---- oracle: full decomposition on the host cores (CPU baseline) and
    # the parity check of the last timed step and of the e2e output
    parity, cpu, res = None, None, None
    if rank == 0 and not args.no_oracle:
        res = oracle_decomposition(V, s, d)
        cpu = cpu_baseline_from(res, E, "oracle run beside the engine")
        parity = check_parity(g, res)
        if e2e is not None:
            if not (np.array_equal(hk, res["kmaxes"]) and np.array_equal(hrows, res["rows"])):
                raise RuntimeError("parity: the e2e output differs from the oracle")
            parity["e2e_output_checked"] = True

    # ---- roofline of the dominant kernel (CUDA events on the engine stream)
    peak, peak_kind = peaks()
    peel_ms = float(np.mean([i["kmax_ms"] for i in infos]))
    rows_ms = float(np.mean([i["rows_ms"] for i in infos]))
    kernels = {"k_peel2": {"ms": peel_ms, "bytes": peel_bytes(V, s, d, None),
                           "model": "per-row peel bytes of kmax + row 0: (12 E + 16 V) + (8 D_0 + 16 I_0 + 24 V)"},
               "k_trans2": {"ms": rows_ms, "bytes": None,
                            "model": "one evaluation per changed value: 8 B per C_k list entry of each change, "
                                     "20 B per change, 4 B per vertex leaving C_k"}}
    roof = None
    if res is not None:
        b_ref, n_changes, n_entries = refinement_bytes(V, s, d, res["kmaxes"], res["rows"])
        kernels["k_trans2"].update(bytes=b_ref, changes=n_changes, entries=n_entries)
        for k in kernels.values():
            k["achieved_gbs"] = k["bytes"] / (k["ms"] / 1000.0) / 1e9 if k["ms"] else None
            k["frac"] = k["achieved_gbs"] / peak if k["achieved_gbs"] else None
        dom = max(kernels, key=lambda k: kernels[k]["ms"])
        sort_b = 12.0 * 2 * E
        expand_b = 4.0 * (K + 1) * V
        b_alg = kernels["k_peel2"]["bytes"] + b_ref + sort_b + expand_b
        roof = {"kernel": dom, "bound": "hbm", "achieved": kernels[dom]["achieved_gbs"], "peak": peak,
                "unit": "GB/s", "frac": kernels[dom]["frac"], "peak_source": peak_kind,
                "traffic": kernel_traffic(dom, args.workload),
                "timing": "CUDA events on the graph's stream around each phase inside dc_decompose; the rows "
                          "phase spans all k_trans2 launches (row segments on concurrent streams joined back)",
                "kernels": kernels,
                "decomposition": {"alg_bytes": b_alg, "ms": ms_per_step,
                                  "achieved_gbs": b_alg / (ms_per_step / 1000.0) / 1e9,
                                  "frac": b_alg / (ms_per_step / 1000.0) / 1e9 / peak,
                                  "model": "k_peel2 + k_trans2 models + list reordering 12 B per list entry + "
                                           "dense rows 4 (kmax+1) V"},
                "engine_counted": {"k_trans2_entries": inf.get("entries", 0), "evals": inf["evals"],
                                   "drops": inf["drops"]}}
    ref = reference_gpu(V, s, d, g) if rank == 0 else None

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": decomp_config(args, w, V, E, K, inf["lmax"], world),
                "engine": {"method": "fused peel (kmax + row 0), rows 1..kmax derived row to row",
                           "tuning": dict(tuning, source=tune_src),
                           "step": "first decomposition of a freshly built handle (CSR/CSC built untimed from "
                                   "the HBM-resident edge list)"},
                "phases_ms": {"peel": peel_ms, "rows": rows_ms, "other": ms_per_step - peel_ms - rows_ms,
                              "of_other": {k: float(np.mean([i[k + "_ms"] for i in infos]))
                                           for k in ("row0", "skyline", "expand")}},
                "step_ms": times, "gpu_launches": int(launches), "roofline": roof, "parity": parity,
                "single_launch_rows": single, "e2e": e2e, "cpu_baseline": cpu, "reference_gpu": ref,
                "clocks": clocks}
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
    ap.add_argument("--no-oracle", action="store_true",
                    help="decomposition: skip the oracle run (CPU baseline, parity check, roofline model)")
    ap.add_argument("--maint-method", type=int, default=0, help="0 scheduler, 1 local, 2 re-peel")
    ap.add_argument("--requests", type=int, default=0, help="serve: number of requests (0: workload default)")
    ap.add_argument("--rate", type=float, default=0.0, help="serve: arrivals per second (0: workload default)")
    ap.add_argument("--workers", type=int, default=0, help="serve: worker threads (0: workload default)")
    ap.add_argument("--shard", choices=["replicas", "rows"], default="replicas",
                    help="decomposition with N > 1: one graph per rank, or the rows of one graph split over ranks")
    ap.add_argument("--no-row-repair", dest="row_repair", action="store_false",
                    help="maintenance: recompute rows 1..R for deletions instead of repairing them in place")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="decomposition: keep the default launch shapes instead of running dc_autotune first")
    ap.add_argument("--tuning", default="",
                    help="decomposition launch shapes instead of the autotuner: "
                         "peel_bps,rows_bps,chunk[,cut1,...] (cuts in per mille of kmax)")
    ap.add_argument("--emulate-ranks", type=int, default=0,
                    help="row sharding of one decomposition over N ranks, run one range after another on one GPU")
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
    if w.get("serve"):
        run_serve(args, w, rank, world, local)
        return
    if w.get("sched"):
        run_sched(args, w, rank, world, local)
        return

    import torch
    import dcore_b200 as dc
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.shard == "rows" or args.emulate_ranks > 1:
        run_row_sharded(args, w, rank, world, local, dist)
        if dist:
            dist.destroy_process_group()
        return

    run_decomposition(args, w, rank, world, local, dist)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
