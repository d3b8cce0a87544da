"""Benchmark: SCC decomposition throughput (GTEPS) on one B200 per rank.

Workload (default): the large mixed-structure graph -- the union of a directed
R-MAT scale-24 graph (edge factor 16, a/b/c/d = .57/.19/.19/.05) and a
4096 x 4096 grid whose edges are oriented by a fair coin with 5% made
bidirectional; self-loops and duplicates removed; seeded synthetic data.
A step is one full SCC decomposition (method 2: Trim1 + global FW-BW +
Trim1/2 + WCC + FW-BW) of that graph, inputs resident in HBM (the CSR and its
transpose are 2.5 GB, far above the 126 MB L2, so no flush is needed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2|rmat24|c1]

Prints one JSON line (rank 0).  value = whole-job GTEPS = edges of all ranks'
graphs / max-over-ranks device time per step; e2e = the same metric through
the C ABI from pinned host CSR arrays (H2D of the forward CSR with the transpose
rebuilt on the device by scc_graph_upload_csr_out, run, D2H of
the canonical labels inside the timed region).  --gpus N > 1 runs N
independent replicas (the path does not shard; no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes as C
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

WORKLOADS = {
    "c2": dict(rmat_scale=24, edge_factor=16, grid_side=4096, seed=2024),
    "rmat24": dict(rmat_scale=24, edge_factor=16, seed=2024),
    "c3": dict(rmat_scale=24, edge_factor=16, num_cycles=1000, cycle_min=3, cycle_max=100000, seed=2024),
    "c1": dict(rmat_scale=16, edge_factor=8, seed=42),
    # smaller cases of the same shapes, for profiler captures
    "rmat22": dict(rmat_scale=22, edge_factor=16, seed=2024),
    "grid4096": dict(grid_side=4096, seed=2024),
    # mid-degree hubs: top-down levels full of items between one warp's and the
    # edge-parallel path's degrees (the block-wide expansion's workload)
    "hubs": dict(hubs_n=1 << 22, hubs=30000, hub_deg=(64, 4000), seed=5),
}
# CPU-baseline sample of the same workload shape at 1/16 of the vertices
CPU_SAMPLES = {
    "c2": dict(rmat_scale=20, edge_factor=16, grid_side=1024, seed=2024),
    "rmat24": dict(rmat_scale=20, edge_factor=16, seed=2024),
    "c3": dict(rmat_scale=20, edge_factor=16, num_cycles=63, cycle_min=3, cycle_max=100000, seed=2024),
    "c1": dict(rmat_scale=16, edge_factor=8, seed=42),
    "rmat22": dict(rmat_scale=18, edge_factor=16, seed=2024),
    "grid4096": dict(grid_side=1024, seed=2024),
    "hubs": dict(hubs_n=1 << 18, hubs=1875, hub_deg=(64, 4000), seed=5),
}
WORKLOAD_NAMES = {
    "c2": "R-MAT s24 ef16 (a=.57,b=.19,c=.19) U 4096x4096 randomly oriented grid (+5% bidirectional)",
    "rmat24": "R-MAT s24 ef16 (a=.57,b=.19,c=.19)",
    "c3": "R-MAT s24 ef16 (a=.57,b=.19,c=.19) + 1,000 planted directed cycles, lengths log-uniform [3, 100,000]",
    "c1": "R-MAT s16 ef8 (a=.57,b=.19,c=.19)",
    "rmat22": "R-MAT s22 ef16 (a=.57,b=.19,c=.19)",
    "grid4096": "4096x4096 randomly oriented grid (+5% bidirectional)",
    "hubs": "4M-vertex random digraph (out-degree 2) + 30,000 hubs of extra out- and in-degree uniform [64, 4000)",
}


# DRAM traffic of the asynchronous drain relative to its algorithmic bytes,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum over all
# launches) of `bench.py --workload grid4096 --steps 1 --warmup 0`: 595.40 MB
# read + written by 9 launches whose algorithmic bytes total 793.8 MB.  The
# full C2 step is too large for that capture; its drain runs the same grid.
ASYNC_TRAFFIC_RATIO = 595.40 / 793.8
ASYNC_TRAFFIC_SOURCE = "ncu dram bytes on the 4096x4096 grid workload (0.750 x algorithmic), scaled per launch"


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_peak_tflops():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons sampled (NVML, every 10 ms) during the timed region.
    Reads only; changes no GPU setting."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device: int):
        self.dev = torch_device
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.stop_flag = threading.Event()
        self.thread = None
        self.handle = None

    def _open(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.dev)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            self.nvml, self.handle = self._open()
            self.max_mhz = self.nvml.nvmlDeviceGetMaxClockInfo(self.handle, self.nvml.NVML_CLOCK_SM)
        except Exception:
            self.handle = None
            return
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        while not self.stop_flag.is_set():
            try:
                self.samples.append(self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
                mask = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def stop(self):
        self.stop_flag.set()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm = self.samples
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(sm)}


def hub_edges(hubs_n, hubs, hub_deg, seed):
    """A random digraph of out-degree 2 on hubs_n vertices plus `hubs` distinct
    vertices with extra out- and in-edges, degrees uniform in hub_deg."""
    rng = np.random.default_rng(seed)
    s = [np.repeat(np.arange(hubs_n, dtype=np.int32), 2)]
    d = [rng.integers(0, hubs_n, 2 * hubs_n, dtype=np.int32)]
    for h in rng.choice(hubs_n, hubs, replace=False):
        k_out, k_in = rng.integers(hub_deg[0], hub_deg[1], 2)
        s += [np.full(k_out, h, np.int32), rng.integers(0, hubs_n, k_in, dtype=np.int32)]
        d += [rng.integers(0, hubs_n, k_out, dtype=np.int32), np.full(k_in, h, np.int32)]
    return hubs_n, np.concatenate(s), np.concatenate(d)


def parse_tuning(text):
    """"bu_alpha=1,cta_deg=256" -> {"bu_alpha": 1, "cta_deg": 256}; "" -> {}."""
    out = {}
    for kv in text.split(","):
        if not kv.strip():
            continue
        k, sep, v = kv.partition("=")
        if not sep:
            raise ValueError(f"tuning entry {kv!r} is not key=value")
        out[k.strip()] = int(v)
    return out


def workload_edges(kw):
    """Seeded edge list (n, src, dst) of a workload, on the host."""
    from dynamicgraphs_scc_b200 import generate_edges_host
    if "hubs" in kw:
        return hub_edges(**kw)
    return generate_edges_host(**kw)


def workload_graph(kw, device):
    """The workload's graph on the device (generated there where it can be)."""
    from dynamicgraphs_scc_b200 import Graph
    if "hubs" in kw:
        n, s, d = hub_edges(**kw)
        return Graph.from_edges(n, s, d, device=device)
    return Graph.generate(**kw, device=device)


def host_csr(kw):
    """Seeded edge list of a workload -> forward CSR on the host (self-loops and
    duplicates removed; the oracle's dedup leaves the edges sorted by (source,
    target), so the CSR is its offsets and targets).  Input preparation for the
    reference's own engine, which builds its reverse edges itself."""
    from oracle import oracle as O
    n, s, d = workload_edges(kw)
    s, d = O.dedup_edges(s, d, n=n)
    b = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(s, minlength=n), out=b[1:])
    return n, b, np.ascontiguousarray(d, np.int32)


# The reference's method per workload.  Method 2 (do_baseline_global_wcc_fb)
# keeps a pool of 65,536 node sets, one per weak component, and takes from it
# with no bound check (init_node_set_pool(65536) in src/scc_weak.cc:35,
# get_node_set_from_pool :24-29): the 4096 x 4096 oriented grid leaves more
# weak components than that after trimming, and method 2 reads past the pool
# and crashes.  On graphs holding that grid the reference arm runs method 1
# (do_baseline_global_fb: Trim1 + global FW-BW + Trim1 + FW-BW), the
# reference's method that completes there.
REF_METHOD = {"c2": 1, "grid4096": 1}
REF_METHOD_NOTE = ("method 2 overruns its 65,536-entry node-set pool (src/scc_weak.cc:24-35) on this graph's "
                   "oriented grid and crashes; method 1 is the reference's method that completes on it")


def run_reference(args, workload, full=True):
    """Reference arm: the reference's own OpenMP pipeline on the host cores, on
    the full workload (full=True) or on the 1/16 sample of CPU_SAMPLES."""
    from oracle import oracle as O
    kw = WORKLOADS[workload] if full else CPU_SAMPLES[workload]
    n, b, a = host_csr(kw)
    threads = os.cpu_count() or 1
    method = REF_METHOD.get(workload, 2) if full else 2
    kind = "reference" if O.ref_available() else "port"
    times = []
    for i in range(args.warmup + args.steps):
        if kind == "reference":
            _, ms = O.ref_method(method, (b, a), threads=threads)
        else:
            t0 = time.perf_counter()
            O.tarjan_canonical(b, a)
            ms = (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            times.append(ms)
    ms = statistics.mean(times)
    gteps = a.size / (ms * 1e-3) / 1e9
    what = "full configuration" if full else "1/16 sample, " + json.dumps(kw)
    sample = f"{WORKLOAD_NAMES[workload]} ({what}): n={n} m={a.size}, method {method}"
    return gteps, ms, dict(value=gteps, unit="GTEPS", cores=threads if kind == "reference" else 1, kind=kind,
                           sample=sample, ms=ms, method=method, n=n, m=int(a.size))


def run_reference_cuda(args, workload):
    """The reference's own CUDA engine (src_CUDA method 2, compiled for sm_100a)
    on this GPU, on the full workload: a comparator, not the drop-in.  Its
    labels are checked against the reference's own Tarjan digest where one is
    recorded (its WCC stops after 100 propagation passes, scc_cuda_weak.cu:489,
    and its host FW-BW takes at most 999,999 work items, scc_cuda_fb_seq2.cu,
    so on long-diameter graphs it may not finish every vertex)."""
    import hashlib
    from oracle import oracle as O
    from dynamicgraphs_scc_b200 import generate_edges_host
    if not O.ref_cuda_available():
        return {"impl": "reference-cuda", "unavailable": "the reference's CUDA engine was not built (oracle/Makefile)"}
    kw = WORKLOADS[workload]
    n, s, d = workload_edges(kw)
    s, d = O.dedup_edges(s, d, n=n)
    csr = O.build_csr(n, s, d)
    m = int(csr[1].size)
    del s, d
    threads = os.cpu_count() or 1
    times, lab = [], None
    for i in range(args.warmup + args.steps):
        lab, ms = O.ref_cuda_method2(csr, threads=threads)
        if i >= args.warmup:
            times.append(ms)
    ms = statistics.mean(times)
    finished = int(np.count_nonzero(lab >= 0))
    canon = O.canonical(np.where(lab >= 0, lab, np.arange(n, dtype=np.int32)).astype(np.int32))
    digest = hashlib.sha256(np.ascontiguousarray(canon, dtype="<i4").tobytes()).hexdigest()
    ref = {}
    p = os.path.join(ROOT, "tests", "golden", "fullsize_digests.json")
    if os.path.exists(p):
        with open(p) as f:
            ref = json.load(f).get(workload, {})
    if not ref and n <= (1 << 22):          # small workloads: the oracle's Tarjan directly
        exp = O.tarjan_canonical(csr[0], csr[1])
        ref = {"labels_sha256": hashlib.sha256(np.ascontiguousarray(exp, dtype="<i4").tobytes()).hexdigest()}
    return {"impl": "reference-cuda", "metric": "SCC GTEPS (edges / end-to-end decomposition time)",
            "value": round(m / (ms * 1e-3) / 1e9, 6), "unit": "GTEPS", "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "int32", "n_gpus": 1,
            "config": {"workload": WORKLOAD_NAMES[workload], "params": kw, "n": n, "m": m, "method": 2,
                       "host_threads": threads,
                       "timing": "host clock over the reference's own timed region (scc_cuda_main.cpp R1..R2)"},
            "vertices_finished": finished,
            "labels_equal_reference_tarjan": (digest == ref.get("labels_sha256")) if ref else None,
            "num_sccs": int(np.count_nonzero(canon == np.arange(n, dtype=np.int32)))}


def train_pivot_model(device):
    """The learned pivot proposer, trained as the configuration asks: records of
    plain runs on 64 seeded R-MAT graphs of scales 18-22 (ef16), then Adam on the
    device.  Returns (model, info)."""
    from dynamicgraphs_scc_b200 import Graph, PivotModel, collect_pivot_records
    t0 = time.perf_counter()
    xs, ts = [], []
    for sd in range(64):
        g = Graph.generate(rmat_scale=18 + sd % 5, edge_factor=16, seed=7000 + sd, device=device)
        x, t = collect_pivot_records(g, capacity=1 << 17, per_round=4096)
        xs.append(x); ts.append(t); g.free()
    x = np.concatenate(xs); t = np.concatenate(ts)
    t1 = time.perf_counter()
    m = PivotModel(seed=0, device=device)
    losses = m.train(x, t, epochs=12, batch=1024, lr=2e-3, seed=0)
    t2 = time.perf_counter()
    info = {"graphs": 64, "records": int(t.size), "target_mean": round(float(t.mean()), 5),
            "target_var": round(float(t.var()), 6), "epochs": 12, "final_loss": round(float(losses[-1]), 6),
            "collect_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2)}
    return m, info


BATCH = dict(num_graphs=4096, n_min=1024, n_max=65536, mean_degree=6.0, rmat_fraction=0.3, seed=4096)


def bench_batched(args, local_rank):
    """4,096 independent uneven graphs decomposed by one persistent launch (each
    block takes whole graphs, largest first) replayed from a captured CUDA graph,
    its launch shape chosen by successive halving; compared with one engine run
    over their disjoint union and with per-graph plain runs of every graph
    (device time of the runs only)."""
    import torch
    from dynamicgraphs_scc_b200 import BatchPlan, Graph, State, batch_autotune
    torch.cuda.set_device(local_rank)
    g, offs = Graph.generate_batch(**{**BATCH, "num_graphs": args.batch_graphs}, device=local_rank)
    n, m = g.num_nodes(), g.num_edges()
    st = State(g)
    t0 = time.perf_counter()
    best, tuned_ms = batch_autotune(g, st, offs)
    tune_s = time.perf_counter() - t0
    plan = BatchPlan(g, st, offs, tuning=best)
    for _ in range(args.warmup):
        plan.run()
    sampler = ClockSampler(local_rank)
    sampler.start()
    runs = [plan.run() for _ in range(args.steps)]
    clocks = sampler.stop()
    ms = statistics.mean(r["ms_total"] for r in runs)
    labels = st.canonical_labels()
    plan.free()
    if args.batch_only:
        print(json.dumps({"metric": "SCC GTEPS, batched uneven graphs (one persistent launch from a CUDA graph)",
                          "value": round(m / (ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "ms_per_step": round(ms, 3),
                          "config": {"graphs": args.batch_graphs, "n": n, "m": m, "autotuned": best}}))
        return
    # the general engine over the disjoint union (many kernel launches, host-driven rounds)
    st.reset(); st.run(2)
    union_runs = []
    for _ in range(max(1, min(args.steps, 3))):
        st.reset()
        union_runs.append(st.run(2))
    union_ms = statistics.mean(r["ms_total"] for r in union_runs)
    union_equal = bool(np.array_equal(st.canonical_labels(), labels))
    # per-graph plain runs
    per_ms = 0.0
    per_kernels = 0
    mismatches = 0
    for i in range(len(offs) - 1):
        sub = g.subgraph(int(offs[i]), int(offs[i + 1]))
        s2 = State(sub)
        s2.run(2)                       # warm-up of this graph's state
        s2.reset()
        r = s2.run(2)
        per_ms += r["ms_total"]
        per_kernels += r["kernels_launched"]
        if not np.array_equal(s2.canonical_labels() + offs[i], labels[offs[i]:offs[i + 1]]):
            mismatches += 1
        s2.free(); sub.free()
    line = {
        "metric": "SCC GTEPS, 4,096 batched uneven graphs (one persistent launch from a CUDA graph)",
        "value": round(m / (ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded per graph)",
        "config": {"workload": f"{args.batch_graphs} graphs, n log-uniform [1024, 65536], out-degree Poisson(6), 30% R-MAT / 70% "
                               "uniform targets, self-loops and duplicates removed", "n": n, "m": m,
                   "autotuned": best, "autotune": {"method": "successive halving (1/8, 1/4, 1/2, all graphs)",
                                                   "seconds": round(tune_s, 2), "best_ms": round(tuned_ms, 3)},
                   "method": "trim1 + FW-BW rounds per graph, one block per graph"},
        "host_submissions_per_run": runs[-1]["host_submissions"], "kernels_per_run": runs[-1]["kernels"],
        "rounds": runs[-1]["rounds"], "max_rounds_one_graph": runs[-1]["max_rounds"],
        "union_engine": {"ms": round(union_ms, 3), "kernels": union_runs[-1]["kernels_launched"],
                         "labels_equal": union_equal, "speedup_of_batched": round(union_ms / ms, 2)},
        "per_graph": {"value": round(m / (per_ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "ms_total": round(per_ms, 2),
                      "kernels": per_kernels, "label_mismatches": mismatches},
        "batched_speedup": round(per_ms / ms, 2),
        "clocks": clocks, "gpu_launches": args.steps,
    }
    print(json.dumps(line))


SERVE = dict(rmat_scale=22, edge_factor=16, seed=2022)


def _tarjan_equal(b, a, labels):
    """Oracle check of one serving snapshot (runs in a spawned worker process)."""
    from oracle import oracle as O
    return bool(np.array_equal(O.tarjan_canonical(b, a), labels))


def _pct(xs, p):
    return xs[min(len(xs) - 1, int(p * (len(xs) - 1) + 0.5))] if xs else None


SUSTAIN_HEADROOM = 3.0


def bench_serving(args, local_rank, batches_n=None, sustain_n=None):
    """Streaming updates against a device-resident R-MAT s22 ef16 graph through the
    serving loop: batches arrive Poisson (mean 2 ms), sizes log-uniform in
    [1e3, 1e6] edges, 70% inserts / 30% deletes of existing edges, endpoints
    degree-proportional (ends of random existing edges); every 100 batches the
    labels are checked against a full Tarjan recomputation of the current graph
    (the checks run in a pool of host processes while serving goes on).

    Two phases.  "configured": the arrival process as configured, which offers
    more than one session's in-order updates can serve, with backpressure (a
    backlog limit in edges, and an age limit) so the queue stays bounded;
    offered, served and shed load are reported.  "sustainable": after the
    queue has drained, the same batch distribution at a mean gap the service
    sustains (SUSTAIN_HEADROOM x the mean service time of the configured
    phase's last 100 admitted batches: the device busy about a third of the
    time, since the service time is heavy-tailed and queueing delay grows with
    its second moment), where p50/p99 describe the system rather than the
    length of the run.  A check waits for the batches before it (serving
    time) and then copies the graph and labels out with the device idle; the
    clocks stop for the copy (rates and wall times leave it out).  Returns the
    JSON line."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    import torch
    from dynamicgraphs_scc_b200 import Graph, Server
    batches_n = args.batches if batches_n is None else batches_n
    sustain_n = args.sustain_batches if sustain_n is None else sustain_n
    pool = ProcessPoolExecutor(max_workers=min(8, os.cpu_count() or 1), mp_context=mp.get_context("spawn"))
    torch.cuda.set_device(local_rank)
    g = Graph.generate(**SERVE, device=local_rank)
    n, m0 = g.num_nodes(), g.num_edges()
    b, a, _, _ = g.csr()
    base_src = np.repeat(np.arange(n, dtype=np.int32), np.diff(b)); base_dst = a
    sv = Server(num_slots=4, hbm_budget_bytes=96 << 30, device=local_rank)
    if args.coalesce > 1:
        sv.set_coalesce(args.coalesce)
    sv.set_admission(args.admit_edges, args.admit_ms)
    sid = sv.add_graph(g)
    rng = np.random.default_rng(2022)
    lo, hi = np.log(1e3), np.log(1e6)

    def make_batch():
        k = int(np.exp(lo + rng.random() * (hi - lo)))
        ki = int(round(0.7 * k)); kd = k - ki
        ii = rng.integers(0, base_src.size, (2, ki))
        dd = rng.integers(0, base_src.size, kd)
        return base_src[ii[0]], base_dst[ii[1]], base_src[dd], base_dst[dd]

    checks = []
    counter = {"batches": 0}

    def run_phase(count, mean_gap_ms):
        results, shed, pending, offered = [], 0, [], 0
        t_last = time.perf_counter()
        gaps = rng.exponential(mean_gap_ms, count)
        t0 = time.perf_counter()
        due = 0.0
        for i in range(count):
            bt = make_batch()
            due += gaps[i] * 1e-3
            delay = t0 + due - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            rid = sv.submit(sid, *bt)
            edges = sum(x.size for x in bt)
            offered += edges
            if rid < 0:
                shed += 1
            else:
                pending.append((rid, edges))
            counter["batches"] += 1
            if counter["batches"] % 100 == 0:
                # the check needs the session idle at this batch: waiting for
                # the queue is serving time; the copy-out that follows leaves
                # the device idle, so the clocks stop for it
                results += [(sv.wait(r), e) for r, e in pending]
                pending = []
                tp = time.perf_counter()
                cb, ca, _, _ = sv.session_csr(sid)
                checks.append(pool.submit(_tarjan_equal, cb, ca, sv.labels(sid)))
                t0 += time.perf_counter() - tp
            t_last = time.perf_counter()
        arrival_s = max(t_last - t0, 1e-9)
        results += [(sv.wait(r), e) for r, e in pending]
        wall = time.perf_counter() - t0
        ok = [(r, e) for r, e in results if r["status"] == 0]
        lat = sorted(r["latency_ms"] for r, _ in ok)
        svc = sorted(r["ms_total"] for r, _ in ok)
        recent = [r["ms_total"] for r, _ in ok[-100:]]
        served_edges = sum(e for _, e in ok)
        return {"batches": count, "mean_gap_ms": round(mean_gap_ms, 3), "admitted": len(results),
                "applied": len(ok), "shed_at_submit": shed,
                "expired_in_queue": sum(r["status"] == 9 for r, _ in results),
                "offered_updates_per_s": round(offered / arrival_s, 1),
                "served_updates_per_s": round(served_edges / wall, 1),
                "latency_ms": {"p50": round(_pct(lat, 0.5), 3) if lat else None,
                               "p99": round(_pct(lat, 0.99), 3) if lat else None,
                               "max": round(lat[-1], 3) if lat else None},
                "service_ms": {"p50": round(_pct(svc, 0.5), 3) if svc else None,
                               "p99": round(_pct(svc, 0.99), 3) if svc else None,
                               "mean": round(float(np.mean(svc)), 3) if svc else None,
                               "mean_last_100": round(float(np.mean(recent)), 3) if recent else None},
                "wall_s": round(wall, 2)}

    t_all = time.perf_counter()
    configured = run_phase(batches_n, 2.0)
    sv.drain()                  # the second phase starts from an empty queue
    # the service time grows with the graph (inserts outnumber deletes), so the
    # sustainable gap follows the latest admitted batches
    gap = SUSTAIN_HEADROOM * (configured["service_ms"]["mean_last_100"] or 2.0)
    sustainable = run_phase(sustain_n, gap) if sustain_n > 0 else None
    sv.drain()
    st = sv.stats()
    cb, _, _, _ = sv.session_csr(sid)
    check_ok = [f.result() for f in checks]
    pool.shutdown()
    sv.free()
    lat_ref = sustainable or configured
    line = {
        "metric": "streaming SCC updates: p50/p99 batch latency (ms) and updates/s",
        "value": configured["served_updates_per_s"], "unit": "updates/s", "n_gpus": 1,
        "steps": configured["applied"] + (sustainable["applied"] if sustainable else 0),
        "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded)",
        "config": {"workload": "R-MAT s22 ef16 base, Poisson(2 ms) arrivals, batch log-uniform [1e3, 1e6], "
                               "70% insert / 30% delete, degree-proportional endpoints",
                   "n": n, "m_before": m0, "m_after": int(cb[-1]), "slots": 4, "coalesce": args.coalesce,
                   "admission": {"max_queued_edges": args.admit_edges, "max_queue_ms": args.admit_ms},
                   "device_updates": st["groups"]},
        "configured": configured,
        "sustainable": sustainable,
        "latency_ms": lat_ref["latency_ms"],
        "tarjan_checks": {"count": len(check_ok), "all_equal": all(check_ok), "every": 100},
        "wall_s": round(time.perf_counter() - t_all, 2),
    }
    return line


def time_steps(st, stream, steps, warmup, mode=0):
    """W untimed decompositions, then K timed ones (CUDA events on the state's stream)."""
    import torch
    for _ in range(warmup):
        st.reset(); st.run(2, mode)
    st.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True); ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    last = None
    for _ in range(steps):
        st.reset()
        last = st.run(2, mode)
    ev1.record(stream)
    st.synchronize()
    return ev0.elapsed_time(ev1) / steps, last


def extra_rmat24(local_rank, steps=10, warmup=3):
    """R-MAT s24 ef16 alone: the configuration whose whole-step roofline target is 40 %."""
    import torch
    from dynamicgraphs_scc_b200 import Graph, State
    g = Graph.generate(**WORKLOADS["rmat24"], device=local_rank)
    n, m = g.num_nodes(), g.num_edges()
    st = State(g)
    stream = torch.cuda.ExternalStream(st.stream(), device=local_rank)
    ms, last = time_steps(st, stream, steps, warmup)
    peak, kind = measured_peak_gbs()
    ach = (16 * m + 20 * n + 8) / (ms * 1e-3) / 1e9
    st.free(); g.free()
    return {"workload": WORKLOAD_NAMES["rmat24"], "n": n, "m": m, "steps": steps, "warmup": warmup,
            "ms_per_step": round(ms, 4), "value": round(m / (ms * 1e-3) / 1e9, 3), "unit": "GTEPS",
            "roofline_step": {"bound": "hbm", "achieved": round(ach, 2), "peak": peak, "peak_kind": kind,
                              "unit": "GB/s", "frac": round(ach / peak, 4)}}


def extra_c3(local_rank, steps=5, warmup=3):
    """Learned vs plain pivot on the planted-cycles configuration, and on the
    mixed configuration (C2), each with labels compared."""
    import torch
    from dynamicgraphs_scc_b200 import Graph, State
    model, info = train_pivot_model(local_rank)
    out = {"pivot_model": info}
    for name in ("c3", "c2"):
        g = Graph.generate(**WORKLOADS[name], device=local_rank)
        m = g.num_edges()
        st = State(g)
        st.set_pivot_model(model)
        # both forms without the one-launch tail, which learned pivots do not use
        st.set_tuning(tail_live=-1)
        stream = torch.cuda.ExternalStream(st.stream(), device=local_rank)
        p_ms, _ = time_steps(st, stream, steps, warmup, 0)
        p_lab = st.canonical_labels()
        l_ms, _ = time_steps(st, stream, steps, warmup, 1)
        eq = bool(np.array_equal(p_lab, st.canonical_labels()))
        # ceiling of any proposer that re-ranks the degree rule's equally good
        # candidates: the same plain run under 15 other tie-breaks of the rule
        salts = []
        for salt in range(1, 16):
            st.set_tuning(pivot_salt=salt)
            ms_s, _ = time_steps(st, stream, 2, 1, 0)
            salts.append(round(ms_s, 4))
            eq = eq and bool(np.array_equal(p_lab, st.canonical_labels()))
        st.set_tuning(pivot_salt=-1)                  # back to the default tie-break
        st.free(); g.free()
        out[name] = {"plain_ms": round(p_ms, 4), "learned_ms": round(l_ms, 4),
                     "learned_speedup": round(p_ms / l_ms, 4), "labels_equal": eq,
                     "plain_gteps": round(m / (p_ms * 1e-3) / 1e9, 3),
                     "learned_gteps": round(m / (l_ms * 1e-3) / 1e9, 3),
                     "tie_break_ceiling": {"other_salts_ms": salts, "best_ms": min(salts),
                                           "median_ms": float(np.median(salts)),
                                           "best_speedup_over_plain": round(p_ms / min(salts), 4)}}
    return out


def default_extras(args, local_rank):
    """Secondary configurations measured in the default run, so that its JSON
    line carries all of the benchmark metric: R-MAT s24's roofline fraction,
    learned vs plain pivot, and the streaming loop's p50/p99."""
    out = {}
    for name, fn in (("rmat24", lambda: extra_rmat24(local_rank)), ("learned_pivot", lambda: extra_c3(local_rank)),
                     ("streaming", lambda: bench_serving(args, local_rank, batches_n=args.extra_batches,
                                                         sustain_n=args.extra_batches // 4))):
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as exc:     # reported, never hidden
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
        out[name + "_s"] = round(time.perf_counter() - t0, 1)
    return out


LEVELS = dict(rmat_scale=24, edge_factor=16, grid_side=4096, seed=2024)          # C2's graph
LEVELS_SAMPLE = dict(rmat_scale=18, edge_factor=16, grid_side=512, seed=2024)     # the reference's sample
LEVELS_BATCH = 100                                                                # inserted edges per batch


def scc_list_ids(labels):
    """scc_list.txt ids of canonical labels: ascending smallest member is the
    order of first appearance over the vertices."""
    _, ids = np.unique(labels, return_inverse=True)
    return ids.astype(np.int32), int(ids.max()) + 1 if ids.size else 0


def bench_levels(args, local_rank):
    """Method 7's preprocessing (create_scc_edges with met_algo 7,
    src/common_main.h:180-262) on C2's decomposition: the condensation DAG of
    the old labels, its topological levels, the levels a batch affects, and the
    condensation with the batch; then the trim shortcut and the run on it.  The
    entry points take and return host arrays, as the reference's vectors, and
    synchronise: host wall clock around each call."""
    import torch
    from dynamicgraphs_scc_b200 import Graph, State, affected_levels, capi, condensation_graph
    torch.cuda.set_device(local_rank)
    g = Graph.generate(**LEVELS, device=local_rank)
    n, m = g.num_nodes(), g.num_edges()
    st = State(g)
    st.run(2)
    ids, k = scc_list_ids(st.canonical_labels())
    rng = np.random.default_rng(7)
    isrc = rng.integers(0, n, LEVELS_BATCH).astype(np.int32)
    idst = rng.integers(0, n, LEVELS_BATCH).astype(np.int32)
    # host arrays in pinned memory, as the end-to-end legs use
    ids = torch.from_numpy(ids).pin_memory().numpy()
    lev_pinned = torch.empty(k, dtype=torch.int32).pin_memory().numpy()

    def levels_into(dag):
        ml = C.c_int32()
        capi.call("scc_topological_levels", dag.handle, capi.i32p(lev_pinned), C.byref(ml))
        return lev_pinned, ml.value

    def bundle():
        t = [time.perf_counter()]
        dag = condensation_graph(g, ids, k)
        t.append(time.perf_counter())
        lev, ml = levels_into(dag)
        t.append(time.perf_counter())
        aff, z = affected_levels(dag, lev, ml, ids, isrc, idst)
        t.append(time.perf_counter())
        cond = condensation_graph(g, ids, k, isrc, idst)
        t.append(time.perf_counter())
        md = dag.num_edges()
        dag.free()
        return cond, lev, ml, aff, z, md, [1e3 * (b - a) for a, b in zip(t, t[1:])]

    for _ in range(args.warmup):
        cond, *_ = bundle()
        cond.free()
    parts = []
    for _ in range(args.steps):
        cond, lev, ml, aff, z, md, p = bundle()
        parts.append(p)
        cond.free()
    part_ms = [statistics.mean(x) for x in zip(*parts)]
    total_ms = sum(part_ms)
    # the trim shortcut and the run over the condensation with the batch
    cond, lev, ml, aff, z, md, _ = bundle()
    cs = State(cond)
    run_ms = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cs.reset()
        fin = cs.finish_unaffected(lev, aff, ml)
        r = cs.run(2)
        if i >= args.warmup:
            run_ms.append(1e3 * (time.perf_counter() - t0))
    cpu = None
    if not args.no_cpu_baseline:
        cpu = levels_reference()
    line = {
        "metric": "method-7 preprocessing (condensation, topological levels, affected levels, batch condensation)",
        "value": round(m / (total_ms * 1e-3) / 1e9, 4), "unit": "Gedges/s (original edges)", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
        "timing": "host wall clock around synchronous entry points (pinned host arrays in and out)",
        "parts_ms": {"condensation": round(part_ms[0], 3), "topological_levels": round(part_ms[1], 3),
                     "affected_levels": round(part_ms[2], 3), "batch_condensation": round(part_ms[3], 3)},
        "shortcut_and_run_ms": round(statistics.mean(run_ms), 3),
        "config": {"workload": "C2 (R-MAT s24 ef16 U 4096x4096 oriented grid) decomposed, then method 7 on its "
                               f"condensation with a {LEVELS_BATCH}-edge batch",
                   "n": n, "m": m, "sccs": k, "condensation_edges": md, "max_level": ml,
                   "unaffected_levels": z, "finished_by_shortcut": fin, "sccs_after": r["num_sccs"]},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


def levels_reference():
    """The reference's own create_scc_edges (met_algo 7; one OpenMP thread, as
    its unlocked push_backs require) on a sample of the same shape, through the
    oracle's build of the reference."""
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from oracle import oracle as O
    from dynamicgraphs_scc_b200 import generate_edges_host
    if not O.ref_available():
        return {"value": None, "unit": "Gedges/s", "cores": 1, "kind": "reference",
                "sample": "reference library not built"}
    n, s, d = generate_edges_host(**LEVELS_SAMPLE)
    s, d = O.dedup_edges(s, d, drop_self_loops=True, n=n)
    csr = O.build_csr(n, s, d)
    ids, k = scc_list_ids(O.tarjan_canonical(csr[0], csr[1]))
    rng = np.random.default_rng(7)
    isrc = rng.integers(0, n, LEVELS_BATCH).astype(np.int32)
    idst = rng.integers(0, n, LEVELS_BATCH).astype(np.int32)
    b, a = O.condensation_csr(ids, k, s, d)
    lev, ml = O.topo_levels(b, a)
    _, z = O.affected_levels(ids, lev, ml, isrc, idst)
    if z == 0:      # its closing loop runs past the end when no level is left unaffected
        return {"value": None, "unit": "Gedges/s", "cores": 1, "kind": "reference",
                "sample": "batch leaves no level unaffected"}
    t0 = time.perf_counter()
    O.ref_method7_levels(n, s, d, isrc, idst, ids, k)
    ms = 1e3 * (time.perf_counter() - t0)
    return {"value": round(s.size / (ms * 1e-3) / 1e9, 5), "unit": "Gedges/s", "cores": 1, "kind": "reference",
            "sample": f"{LEVELS_SAMPLE} n={n} m={s.size}: {ms:.1f} ms"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-cuda"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c4", "c5", "levels"])
    ap.add_argument("--tune-trials", type=int, default=8)
    ap.add_argument("--batch-graphs", type=int, default=4096, help="c4: graphs in the batch")
    ap.add_argument("--batch-only", action="store_true", help="c4: skip the union-engine and per-graph comparisons")
    ap.add_argument("--batches", type=int, default=10000, help="c5: batches at the configured arrival rate")
    ap.add_argument("--sustain-batches", type=int, default=2000,
                    help="c5: batches at a rate the service sustains (0 = skip)")
    ap.add_argument("--admit-edges", type=int, default=4000000,
                    help="c5: backlog limit in queued edges (0 = none)")
    ap.add_argument("--admit-ms", type=float, default=2000.0, help="c5: age limit of a queued batch (0 = none)")
    ap.add_argument("--coalesce", type=int, default=1, help="c5: queued batches of a session composed per update")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the secondary configurations of the default run (R-MAT s24, learned pivot, streaming)")
    ap.add_argument("--extra-batches", type=int, default=1000, help="streaming batches measured in the default run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default="",
                    help="comma-separated scc_tuning fields for the engine arm, e.g. bu_alpha=1,cta_deg=256")
    ap.add_argument("--ref-sample", action="store_true",
                    help="reference arm: time the 1/16 sample instead of the full configuration")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.workload == "c5":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no streaming mode (one "
                                  "update file per process, methods 5-11)"}))
            return
        if rank == 0:
            print(json.dumps(bench_serving(args, local_rank)))
        return

    if args.workload == "levels":
        if rank == 0:
            if args.impl == "reference":
                cpu = levels_reference()
                print(json.dumps({"impl": "reference", "metric": "method-7 preprocessing (create_scc_edges)",
                                  "value": cpu["value"], "unit": cpu["unit"], "cpu_baseline": cpu,
                                  "e2e": {"value": cpu["value"], "unit": cpu["unit"], "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}))
            else:
                bench_levels(args, local_rank)
        return

    if args.workload == "c4":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the batched configuration is measured "
                                  "against per-graph runs of this engine; the reference has no batched mode"}))
            return
        if rank == 0:
            bench_batched(args, local_rank)
        return

    if args.impl == "reference-cuda":
        if rank == 0:
            print(json.dumps(run_reference_cuda(args, args.workload)))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        gteps, ms, cpu = run_reference(args, args.workload, full=not args.ref_sample)
        line = {"metric": "SCC GTEPS (edges / end-to-end decomposition time)", "value": round(gteps, 6),
                "unit": "GTEPS", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
                "config": {"workload": WORKLOAD_NAMES[args.workload], "params": WORKLOADS[args.workload],
                           "n": cpu["n"], "m": cpu["m"], "method": cpu["method"],
                           "parallelism": f"host cores x{cpu['cores']} (rank 0 only)"},
                "same_config": not args.ref_sample,
                "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": round(gteps, 6), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if cpu["method"] != 2:
            line["method_note"] = REF_METHOD_NOTE
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local_rank)
    from dynamicgraphs_scc_b200 import Graph, State, capi
    from dynamicgraphs_scc_b200.replicas import reduce_replicas

    kw = WORKLOADS[args.workload]
    learned = args.workload == "c3"            # the learned-pivot configuration
    model, model_info = (train_pivot_model(local_rank) if learned else (None, None))
    g = workload_graph(kw, local_rank)
    n, m = g.num_nodes(), g.num_edges()
    st = State(g)
    tuning = parse_tuning(args.tuning)
    if tuning:
        st.set_tuning(**tuning)
    if model is not None:
        st.set_pivot_model(model)
        st.set_tuning(tail_live=-1)        # both forms without the one-launch tail, which learned pivots do not use
    pivot_mode = 1 if learned else 0
    stream = torch.cuda.ExternalStream(st.stream(), device=local_rank)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(mode, sampler=None):
        """W untimed steps, then K steps bracketed by barrier + synchronize and
        CUDA events on the state's stream; max over ranks."""
        for _ in range(args.warmup):
            st.reset()
            st.run(2, mode)
        st.synchronize()
        if sampler is not None:
            sampler.start()
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        kernels = 0
        phase = []
        capi.call("scc_state_profile", st.handle, 1)   # time the dominant kernel's launches on this stream
        ev0.record(stream)
        for _ in range(args.steps):
            st.reset()
            stats = st.run(2, mode)
            kernels += stats["kernels_launched"] + 3
            phase.append(stats)
        ev1.record(stream)
        st.synchronize()
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop() if sampler is not None else None
        l_ms, l_launch, l_items, l_edges = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
        capi.call("scc_state_profile_read", st.handle, C.byref(l_ms), C.byref(l_launch), C.byref(l_items),
                  C.byref(l_edges))
        capi.call("scc_state_profile", st.handle, 0)
        ms, _ = reduce_replicas(ev0.elapsed_time(ev1) / args.steps, m, dist, f"cuda:{local_rank}")
        return ms, kernels, phase, clocks, (l_ms, l_launch, l_items, l_edges)

    plain = None
    if learned:                                 # the plain-pivot form on the same GPU, for the comparison
        p_ms, _, p_phase, _, _ = timed(0)
        plain_labels = st.canonical_labels() if rank == 0 else None
        plain = {"value": round(m * world / (p_ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "ms_per_step": round(p_ms, 4),
                 "fb_rounds": p_phase[-1]["fb_rounds"], "traversal_steps": p_phase[-1]["traversal_steps"]}
    ms, kernels, phase, clocks, ledger = timed(pivot_mode, ClockSampler(local_rank))
    l_ms, l_launch, l_items, l_edges = ledger
    if learned and rank == 0:
        plain["labels_equal_learned"] = bool(np.array_equal(plain_labels, st.canonical_labels()))
    _, total_edges = reduce_replicas(ms, m, dist, f"cuda:{local_rank}")
    gteps = total_edges / (ms * 1e-3) / 1e9

    # roofline of the whole step (algorithmic bytes 16M + 20N + 8)
    peak, peak_kind = measured_peak_gbs()
    b_alg = 16 * m + 20 * n + 8
    achieved = b_alg / (ms * 1e-3) / 1e9
    # dominant kernel: the asynchronous reachability drain.  Algorithmic bytes:
    # 13 B per expanded item (offset pair, colour, mark) + 9 B per scanned edge
    # (neighbour id, its colour, its mark).
    kernel_roofline = None
    if l_launch.value > 0 and l_ms.value > 0:
        k_bytes = (13 * l_items.value + 9 * l_edges.value) / l_launch.value
        k_ms = l_ms.value / l_launch.value
        k_ach = k_bytes / (k_ms * 1e-3) / 1e9
        kernel_roofline = {"bound": "hbm", "kernel": "k_reach_async", "achieved": round(k_ach, 2), "peak": peak,
                           "peak_kind": peak_kind, "unit": "GB/s", "frac": round(k_ach / peak, 5),
                           "traffic": int(ASYNC_TRAFFIC_RATIO * k_bytes), "traffic_source": ASYNC_TRAFFIC_SOURCE,
                           "bytes_per_launch": int(k_bytes), "ms_per_launch": round(k_ms, 4),
                           "launches": l_launch.value, "share_of_step": round(l_ms.value / (ms * args.steps), 4)}

    # e2e: host CSR (pinned) -> H2D -> run -> canonical labels D2H, through the C ABI
    b, a, rb, ra = g.csr()
    hb = torch.from_numpy(b).pin_memory(); ha = torch.from_numpy(a).pin_memory()
    labels = torch.empty(n, dtype=torch.int32).pin_memory()
    lib = capi.lib()
    e2e_ms = []
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # forward CSR across the bus; the transpose is rebuilt on the device
        capi.call("scc_graph_upload_csr_out", g.handle, hb.data_ptr(), ha.data_ptr(), st.stream())
        st.reset()
        st.run(2, pivot_mode)
        capi.call("scc_canonical_labels", st.handle, C.cast(labels.data_ptr(), C.POINTER(C.c_int32)))
        e1.record(stream)
        st.synchronize()
        if i > 0:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e = statistics.mean(e2e_ms) if e2e_ms else float("nan")
    e2e, _ = reduce_replicas(e2e, m, dist, f"cuda:{local_rank}")
    e2e_gteps = total_edges / (e2e * 1e-3) / 1e9 if e2e_ms else None
    h2d = 4 * ((n + 1) + m)
    d2h = 4 * n

    # e2e, pipelined: the same steps (CSR in, decomposition, labels out) with two
    # resident graphs, step i+1's CSR-only upload issued on its own stream before
    # step i's run, so the PCIe transfer overlaps the decomposition
    pipe = None
    if args.e2e_steps > 0:
        g2 = Graph.from_csr(b, a, device=local_rank)
        st2 = State(g2)
        if learned:
            st2.set_pivot_model(model)
            st2.set_tuning(tail_live=-1)
        pair = [(g, st), (g2, st2)]
        lab_dev = [torch.empty(n, dtype=torch.int32, device=f"cuda:{local_rank}") for _ in range(2)]
        lab_host = [torch.empty(n, dtype=torch.int32).pin_memory() for _ in range(2)]
        streams = [torch.cuda.ExternalStream(sk.stream(), device=local_rank) for _, sk in pair]

        def upload(k):
            gk, sk = pair[k % 2]
            capi.call("scc_graph_upload_csr_out", gk.handle, hb.data_ptr(), ha.data_ptr(), sk.stream())

        def pipelined(steps):
            upload(0)
            for i in range(steps):
                if i + 1 < steps:
                    upload(i + 1)
                k = i % 2
                _, sk = pair[k]
                sk.reset()
                sk.run(2, pivot_mode)
                # labels to the host on this graph's stream, overlapping the next decomposition
                capi.call("scc_canonical_labels_device", sk.handle,
                          C.cast(lab_dev[k].data_ptr(), C.POINTER(C.c_int32)))
                with torch.cuda.stream(streams[k]):
                    lab_host[k].copy_(lab_dev[k], non_blocking=True)

        p_steps = max(10, 2 * args.e2e_steps)
        pipelined(4)                                   # warm-up (both graphs, the pool's blocks)
        barrier()
        torch.cuda.synchronize()
        s_a = torch.cuda.ExternalStream(st.stream(), device=local_rank)
        s_b = torch.cuda.ExternalStream(st2.stream(), device=local_rank)
        p0 = torch.cuda.Event(enable_timing=True)
        p0.record(s_a)
        pipelined(p_steps)
        pa = torch.cuda.Event(enable_timing=True); pb = torch.cuda.Event(enable_timing=True)
        pa.record(s_a); pb.record(s_b)
        torch.cuda.synchronize()
        p_ms = max(p0.elapsed_time(pa), p0.elapsed_time(pb)) / p_steps
        p_ms, _ = reduce_replicas(p_ms, m, dist, f"cuda:{local_rank}")
        pipe = {"value": round(total_edges / (p_ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "ms_per_step": round(p_ms, 3),
                "steps": p_steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "method": "every step copies its CSR in and its labels out; step i+1's upload, and step i's "
                          "labels copy, run on the two resident graphs' streams during the neighbouring "
                          "decomposition (pipeline fill included; all copies finish inside the timed region)"}
        # release the tensors used on the second graph's stream before that stream goes
        torch.cuda.synchronize()
        del lab_dev, lab_host, streams, s_a, s_b
        st2.free(); g2.free()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            _, _, cpu = run_reference(argparse.Namespace(steps=1, warmup=0), args.workload, full=False)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as exc:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "GTEPS", "cores": 0, "kind": "reference", "sample": f"failed: {exc}"}

    extras = None
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_extras:
        st.free(); g.free()                 # the headline graph is done with
        extras = default_extras(args, local_rank)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    last = phase[-1]
    line = {
        "metric": "SCC GTEPS (edges / end-to-end decomposition time)",
        "value": round(gteps, 4), "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded generator, same shapes as the benchmark configuration)",
        "config": {"workload": WORKLOAD_NAMES[args.workload], "params": kw, "n": n, "m": m, "method": 2,
                   "pivot": ("learned (MLP 8-64-64-1, BF16 weights, re-ranks the in*out candidates)" if learned
                             else "max in*out degree"),
                   "parallelism": f"replicas x{world}", "l2": "inputs (CSR+transpose) > L2; no flush",
                   **({"tuning": tuning} if tuning else {})},
        "roofline": kernel_roofline,
        "roofline_step": {"bound": "hbm", "scope": "whole step (16M+20N+8 algorithmic bytes)",
                          "achieved": round(achieved, 2), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                          "frac": round(achieved / peak, 5)},
        "e2e": {"value": round(e2e_gteps, 4) if e2e_gteps else None, "unit": "GTEPS",
                "ms_per_step": round(e2e, 3) if e2e_ms else None,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "e2e_pipelined": pipe,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": kernels,
        "phases_ms": {k: round(last[k], 3) for k in ("ms_trim1", "ms_global_fb", "ms_trim12", "ms_wcc", "ms_fb")},
        "stats": {k: last[k] for k in ("num_sccs", "first_scc_size", "trimmed_first", "trimmed_second",
                                        "num_wcc_classes", "traversal_steps")},
    }
    if extras is not None:
        line["extras"] = extras
    if learned:
        line["metric"] = "SCC GTEPS, learned pivot (plain pivot beside it)"
        line["plain_pivot"] = plain
        line["learned_speedup"] = round(plain["ms_per_step"] / ms, 4)
        line["pivot_model"] = model_info
        # the inference kernel alone: tensor-core roofline (2 x 4,672 useful FLOPs per vertex scored)
        rows = 1 << 22
        mlp_ms = model.bench_inference(rows, 20)
        tflops = 2 * 4672 * rows / (mlp_ms * 1e-3) / 1e12
        tpeak, tkind = measured_peak_tflops()
        line["mlp_roofline"] = {"bound": "tensor", "kernel": "k_mlp_score_tc", "rows": rows,
                                "ms_per_launch": round(mlp_ms, 4), "achieved": round(tflops, 3), "peak": tpeak,
                                "peak_kind": tkind, "unit": "TFLOP/s", "frac": round(tflops / tpeak, 5),
                                "rows_per_s": round(rows / (mlp_ms * 1e-3), 1)}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
