"""Benchmark: Louvain edges/s per pass (and final Q) on the power-law
co-purchase-like workload (334,863 vertices, ~925k undirected unit-weight
edges, Chung-Lu degrees exponent 2.3 / max 550, planted communities mu=0.3,
seed 0, min gain 1e-6), on 1..N B200s.

One step = one complete Louvain run (every level until the first pass of a
phase gains less than min gain).  edges/s per pass = sum over passes of the
pass's stored adjacency entries / time.

  value      inputs resident in HBM (lv_run_device), device time of K steps
             measured with CUDA events on the engine's stream, L2 flushed
             (256 MB write) between steps outside the timed events
  e2e        same metric through the C ABI with host buffers (lv_run +
             lv_get_assignment: CSR upload and assignment download inside)
  roofline   the kernel group with the largest device time, from K further
             steps run with a CUDA event pair around every launch group
             (on the engine's stream): algorithmic bytes / event time,
             against the measured HBM copy bandwidth
  cpu_baseline  the reference's CPU path (louvian.py restated in C by the
             oracle, FP64; its move decisions spread over all host
             threads -- every bucket is one Jacobi step -- with results
             identical to the single-threaded restatement) on the same graph
N > 1 (torchrun): every rank runs its own replica (the single-graph path
does not shard); value = edges of all ranks / max-over-ranks time.
  batched    (N=1) the batched form on 4,096 SBM graphs against the plain
             engine looped over the same graphs: graphs/s of each, and whether
             every partition is identical
  served     (N=1) the served form (continuous batching, 120 GB budget) on
             2,000 R-MAT / LFR-style requests: saturated capacity (all queued
             at t=0) in graphs/s, and p50/p99 latency under Poisson arrivals
             at 200/s, both against the plain engine run per request
  hbm_scale  (N=1) the plain engine on R-MAT scale 24 (16.8 M vertices,
             521 M entries): ms per run, edges/s per pass and the dominant
             move group's roofline; then, untimed, one run with FP64 gains
             and the oracle's louvian.py restatement on the same graph (its
             final Q, and how far each engine mode is from it)
--impl reference: the reference's CPU implementation (oracle port) alone.
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
sys.path.insert(0, os.path.join(ROOT, "louvain-community-detection_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

import lvgen  # noqa: E402

METRIC = "Louvain edges/s per pass & final Q; batched graphs/s & p99 vs plain, 1 B200"
UNIT = "edges/s"
MIN_GAIN = 1e-6


def workload(name: str):
    if name == "powerlaw":
        n, s, d, w = lvgen.planted_powerlaw(seed=0)
        desc = {"workload": "planted power-law co-purchase-like graph",
                "n_vertices": n, "gamma": 2.3, "max_degree": 550, "mu": 0.3,
                "weights": "unit FP32", "seed": 0}
    elif name == "banded":
        n, s, d, w = lvgen.banded_fem(seed=0)
        desc = {"workload": "banded FEM-like matrix", "n_vertices": n,
                "half_band": 60, "weights": "U(0.1,1.0) FP32", "seed": 0}
    elif name.startswith("rmat"):
        scale = int(name[4:])
        n, s, d, w = lvgen.rmat(scale, seed=0)
        desc = {"workload": f"R-MAT scale {scale}", "n_vertices": n,
                "abcd": [0.57, 0.19, 0.19, 0.05], "weights": "unit FP32", "seed": 0}
    else:
        raise SystemExit(f"unknown workload {name}")
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    desc.update({"n_edges": int(len(s)), "n_entries": int(len(col)),
                 "min_gain": MIN_GAIN, "rule": "louvian.py (max_gain > 0)"})
    return n, off, col, ww, desc


class ClockSampler:
    """nvidia-smi samples during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200", "-i", self.gpu_id],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax = float(parts[2].split()[0])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_group: str):
    """DRAM bytes per launch of a kernel group from the committed ncu
    summary (profiles/ncu_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(kernel_group, {}).get("dram_bytes_per_launch")


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(n, off, col, ww, budget_s=12.0):
    """The reference's CPU path (louvian.py's algorithm, restated in C by the
    oracle: FP64, first-seen row order), on every host thread, on the same
    graph, repeated until about `budget_s` seconds of CPU work."""
    import pyoracle

    threads = host_threads()
    pyoracle.set_threads(threads)
    g = pyoracle.CSR(n, off, col, ww.astype(np.float64))
    runs, t_tot, edges = 0, 0.0, 0
    q = None
    while t_tot < budget_s or runs == 0:
        t0 = time.perf_counter()
        r = pyoracle.louvain(g, MIN_GAIN, rule="py", prec="fp64", rows="first_seen")
        t_tot += time.perf_counter() - t0
        edges += sum(l.passes * l.n_entries for l in r.levels)
        q = r.q
        runs += 1
        if runs >= 50:
            break
    pyoracle.set_threads(1)
    return {"value": edges / t_tot, "unit": UNIT, "cores": threads, "kind": "port",
            "host_threads": os.cpu_count(),
            "sample": f"full workload, {runs} complete runs ({t_tot:.1f} s) on {threads} of "
                      f"{os.cpu_count()} host threads",
            "final_q": q}


def batched_measure(stream, count: int, steps: int = 2, apply_launch: bool = False):
    """Batched form on the SBM batch workload (count graphs, sizes
    log-uniform 64..65,536, 4-32 equal blocks, mean degree 16,
    p_in/p_out = 20, weights U(0.5, 1.5), generated on the device):
    graphs/s of one batched run (lv_batch_run_device) against the plain
    engine looped over the same device-resident graphs (lv_run_device per
    graph), and whether every graph's partition is identical."""
    import torch

    import lvb200

    goff, off, col, w, n_edges = lvgen.sbm_batch_device(count, seed=0)
    N, E = int(goff[-1]), int(col.numel())
    out = torch.zeros(N, dtype=torch.int32, device="cuda")
    out_plain = torch.zeros(N, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    res = {"workload": "SBM batch", "graphs": count, "n_vertices": N,
           "n_edges": int(n_edges), "n_entries": E, "sizes": "log-uniform 64..65536",
           "blocks": "4..32", "mean_degree": 16, "p_in/p_out": 20,
           "weights": "U(0.5,1.5) FP32", "seed": 0}
    with torch.cuda.stream(stream):
        eng = lvb200.Engine(stream=stream.cuda_stream, apply_launch=apply_launch)
        # kernel variants tuned on the union's level 0 (untimed)
        eng.load_device(N, E, off.data_ptr(), col.data_ptr(), w.data_ptr())
        res["tuning"] = {str(b): k for b, (k, _) in eng.autotune().items()}

        def batch_step():
            return eng.batch_run_device(goff, N, E, off.data_ptr(), col.data_ptr(),
                                        w.data_ptr(), MIN_GAIN, out.data_ptr())

        batch_step()  # warm-up: buffers, graph instantiation paths
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            q_b, lv_b, r = batch_step()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        eng.close()
        # plain engine looped over the same graphs (local CSR views)
        loff, lcol = lvgen.localize_batch(goff, off, col)
        eoff = off[torch.from_numpy(goff.astype(np.int64)).cuda()].cpu().numpy()
        plain = lvb200.Engine(stream=stream.cuda_stream, apply_launch=apply_launch)
        q_p = np.zeros(count)

        def one(g):
            n = int(goff[g + 1] - goff[g])
            b0, e0, e1 = int(goff[g]), int(eoff[g]), int(eoff[g + 1])
            return plain.run_device(n, e1 - e0, loff.data_ptr() + 8 * (b0 + g),
                                    lcol.data_ptr() + 4 * e0, w.data_ptr() + 4 * e0,
                                    MIN_GAIN, out_plain.data_ptr() + 4 * b0)

        one(int(np.argmax(goff[1:] - goff[:-1])))  # warm-up at the largest size
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for g in range(count):
            q_p[g] = one(g).modularity
        b.record(stream)
        torch.cuda.synchronize()
        plain_ms = a.elapsed_time(b)
        plain.close()
    o1, o2 = out.cpu().numpy(), out_plain.cpu().numpy()
    batch_ms = min(ms)
    res.update({
        "batched_ms": batch_ms, "batched_graphs_per_s": count / (batch_ms / 1000.0),
        "plain_looped_ms": plain_ms, "plain_looped_graphs_per_s": count / (plain_ms / 1000.0),
        "speedup": plain_ms / batch_ms,
        "partitions_identical": bool(np.array_equal(o1, o2)),
        "max_abs_dq": float(np.max(np.abs(q_b - q_p))),
        "levels_max": int(lv_b.max()), "mean_q": float(q_b.mean()),
    })
    return res


def hbm_scale_measure(stream, scale: int, steps: int = 2, oracle_check: bool = True,
                      apply_launch: bool = False, use_graphs: bool = True):
    """The plain engine at HBM scale: R-MAT (a, b, c, d = 0.57, 0.19, 0.19,
    0.05, edge factor 16, duplicates merged, unit weights) generated on the
    device; edges/s per pass over `steps` device-timed runs after one
    warm-up, then one run with a CUDA event pair around every launch group
    for the dominant move group's algorithmic GB/s against the HBM peak."""
    import torch

    import lvb200

    n, off, col, w, m = lvgen.rmat_device(scale, seed=0)
    nnz = int(col.numel())
    asg = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    res = {"workload": f"R-MAT scale {scale}", "n_vertices": n, "n_edges": int(m),
           "n_entries": nnz, "abcd": [0.57, 0.19, 0.19, 0.05], "weights": "unit FP32",
           "seed": 0}
    with torch.cuda.stream(stream):
        eng = lvb200.Engine(stream=stream.cuda_stream, apply_launch=apply_launch,
                            use_graphs=use_graphs)
        eng.load_device(n, nnz, off.data_ptr(), col.data_ptr(), w.data_ptr())
        res["tuning"] = {str(b): k for b, (k, _) in eng.autotune().items()}

        def step():
            return eng.run_device(n, nnz, off.data_ptr(), col.data_ptr(), w.data_ptr(),
                                  MIN_GAIN, asg.data_ptr())

        step()
        torch.cuda.synchronize()
        ms, edges, r = [], 0, None
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r = step()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
            edges += r.edges_processed
        levels = eng.levels()
        eng.set_profiling(True)
        eng.reset_kernel_stats()
        step()
        torch.cuda.synchronize()
        eng.set_profiling(False)
        kstats = eng.kernel_stats()
        eng.close()
        check = None
        if oracle_check:  # untimed: FP64 gains, then the oracle on the host
            eng64 = lvb200.Engine(stream=stream.cuda_stream, gain="fp64")
            r64 = eng64.run_device(n, nnz, off.data_ptr(), col.data_ptr(), w.data_ptr(),
                                   MIN_GAIN, asg.data_ptr())
            torch.cuda.synchronize()
            asg64 = asg.cpu().numpy().view(np.uint32).copy()
            eng64.close()
            check = {"engine_fp64_q": r64.modularity}
            h_off = off.cpu().numpy().view(np.uint64)
            h_col = col.cpu().numpy().view(np.uint32)
            h_w = w.cpu().numpy()
    del off, col, w, asg
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if check is not None:
        import pyoracle

        threads = host_threads()
        pyoracle.set_threads(threads)
        t0 = time.perf_counter()
        g = pyoracle.CSR(n, h_off, h_col, h_w.astype(np.float64))
        del h_w
        ref = pyoracle.louvain(g, MIN_GAIN, rule="py", prec="fp64", rows="first_seen")
        pyoracle.set_threads(1)
        check.update({
            "oracle": "louvian.py restated (FP64 gains, louvian.py's stop rule)",
            "oracle_q": ref.q, "oracle_s": time.perf_counter() - t0,
            "oracle_threads": threads,
            "abs_dq_fp32_mode": abs(r.modularity - ref.q),
            "abs_dq_fp64_mode": abs(check["engine_fp64_q"] - ref.q),
            "fp64_mode_partition_identical": bool(np.array_equal(asg64, ref.assignment)),
            "oracle_passes": [l.passes for l in ref.levels],
        })
        del g
    peak, peak_kind = measured_peak()
    moves = {k: v for k, v in kstats.items() if k.startswith("move") or k == "modularity"}
    name, st = max(moves.items(), key=lambda kv: kv[1]["total_ms"])
    launches_k = max(st["launches"], 1)
    achieved = (st["bytes"] / launches_k) / (st["total_ms"] / launches_k / 1000.0) / 1e9
    res.update({
        "ms_per_run": sum(ms) / len(ms), "edges_per_s_per_pass": edges / (sum(ms) / 1000.0),
        "final_q": r.modularity, "levels": len(levels),
        "passes": [l["passes"] for l in levels],
        "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "bytes_per_launch": st["bytes"] / launches_k,
                     "ms_per_launch": st["total_ms"] / launches_k},
        "kernel_ms": {k: round(v["total_ms"], 3) for k, v in kstats.items()},
    })
    if check is not None:
        res["oracle_check"] = check
    return res


def served_requests(count: int, seed: int):
    """The served workload's requests (seeded): half R-MAT graphs of scale
    U{10..21} (1,024 .. 2,097,152 vertices), half LFR-style graphs with
    log-uniform 1k .. 2M vertices and mixing mu ~ U(0.1, 0.5); unit FP32
    weights.  Generated on the device, kept as host graphs (the requests
    arrive from the host).  Returns [(graph, n, entries, kind)]."""
    import torch

    import lvb200

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        gseed = seed * 100_003 + i
        if rng.random() < 0.5:
            scale = int(rng.integers(10, 22))
            n, off, col, w, _ = lvgen.rmat_device(scale, seed=gseed)
            kind = f"rmat{scale}"
        else:
            n = int(np.exp(rng.uniform(np.log(1_000), np.log(2_000_000))))
            mu = float(rng.uniform(0.1, 0.5))
            (n, off, col, w, _), _ = lvgen.lfr_device(n, mu, seed=gseed)
            kind = "lfr"
        g = lvb200.Graph.from_csr(n, off.cpu().numpy().view(np.uint64),
                                  col.cpu().numpy().view(np.uint32), w.cpu().numpy())
        out.append((g, n, int(col.numel()), kind))
        del off, col, w
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def served_measure(count: int, rate: float, budget: int, distinct: int, seed: int = 0):
    """Served form on `count` requests whose graphs are drawn (seeded, with
    repetition) from `distinct` generated request graphs.  Two runs of the
    server: every request queued at t=0 (saturated capacity: graphs/s over
    the makespan), and Poisson arrivals at `rate` per second (latency =
    result time - arrival, p50/p99).  Against them the plain engine run per
    request through lv_run (host graphs, as the server's): its graphs/s from
    the summed run times, and the latencies a first-come-first-served single
    engine gives for the same arrivals.  Every served partition is compared
    with its graph's plain run."""
    pool = served_requests(distinct, seed)
    rng = np.random.default_rng(seed + 2)
    pick = rng.integers(0, len(pool), size=count)
    reqs = [pool[i] for i in pick]
    arrivals = np.cumsum(np.random.default_rng(seed + 1).exponential(1.0 / rate, size=count))
    return served_report(pool, pick, reqs, arrivals, rate, budget)


def serve_run(reqs, arrivals, budget, lanes=4):
    """Replays the arrivals against a server with its default lanes (two
    union lanes for smaller graphs, two solo lanes for larger ones, each
    stepped by a worker thread); arrivals None queues every request at
    t=0.  Returns (results by request, completion times, steps, most graphs
    resident at once)."""
    import lvb200

    count = len(reqs)
    with lvb200.Server(MIN_GAIN, budget, lanes=lanes, background=True) as server:
        # warm-up request (kernel set-up, first graph instantiations)
        server.submit(reqs[0][0], n_vertices=reqs[0][1])
        server.drain()
        ticket_of, done, done_t = {}, {}, np.zeros(count)
        max_res, i = 0, 0
        t0 = time.perf_counter()
        if arrivals is None:
            arrivals = np.zeros(count)
        while len(done) < count:
            now = time.perf_counter() - t0
            while i < count and arrivals[i] <= now:
                ticket_of[server.submit(reqs[i][0], n_vertices=reqs[i][1])] = i
                i += 1
            wait_s = (arrivals[i] - now) if i < count else 0.05
            server.wait(max(1, int(wait_s * 1000)))
            max_res = max(max_res, server.stats()["resident"])
            t = time.perf_counter() - t0
            while (x := server.poll()) is not None:
                j = ticket_of[x.ticket]
                done[j] = x
                done_t[j] = t
        stats = server.stats()
    return done, done_t, int(stats["steps"]), max_res


def served_report(pool, pick, reqs, arrivals, rate, budget):
    import lvb200

    count = len(reqs)
    # saturated: everything queued at t=0
    done_s, done_ts, _, max_res_s = serve_run(reqs, None, budget)
    makespan_s = float(done_ts.max())
    # Poisson arrivals
    done, done_t, steps, max_res = serve_run(reqs, arrivals, budget)
    lat = (done_t - arrivals) * 1000.0
    makespan = float(done_t.max() - arrivals[0])
    # plain engine, one run per distinct graph (its service time and result)
    eng = lvb200.Engine()
    eng.run(pool[0][0], MIN_GAIN)
    svc_pool, res_pool = np.zeros(len(pool)), []
    for k, (g, n, e, kind) in enumerate(pool):
        t = time.perf_counter()
        res = eng.run(g, MIN_GAIN)
        svc_pool[k] = time.perf_counter() - t
        res_pool.append(res)
    eng.close()
    svc = svc_pool[pick]
    same, dq = 0, 0.0
    for j in range(count):
        res = res_pool[pick[j]]
        same += int(np.array_equal(res.assignment, done[j].assignment) and
                    np.array_equal(res.assignment, done_s[j].assignment))
        dq = max(dq, abs(res.modularity - done[j].modularity),
                 abs(res.modularity - done_s[j].modularity))
    end, plain_lat = 0.0, np.zeros(count)
    for j in range(count):  # first come first served on one engine
        end = max(end, arrivals[j]) + svc[j]
        plain_lat[j] = (end - arrivals[j]) * 1000.0
    by_lane = []
    for ln in sorted({x.lane for x in done.values()}):
        idx = [j for j in range(count) if done[j].lane == ln]
        by_lane.append({"lane": ln, "requests": len(idx),
                        "p50_ms": float(np.percentile(lat[idx], 50)),
                        "p99_ms": float(np.percentile(lat[idx], 99))})
    kinds = {}
    for _, _, _, k in reqs:
        kinds[k] = kinds.get(k, 0) + 1
    plain_gps = count / float(svc.sum())
    return {
        "workload": "served requests", "requests": count,
        "distinct_graphs": len(pool),
        "requests_note": "graphs drawn with repetition from the distinct seeded request "
                         "graphs; every request runs in full",
        "arrivals": f"Poisson {rate}/s",
        "mix": "50% R-MAT scale U{10..21}, 50% LFR-style n log-U[1k,2M] mu U(0.1,0.5)",
        "kinds": kinds, "total_entries": int(sum(r[2] for r in reqs)),
        "total_vertices": int(sum(r[1] for r in reqs)), "budget_gb": budget / 1e9,
        "lanes": "2 union lanes (<= 2^18, <= 2^22 entries; 10/30% of the budget), "
                 "2 solo lanes for larger graphs (30% each), worker threads",
        "saturated": {"graphs_per_s": count / makespan_s, "makespan_s": makespan_s,
                      "plain_graphs_per_s": plain_gps,
                      "speedup_graphs_per_s": (count / makespan_s) / plain_gps,
                      "max_resident": int(max_res_s)},
        "poisson": {"graphs_per_s": count / makespan, "makespan_s": makespan,
                    "p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99)),
                    "plain_p50_ms": float(np.percentile(plain_lat, 50)),
                    "plain_p99_ms": float(np.percentile(plain_lat, 99)),
                    "max_resident": int(max_res), "steps": steps, "by_lane": by_lane},
        "plain_looped": {"graphs_per_s": plain_gps, "total_s": float(svc.sum())},
        "partitions_identical": f"{same}/{count}", "max_abs_dq": dq,
    }


def run_reference(args, rank, world):
    n, off, col, ww, desc = workload(args.workload)
    if rank != 0:
        return
    import pyoracle

    threads = host_threads()
    pyoracle.set_threads(threads)
    g = pyoracle.CSR(n, off, col, ww.astype(np.float64))
    for _ in range(args.warmup):
        pyoracle.louvain(g, MIN_GAIN, rule="py", prec="fp64", rows="first_seen")
    times, edges, q = [], 0, None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = pyoracle.louvain(g, MIN_GAIN, rule="py", prec="fp64", rows="first_seen")
        times.append(time.perf_counter() - t0)
        edges += sum(l.passes * l.n_entries for l in r.levels)
        q = r.q
    total = sum(times)
    value = edges / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(desc, parallelism=f"replicas only ({threads} CPU threads)",
                       l2="n/a (CPU)"),
        "final_q": q,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "host_threads": os.cpu_count(),
                         "sample": f"full workload, {args.steps} timed runs on {threads} of "
                                   f"{os.cpu_count()} host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def combine_replicas(ms: float, edges: float, device: str):
    """Replicas on N ranks: the job's time is the slowest rank's (max over
    ranks), its work the edges every rank processed (sum).  Every rank
    calls it at the same point."""
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item()), sum_over_ranks(float(edges), device)


def sum_over_ranks(x: float, device: str) -> float:
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t)
    return float(t.item())


def run_engine(args, rank, world):
    import torch

    import lvb200

    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    dev = torch.cuda.current_device()
    n, off, col, ww, desc = workload(args.workload)
    nnz = len(col)
    stream = torch.cuda.Stream()
    d_off = torch.from_numpy(off.view(np.int64)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_w = torch.from_numpy(ww).cuda()
    d_asg = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB
    torch.cuda.synchronize()
    eng = lvb200.Engine(device=dev, rule="py", stream=stream.cuda_stream,
                        use_graphs=not args.no_graphs, apply_launch=args.apply_launch)
    tuning = None
    if not args.no_tune:  # kernel variant per bucket, timed on level 0 (untimed)
        with torch.cuda.stream(stream):
            eng.load_device(n, nnz, d_off.data_ptr(), d_col.data_ptr(), d_w.data_ptr())
            tuning = {str(b): k for b, (k, _) in eng.autotune().items()}

    def step():
        return eng.run_device(n, nnz, d_off.data_ptr(), d_col.data_ptr(),
                              d_w.data_ptr(), MIN_GAIN, d_asg.data_ptr())

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        props = torch.cuda.get_device_properties(dev)
        gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(dev)
        launches0 = lvb200.launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        edges, q, levels = 0, None, None
        with ClockSampler(gpu_id) as clocks:
            for i in range(args.steps):
                flush.zero_()  # evict the previous step's working set from L2
                ev[i][0].record(stream)
                r = step()
                ev[i][1].record(stream)
                edges += r.edges_processed
                q = r.modularity
            torch.cuda.synchronize()
        launches = lvb200.launch_count() - launches0
        levels = eng.levels()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        # kernel timing: K more steps with a CUDA event pair around every
        # launch group (the pass loop then replays a captured pass per pass,
        # since event nodes cannot sit inside the graph's WHILE body)
        eng.set_profiling(True)
        eng.reset_kernel_stats()
        prof_ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        prof_ev[0].record(stream)
        for i in range(args.steps):
            flush.zero_()
            step()
        prof_ev[1].record(stream)
        torch.cuda.synchronize()
        eng.set_profiling(False)
        kstats = eng.kernel_stats()
        prof_ms = prof_ev[0].elapsed_time(prof_ev[1]) / args.steps
        if world > 1:
            torch.distributed.barrier()
            ms, edges_all = combine_replicas(ms, edges, "cuda")
        else:
            edges_all = float(edges)
        value = edges_all / (ms / 1000.0)

        # e2e: host buffers through lv_run (+ assignment download)
        g = lvb200.Graph.from_csr(n, off, col, ww)
        e2e_times, e2e_edges = [], 0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rr = eng.run(g, MIN_GAIN)  # includes lv_get_assignment
            e2e_times.append(time.perf_counter() - t0)
            e2e_edges += rr.edges_processed
        e2e_value = e2e_edges / sum(e2e_times)
        if world > 1:
            e2e_value = sum_over_ranks(e2e_value, "cuda")  # replicas: throughputs add up

    eng.close()
    batched = served = hbm = None
    if world == 1 and args.batch_graphs > 0:
        batched = batched_measure(stream, args.batch_graphs, apply_launch=args.apply_launch)
    if world == 1 and args.serve_requests > 0:
        served = served_measure(args.serve_requests, args.serve_rate,
                                int(args.serve_budget_gb * 1e9),
                                min(args.serve_distinct, args.serve_requests))
    if world == 1 and args.hbm_scale > 0:
        hbm = hbm_scale_measure(stream, args.hbm_scale, oracle_check=not args.no_oracle_check,
                                apply_launch=args.apply_launch, use_graphs=not args.no_graphs)
    if rank != 0:
        return
    # roofline of the dominant kernel group
    peak, peak_kind = measured_peak()
    dom = max(kstats.items(), key=lambda kv: kv[1]["total_ms"])
    name, st = dom
    launches_k = max(st["launches"], 1)
    achieved = (st["bytes"] / launches_k) / (st["total_ms"] / launches_k / 1000.0) / 1e9
    traffic = ncu_traffic(name)
    cpu = cpu_baseline(n, off, col, ww) if world == 1 and not args.no_cpu_baseline else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(desc, parallelism="replicas only" if world > 1 else "single GPU",
                       l2="flushed (256 MB write) between timed steps",
                       pass_loop="host loop" if args.no_graphs else "CUDA graph WHILE node",
                       apply=("a launch per bucket" if args.apply_launch
                              else "in the bucket steps (second state copy)"),
                       tuning=tuning or "defaults"),
        "final_q": q,
        "levels": [{"V": l["n_vertices"], "E": l["n_entries"], "passes": l["passes"],
                    "prepare_ms": round(l["prepare_ms"], 4),
                    "move_ms": round(l["move_ms"], 4),
                    "aggregate_ms": round(l["aggregate_ms"], 4)}
                   for l in levels],
        "profiled_ms_per_step": prof_ms,
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int((n + 1) * 8 + nnz * 8),
                "d2h_bytes_per_step": int(n * 4)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "traffic": traffic,
                     "bytes_per_launch": st["bytes"] / launches_k,
                     "ms_per_launch": st["total_ms"] / launches_k},
        "kernel_ms": {k: round(v["total_ms"], 4) for k, v in kstats.items()},
        "clocks": clocks.summary(),
    }
    if batched:
        line["batched"] = batched
    if served:
        line["served"] = served
    if hbm:
        line["hbm_scale"] = hbm
    if cpu:
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind",
                                                    "host_threads", "sample")}
        line["cpu_baseline"]["final_q"] = cpu["final_q"]
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="powerlaw")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default move kernel of every bucket (no lv_autotune)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="run each level's pass loop from the host instead of a CUDA graph "
                         "WHILE node, in the headline and HBM-scale legs (same kernels; ncu "
                         "cannot profile kernels inside graphs with conditional nodes)")
    ap.add_argument("--hbm-scale", type=int, default=24,
                    help="R-MAT scale of the HBM-scale plain-engine measurement (0: skip)")
    ap.add_argument("--apply-launch", action="store_true",
                    help="apply each bucket's moves in a launch of its own (lv_config.apply_launch) "
                         "instead of inside the bucket steps")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline leg (profiling runs)")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the untimed FP64-gain run and host oracle on the HBM-scale graph")
    ap.add_argument("--batch-graphs", type=int, default=4096,
                    help="graphs of the batched-form measurement (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests of the served-form measurement (0: skip)")
    ap.add_argument("--serve-distinct", type=int, default=400,
                    help="distinct request graphs the served requests are drawn from")
    ap.add_argument("--serve-rate", type=float, default=200.0,
                    help="Poisson arrival rate of the served requests, per second")
    ap.add_argument("--serve-budget-gb", type=float, default=120.0,
                    help="device memory budget of the server")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    if world > 1 and args.impl == "b200":
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group(
            "nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_engine(args, local if world > 1 else 0, world)
    finally:
        if world > 1 and args.impl == "b200":
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
