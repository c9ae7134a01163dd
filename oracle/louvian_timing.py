"""Times the reference's own CPU path, louvian.py, per pass -- test and
measurement infrastructure only (it runs where the reference checkout is,
not on the GPU box; bench.py's CPU baseline there is the oracle's
restatement, which this script also times on the same graph for the
ratio between the two).

    python oracle/louvian_timing.py --ref $LOUVAIN_REFERENCE_DIR/louvian.py \
        [--workload banded|powerlaw-small] [--min-gain 1e-6]

louvian.py is imported unmodified; its Graph.modularity_optimization and
Graph._compute_modularity are wrapped to count passes and time every phase
(louvian.py:75-99 is the pass loop, louvian.py:218-232 the level loop).
Prints one JSON line: per level the vertices, stored entries, passes and
seconds, the final modularity, and edges/s per pass for louvian.py and
for the oracle.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "louvain-community-detection_b200",
                                "python"))

import lvgen  # noqa: E402
import pyoracle  # noqa: E402


def load_reference(path):
    spec = importlib.util.spec_from_file_location("louvian_ref", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload(name):
    if name == "banded":
        return lvgen.banded_fem(seed=0)
    if name == "powerlaw-small":
        return lvgen.planted_powerlaw(n=20_000, target_edges=55_000, seed=0)
    raise SystemExit(f"unknown workload {name}")


def time_louvian(mod, path, min_gain):
    """Runs louvian.py's level loop (its main(), louvian.py:218-232) with
    per-pass counting; returns (levels, final Q, seconds)."""
    levels = []
    orig_opt = mod.Graph.modularity_optimization
    orig_q = mod.Graph._compute_modularity

    def counting_q(self):
        self._lv_passes = getattr(self, "_lv_passes", 0) + 1
        return orig_q(self)

    def timed_opt(self, threshold):
        self._lv_passes = 0
        entries = sum(len(e) for e in self.edges)
        t0 = time.perf_counter()
        r = orig_opt(self, threshold)
        # the sweep before the first pass is not a pass
        levels.append({"V": self.vert_n, "E": entries, "passes": max(0, self._lv_passes - 1),
                       "s": time.perf_counter() - t0})
        return r

    mod.Graph.modularity_optimization = timed_opt
    mod.Graph._compute_modularity = counting_q
    try:
        g = mod.Graph()
        g.parse_graph(path)
        aggr = mod.CommAggregation()
        t0 = time.perf_counter()
        import io
        import contextlib
        out = io.StringIO()
        with contextlib.redirect_stdout(out):  # louvian.py prints Q itself
            while g.modularity_optimization(min_gain):
                aggr.contract(g)
        total = time.perf_counter() - t0
        q = float(out.getvalue().split()[-1]) if out.getvalue().split() else None
    finally:
        mod.Graph.modularity_optimization = orig_opt
        mod.Graph._compute_modularity = orig_q
    return levels, q, total


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.path.join(
        os.environ.get("LOUVAIN_REFERENCE_DIR", "/root/reference"), "louvian.py"))
    ap.add_argument("--workload", default="banded")
    ap.add_argument("--min-gain", type=float, default=1e-6)
    args = ap.parse_args()
    n, s, d, w = workload(args.workload)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "g.mtx")
        lvgen.write_mtx(path, n, s, d, w)
        mod = load_reference(args.ref)
        levels, q_ref, total = time_louvian(mod, path, args.min_gain)
        g = pyoracle.read_mtx(path, as_float=False)
    t0 = time.perf_counter()
    r = pyoracle.louvain(g, args.min_gain, rule="py", prec="fp64", rows="first_seen")
    t_or = time.perf_counter() - t0
    pass_entries = sum(l["passes"] * l["E"] for l in levels)
    or_entries = sum(l.passes * l.n_entries for l in r.levels)
    print(json.dumps({
        "workload": args.workload, "n_vertices": n, "n_edges": int(len(s)),
        "louvian_py": {"levels": levels, "final_q": q_ref, "seconds": total,
                       "edges_per_s_per_pass": pass_entries / total, "cores": 1},
        "oracle": {"final_q": r.q, "seconds": t_or,
                   "edges_per_s_per_pass": or_entries / t_or, "cores": 1},
        "oracle_speedup": total / t_or,
    }))


if __name__ == "__main__":
    main()
