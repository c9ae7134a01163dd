"""Generates the golden fixtures under tests/golden/ by running the
reference's own CPU implementation (louvian.py, imported unmodified from the
reference checkout) on small seeded graphs.

Run in a checkout where the reference is present:
    python tests/golden/make_golden.py [--ref $LOUVAIN_REFERENCE_DIR]

For every graph it writes `<name>.mtx` (the input, readable by both the
reference CLI and louvian.py) and `<name>.json` with what louvian.py
computed: per level the vertex count, the per-pass modularity values and
the pass count, the final modularity, and the final community of every
vertex.  louvian.py numbers vertices from 1 and adds an isolated vertex 0
(louvian.py:33); that vertex always stays alone in community 0, so the
fixture stores sizes and community ids with it removed (ids shifted by -1),
which is how a reader with the reference CLI's semantics numbers them.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "louvain-community-detection_b200",
                                "python"))
import lvgen  # noqa: E402

GAIN = 1e-6


def graphs():
    """(name, n, src, dst, w, description)"""
    out = []
    n, s, d, w = lvgen.two_cliques_bridge(5)
    out.append(("two_cliques", n, s, d, w, "two 5-cliques joined by a bridge"))
    n, s, d, w = lvgen.ring_of_cliques(8, 6)
    out.append(("ring_of_cliques", n, s, d, w, "ring of eight 6-cliques"))
    n, s, d, w = lvgen.banded_fem(n=600, half_band=30, target_entries=20000, seed=1)
    out.append(("banded_small", n, s, d, w,
                "banded FEM-like, n=600, half-band 30, weights U(0.1,1)"))
    n, s, d, w = lvgen.planted_powerlaw(n=3000, target_edges=9000, max_deg=400,
                                        comm_min=8, comm_max=300, seed=2)
    out.append(("planted_small", n, s, d, w,
                "Chung-Lu power law 2.3 + planted communities, unit weights"))
    n, s, d, w = lvgen.planted_powerlaw(n=2500, target_edges=8000, max_deg=300,
                                        comm_min=8, comm_max=200, seed=3,
                                        unit=False)
    out.append(("planted_weighted", n, s, d, w,
                "Chung-Lu power law + planted communities, weights U(0.5,1.5)"))
    n, s, d, w = lvgen.rmat(11, edge_factor=8, seed=4)
    out.append(("rmat11", n, s, d, w, "R-MAT scale 11, edge factor 8, unit"))
    n, s, d, w = lvgen.sbm(2000, 8, mean_deg=16, seed=5)
    out.append(("sbm_small", n, s, d, w, "SBM 2000 vertices, 8 blocks"))
    n, s, d, w = lvgen.star(1000, seed=6)
    out.append(("star1000", n, s, d, w, "star with 1000 leaves (hub, shared table)"))
    # hub beyond the shared-memory class plus a ring among the leaves
    rng = np.random.default_rng(7)
    leaves = 3000
    s = np.concatenate([np.zeros(leaves, np.int64), np.arange(1, leaves)])
    d = np.concatenate([np.arange(1, leaves + 1), np.arange(2, leaves + 1)])
    w = rng.uniform(0.5, 1.5, len(s)).astype(np.float32)
    out.append(("hub3000", leaves + 1, s, d, w,
                "hub of degree 3000 (global table) plus a path through its leaves"))
    # self-loops, duplicate entries, isolated vertices, mixed weights
    s = np.array([0, 1, 2, 0, 3, 4, 4, 5, 6, 2, 7, 7, 1, 8])
    d = np.array([1, 2, 0, 0, 4, 5, 3, 5, 7, 1, 6, 7, 0, 9])
    w = np.array([1.0, 2.0, 0.5, 0.25, 1.5, 1.0, 2.0, 3.0, 1.0, 0.75, 2.5, 1.25,
                  0.5, 1.0], np.float32)
    out.append(("loops_dups_isolated", 12, s, d, w,
                "self-loops, repeated pairs, isolated vertices 10 and 11"))
    return out


def run_louvian(louvian, path):
    g = louvian.Graph()
    aggr = louvian.CommAggregation()
    g.parse_graph(path)
    n_in = g.vert_n - 1
    assignment = list(range(g.vert_n))  # louvian.py vertex -> current vertex
    levels = []
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        while True:
            start = len(buf.getvalue().splitlines())
            v_level = g.vert_n
            more = g.modularity_optimization(GAIN)
            lines = buf.getvalue().splitlines()[start:]
            # every pass prints "Q_new Q_old"; a failing first pass adds "Q_old"
            trace = [float(x.split()[0]) for x in lines if len(x.split()) == 2]
            q_start = float(lines[0].split()[1])
            levels.append({"n_vertices": v_level - 1, "passes": len(trace),
                           "q_trace": trace, "q_start": q_start,
                           "moved": bool(more)})
            if not more:
                q_final = float(lines[-1].split()[0])
                break
            comm = list(g.comm)
            aggr.contract(g)
            new_id = aggr.new_id
            assignment = [new_id[comm[a]] for a in assignment]
    part = [a - 1 for a in assignment[1:]]
    assert all(p >= 0 for p in part)
    assert len(part) == n_in
    return {"q_final": q_final, "levels": levels, "assignment": part,
            "n_communities": levels[-1]["n_vertices"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("LOUVAIN_REFERENCE_DIR", "/root/reference"))
    args = ap.parse_args()
    sys.path.insert(0, args.ref)
    import louvian  # the reference's CPU path, unmodified

    index = []
    for name, n, s, d, w, desc in graphs():
        path = os.path.join(HERE, name + ".mtx")
        lvgen.write_mtx(path, n, s, d, w)
        res = run_louvian(louvian, path)
        res.update({"name": name, "description": desc, "min_gain": GAIN,
                    "n_vertices": int(n), "n_edge_lines": int(len(s)),
                    "generator": "tests/golden/make_golden.py",
                    "reference": "louvian.py (upicine/louvain-community-detection)"})
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(res, f, indent=None, separators=(",", ":"))
        index.append(name)
        print(f"{name:22s} V={n:6d} lines={len(s):7d} Q={res['q_final']!r} "
              f"levels={[l['n_vertices'] for l in res['levels']]}")
    # the same graph written 0-based and with comment/banner lines: the
    # reference CLI's reader must build the identical CSR (utils.cu:132-166)
    n, s, d, w = lvgen.two_cliques_bridge(5)
    lvgen.write_mtx(os.path.join(HERE, "two_cliques_zero_based.mtx"), n, s, d, w,
                    one_based=False)
    lvgen.write_mtx(os.path.join(HERE, "two_cliques_banner.mtx"), n, s, d, w,
                    banner=True, comments=[" written by make_golden.py", ""])
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump({"graphs": index, "min_gain": GAIN}, f, indent=1)


if __name__ == "__main__":
    main()
