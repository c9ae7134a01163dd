"""Runs the engine on one synthetic workload and prints what it did.

    python louvain-community-detection_b200/python/run_case.py \
        --workload powerlaw|banded|rmat<S>|rmatdev<S> [--rule py|cuda]
        [--no-graphs] [--runs N] [--min-gain G] [--timing]

`rmat<S>` builds R-MAT scale S on the host (numpy), `rmatdev<S>` on the GPU
(needed for S >= 22).  The CSR stays in device memory and the run goes
through lv_run_device.  Also the target of the ncu captures summarised
under profiles/.
"""
import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402


def device_workload(name):
    import torch

    import lvgen

    if name.startswith("rmatdev"):
        n, off, col, w, m = lvgen.rmat_device(int(name[7:]), seed=0)
        return n, off, col, w, m
    if name == "powerlaw":
        n, s, d, w = lvgen.planted_powerlaw(seed=0)
    elif name == "banded":
        n, s, d, w = lvgen.banded_fem(seed=0)
    elif name.startswith("rmat"):
        n, s, d, w = lvgen.rmat(int(name[4:]), seed=0)
    else:
        raise SystemExit(f"unknown workload {name}")
    off, col, ww = lvgen.csr_from_edges(n, s, d, w)
    return (n, torch.from_numpy(off.view(np.int64)).cuda(),
            torch.from_numpy(col.view(np.int32)).cuda(), torch.from_numpy(ww).cuda(),
            len(s))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="powerlaw")
    ap.add_argument("--rule", default="py", choices=["py", "cuda"])
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--runs", type=int, default=1)
    ap.add_argument("--min-gain", type=float, default=1e-6)
    ap.add_argument("--timing", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="time every launch group with CUDA events")
    args = ap.parse_args()
    import torch

    import lvb200

    t0 = time.perf_counter()
    n, off, col, w, m = device_workload(args.workload)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    nnz = col.numel()
    print(f"workload={args.workload} V={n} edges={m} entries={nnz} gen_s={gen_s:.1f}")
    asg = torch.empty(n, dtype=torch.int32, device="cuda")
    with lvb200.Engine(rule=args.rule, use_graphs=not args.no_graphs) as e:
        e.set_profiling(args.profile)
        for i in range(args.runs):
            e.reset_kernel_stats()
            t0 = time.perf_counter()
            r = e.run_device(n, nnz, off.data_ptr(), col.data_ptr(), w.data_ptr(),
                             args.min_gain, asg.data_ptr())
            dt = time.perf_counter() - t0
            print(f"run {i}: Q={r.modularity:.10f} levels={r.n_levels} "
                  f"communities={r.n_communities} alg_ms={r.alg_ms:.3f} wall_ms={dt*1e3:.3f} "
                  f"edges/s per pass={r.edges_processed / (r.alg_ms / 1e3):.4g}")
        if args.timing:
            for lv in e.levels():
                print("  level V={n_vertices} E={n_entries} passes={passes} "
                      "prepare_ms={prepare_ms:.3f} move_ms={move_ms:.3f} "
                      "aggregate_ms={aggregate_ms:.3f} q_end={q_end:.8f}".format(**lv))
        if args.profile:
            for name, st in e.kernel_stats().items():
                if st["launches"]:
                    gbs = st["bytes"] / (st["total_ms"] / 1e3) / 1e9
                    print(f"  kernel {name:11s} launches={st['launches']:5d} "
                          f"ms={st['total_ms']:9.3f} avg_us={1e3 * st['total_ms'] / st['launches']:9.2f} "
                          f"alg_GB/s={gbs:8.1f}")


if __name__ == "__main__":
    main()
