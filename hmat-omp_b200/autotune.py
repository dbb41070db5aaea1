"""Offline tile autotuner for the batched GEMM steps.

Runs a workload once per tile choice (tile width BN of the warp-tiled kernel in
{32, 64, 96, 128}, its shape (default, 64-row tiles, 8 x 8 outputs per lane for FP64,
96-row tiles),
tc on/off: the tcgen05 kernel for the FP32 batches the accuracy policy lets on it, the
FP64 MMA kernel for FP64 batches) with the choice forced on every batch (HM_TILE_FORCE), times
every GEMM step with the library's profiler, and keeps, per batch signature, the fastest
choice when it beats the built-in heuristic by more than --margin.  The result is a JSON
table {"signature": [bn, small, tc], ...} that the library reads from tile_table.json
beside it (or from HM_TILE_TABLE) when it plans an operator.

    python hmat-omp_b200/autotune.py --workload headline hss --out hmat-omp_b200/tile_table.json

Workloads: "headline" = mixed and FP64 factor + solve of the 2-D Coulomb operator
(N = 2^18, leaf 256, ranks <= 96, 64 RHS); "hss" = FP64 factor + solve of the Gaussian
HSS operator (N = 65536, leaf 128, 32 RHS).  Each child process plans its operator with
the forced choice, runs one untimed factor + solve, then --reps profiled ones; a step's
time is the sum over its records in one repetition, minimum over repetitions.
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CHOICES = [(bn, sm, tc) for bn, sm, tc in itertools.product((32, 64, 96, 128), (0, 1, 2, 3), (0, 1))]


def _headline(H):
    rng = np.random.default_rng(3)
    N = 1 << 18
    p = rng.random((N, 2))
    p = np.ascontiguousarray(p[H.morton_order(p)])
    ops = []
    for prec in (H.MIXED, H.FP64):
        h = H.HODLRMatrix(1e-10, rsvd_rank=96, oversample=10, max_rank=96, sketch=H.SKETCH_DEVICE_NORMAL, seed=0,
                          precision=prec, ir_tol=1e-10, ir_max_iter=30)
        h.build_from_kernel(H.KERNEL_COULOMB, p, [1e-3, 4.0], 256)
        ops.append((h, np.random.default_rng(5).standard_normal((N, 64))))
    return ops


def _hss(H):
    N = 65536
    x = np.sort(np.random.default_rng(2).random(N))
    h = H.HSSMatrix(1e-10, rsvd_rank=64, max_rank=64, oversample=10, sketch=H.SKETCH_DEVICE_NORMAL, seed=0,
                    refine_steps=1)
    h.build_from_kernel(H.KERNEL_GAUSSIAN, x, [0.05, 1e-2], 128)
    return [(h, np.random.default_rng(5).standard_normal((N, 32)))]


WORKLOADS = {"headline": _headline, "hss": _hss}


def child(workload: str, reps: int) -> dict:
    """Per signature: (effective choice, best summed ms) for one forced choice."""
    sys.path.insert(0, HERE)
    import hmat_b200 as H
    if not os.environ.get("HM_TILE_FORCE"):
        H.tile_table_load("")   # the built-in heuristics, not a previous table
    ops = WORKLOADS[workload](H)
    for h, b in ops:
        h.factor()
        h.solve(b)
    best: dict[str, list] = {}
    for _ in range(reps):
        tot: dict[str, list] = {}
        for h, b in ops:
            H.profile_enable(True)
            h.factor()
            h.solve(b)
            seq = H.profile_sequence()
            H.profile_enable(False)
            for rec in seq:
                tag = rec[5] if len(rec) > 5 else ""
                if "#" not in tag:
                    continue
                sig, ch = tag.split("#")
                t = tot.setdefault(sig, [ch, 0.0])
                t[1] += rec[2]
        for sig, (ch, ms) in tot.items():
            if sig not in best or ms < best[sig][1]:
                best[sig] = [ch, ms]
    return best


def run_child(workload: str, choice, reps: int) -> dict:
    env = dict(os.environ)
    env.pop("HM_TILE_FORCE", None)
    if choice is not None:
        env["HM_TILE_FORCE"] = ",".join(map(str, choice))
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", workload, "--reps", str(reps)],
                         env=env, capture_output=True, text=True)
    if out.returncode != 0:   # e.g. a choice under which the mixed refinement stops converging
        print(f"choice {choice}: child failed: {out.stderr.strip().splitlines()[-1:]}", file=sys.stderr)
        return {}
    return json.loads(out.stdout.strip().splitlines()[-1])


def select(base: dict, runs: list, margin: float, table: dict) -> dict:
    """Fold child results into `table` (updated in place) and return a per-signature report.
    base: {sig: [choice, ms]} of the heuristic run; runs: the forced runs' results.  A
    signature gets an entry only when its fastest effective choice differs from the
    heuristic's and beats it by more than `margin`; otherwise any old entry is dropped."""
    cands = {sig: {} for sig in base}
    for res in runs:
        for sig, (eff, ms) in res.items():
            if sig in cands:
                cands[sig][eff] = min(ms, cands[sig].get(eff, float("inf")))
    report = {}
    for sig, (eff0, ms0) in base.items():
        eff, ms = min(cands[sig].items(), key=lambda kv: kv[1]) if cands[sig] else (eff0, ms0)
        report[sig] = {"heuristic": [eff0, round(ms0, 4)], "best": [eff, round(ms, 4)]}
        if ms < (1.0 - margin) * ms0 and eff != eff0:
            table[sig] = [int(v) for v in eff.split(",")]
        else:
            table.pop(sig, None)
    return report


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", nargs="+", default=["headline"], choices=sorted(WORKLOADS))
    ap.add_argument("--out", default=os.path.join(HERE, "tile_table.json"))
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--margin", type=float, default=0.03, help="keep a choice only if this much faster")
    ap.add_argument("--child", default=None)
    args = ap.parse_args()
    if args.child:
        print(json.dumps(child(args.child, args.reps)))
        return
    table = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            table = json.load(f)
    report = {}
    for wl in args.workload:
        base = run_child(wl, None, args.reps)
        runs = [run_child(wl, ch, args.reps) for ch in CHOICES]
        report.update(select(base, runs, args.margin, table))
    with open(args.out, "w") as f:
        json.dump(dict(sorted(table.items())), f, indent=1)
        f.write("\n")
    print(json.dumps({"entries": len(table), "report": report}, indent=1))


if __name__ == "__main__":
    main()
