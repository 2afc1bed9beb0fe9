"""Iteration counts of the reference algorithm on the 64 members of the batched 3D workload.

The batched workload (64 sliding ice streams, n ~ U{64..256} vertices per side, 11 levels,
seeded log-normal basal friction each; Chronopoulos-Gear PCG, SIA preconditioner, tol 1e-8,
ncheck 5) takes about two hours of single-core time to solve in full with the reference's
algorithm on the CPU, far too long for a benchmark run.  bench.py's CPU arms therefore time a bounded number of iterations of each member and scale
by the number of iterations a full solve takes.  This script computes those counts once, by
running the oracle (the reference's algorithm and summation order, FP64) to convergence on
every member, and writes them to cfg4_niters.json beside it.

    python oracle/cfg4_niters.py [--procs N]

Test infrastructure: nothing in the product path reads the file.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "cfg4_niters.json")
TOL, NCHECK, MAXITERS, PRECOND = 1e-8, 5, 4000, 2


def _solve(args):
    n, seed = args
    sys.path.insert(0, ROOT)
    import oracle
    from cism_b200 import assembly as asm
    P = asm.batch_member(n, seed)
    t0 = time.perf_counter()
    st, xu, xv, err, nit = oracle.pcg("chrongear", P, PRECOND, ncheck=NCHECK, tol=TOL, maxiters=MAXITERS,
                                      summode=oracle.SUM_SEQ)
    return seed, n, int(st), float(err), int(nit), time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    sys.path.insert(0, ROOT)
    import oracle
    from cism_b200 import assembly as asm
    oracle.build()
    sizes = asm.batch_sizes(64)
    jobs = sorted([(n, s) for s, n in enumerate(sizes)], key=lambda a: -a[0])  # largest first
    with mp.get_context("spawn").Pool(args.procs) as pool:
        res = pool.map(_solve, jobs, chunksize=1)
    res.sort()
    out = {"workload": "64 sliding 3D ice streams, n ~ U{64..256}^2 x 11 levels (assembly.batch_sizes(64), "
                       "batch_member(n, seed)), Chronopoulos-Gear + SIA precond, tol 1e-8, ncheck 5",
           "summation": "reference order (oracle SUM_SEQ), FP64",
           "sizes": [r[1] for r in res], "status": [r[2] for r in res], "err": [r[3] for r in res],
           "niters": [r[4] for r in res], "cpu_s": [round(r[5], 1) for r in res]}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {OUT}: niters {min(out['niters'])}..{max(out['niters'])}, "
          f"max err {max(out['err']):.3e}, cpu {sum(out['cpu_s']):.0f} s")


if __name__ == "__main__":
    main()
