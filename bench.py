"""Benchmark: solves/sec (and p50/p99 latency) to a 1e-8 FP64 relative residual, vs the plain
FP64 GPU PCG.

Workload (default, one GPU): the batched configuration, 64 uneven 3D Blatter-Pattyn systems
(sliding ice streams, n ~ U{64..256} vertices per side, 11 levels, each with its own seeded
log-normal basal friction, first-Picard assembly), Chronopoulos-Gear PCG with the SIA
preconditioner, tol 1e-8.  Synthetic data: the reference runs no public dataset for this path.

Our arm ("ours"): the mixed-precision Chronopoulos-Gear solver (FP32 recurrences, FP64 x, dot
products and residual replacement every 5 iterations) over all 64 device-resident systems in one
persistent launch, captured in a CUDA graph; a step is one replay (64 solves from x0 = 0).  Beside
it in the same line: the plain FP64 GPU PCG (the reference algorithm statement by statement,
bit-identical to the oracle) one system after another, the mixed solver one system at a time, a
1-core CPU baseline, and the like-for-like plain FP64 comparison on the 401x401 2D SSA
configuration (GPU against 1 CPU core).  The inputs (~10 GB of FP32 and ~20 GB of FP64 matrices)
are larger than L2.  `e2e` is the same metric through the batch API with host buffers: every
member's A and b uploaded from pinned host memory, the batched solve, every x downloaded.

Reference arm (`--impl reference`): the CPU restatement of the reference PCG (oracle/, FP64,
the reference's summation order) on all host cores for the same 64 members; each step is a
bounded sample scaled to full solves by the members' iteration counts (oracle/cfg4_niters.json).

Other workloads: --workload cfg2 (the 401x401 2D SSA system, mixed solver, single solves),
cfg5 (the served Poisson stream), --mode profile (the commands the ncu summaries capture).

Launch: python bench.py [--gpus N --steps K --warmup W] (torchrun for N > 1: each rank solves
its own replica of the workload, scaling "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "solves/sec and p50/p99 latency at 1e-8 rel. residual vs plain FP64 GPU PCG"
UNIT = "solves/s"
WORKLOAD = "cfg2: 2D SSA 401x401 nodes, dx=1 km, Chronopoulos-Gear PCG + diagonal (Jacobi) precond, tol 1e-8"
TOL, NCHECK, MAXITERS, PRECOND = 1e-8, 5, 20000, 1
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def make_problem(workload="cfg2"):
    from cism_b200 import assembly as asm
    if workload == "cfg2":
        return asm.ssa_random(ewn=401, nsn=401, dx=1000.0, seed=7)
    if workload == "cfg3":   # 201x201x11 ice stream, no-slip bed
        return asm.ice_stream(ewn=201, nsn=201, nz=11, dx=2000.0)
    if workload == "dome":   # cfg1: 31x31x11 dome
        return asm.dome()
    raise ValueError(workload)


PROFILE_PRECOND = {"cfg2": 1, "cfg3": 2, "dome": 2}


def run_profile(args):
    """Only the product path (mixed solves) on one workload: the command ncu captures."""
    import torch
    import cism_b200 as cg
    from cism_b200 import build
    build.build()
    torch.zeros(1, device="cuda")  # CUDA context up before any timing
    cg.set_mixed_layout(cg.MIXED_LAYOUT_FULL if args.layout == "full" else cg.MIXED_LAYOUT_AUTO)
    if args.workload == "cfg4":  # the first --batch members of cfg4 through one graph-captured launch
        from cism_b200 import assembly as asm
        sizes = asm.batch_sizes(64)[:args.batch]
        solvers = [cg.DeviceSolver(P) for P in cfg4_problems(os.cpu_count() or 1, args.batch)]
        B = cg.GraphBatch(solvers, precond=args.precond, ncheck=NCHECK, tol=TOL, maxiters=4000)
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            B.run()
            errs, nits, sts = B.wait()
            wall = time.perf_counter() - t0
        print(f"profile workload=cfg4 batch={len(sizes)} precond={args.precond} sizes={sizes} niters={list(nits)} "
              f"niters_sum={int(sum(nits))} err_max={max(errs):.3e} "
              f"wall_ms={1e3 * wall:.1f}")
        print("tile heights:", cg.tile_table())
        B.close()
        if args.fp64:  # the plain FP64 solver on the same members, one after another
            t0 = time.perf_counter()
            n64 = 0
            for S in solvers:
                e, n = S.solve(cg.ALG_CHRONGEAR, args.precond, NCHECK, TOL, 4000)
                n64 += n
            print(f"fp64 plain: precond={args.precond} niters_sum={n64} wall_ms={1e3 * (time.perf_counter() - t0):.1f}")
        return 0
    P = make_problem(args.workload)
    S = cg.DeviceSolver(P)
    pc = PROFILE_PRECOND[args.workload]
    for k in range(args.warmup):
        e, n = S.solve(cg.ALG_MIXED_CHRONGEAR, pc, NCHECK, TOL, MAXITERS)
    S.profile(True)
    t0 = time.perf_counter()
    for k in range(args.steps):
        e, n = S.solve(cg.ALG_MIXED_CHRONGEAR, pc, NCHECK, TOL, MAXITERS)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / max(args.steps, 1)
    ms, nl, by = S.profile_read()
    print("tile heights:", cg.tile_table())
    print(f"profile workload={args.workload} precond={pc} niters={n} err={e:.3e} unknowns={P.n_unknowns} "
          f"kernel_ms={ms / max(nl, 1):.3f} wall_ms={1e3 * wall:.3f} GB/s={by / (ms / max(nl, 1) / 1e3) / 1e9:.1f}")
    if args.fp64:
        t0 = time.perf_counter()
        e, n = S.solve(cg.ALG_CHRONGEAR, pc, NCHECK, TOL, MAXITERS)
        print(f"fp64 plain: niters={n} err={e:.3e} wall_ms={1e3 * (time.perf_counter() - t0):.3f}")
    return 0


# ---------------------------------------------------------------------------
# batched workload (the default line): 64 uneven 3D solves in one graph-captured launch
# ---------------------------------------------------------------------------
CFG4_WORKLOAD = ("cfg4: 64 uneven 3D BP solves, n~U{64..256}^2 x 11 levels, own seeded log-normal beta each, "
                 "Chronopoulos-Gear + SIA precond, tol 1e-8")
CFG4_PRECOND, CFG4_MAXIT = 2, 4000
CFG4_NITERS = os.path.join(ROOT, "oracle", "cfg4_niters.json")


def _make_member(args):
    from cism_b200 import assembly as asm
    n, seed = args
    return asm.batch_member(n, seed)


def cfg4_problems(procs, count=64):
    """The first `count` of the 64 members (seeded sizes and fields), generated in a pool of spawned
    processes."""
    import multiprocessing as mp
    from cism_b200 import assembly as asm
    sizes = asm.batch_sizes(64)[:count]
    with mp.get_context("spawn").Pool(max(1, min(len(sizes), procs))) as pool:
        return pool.map(_make_member, [(n, s) for s, n in enumerate(sizes)])


def cfg4_reference_niters():
    """Full-solve iteration counts of the reference algorithm (oracle, reference order) per member."""
    try:
        with open(CFG4_NITERS) as f:
            d = json.load(f)
        return [int(v) for v in d["niters"]]
    except Exception:
        return None


def active_nodes(P):
    return int(np.count_nonzero(P.active_vertex)) * (P.nz if P.kind == "3d" else 1)


def mixed_bytes(P, niters, ncheck=NCHECK, half=False):
    """Algorithmic HBM bytes of one mixed solve: FP32 iterations x (4*NC*4 + 112 + 24 SIA / +8 diag) and
    FP64 checks x (4*NC*8 + 40) per active node, NC the couplings stored per node (27 in 3D, 14 for
    the symmetric half of an exactly symmetric 3D matrix, 9 in 2D)."""
    nc = (14 if half else 27) if P.kind == "3d" else 9
    pre = 24 if P.kind == "3d" else 8
    checks = int(niters) // ncheck + (1 if niters >= 5 else 0)
    return active_nodes(P) * (float(niters) * (4 * nc * 4 + 112 + pre) + checks * (4 * nc * 8 + 40))


def cpu_cost_sample(P, precond, alg="chrongear", short=2, long=7):
    """Seconds of the oracle (reference algorithm and order, FP64) for `short` and `long` iterations
    of one system: their difference gives the cost of an iteration, the rest the set-up."""
    import oracle
    t0 = time.perf_counter()
    oracle.pcg(alg, P, precond, ncheck=NCHECK, tol=0.0, maxiters=short, summode=oracle.SUM_SEQ)
    t1 = time.perf_counter()
    oracle.pcg(alg, P, precond, ncheck=NCHECK, tol=0.0, maxiters=long, summode=oracle.SUM_SEQ)
    t2 = time.perf_counter()
    per_iter = max((t2 - t1) - (t1 - t0), 1e-9) / (long - short)
    setup = max((t1 - t0) - short * per_iter, 0.0)
    return setup, per_iter


def cfg4_cpu_baseline(probs, niters):
    """The oracle on 1 core, a bounded sample: 2 and 7 iterations of every 8th member (by size),
    per-node set-up and iteration costs scaled to every member's full-solve iteration count."""
    import oracle
    oracle.build()
    order = sorted(range(len(probs)), key=lambda i: active_nodes(probs[i]))
    pick = order[::8]
    t0 = time.perf_counter()
    su = it = nn = 0.0
    for i in pick:
        s, p = cpu_cost_sample(probs[i], CFG4_PRECOND)
        n = active_nodes(probs[i])
        su, it, nn = su + s, it + p, nn + n
    dt = time.perf_counter() - t0
    su_pn, it_pn = su / nn, it / nn
    total = sum(active_nodes(P) * (su_pn + k * it_pn) for P, k in zip(probs, niters))
    return {"value": len(probs) / total, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"2 and 7 Chronopoulos-Gear iterations of {len(pick)} of the 64 members ({dt:.1f} s, 1 core, "
                      "reference algorithm and summation order in FP64), per-node set-up and iteration costs "
                      "scaled to each member's full-solve iteration count (oracle/cfg4_niters.json)",
            "solve_s_total": total}


def cfg2_side(stream, flush):
    """The like-for-like plain FP64 comparison on cfg2 (the 401x401 2D SSA system, Chronopoulos-Gear
    + Jacobi): the FP64 GPU PCG (bit-exact with the oracle) against the oracle on 1 core."""
    import torch
    import cism_b200 as cg
    import oracle
    P = make_problem("cfg2")
    S = cg.DeviceSolver(P, stream=stream.cuda_stream)
    try:
        S.solve(cg.ALG_CHRONGEAR, PRECOND, NCHECK, TOL, 5)  # workspace
        ms = []
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                e, n = S.solve(cg.ALG_CHRONGEAR, PRECOND, NCHECK, TOL, MAXITERS)
                b.record(stream)
            stream.synchronize()
            ms.append(a.elapsed_time(b))
    finally:
        S.close()
    oracle.build()
    setup, per_iter = cpu_cost_sample(P, PRECOND, short=20, long=220)
    cpu_s = setup + n * per_iter
    gpu_s = float(np.median(ms)) / 1e3
    return {"workload": WORKLOAD, "fp64_gpu_solves_per_s": 1.0 / gpu_s, "fp64_gpu_ms": 1e3 * gpu_s, "niters": n,
            "err": e, "cpu_1core_solves_per_s": 1.0 / cpu_s,
            "cpu_sample": "20 and 220 iterations of the oracle (reference algorithm and order, FP64, 1 core), "
                          f"scaled to {n} iterations", "gpu_over_cpu": cpu_s / gpu_s}


def run_cfg4(args):
    """64 sliding 3D ice streams, n ~ U{64..256} vertices per side, 11 levels, each with its own seeded
    log-normal friction; SIA preconditioner, tol 1e-8.  A step = one replay of the CUDA graph that runs
    all 64 solves from x0 = 0 in one persistent launch of the mixed-precision kernel."""
    import tempfile
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    # the tile tuner times this workload's own systems (a table left by earlier processes on the
    # machine, e.g. small test batches, would otherwise decide the batch tile floor)
    tile_cache = os.path.join(tempfile.mkdtemp(prefix="cismgpu-bench-"), "tiles.txt")
    os.environ["CISMGPU_TILE_CACHE"] = tile_cache
    t0 = time.perf_counter()
    probs = cfg4_problems(max(1, (os.cpu_count() or 1) // world))
    t_gen = time.perf_counter() - t0
    import cism_b200 as cg
    from cism_b200 import build
    build.build()
    cg.load_library()
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    solvers = [cg.DeviceSolver(P, stream=stream.cuda_stream) for P in probs]
    pc, maxit, n = CFG4_PRECOND, CFG4_MAXIT, len(probs)
    nodes = sum(active_nodes(P) for P in probs)

    def timed_each(alg):
        """Each member alone, one after another (device time by CUDA events on the solve stream)."""
        ms, out = 0.0, []
        for S in solvers:
            S.solve(alg, pc, NCHECK, TOL, 5)  # workspace and FP32 copies of this algorithm
        for S in solvers:
            with torch.cuda.stream(stream):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                e, k = S.solve(alg, pc, NCHECK, TOL, maxit)
                b.record(stream)
            stream.synchronize()
            ms += a.elapsed_time(b)
            out.append((e, k, S.x()))
        return ms, out

    # plain FP64 GPU PCG (reference algorithm, bit-exact with the oracle), one system after another
    fp64_ms, fp64 = timed_each(cg.ALG_CHRONGEAR)
    n64 = [k for _, k, _ in fp64]
    # the mixed solver one system at a time
    one_ms, _ = timed_each(cg.ALG_MIXED_CHRONGEAR)

    # the product path: one graph-captured persistent launch over all 64 members
    B = cg.GraphBatch(solvers, precond=pc, ncheck=NCHECK, tol=TOL, maxiters=maxit, stream=stream.cuda_stream)
    for _ in range(max(args.warmup, 3)):
        B.run()
        B.wait()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    errs = nits = None
    for k in range(args.steps):
        evs[k][0].record(stream)
        B.run()
        evs[k][1].record(stream)
        errs, nits, sts = B.wait()
        assert not np.any(sts), sts
    t_end.record(stream)
    stream.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(t_start.elapsed_time(t_end), pg, "cuda")
    step_ms = [a.elapsed_time(b) for a, b in evs]
    xb = [S.x() for S in solvers]
    half = [S.mixed_symmetric_half() for S in solvers]
    B.close()
    rel = max(math.sqrt(float(np.sum((a[0] - b[2][0]) ** 2) + np.sum((a[1] - b[2][1]) ** 2))) /
              math.sqrt(float(np.sum(b[2][0] ** 2) + np.sum(b[2][1] ** 2))) for a, b in zip(xb, fp64))
    value = whole_job_rate(world, args.steps * n, total_ms)
    by = sum(mixed_bytes(P, it, half=h) for P, it, h in zip(probs, nits, half))
    peak, peak_kind = hbm_peak()
    achieved = by / (float(np.mean(step_ms)) / 1e3) / 1e9

    # the same members with the tridiagonal line preconditioner (precond 3, local form): the mixed
    # batch (one graph replay after a warm-up) against the plain FP64 solver one system at a time
    lines = None
    if world == 1:
        BL = cg.GraphBatch(solvers, precond=3, ncheck=NCHECK, tol=TOL, maxiters=maxit, stream=stream.cuda_stream)
        BL.run()
        BL.wait()
        with torch.cuda.stream(stream):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            BL.run()
            b.record(stream)
        el, nl, sl = BL.wait()
        assert not np.any(sl), sl
        line_ms = a.elapsed_time(b)
        BL.close()
        l64_ms, l64_it = 0.0, 0
        for S in solvers:
            S.solve(cg.ALG_CHRONGEAR, 3, NCHECK, TOL, 5)  # line factors and workspace
            with torch.cuda.stream(stream):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                e, k = S.solve(cg.ALG_CHRONGEAR, 3, NCHECK, TOL, maxit)
                b.record(stream)
            stream.synchronize()
            l64_ms += a.elapsed_time(b)
            l64_it += k
        lines = {"precond": "3 (tridiagonal line, local form)", "solves_per_s": n / (line_ms / 1e3),
                 "ms_per_replay": line_ms, "niters_sum": int(np.sum(nl)), "err_max": float(np.max(el)),
                 "fp64_plain_solves_per_s": n / (l64_ms / 1e3), "fp64_plain_niters_sum": int(l64_it),
                 "speedup_vs_fp64_plain": l64_ms / line_ms,
                 "note": "same 64 members; mixed: one graph replay of the batch (CUDA events); FP64: the reference "
                         "algorithm one system at a time (CUDA events)"}

    # end to end through the batch API with host buffers: per step every member's A and b are
    # uploaded from pinned host memory (cismgpu_solver_set_system), all 64 are solved in one
    # persistent launch (cismgpu_solver_solve_batch) and every x comes back to host memory
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    host = [tuple(pin(a) for a in (P.Auu, P.Auv, P.Avu, P.Avv, P.bu, P.bv)) for P in probs]
    xout = [(pin(np.zeros_like(P.bu)), pin(np.zeros_like(P.bv))) for P in probs]
    e2e_ms = []
    for k in range(3):
        torch.cuda.synchronize()
        ta = time.perf_counter()
        for S, h in zip(solvers, host):
            S.set_system(*h, x0_from_solution=False)
        ee, kk, ss = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, pc, NCHECK, TOL, maxit,
                                    stream=stream.cuda_stream)
        assert not np.any(ss), ss
        for S, (xu, xv) in zip(solvers, xout):
            S.x_into(xu, xv)
        tb = time.perf_counter()
        if k > 0:  # the first round re-creates the FP32 copies' workspace
            e2e_ms.append(1e3 * (tb - ta))
    h2d = sum(sum(a.nbytes for a in h) for h in host)
    d2h = sum(xu.nbytes + xv.nbytes for xu, xv in xout)
    e2e_rate = world * n * 1e3 / float(np.mean(e2e_ms))
    for S in solvers:
        S.close()

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return 0
    counts = cfg4_reference_niters() or n64
    cpu = cfg4_cpu_baseline(probs, counts) if world == 1 else None
    side = cfg2_side(stream, flush) if world == 1 else None
    fp64_rate = n / (fp64_ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 recurrences + f64 x/dots/residual", "data": "synthetic",
        "config": {"workload": CFG4_WORKLOAD, "solver": "one CUDA-graph-captured persistent launch (k_mixed_dyn)",
                   "l2": "inputs larger than L2 (FP32 matrices ~10 GB, FP64 ~20 GB)", "nodes": nodes,
                   "parallelism": f"replicas x{world}", "generation_s": round(t_gen, 1)},
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
        "niters": {"min": int(np.min(nits)), "max": int(np.max(nits)), "sum": int(np.sum(nits)),
                   "fp64_sum": int(sum(n64))},
        "err_max": float(np.max(errs)), "err_vs_fp64_solution_max": rel,
        "fp64_plain": {"solves_per_s": fp64_rate, "ms_for_all": fp64_ms,
                       "solver": "reference Chronopoulos-Gear statement by statement, FP64, one system at a time"},
        "speedup_vs_fp64_plain": value / world / fp64_rate,
        "mixed_one_at_a_time": {"solves_per_s": n / (one_ms / 1e3), "ms_for_all": one_ms},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": cfg4_traffic(by), "peak_kind": peak_kind,
                     "kernel": "k_mixed_dyn<27,16> (the whole batch in one launch; the graph's other kernels are "
                               "64 halo resets and one result copy)",
                     "note": "achieved = algorithmic bytes of the replay (per active node: FP32 iterations x "
                             "(16 B x stored couplings + 136 B) + FP64 checks x (32 B x stored couplings + 40 B); "
                             f"{sum(half)} of {n} members stored as the symmetric half, 14 of 27 couplings) / mean "
                             "replay time by CUDA events; traffic = ncu DRAM bytes of the 4-member batch "
                             "(profiles/k_mixed_dyn_cfg4_batch4.md) scaled by algorithmic bytes"},
        "algorithmic_bytes_per_step": by,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_rate, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": float(np.mean(e2e_ms)),
                "path": "cismgpu_solver_set_system x64 (pinned host A, b) + cismgpu_solver_solve_batch + "
                        "cismgpu_solver_get_x x64, host wall clock"},
        "cfg2_fp64_gpu_vs_cpu": side,
        "line_preconditioner": lines,
        "tile_heights": [ln for ln in cg.tile_table() if ln.startswith("batch:")],
        "gpu_launches": (n + 2) * args.steps, "clocks": clk,
    }
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# served workload: a Poisson stream of 2D SSA and 3D BP requests
# ---------------------------------------------------------------------------
def _make_served(args):
    from cism_b200 import assembly as asm
    kind, n, nz, seed = args
    if kind == "2d":
        return asm.ssa_random(ewn=n, nsn=n, dx=1000.0, seed=seed, name=f"ssa{n}")
    return asm.ice_stream(ewn=n, nsn=n, nz=nz, dx=2000.0, seed=seed, name=f"bp{n}x{nz}")


def _fifo(arrivals, service):
    """Completion latencies of one FIFO server with the given service times."""
    t, lat = 0.0, []
    for a, s in zip(arrivals, service):
        t = max(t, a) + s
        lat.append(t - a)
    return lat


def run_serve(args):
    """A seeded Poisson stream (mean 200 req/s) of 2D SSA (96^2..1025^2 vertices, diagonal
    precond) and 3D BP ice streams (48^2..384^2 vertices x 5..21 levels, no-slip bed, SIA
    precond), served by the continuous-batching loop under a 150 GB HBM budget; latency is
    submit to x back in host memory.  Requests draw from a seeded pool of distinct systems
    (every request gets its own device copy).  Beside it: the same stream through a FIFO
    queue of one-shot reference-signature calls, plain FP64 and mixed, with service times
    measured per pool system."""
    import multiprocessing as mp
    rng = np.random.default_rng(2024)
    pool_spec = [("2d", int(rng.integers(96, 1026)), 1, 100 + k) for k in range(args.pool)]
    pool_spec += [("3d", int(rng.integers(48, 385)), int(rng.integers(5, 22)), 200 + k) for k in range(args.pool)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(min(len(pool_spec), os.cpu_count() or 1)) as pool:
        probs = pool.map(_make_served, pool_spec)
    t_gen = time.perf_counter() - t0
    import cism_b200 as cg
    from cism_b200 import build
    from cism_b200 import assembly as asm
    build.build()
    pcs = [1 if P.kind == "2d" else 2 for P in probs]
    nreq = args.requests
    arrivals = np.cumsum(rng.exponential(1.0 / 200.0, nreq))
    arrivals -= arrivals[0]
    which = rng.integers(0, len(probs), nreq)
    maxit = 20000

    def oneshot(P, pc, alg):
        prev = cg.set_oneshot_algorithm(alg)
        try:
            xu, xv = np.zeros_like(P.bu), np.zeros_like(P.bv)
            t = time.perf_counter()
            if P.kind == "3d":
                cg.pcg_solver_chrongear_3d(P.nx, P.ny, P.nz, P.par, asm.indxA_2d(), asm.indxA_3d(), P.active_vertex,
                                           P.Auu, P.Auv, P.Avu, P.Avv, P.bu, P.bv, xu, xv, pc, NCHECK, TOL, maxit)
            else:
                cg.pcg_solver_chrongear_2d(P.nx, P.ny, P.par, asm.indxA_2d(), P.active_vertex, P.Auu, P.Auv, P.Avu,
                                           P.Avv, P.bu, P.bv, xu, xv, pc, NCHECK, TOL, maxit)
            return time.perf_counter() - t, (xu, xv)
        finally:
            cg.set_oneshot_algorithm(prev)

    svc64, svcmx, x64 = [], [], []
    for P, pc in zip(probs, pcs):
        oneshot(P, pc, cg.ALG_CHRONGEAR)  # warm the workspace
        dt, x = oneshot(P, pc, cg.ALG_CHRONGEAR)
        svc64.append(dt)
        x64.append(x)
        oneshot(P, pc, cg.ALG_MIXED_CHRONGEAR)
        svcmx.append(oneshot(P, pc, cg.ALG_MIXED_CHRONGEAR)[0])
    S = cg.Server(hbm_budget_bytes=150 * 10**9, epoch_steps=args.epoch_steps)
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    ids = []
    start = time.perf_counter()
    for k in range(nreq):
        dt = arrivals[k] - (time.perf_counter() - start)
        if dt > 0:
            time.sleep(dt)
        ids.append(S.submit(probs[which[k]], precond=pcs[which[k]], tol=TOL, maxiters=maxit))
    S.drain()
    wall = time.perf_counter() - start
    clk = clocks.stop()
    infos = [S.poll(i) for i in ids]
    bad = [i["status"] for i in infos if i["status"] != 0]
    if bad:
        raise RuntimeError(f"served requests failed: {bad[:8]}")
    lat = np.array([i["latency_ms"] for i in infos])
    errs = np.array([i["err"] for i in infos])
    rel = 0.0
    for k, rid in enumerate(ids):
        xu, xv, _ = S.result(rid)
        au, av = x64[which[k]]
        rel = max(rel, math.sqrt(float(np.sum((xu - au) ** 2) + np.sum((xv - av) ** 2))) /
                  math.sqrt(float(np.sum(au ** 2) + np.sum(av ** 2))))
    st = S.stats()
    S.close()
    lat64 = 1e3 * np.array(_fifo(arrivals, [svc64[w] for w in which]))
    latmx = 1e3 * np.array(_fifo(arrivals, [svcmx[w] for w in which]))
    value = nreq / wall
    fp64_rate = nreq / max(float(np.max(arrivals + lat64 / 1e3)), 1e-9)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": nreq, "warmup": 0,
        "ms_per_step": 1e3 * wall / nreq, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 recurrences + f64 x/dots/residual", "data": "synthetic",
        "config": {"workload": f"cfg5: {nreq} requests, Poisson mean 200 req/s, 2D SSA 96^2..1025^2 (diag) and 3D BP "
                               f"48^2..384^2 x 5..21 levels (SIA), pool of {len(probs)} seeded systems, "
                               "HBM budget 150 GB, tol 1e-8",
                   "solver": f"continuous-batching serving loop, epochs of {args.epoch_steps} steps",
                   "generation_s": round(t_gen, 1)},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "mean": float(np.mean(lat))},
        "err_max": float(np.max(errs)), "err_vs_fp64_solution_max": rel,
        "fp64_plain_fifo": {"solves_per_s": fp64_rate,
                            "latency_ms": {"p50": float(np.percentile(lat64, 50)), "p99": float(np.percentile(lat64, 99))},
                            "solver": "one-shot cismgpu_pcg_chrongear_* calls (FP64 reference statements), FIFO"},
        "mixed_one_at_a_time_fifo": {"solves_per_s": nreq / max(float(np.max(arrivals + latmx / 1e3)), 1e-9),
                                     "latency_ms": {"p50": float(np.percentile(latmx, 50)),
                                                    "p99": float(np.percentile(latmx, 99))}},
        "speedup_vs_fp64_plain": value / fp64_rate,
        "pool_service_ms": [{"system": P.name, "kind": P.kind, "nz": int(P.nz) if P.kind == "3d" else 1,
                             "precond": pc, "fp64_ms": round(1e3 * a, 2), "mixed_ms": round(1e3 * b, 2),
                             "requests": int(np.count_nonzero(which == w))}
                            for w, (P, pc, a, b) in enumerate(zip(probs, pcs, svc64, svcmx))],
        "server": {"epochs": st["epochs"]},
        "clocks": clk,
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# on-device assembly of a Picard iteration's 3D system (the step the upload replaces)
# ---------------------------------------------------------------------------
def run_asm3d(args):
    """cismgpu_solver_assemble_system_3d on the cfg3 grid (201x201 vertices x 11 levels, the ice
    stream): stiffness with the nonlinear (Glen) viscosity from a velocity field, local basal
    friction, the gravitational load as b, no-slip Dirichlet rows at the bed, staggered halo.
    Device time by CUDA events on the handle's stream, against the upload of the same assembled
    system from pinned host memory (cismgpu_solver_set_system), the host-to-device traffic the
    on-device assembly removes.  A step is one assembly."""
    import math as _m
    import torch
    import cism_b200 as cg
    from cism_b200 import assembly as asm
    from cism_b200 import build
    build.build()
    torch.cuda.set_device(0)
    ewn, nz, dx = 201, 11, 2000.0
    P = asm.ice_stream(ewn=ewn, nsn=ewn, nz=nz, dx=dx)
    nx, ny = P.nx, P.ny
    rng = np.random.default_rng(3)
    x = (np.arange(nx) + 0.5) * dx
    usrf0 = 3000.0 - x * _m.tan(_m.radians(0.5))
    topg = usrf0[None, :] - 1500.0 + 0.05 * 1500.0 * asm.smooth_field((ny, nx), 4.0, rng)
    usrf = np.broadcast_to(usrf0[None, :], (ny, nx)).copy()
    thck = np.where(asm._ice_interior(ny, nx), usrf - topg, 0.0)
    usrf = np.where(thck > 0, usrf, topg)
    ac, av = asm.active_masks(thck)
    sigma = asm.glide_sigma(nz)
    xV = np.broadcast_to(np.arange(nx - 1) * dx, (ny - 1, nx - 1)).copy()
    yV = np.broadcast_to((np.arange(ny - 1) * dx)[:, None], (ny - 1, nx - 1)).copy()
    stagusrf, stagthck = asm.stagger(usrf, thck > 1.0), asm.stagger(thck, thck > 1.0)
    ff = np.full((ny, nx, nz - 1), 0.5 * 1.0e-16 ** (-1.0 / 3.0))
    beta = asm.lognormal_beta((ny - 1, nx - 1), 7)
    lsrf = usrf - thck
    u0 = 30.0 * rng.standard_normal((ny - 1, nx - 1, nz))
    v0 = 30.0 * rng.standard_normal((ny - 1, nx - 1, nz))
    stream = torch.cuda.Stream()
    S = cg.DeviceSolver(P, x0=(u0, v0), stream=stream.cuda_stream)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    # the call's inputs in pinned host memory, as the upload it is compared with
    geo = tuple(pin(a) for a in (sigma, ac.astype(np.int32), av.astype(np.int32), xV, yV, stagusrf, stagthck, ff))
    load = (pin(P.bu), pin(P.bv))
    beta, lsrf = pin(beta), pin(lsrf)

    def assemble():
        return S.assemble_system(2, dx, dx, *geo, load[0], load[1], beta=beta, lsrf=lsrf)

    host = [pin(a) for a in (P.Auu, P.Auv, P.Avu, P.Avv, P.bu, P.bv)]
    for _ in range(max(args.warmup, 3)):
        assemble()
        S.set_system(*host, x0_from_solution=False)
    a_ms, u_ms, w_ms = [], [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            t0 = time.perf_counter()
            e[0].record(stream)
            assemble()
            e[1].record(stream)
            t1 = time.perf_counter()
            e[2].record(stream)
            S.set_system(*host, x0_from_solution=False)
            e[3].record(stream)
        stream.synchronize()
        a_ms.append(e[0].elapsed_time(e[1]))
        u_ms.append(e[2].elapsed_time(e[3]))
        w_ms.append(1e3 * (t1 - t0))
    S.close()
    nodes = int(np.count_nonzero(av)) * nz
    up_bytes = sum(a.nbytes for a in host)
    am = float(np.median(a_ms))
    line = {
        "metric": "on-device assembly of one Picard iteration's 3D system", "value": 1e3 / am, "unit": "systems/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": am, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cfg3 grid: {ewn}x{ewn} vertices x {nz} levels ice stream, nonlinear Glen viscosity "
                               "from a velocity field, local basal friction, gravitational load, staggered halo",
                   "active_nodes": nodes},
        "assemble_ms": {"device_median": am, "wall_median": float(np.median(w_ms)),
                        "note": "CUDA events on the handle's stream around cismgpu_solver_assemble_system_3d "
                                "(inputs' host-to-device copies from pinned memory, the kernels, the efvs "
                                "download, the call's host steps)"},
        "upload_ms": {"device_median": float(np.median(u_ms)), "bytes": int(up_bytes),
                      "GB_per_s": up_bytes / (float(np.median(u_ms)) / 1e3) / 1e9,
                      "note": "the same system assembled on the host and uploaded from pinned memory "
                              "(cismgpu_solver_set_system)"},
        "speedup_vs_upload": float(np.median(u_ms)) / am,
    }
    print(json.dumps(line))
    return 0


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def cfg4_traffic(algorithmic_bytes):
    """DRAM bytes of one cfg4 replay: the dram__bytes_read.sum + write.sum of an ncu capture of the
    first 4 members' batch (profiles/traffic.json; the full 64-member launch runs ~6 s, too long to
    capture), scaled by the ratio of the replay's algorithmic bytes to the capture's."""
    rec = ncu_traffic("k_mixed_dyn<27,16>:cfg4-batch4")
    if not isinstance(rec, dict) or not rec.get("algorithmic_bytes"):
        return None
    return rec["dram_bytes"] / rec["algorithmic_bytes"] * algorithmic_bytes


def ncu_traffic(kernel_key):
    """Per-launch DRAM bytes (dram__bytes_read.sum + write.sum of one ncu capture) of a kernel,
    as recorded in profiles/traffic.json beside the capture summaries, or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(total_ms, pg, device="cuda"):
    """The slowest rank's timed region (every rank passes its own, every rank gets the max).
    pg is torch.distributed (an initialised default group) or None for one process."""
    if not pg:
        return float(total_ms)
    import torch
    t = torch.tensor([float(total_ms)], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, total_ms):
    """Solves per second of the whole job: every rank (one replica per GPU) solved `steps`
    systems within the slowest rank's total_ms."""
    return world * steps / (total_ms / 1e3)


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement on all host cores
# ---------------------------------------------------------------------------
def _ref_cfg4_worker(args):
    """One host core's share of the cfg4 members: generate them, then `rounds` samples of each
    (2 and 7 iterations of the oracle: set-up and per-iteration seconds)."""
    jobs, rounds = args
    import oracle
    from cism_b200 import assembly as asm
    probs = [(i, asm.batch_member(nn, i)) for i, nn in jobs]
    out = []
    for _ in range(rounds):
        out.append({i: cpu_cost_sample(P, CFG4_PRECOND) for i, P in probs})
    return out


def run_reference(args):
    """The reference's algorithm on the host cores for the same workload: the C++ restatement of
    pcg_solver_chrongear_3d (oracle/, FP64, the reference's summation order), one member per core
    at a time over all cores.  A step is a bounded sample (2 and 7 iterations of every member, all
    cores busy), scaled to each member's full-solve iteration count; the whole-workload time is the
    members' summed solve time divided by the cores (64 members on far fewer cores pack evenly)."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    if args.workload == "cfg2":
        return run_reference_cfg2(args)
    import multiprocessing as mp
    import oracle
    from cism_b200 import assembly as asm
    oracle.build()
    counts = cfg4_reference_niters()
    if counts is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/cfg4_niters.json (full-solve iteration counts) "
                                                               "missing: run oracle/cfg4_niters.py"}))
        return 0
    cores = os.cpu_count() or 1
    sizes = asm.batch_sizes(64)
    order = sorted(range(len(sizes)), key=lambda i: -sizes[i])
    shares = [[] for _ in range(cores)]
    for r, i in enumerate(order):  # snake order: similar work per core
        c = r % (2 * cores)
        shares[c if c < cores else 2 * cores - 1 - c].append((i, sizes[i]))
    rounds = max(args.warmup, 0) + args.steps
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ref_cfg4_worker, [(sh, rounds) for sh in shares if sh])
    wall = time.perf_counter() - t0
    rates, step_s = [], []
    for r in range(max(args.warmup, 0), rounds):
        total = 0.0
        for wres in res:
            for i, (su, it) in wres[r].items():
                total += su + counts[i] * it
        step_s.append(total / cores)
        rates.append(len(sizes) / (total / cores))
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * float(np.median(step_s)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": CFG4_WORKLOAD,
                   "solver": f"C++ restatement of the reference PCG (oracle/), {cores} cores: FP64, reference "
                             "summation order, one member per core at a time"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"per step: 2 and 7 Chronopoulos-Gear iterations of each of the 64 members on "
                                   f"{cores} cores at once, set-up and per-iteration seconds scaled to each member's "
                                   f"full-solve count (oracle/cfg4_niters.json, {sum(counts)} iterations in all); "
                                   f"whole run {wall:.0f} s incl. generation"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


_WORKER_PROBLEM = None


def _ref_worker(niters):
    global _WORKER_PROBLEM
    import oracle
    if _WORKER_PROBLEM is None:
        _WORKER_PROBLEM = make_problem()
    P = _WORKER_PROBLEM
    t0 = time.perf_counter()
    oracle.pcg("chrongear", P, PRECOND, ncheck=NCHECK, tol=0.0, maxiters=niters, summode=oracle.SUM_SEQ)
    return time.perf_counter() - t0


def run_reference_cfg2(args):
    """cfg2 (--workload cfg2): the C++ restatement on all host cores, one independent solve per core."""
    import multiprocessing as mp
    import oracle
    oracle.build()
    world = dist_setup(args)[0]
    cores = os.cpu_count() or 1
    P = make_problem()
    st, xu, xv, err, nfull = oracle.pcg("chrongear", P, PRECOND, ncheck=NCHECK, tol=TOL, maxiters=MAXITERS,
                                        summode=oracle.SUM_SEQ)
    sample_iters = 100
    with mp.get_context("spawn").Pool(cores) as pool:
        for _ in range(max(args.warmup, 0)):
            pool.map(_ref_worker, [10] * cores)
        rates = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            times = pool.map(_ref_worker, [sample_iters] * cores)
            per_iter = max(times) / sample_iters
            rates.append(cores / (per_iter * nfull))
        wall = time.perf_counter() - t0
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "solver": f"C++ restatement of the reference PCG (oracle/), {cores} cores, FP64, reference order"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{sample_iters} Chronopoulos-Gear iterations per core per step, scaled to the "
                                   f"{nfull} iterations of a full solve to 1e-8 (err {err:.2e})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def cpu_baseline_sample(P, niters_full):
    """The oracle (reference order, FP64) on one core, a bounded sample scaled to a full solve."""
    import oracle
    oracle.build()
    sample = 600
    t0 = time.perf_counter()
    oracle.pcg("chrongear", P, PRECOND, ncheck=NCHECK, tol=0.0, maxiters=sample, summode=oracle.SUM_SEQ)
    dt = time.perf_counter() - t0
    per_iter = dt / sample
    return {"value": 1.0 / (per_iter * niters_full), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{sample} Chronopoulos-Gear iterations ({dt:.1f} s) on 1 core, scaled to the {niters_full} "
                      f"iterations the FP64 reference algorithm takes to reach 1e-8"}


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    import cism_b200 as cg
    from cism_b200 import build
    build.build()
    cg.load_library()
    P = make_problem()
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    S = cg.DeviceSolver(P, stream=stream.cuda_stream)

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    # --- warm-up of the product path ---
    for w in range(max(args.warmup, 3)):
        with torch.cuda.stream(stream):
            flush.fill_(float(-w))  # also loads torch's fill kernel before the timed region
            S.solve(cg.ALG_MIXED_CHRONGEAR, PRECOND, NCHECK, TOL, MAXITERS)
    stream.synchronize()

    # --- timed region ---
    S.profile(True)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    errs, nits = [], []
    with torch.cuda.stream(stream):
        t_start.record(stream)
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            e, n = S.solve(cg.ALG_MIXED_CHRONGEAR, PRECOND, NCHECK, TOL, MAXITERS)
            evs[k][1].record(stream)
            errs.append(e)
            nits.append(n)
        t_end.record(stream)
    stream.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(total_ms, pg, "cuda")
    prof_ms, prof_n, prof_bytes = S.profile_read()
    S.profile(False)
    xm = S.x()  # the mixed solution, before the FP64 solves below overwrite x
    # --- plain FP64 GPU PCG (reference algorithm, bit-identical to the oracle) ---
    with torch.cuda.stream(stream):
        e64, n64 = S.solve(cg.ALG_CHRONGEAR, PRECOND, NCHECK, TOL, MAXITERS)  # warm
    x64 = S.x()
    fp64_ms = []
    for _ in range(2):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            S.solve(cg.ALG_CHRONGEAR, PRECOND, NCHECK, TOL, MAXITERS)
            ev1.record(stream)
        stream.synchronize()
        fp64_ms.append(ev0.elapsed_time(ev1))
    fp64_solve_ms = float(np.median(fp64_ms))

    num = math.sqrt(float(np.sum((xm[0] - x64[0]) ** 2) + np.sum((xm[1] - x64[1]) ** 2)))
    den = math.sqrt(float(np.sum(x64[0] ** 2) + np.sum(x64[1] ** 2)))
    err_vs_fp64 = num / den

    value = whole_job_rate(world, args.steps, total_ms)
    peak, peak_kind = hbm_peak()
    avg_launch_ms = prof_ms / max(prof_n, 1)
    achieved = prof_bytes / (avg_launch_ms / 1e3) / 1e9 if prof_n else None
    traffic = ncu_traffic("k_mixed<9,1>:cfg2")

    # --- end to end through the reference-signature C-ABI call, pinned host buffers ---
    e2e = None
    if True:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        Auu, Auv, Avu, Avv = pin(P.Auu), pin(P.Auv), pin(P.Avu), pin(P.Avv)
        bu, bv, act = pin(P.bu), pin(P.bv), pin(P.active_vertex)
        xu, xv = pin(np.zeros_like(P.bu)), pin(np.zeros_like(P.bv))
        from cism_b200 import assembly as asm
        i2 = asm.indxA_2d()
        prev = cg.set_oneshot_algorithm(cg.ALG_MIXED_CHRONGEAR)
        e2e_ms = []
        try:
            for k in range(max(2, args.steps // 2) + 1):
                xu[...] = 0.0
                xv[...] = 0.0
                flush.fill_(1.0)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                cg.pcg_solver_chrongear_2d(P.nx, P.ny, P.par, i2, act, Auu, Auv, Avu, Avv, bu, bv, xu, xv, PRECOND,
                                           NCHECK, TOL, MAXITERS)
                dt = time.perf_counter() - t0
                if k > 0:  # the first call allocates the workspace
                    e2e_ms.append(1e3 * dt)
        finally:
            cg.set_oneshot_algorithm(prev)
        h2d = sum(a.nbytes for a in (Auu, Auv, Avu, Avv, bu, bv, xu, xv, act)) + 9 * 4
        d2h = xu.nbytes + xv.nbytes
        e2e = {"value": world * 1e3 / float(np.mean(e2e_ms)), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_solve": float(np.mean(e2e_ms)),
               "path": "cismgpu_pcg_chrongear_2d (reference signature), mixed algorithm, pinned host buffers"}

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return 0
    cpu = cpu_baseline_sample(P, n64) if world == 1 else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 recurrences + f64 x/dots/residual", "data": "synthetic",
        "config": {"workload": WORKLOAD, "solver": "mixed-precision persistent Chronopoulos-Gear (one launch per solve)",
                   "l2": "flushed (256 MiB write) before every solve", "parallelism": f"replicas x{world}",
                   "unknowns": P.n_unknowns},
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
        "niters": int(np.median(nits)), "err": float(max(errs)), "err_vs_fp64_solution": err_vs_fp64,
        "fp64_plain": {"solves_per_s": 1e3 / fp64_solve_ms, "ms_per_solve": fp64_solve_ms, "niters": n64,
                       "err": e64, "solver": "reference Chronopoulos-Gear statement by statement, FP64"},
        "speedup_vs_fp64_plain": value / world / (1e3 / fp64_solve_ms),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": "k_mixed<9,1> (whole solve in one cooperative launch)",
                     "peak_kind": peak_kind,
                     "note": "algorithmic bytes = FP32 iterations x 264 B + FP64 checks x 328 B per active vertex; "
                             "the 2D working set (~40 MB) stays in L2 across iterations"},
        "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": 3 * args.steps, "clocks": clk,
    }
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default: 5 for cfg4, else 10)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="bench", choices=["bench", "profile"])
    ap.add_argument("--workload", default="cfg4", choices=["cfg2", "cfg3", "dome", "cfg4", "cfg5", "asm3d"])
    ap.add_argument("--requests", type=int, default=96, help="cfg5: number of requests")
    ap.add_argument("--pool", type=int, default=8, help="cfg5: distinct systems per kind")
    ap.add_argument("--epoch-steps", type=int, default=64, help="cfg5: steps per serving epoch")
    ap.add_argument("--batch", type=int, default=64, help="cfg4: number of systems")
    ap.add_argument("--fp64", action="store_true", help="profile mode: also time one plain FP64 solve")
    ap.add_argument("--precond", type=int, default=2, help="profile mode, cfg4: preconditioner of the batch")
    ap.add_argument("--layout", default="auto", choices=["auto", "full"],
                    help="profile mode: mixed matrix layout (auto: symmetric half when exactly symmetric)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 5 if args.workload == "cfg4" else 10
    if args.mode == "profile":
        return run_profile(args)
    if args.workload == "cfg4" and args.impl == "ours":
        return run_cfg4(args)
    if args.workload == "cfg5":
        return run_serve(args)
    if args.workload == "asm3d":
        return run_asm3d(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
