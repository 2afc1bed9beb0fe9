"""The continuous-batching serving loop (cismgpu_server_*), called through the C ABI.

Each request's result must be bit-identical whether it is served alone or in a mix
(requests of different kinds and sizes, submitted while others are on the GPU; 2D and 3D
requests in the same multi-class launch), must reach
the FP64 tolerance, and must agree with the FP64 oracle within the accuracy that tolerance
implies.  Admission respects the HBM budget.
"""
import time

import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests import problems

pytestmark = pytest.mark.gpu


def mix():
    return [
        (asm.ssa_random(ewn=61, nsn=57, seed=3), 1),
        (asm.batch_member(24, seed=5, nz=7), 2),
        (problems.slab_3d(seed=5, sliding=False), 1),
        (asm.ssa_random(ewn=90, nsn=70, seed=9), 1),
        (asm.batch_member(31, seed=6, nz=19), 2),   # nz > 16: the second kernel class
        (asm.dome(), 2),
    ]


def serve_alone(P, pc):
    S = cg.Server(hbm_budget_bytes=4 * 10**9, epoch_steps=16)
    try:
        rid = S.submit(P, precond=pc, tol=1e-8, maxiters=5000)
        S.drain()
        xu, xv, info = S.result(rid)
        return xu.copy(), xv.copy(), info
    finally:
        S.close()


def test_served_alone_equals_mix(gpu_lib):
    cases = mix()
    alone = [serve_alone(P, pc) for P, pc in cases]
    S = cg.Server(hbm_budget_bytes=4 * 10**9, epoch_steps=16)
    try:
        ids = [S.submit(P, precond=pc, tol=1e-8, maxiters=5000) for P, pc in cases[:3]]
        time.sleep(0.02)  # the rest arrive while the first ones are on the GPU
        ids += [S.submit(P, precond=pc, tol=1e-8, maxiters=5000) for P, pc in cases[3:]]
        S.drain()
        assert S.stats()["epochs"] > 1
        launches, multi = S.launch_stats()
        assert multi >= 1 and launches >= S.stats()["epochs"]  # 2D and 3D requests in one launch
        for (P, pc), rid, (au, av, ainfo) in zip(cases, ids, alone):
            xu, xv, info = S.result(rid)
            assert info["status"] == 0 and ainfo["status"] == 0
            assert info["err"] < 1e-8
            assert info["err"] == ainfo["err"] and info["niters"] == ainfo["niters"]
            np.testing.assert_array_equal(xu, au)
            np.testing.assert_array_equal(xv, av)
            assert info["latency_ms"] >= info["queue_ms"] >= 0.0
    finally:
        S.close()
    P, pc = cases[0]
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, pc, tol=1e-8, maxiters=5000)
    from tests.test_gpu_mixed import rel
    assert rel(alone[0][:2], (ou, ov), P) < 1e-5


def test_server_budget(gpu_lib):
    """A budget that holds one request at a time still serves them all, one after another; a
    request larger than the budget fails with CISMGPU_ENOMEM without stopping the others."""
    P = asm.ssa_random(ewn=61, nsn=57, seed=3)
    big = asm.ssa_random(ewn=150, nsn=140, seed=4)
    S = cg.Server(hbm_budget_bytes=14 * 10**6, epoch_steps=32)  # one small request (~12.3 MB) at a time
    try:
        ids = [S.submit(P, precond=1, tol=1e-8, maxiters=5000) for _ in range(3)]
        bid = S.submit(big, precond=1, tol=1e-8, maxiters=5000)
        S.drain()
        infos = [S.poll(i) for i in ids]
        assert all(i["status"] == 0 and i["err"] < 1e-8 for i in infos)
        assert S.poll(bid)["status"] == 7
        assert S.stats()["bytes_in_use"] == 0
        # one at a time: each waited for the previous one
        q = sorted(i["queue_ms"] for i in infos)
        assert q[2] > q[0]
    finally:
        S.close()


def test_large_2d_request_alone_equals_mix(gpu_lib):
    """A 2D request large enough for the single-solve kernel's own launches (>= 65536 owned
    vertices) gives the same bits served alone and served beside 3D and small 2D requests."""
    big = (asm.ssa_random(ewn=300, nsn=240, seed=21), 1)
    others = [(asm.batch_member(30, seed=8, nz=7), 2), (asm.ssa_random(ewn=50, nsn=44, seed=22), 1)]
    au, av, ainfo = serve_alone(*big)
    S = cg.Server(hbm_budget_bytes=4 * 10**9, epoch_steps=16)
    try:
        ids = [S.submit(P, precond=pc, tol=1e-8, maxiters=5000) for P, pc in [big] + others]
        S.drain()
        xu, xv, info = S.result(ids[0])
        assert info["status"] == 0 and ainfo["status"] == 0 and info["err"] < 1e-8
        assert info["err"] == ainfo["err"] and info["niters"] == ainfo["niters"]
        np.testing.assert_array_equal(xu, au)
        np.testing.assert_array_equal(xv, av)
        assert all(S.poll(i)["status"] == 0 for i in ids)
    finally:
        S.close()
