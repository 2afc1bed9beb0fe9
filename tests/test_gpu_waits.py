"""The bounded device waits of the mixed-precision kernels, exercised without any fault.

Every spin-wait in those kernels (a CTA waiting for another CTA's step record, or for a
solve's broadcast scalars) gives up after a bounded number of SM cycles, sets the launch's
abort word and leaves; the host then reports CISMGPU_ETIMEOUT.  The test hook
cismgpu_test_set_device_waits shortens the bound and makes tile 0 of every solve withhold
its record of one step -- a flag that nothing else sets -- so the waits for it run out.
Each test then checks that the same handle, batch or server solves correctly afterwards,
bit for bit as before.
"""
import numpy as np
import pytest

import cism_b200 as cg
from cism_b200 import assembly as asm
from tests import problems

pytestmark = pytest.mark.gpu

ETIMEOUT = 6
SHORT = 2_000_000  # SM cycles, about 1 ms


@pytest.fixture
def waits(gpu_lib):
    cg.debug_set_device_waits(0, 0)
    yield cg.debug_set_device_waits
    cg.debug_set_device_waits(0, 0)


def same(a, b):
    return a[0] == b[0] and np.array_equal(a[1][0], b[1][0]) and np.array_equal(a[1][1], b[1][1])


def test_single_solve_times_out_and_recovers(waits):
    P = asm.dome()
    S = cg.DeviceSolver(P)
    try:
        ref = S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 200), S.x()
        assert ref[0][0] < 1e-8
        waits(SHORT, 3)
        with pytest.raises(cg.CismGpuError) as e:
            S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 200)
        assert e.value.status == ETIMEOUT
        waits(0, 0)
        again = S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 200), S.x()
        assert same(again, ref)
    finally:
        S.close()


def test_batch_times_out_and_recovers(waits):
    probs = [asm.dome(), problems.slab_3d(seed=5, sliding=False)]
    solvers = [cg.DeviceSolver(P) for P in probs]
    try:
        e0, n0, s0 = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 400)
        assert not np.any(s0)
        x0 = [S.x() for S in solvers]
        waits(SHORT, 4)
        e1, n1, s1 = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 400)
        assert list(s1) == [ETIMEOUT, ETIMEOUT]
        waits(0, 0)
        e2, n2, s2 = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 400)
        assert not np.any(s2) and np.array_equal(e2, e0) and np.array_equal(n2, n0)
        for S, x in zip(solvers, x0):
            xu, xv = S.x()
            assert np.array_equal(xu, x[0]) and np.array_equal(xv, x[1])
        # the graph-captured form reads the same bound at each replay
        B = cg.GraphBatch(solvers, precond=2, ncheck=5, tol=1e-8, maxiters=400)
        try:
            waits(SHORT, 4)
            B.run()
            assert list(B.wait()[2]) == [ETIMEOUT, ETIMEOUT]
            waits(0, 0)
            B.run()
            e3, n3, s3 = B.wait()
            assert not np.any(s3) and np.array_equal(e3, e0) and np.array_equal(n3, n0)
        finally:
            B.close()
    finally:
        for S in solvers:
            S.close()


def test_server_retires_timed_out_request_and_serves_the_next(waits):
    P = asm.dome()
    srv = cg.Server(hbm_budget_bytes=2 * 10**9, epoch_steps=64)
    try:
        ok = srv.submit(P, precond=2, tol=1e-8, maxiters=200)
        srv.drain()
        ref_u, ref_v, info = srv.result(ok)
        assert info["status"] == 0
        waits(SHORT, 3)
        bad = srv.submit(P, precond=2, tol=1e-8, maxiters=200)
        srv.drain()
        assert srv.poll(bad)["status"] == ETIMEOUT
        waits(0, 0)
        good = srv.submit(P, precond=2, tol=1e-8, maxiters=200)
        srv.drain()
        xu, xv, info = srv.result(good)
        assert info["status"] == 0
        assert np.array_equal(xu, ref_u) and np.array_equal(xv, ref_v)
    finally:
        srv.close()
