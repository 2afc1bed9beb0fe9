"""FP64 solves with parallel%reprosum, through the C ABI, against the oracle's restatement of
the reference's reprosum path (oracle.SUM_REPRO): every global sum of the standard and
Chronopoulos-Gear solvers is cism_reprosum_calc's sum (libglimmer/parallel_mpi.F90:6703-6738),
so x (halo entries included), err, niters and status must be bit-identical.
"""
import copy
import math

import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests import problems
from tests.test_gpu_parity import assert_bitexact, gpu_solve

pytestmark = pytest.mark.gpu


def with_reprosum(P):
    Q = copy.copy(P)
    Q.par = dict(P.par, reprosum=1)
    return Q


@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
def test_3d_reprosum_bitexact(gpu_lib, alg, precond):
    P = with_reprosum(problems.slab_3d(seed=5, sliding=False))
    x0 = problems.random_x0(P, seed=7, scale=10.0)
    o = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=300, summode=oracle.SUM_REPRO, x0=x0)
    g = gpu_solve(alg, P, precond, tol=1e-8, maxiters=300, x0=x0)
    assert o[0] == 0 and o[3] < 1e-8
    assert_bitexact(g, o)


@pytest.mark.parametrize("precond", [2, 3, 4])
def test_3d_reprosum_breakdown(gpu_lib, precond):
    """A first pass whose sums meet NaN: the reproducible sum of non-finite summands is their
    IEEE sum, so alpha = NaN ends the solve with EBREAKDOWN_ALPHA after one iteration."""
    P = with_reprosum(problems.slab_3d(seed=3, boundary_ice=True, bc="outflow"))
    x0 = problems.random_x0(P, seed=7, scale=10.0)
    o = oracle.pcg("chrongear", P, precond, tol=1e-8, maxiters=300, summode=oracle.SUM_REPRO, x0=x0)
    g = gpu_solve("chrongear", P, precond, tol=1e-8, maxiters=300, x0=x0)
    assert o[0] == 2 and o[4] == 1  # CISMGPU_EBREAKDOWN_ALPHA
    assert_bitexact(g, o)


@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 3, 4])
@pytest.mark.parametrize("bc", ["periodic", "no_ice"])
def test_2d_reprosum_bitexact(gpu_lib, alg, precond, bc):
    P = with_reprosum(problems.slab_2d(seed=2, boundary_ice=True, bc=bc))
    x0 = problems.random_x0(P, seed=8, scale=10.0)
    o = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=400, summode=oracle.SUM_REPRO, x0=x0)
    g = gpu_solve(alg, P, precond, tol=1e-8, maxiters=400, x0=x0)
    assert_bitexact(g, o)


def test_dome_reprosum_bitexact(gpu_lib):
    """The 31x31x11 dome with the reference's defaults (Chronopoulos-Gear, SIA preconditioner)."""
    P = with_reprosum(asm.dome())
    o = oracle.pcg("chrongear", P, 2, maxiters=400, summode=oracle.SUM_REPRO)
    g = gpu_solve("chrongear", P, 2, maxiters=400)
    assert g[0] == 0 and g[3] < 1e-8
    assert_bitexact(g, o)


def test_reprosum_fixed_iterations(gpu_lib):
    """tol = 0 runs every iteration to maxiters: the trajectories agree at each stopping point."""
    P = with_reprosum(problems.slab_2d(seed=5))
    for n in (1, 2, 7):
        o = oracle.pcg("chrongear", P, 1, tol=0.0, maxiters=n, summode=oracle.SUM_REPRO)
        g = gpu_solve("chrongear", P, 1, tol=0.0, maxiters=n)
        assert_bitexact(g, o)


def test_reprosum_handle_solve_matches_oneshot(gpu_lib):
    """A device-resident system created with reprosum set solves with the reproducible sums."""
    P = with_reprosum(problems.slab_3d(seed=4))
    o = oracle.pcg("standard", P, 2, tol=1e-8, maxiters=300, summode=oracle.SUM_REPRO)
    s = cg.DeviceSolver(P)
    try:
        err, nit = s.solve(cg.ALG_STANDARD, 2, 5, 1e-8, 300)
        xu, xv = s.x()
    finally:
        s.close()
    assert nit == o[4] and (err == o[3] or (math.isnan(err) and math.isnan(o[3])))
    np.testing.assert_array_equal(xu, o[1])
    np.testing.assert_array_equal(xv, o[2])
