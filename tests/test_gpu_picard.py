"""The steps around the solve in a Picard iteration, called through the C ABI:
compute_residual_vector and compute_residual_velocity (glissade_velo_higher.F90), one-shot
and on a device-resident handle whose A, b and x stay in HBM between iterations.

Bars: bit-exact against the oracle with the device's summation tree (oracle.SUM_DDTREE) for
every array and norm; max-type velocity residuals are exact in any order; against the
reference's sequential order the norms agree within 1e-13 relative.
"""
import math

import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests import problems

pytestmark = pytest.mark.gpu

CASES = [
    ("3d-periodic", lambda: problems.slab_3d(seed=41, boundary_ice=True, bc="periodic")),
    ("3d-noice", lambda: problems.slab_3d(seed=42, boundary_ice=True, bc="no_ice")),
    ("2d-outflow", lambda: problems.slab_2d(seed=43, boundary_ice=True, bc="outflow")),
    ("2d-interior", lambda: problems.slab_2d(seed=44)),
]


def gpu_residual_vector(P, u, v):
    if P.kind == "3d":
        return cg.compute_residual_vector_3d(P.nx, P.ny, P.nz, P.par, asm.indxA_3d(), P.active_vertex, P.Auu,
                                             P.Auv, P.Avu, P.Avv, P.bu, P.bv, u, v)
    return cg.compute_residual_vector_2d(P.nx, P.ny, P.par, asm.indxA_2d(), P.active_vertex, P.Auu, P.Auv,
                                         P.Avu, P.Avv, P.bu, P.bv, u, v)


def gpu_residual_velocity(P, which, u, v, us, vs):
    if P.kind == "3d":
        return cg.compute_residual_velocity_3d(which, P.nx, P.ny, P.nz, P.par, u, v, us, vs)
    return cg.compute_residual_velocity_2d(which, P.nx, P.ny, P.par, u, v, us, vs)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_residual_vector_bitexact(gpu_lib, case):
    P = case[1]()
    rng = np.random.default_rng(7)
    u, v = rng.standard_normal(P.bu.shape) * 50, rng.standard_normal(P.bv.shape) * 50
    g = gpu_residual_vector(P, u, v)
    o = oracle.residual_vector(P, u, v, summode=oracle.SUM_DDTREE)
    np.testing.assert_array_equal(g[0], o[0])
    np.testing.assert_array_equal(g[1], o[1])
    assert g[2] == o[2] and g[3] == o[3]
    s = oracle.residual_vector(P, u, v, summode=oracle.SUM_SEQ)
    assert abs(g[2] - s[2]) <= 1e-13 * s[2] and abs(g[3] - s[3]) <= 1e-13 * s[3]


@pytest.mark.parametrize("which", [0, 1, 2, 4])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_residual_velocity_bitexact(gpu_lib, case, which):
    P = case[1]()
    rng = np.random.default_rng(8)
    u, v = rng.standard_normal(P.bu.shape), rng.standard_normal(P.bv.shape)
    u.reshape(-1)[::7] = 0.0
    v.reshape(-1)[::7] = 0.0  # some zero speeds: skipped
    us, vs = u * (1 + 0.2 * rng.random(u.shape)), v * (1 - 0.2 * rng.random(v.shape))
    g = gpu_residual_velocity(P, which, u, v, us, vs)
    assert g == oracle.residual_velocity(P, which, u, v, us, vs, summode=oracle.SUM_DDTREE)
    seq = oracle.residual_velocity(P, which, u, v, us, vs, summode=oracle.SUM_SEQ)
    assert (g == seq) if which != 2 else abs(g - seq) <= 1e-13 * seq


@pytest.mark.parametrize("kind", ["3d", "2d"])
def test_device_resident_picard_steps(gpu_lib, kind):
    """Two Picard iterations on one handle: after set_system the residual of the last solution
    with the new system, and after the next solve the velocity residual against the guess it
    started from, equal the one-shot calls on the same host arrays bit for bit."""
    P = problems.slab_3d(seed=45) if kind == "3d" else problems.slab_2d(seed=45)
    S = cg.DeviceSolver(P)
    S.solve(cg.ALG_CHRONGEAR, 1, 5, 1e-10, 400)
    x1 = S.x()
    # the next iteration's system: coefficients scaled (still symmetric positive definite)
    A2 = [a * 1.07 for a in (P.Auu, P.Auv, P.Avu, P.Avv)]
    b2u, b2v = P.bu * 0.95, P.bv * 0.95
    S.set_system(*A2, b2u, b2v, x0_from_solution=True)
    Q = problems.slab_3d(seed=45) if kind == "3d" else problems.slab_2d(seed=45)
    Q.Auu, Q.Auv, Q.Avu, Q.Avv, Q.bu, Q.bv = A2[0], A2[1], A2[2], A2[3], b2u, b2v
    ru, rv, l2, l2r = S.residual_vector()
    want = gpu_residual_vector(Q, x1[0], x1[1])
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert (l2, l2r) == (want[2], want[3])
    assert S.residual_vector(arrays=False)[2:] == (l2, l2r)
    with pytest.raises(cg.CismGpuError):
        S.residual_velocity(1)  # no solve since the system was set
    err, nit = S.solve(cg.ALG_CHRONGEAR, 1, 5, 1e-10, 400)
    x2 = S.x()
    # the solve started from x1: the same as a one-shot solve of Q from x1
    xu, xv = x1[0].copy(), x1[1].copy()
    if kind == "3d":
        e2, n2 = cg.pcg_solver_chrongear_3d(Q.nx, Q.ny, Q.nz, Q.par, asm.indxA_2d(), asm.indxA_3d(),
                                            Q.active_vertex, *A2, b2u, b2v, xu, xv, 1, 5, 1e-10, 400)
    else:
        e2, n2 = cg.pcg_solver_chrongear_2d(Q.nx, Q.ny, Q.par, asm.indxA_2d(), Q.active_vertex, *A2, b2u, b2v,
                                            xu, xv, 1, 5, 1e-10, 400)
    assert (err, nit) == (e2, n2)
    np.testing.assert_array_equal(x2[0], xu)
    for which in (0, 1, 2):
        assert S.residual_velocity(which) == gpu_residual_velocity(Q, which, x2[0], x2[1], x1[0], x1[1])
    # after the solve the residual vector is that of the new solution
    assert S.residual_vector(arrays=False)[2] == gpu_residual_vector(Q, x2[0], x2[1])[2]
    S.close()


def test_accelerated_picard_save_restore(gpu_lib):
    """evaluate_accelerated_picard's saved state on a handle: after save, a new system and a
    solve, restore brings back the saved velocity and A (b stays the latest, as in the
    reference); the residual and the next solve equal the one-shot calls on (A1, b2) from x1."""
    P = problems.slab_3d(seed=46)
    S = cg.DeviceSolver(P)
    with pytest.raises(cg.CismGpuError):
        S.restore()  # nothing saved yet
    S.solve(cg.ALG_CHRONGEAR, 1, 5, 1e-10, 400)
    x1 = S.x()
    S.save()
    A2 = [a * 1.07 for a in (P.Auu, P.Auv, P.Avu, P.Avv)]
    b2u, b2v = P.bu * 0.95, P.bv * 0.95
    S.set_system(*A2, b2u, b2v, x0_from_solution=True)
    S.solve(cg.ALG_CHRONGEAR, 1, 5, 1e-10, 400)
    S.restore()
    Q = problems.slab_3d(seed=46)
    Q.bu, Q.bv = b2u, b2v
    ru, rv, l2, l2r = S.residual_vector()
    want = gpu_residual_vector(Q, x1[0], x1[1])
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert (l2, l2r) == (want[2], want[3])
    err, nit = S.solve(cg.ALG_CHRONGEAR, 1, 5, 1e-10, 400)
    xu, xv = x1[0].copy(), x1[1].copy()
    e2, n2 = cg.pcg_solver_chrongear_3d(Q.nx, Q.ny, Q.nz, Q.par, asm.indxA_2d(), asm.indxA_3d(), Q.active_vertex,
                                        Q.Auu, Q.Auv, Q.Avu, Q.Avv, b2u, b2v, xu, xv, 1, 5, 1e-10, 400)
    assert (err, nit) == (e2, n2)
    np.testing.assert_array_equal(S.x()[0], xu)
    np.testing.assert_array_equal(S.x()[1], xv)
    # the mixed solver after a restore works on the restored matrix (its FP32 copy rebuilt)
    S.restore()
    em, nm = S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 2000)
    assert em < 1e-8
    S.close()
