"""A second, independent restatement of one reference solver, in plain Python, against the oracle.

The oracle (oracle/pcg_oracle.cpp) is a C++ restatement of glissade_velo_higher_pcg.F90.  This file
restates pcg_solver_standard_2d with the diagonal preconditioner once more, statement by statement
from the reference source, in Python floats (IEEE binary64, no fused multiply-add, left-to-right
evaluation as in Fortran): the staggered halo update on one rank (staggered_parallel_halo_real8_2d,
libglimmer/parallel_mpi.F90:10609-10769), matvec_multiply_structured_2d (:5656-5773), the
non-reprosum global sum (parallel_global_sum_stagger_real8_2d, parallel_mpi.F90:6620-6637),
setup_preconditioner_diag_2d (:4199-4243) and the solver loop (:385-808).  Two restatements written
separately that agree bit for bit at every iteration count rule out transcription slips in either.
"""
import math

import numpy as np
import pytest

import oracle
from cism_b200 import assembly as asm
from tests import problems


def _halo(a, par):
    """staggered_parallel_halo on one rank: with periodic_bc the exchanges go to the rank itself
    (east/west on the owned rows, then north/south on whole columns); outflow and no_ice zero the
    edges of the global domain.  lhalo = 2, uhalo = 1.  a is (NY, NX), a[j-1, i-1] = a(i, j)."""
    NY, NX = a.shape
    jlo, jhi = par["staggered_jlo"], par["staggered_jhi"]
    if par["periodic_bc"]:
        rows = slice(jlo - 1, jhi)
        wsend = a[rows, 2:3].copy()          # a(1+lhalo : lhalo+uhalo, jlo:jhi)
        esend = a[rows, NX - 3:NX - 1].copy()  # a(NX-uhalo-lhalo+1 : NX-uhalo, jlo:jhi)
        a[rows, NX - 1:NX] = wsend           # erecv (from self as the east neighbour)
        a[rows, 0:2] = esend                 # wrecv
        ssend = a[2:3, :].copy()             # a(:, 1+lhalo : lhalo+uhalo)
        nsend = a[NY - 3:NY - 1, :].copy()   # a(:, NY-uhalo-lhalo+1 : NY-uhalo)
        a[NY - 1:NY, :] = ssend              # nrecv
        a[0:2, :] = nsend                    # srecv
    if par["outflow_bc"]:
        a[:, 0:1] = 0.0
        a[:, NX - 1:NX] = 0.0
        a[0:1, :] = 0.0
        a[NY - 1:NY, :] = 0.0
    elif par["no_ice_bc"]:
        a[:, 0:2] = 0.0
        a[:, NX - 2:NX] = 0.0
        a[0:2, :] = 0.0
        a[NY - 2:NY, :] = 0.0


def _m(iA, jA):
    """indxA_2d(iA, jA) - 1 for the standard map (1..9, iA fastest)."""
    return (iA + 1) + 3 * (jA + 1)


def _matvec(P, xu, xv):
    par = P.par
    NY, NX = xu.shape
    act = P.active_vertex
    yu = np.zeros_like(xu)
    yv = np.zeros_like(xv)
    for jA in (-1, 0, 1):
        for iA in (-1, 0, 1):
            m = _m(iA, jA)
            for j in range(par["staggered_jlo"], par["staggered_jhi"] + 1):
                for i in range(par["staggered_ilo"], par["staggered_ihi"] + 1):
                    if act[j - 1, i - 1] and 1 <= i + iA <= NX and 1 <= j + jA <= NY:
                        x1 = float(xu[j + jA - 1, i + iA - 1])
                        x2 = float(xv[j + jA - 1, i + iA - 1])
                        yu[j - 1, i - 1] = (float(yu[j - 1, i - 1]) + float(P.Auu[m, j - 1, i - 1]) * x1) + \
                            float(P.Auv[m, j - 1, i - 1]) * x2
                        yv[j - 1, i - 1] = (float(yv[j - 1, i - 1]) + float(P.Avu[m, j - 1, i - 1]) * x1) + \
                            float(P.Avv[m, j - 1, i - 1]) * x2
    return yu, yv


def _gsum(P, a1, a2):
    par = P.par
    s = 0.0
    for j in range(par["staggered_jlo"], par["staggered_jhi"] + 1):
        for i in range(par["staggered_ilo"], par["staggered_ihi"] + 1):
            s = (s + float(a1[j - 1, i - 1])) + float(a2[j - 1, i - 1])
    return s


def pcg_standard_2d_diag(P, maxiters, ncheck=5, tol=1e-8):
    """pcg_solver_standard_2d, precond = HO_PRECOND_DIAG, from x0 = 0; returns (xu, xv, err, niters)."""
    par = P.par
    bu, bv = P.bu.astype(np.float64), P.bv.astype(np.float64)
    xu, xv = np.zeros_like(bu), np.zeros_like(bv)
    adu, adv = P.Auu[_m(0, 0)], P.Avv[_m(0, 0)]
    _halo(xu, par)
    _halo(xv, par)
    zu, zv = _matvec(P, xu, xv)
    ru, rv = bu - zu, bv - zv
    niters = maxiters
    eta0 = 1.0
    du, dv = np.zeros_like(bu), np.zeros_like(bv)
    l2_rhs = math.sqrt(_gsum(P, bu * bu, bv * bv))
    err = float("nan")
    for it in range(1, maxiters + 1):
        zu = np.divide(ru, adu, out=np.zeros_like(ru), where=adu != 0.0)
        zv = np.divide(rv, adv, out=np.zeros_like(rv), where=adv != 0.0)
        eta1 = _gsum(P, ru * zu, rv * zv)
        beta = eta1 / eta0
        du = zu + beta * du
        dv = zv + beta * dv
        _halo(du, par)
        _halo(dv, par)
        qu, qv = _matvec(P, du, dv)
        eta0 = eta1
        eta2 = _gsum(P, du * qu, dv * qv)
        alpha = eta1 / eta2
        xu = xu + alpha * du
        xv = xv + alpha * dv
        ru = ru - alpha * qu
        rv = rv - alpha * qv
        if it % ncheck == 0 or it == 5:
            _halo(xu, par)
            _halo(xv, par)
            zu, zv = _matvec(P, xu, xv)
            ru, rv = bu - zu, bv - zv
            err = math.sqrt(_gsum(P, ru * ru, rv * rv)) / l2_rhs
            if err < tol:
                niters = it
                break
    return xu, xv, err, niters


CASES = [
    ("slab-periodic", lambda: problems.slab_2d(seed=1)),
    ("slab-outflow-boundary-ice", lambda: problems.slab_2d(seed=2, boundary_ice=True, bc="outflow")),
    ("slab-no-ice", lambda: problems.slab_2d(seed=3, boundary_ice=True, bc="no_ice")),
    ("ssa-interior", lambda: asm.ssa_random(ewn=14, nsn=12, seed=5)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("maxiters", [3, 12, 400])
def test_second_restatement_matches_oracle(name, make, maxiters):
    """Bit-identical x, err and niters at fixed iteration counts and through convergence."""
    P = make()
    xu, xv, err, nit = pcg_standard_2d_diag(P, maxiters)
    st, ou, ov, oerr, onit = oracle.pcg("standard", P, 1, tol=1e-8, maxiters=maxiters, summode=oracle.SUM_SEQ)
    assert st == 0
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)
