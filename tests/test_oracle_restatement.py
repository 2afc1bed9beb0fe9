"""A second, independent restatement of reference solvers, in Python, against the oracle.

The oracle (oracle/pcg_oracle.cpp) is a C++ restatement of glissade_velo_higher_pcg.F90.  This file
restates pcg_solver_standard_2d (diagonal preconditioner), pcg_solver_standard_3d,
pcg_solver_chrongear_2d and pcg_solver_chrongear_3d (no, diagonal, SIA and local tridiagonal line
preconditioners) once more, statement by statement
from the reference source, in IEEE binary64 with no fused multiply-add and Fortran's left-to-right
evaluation: the staggered halo update on one rank (staggered_parallel_halo_real8_2d/_3d,
libglimmer/parallel_mpi.F90:10609-10936), matvec_multiply_structured_2d/_3d (:5656-5773,
:5528-5652), the non-reprosum global sums (parallel_global_sum_stagger_real8_2d/_3d and their
two-field forms, parallel_mpi.F90:6620-6637, 6770-6790, 6904, 7042), the diagonal and SIA
preconditioners (setup_preconditioner_diag_2d/_3d, setup_preconditioner_sia_3d :3647-3733,
easy_sia_solver and tridiag_solver :5777-5922, setup_preconditioner_tridiag_local_2d/_3d
:3737-3830, :4247-4392, tridiag_solver_local_2d/_3d :4917-5100, :4524-4655, and the global forms)
and the solver loops, plus the residual steps of the Picard loop (compute_residual_vector_2d/_3d and
compute_residual_velocity_2d/_3d, glissade_velo_higher.F90:9502-9894, 10188-10446) and the stiffness
assembly (assemble_stiffness_matrix_3d :5382-5643, the SSA branch of assemble_stiffness_matrix_2d
:4961-5378, with the basis-function derivatives, viscosities, element matrices and scatters).  Element-wise statements use
numpy arrays (one IEEE operation per element); the 3D matvec runs over all nodes at once but adds
each node's couplings in the reference's order; the global sums are sequential Python loops.  Two
restatements written separately that agree bit for bit at every iteration count rule out
transcription slips in either.
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
    edges of the global domain.  lhalo = 2, uhalo = 1.  a is (NY, NX) or (NY, NX, nz), a[j-1, i-1]
    = a(i, j) (all levels of the column in 3D, as the 3D routine exchanges whole columns)."""
    NY, NX = a.shape[:2]
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
    return np.float64(s)  # the solvers' scalars then divide as IEEE (inf, NaN), as the reference's do


def _tri_setup_2d(P, U, V, glob=False):
    """setup_preconditioner_tridiag_local_2d (:4247-4392) on coefficient planes U = Auu, V = Avv
    ((9, NY, NX), 0-based m = indxA_2d - 1): u lines along i with the couplings (-1,0), (0,0),
    (1,0), v lines along j with (0,-1), (0,0), (0,1); a zero diagonal becomes 1 with zero
    off-diagonals; forward elimination over the owned range; a zero pivot is GM_FATAL (raises)."""
    par = P.par
    ilo, ihi, jlo, jhi = par["staggered_ilo"], par["staggered_ihi"], par["staggered_jlo"], par["staggered_jhi"]
    out = {}
    for comp, A, offs in (("u", U, ((-1, 0), (0, 0), (1, 0))), ("v", V, ((0, -1), (0, 0), (0, 1)))):
        sub, dg, sp = (A[_m(*o)].astype(np.float64).copy() for o in offs)
        zero = dg == 0.0
        dg[zero], sub[zero], sp[zero] = 1.0, 0.0, 0.0
        om, den = np.zeros_like(dg), np.zeros_like(dg)
        lines = range(jlo, jhi + 1) if comp == "u" else range(ilo, ihi + 1)
        for ln in lines:
            pos = list(range(ilo, ihi + 1)) if comp == "u" else list(range(jlo, jhi + 1))
            at = (lambda q: (ln - 1, q - 1)) if comp == "u" else (lambda q: (q - 1, ln - 1))
            om[at(pos[0])] = float(sp[at(pos[0])]) / float(dg[at(pos[0])])
            for a, b in zip(pos[:-1], pos[1:]):
                d = float(dg[at(b)]) - float(sub[at(b)]) * float(om[at(a)])
                if d == 0.0:
                    raise ZeroDivisionError("divzero in setup_preconditioner_tridiag_local_2d")
                den[at(b)] = 1.0 / d
                om[at(b)] = float(sp[at(b)]) * float(den[at(b)])
            if glob:  # setup_preconditioner_tridiag_global_2d (:4396-4520): the reverse recurrence's check
                ouh = float(sub[at(pos[-1])]) / float(dg[at(pos[-1])])
                for q in reversed(pos[:-1]):
                    duh = float(dg[at(q)]) - float(sp[at(q)]) * ouh
                    if duh == 0.0:
                        raise ZeroDivisionError("divzero in setup_preconditioner_tridiag_global_2d")
                    ouh = float(sub[at(q)]) / duh
        out[comp] = (1.0 / dg, sub, om, den)
    return out


def _tri_solve_2d(P, T, bu, bv, glob=False):
    """tridiag_solver_local_2d (:4917-5100): gamma forward over the owned range, back substitution
    from the last owned position down to the array's first (omega and gamma are zero below)."""
    par = P.par
    ilo, ihi, jlo, jhi = par["staggered_ilo"], par["staggered_ihi"], par["staggered_jlo"], par["staggered_jhi"]
    res = []
    for comp, b in (("u", bu), ("v", bv)):
        adg, sub, om, den = T[comp]
        x, gam = np.zeros_like(b), np.zeros_like(b)
        lines = range(jlo, jhi + 1) if comp == "u" else range(ilo, ihi + 1)
        for ln in lines:
            lo, hi = (ilo, ihi) if comp == "u" else (jlo, jhi)
            at = (lambda q: (ln - 1, q - 1)) if comp == "u" else (lambda q: (q - 1, ln - 1))
            gam[at(lo)] = float(b[at(lo)]) * float(adg[at(lo)])
            for q in range(lo + 1, hi + 1):
                gam[at(q)] = (float(b[at(q)]) - float(sub[at(q)]) * float(gam[at(q - 1)])) * float(den[at(q)])
            x[at(hi)] = gam[at(hi)]
            # the global form (tridiag_solver_global_2d on one task: the particular solution of the
            # owned block, zero elsewhere, :5291-5519) stops at the owned range
            for q in range(hi - 1, (lo - 1) if glob else 0, -1):
                x[at(q)] = float(gam[at(q)]) - float(om[at(q)]) * float(x[at(q + 1)])
        res.append(x)
    return res[0], res[1]


def _vsum_planes(P, A, glob=False):
    """setup_preconditioner_tridiag_local_3d (:3737-3830): per column the sums over levels of the
    three vertical offsets of each horizontal coupling, ((s + A(m)) + A(m+9)) + A(m+18); inactive
    columns get the identity (centre 1, the rest 0)."""
    nz = A.shape[2]
    out = np.zeros((9,) + A.shape[:2])
    for m in range(9):
        acc = np.zeros(A.shape[:2])
        for k in range(nz):
            acc = ((acc + A[:, :, k, m]) + A[:, :, k, m + 9]) + A[:, :, k, m + 18]
        out[m] = acc
    inact = P.active_vertex == 0
    if glob:  # setup_preconditioner_tridiag_global_3d (:3937-4195): the centre only, then the halo
        out[4, inact] = 1.0  # update of every summed plane (:4056-4057)
        for m in range(9):
            _halo(out[m], P.par)
    else:
        out[:, inact] = 0.0
        out[4, inact] = 1.0
    return out


def _line_rhs_3d(r):
    """sum(r(:, i, j)) in level order."""
    acc = np.zeros(r.shape[:2])
    for k in range(r.shape[2]):
        acc = acc + r[:, :, k]
    return acc


def pcg_standard_2d_diag(P, maxiters, ncheck=5, tol=1e-8, precond=1, x0=None):
    """pcg_solver_standard_2d with precond 0 (none), 1 (diagonal), 3/4 (local/global tridiagonal
    lines, then the halo of z) or 2, which takes no branch in 2D and leaves z as it is: the zeros
    set before the loop (:424-428), so the first alpha is 0/0.  From x0 (default 0); returns (xu, xv, err,
    niters)."""
    par = P.par
    bu, bv = P.bu.astype(np.float64), P.bv.astype(np.float64)
    if x0 is None:
        xu, xv = np.zeros_like(bu), np.zeros_like(bv)
    else:
        xu, xv = np.array(x0[0], dtype=np.float64, copy=True), np.array(x0[1], dtype=np.float64, copy=True)
    adu, adv = P.Auu[_m(0, 0)], P.Avv[_m(0, 0)]
    T = _tri_setup_2d(P, P.Auu, P.Avv, glob=precond == 4) if precond in (3, 4) else None
    _halo(xu, par)
    _halo(xv, par)
    zu, zv = _matvec(P, xu, xv)
    ru, rv = bu - zu, bv - zv
    niters = maxiters
    eta0 = 1.0
    du, dv = np.zeros_like(bu), np.zeros_like(bv)
    zu, zv = np.zeros_like(bu), np.zeros_like(bv)
    l2_rhs = np.sqrt(_gsum(P, bu * bu, bv * bv))
    err = float("nan")
    for it in range(1, maxiters + 1):
        if precond == 2:
            pass
        elif precond in (3, 4):
            zu, zv = _tri_solve_2d(P, T, ru, rv, glob=precond == 4)
            _halo(zu, par)
            _halo(zv, par)
        elif precond == 0:
            zu, zv = ru.copy(), rv.copy()
        else:
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
        if eta1 != eta1 or alpha != alpha:  # eta1 = NaN or alpha = NaN: GM_FATAL
            return xu, xv, err, -it
        xu = xu + alpha * du
        xv = xv + alpha * dv
        ru = ru - alpha * qu
        rv = rv - alpha * qv
        if it % ncheck == 0 or it == 5:
            _halo(xu, par)
            _halo(xv, par)
            zu, zv = _matvec(P, xu, xv)
            ru, rv = bu - zu, bv - zv
            err = np.sqrt(_gsum(P, ru * ru, rv * rv)) / l2_rhs
            if err < tol:
                niters = it
                break
    return xu, xv, err, niters


def _gsum2(P, a1, b1, a2, b2):
    """The two-field form (nflds = 2, parallel_mpi.F90:6904): each field summed on its own."""
    return _gsum(P, a1, b1), _gsum(P, a2, b2)


def _precond(P, precond, ru, rv, T=None, z=None):
    if precond == 0:
        return ru.copy(), rv.copy()
    if precond == 2:  # no branch of the 2D solvers takes it: z keeps its contents
        return z[0].copy(), z[1].copy()
    if precond in (3, 4):
        zu, zv = _tri_solve_2d(P, T, ru, rv, glob=precond == 4)
        _halo(zu, P.par)
        _halo(zv, P.par)
        return zu, zv
    adu, adv = P.Auu[_m(0, 0)], P.Avv[_m(0, 0)]
    return (np.divide(ru, adu, out=np.zeros_like(ru), where=adu != 0.0),
            np.divide(rv, adv, out=np.zeros_like(rv), where=adv != 0.0))


def pcg_chrongear_2d(P, precond, maxiters, ncheck=5, tol=1e-8, x0=None):
    """pcg_solver_chrongear_2d (:1541-2628) with precond 0-4, from x0 (default 0): the first pass
    (:1913-2227), then iterations 2.. with one two-field sum each; with the line preconditioner at
    most 100 iterations (maxiters_tridiag, :1703-1732).  Precond 2 takes no branch: z keeps A x0
    from the first pass's matvec, later A x from the last convergence check.  Returns (xu, xv,
    err, niters)."""
    par = P.par
    T = None
    if precond in (3, 4):
        T = _tri_setup_2d(P, P.Auu, P.Avv, glob=precond == 4)
        maxiters = 100
    bu, bv = P.bu.astype(np.float64), P.bv.astype(np.float64)
    if x0 is None:
        xu, xv = np.zeros_like(bu), np.zeros_like(bv)
    else:
        xu, xv = np.array(x0[0], dtype=np.float64, copy=True), np.array(x0[1], dtype=np.float64, copy=True)
    du, dv = np.zeros_like(bu), np.zeros_like(bv)
    l2_rhs = np.sqrt(_gsum(P, bu * bu, bv * bv))
    _halo(xu, par)
    _halo(xv, par)
    zu, zv = _matvec(P, xu, xv)
    ru, rv = bu - zu, bv - zv
    _halo(ru, par)
    _halo(rv, par)
    zu, zv = _precond(P, precond, ru, rv, T, (zu, zv))
    w1u, w1v = ru * zu, rv * zv
    du, dv = zu.copy(), zv.copy()
    qu, qv = _matvec(P, du, dv)
    rho_old, sigma = _gsum2(P, w1u, w1v, du * qu, dv * qv)
    _halo(qu, par)
    _halo(qv, par)
    alpha = rho_old / sigma
    if alpha != alpha:  # 'solver has failed, alpha = NaN', GM_FATAL
        return xu, xv, float("nan"), -1
    xu = xu + alpha * du
    xv = xv + alpha * dv
    ru = ru - alpha * qu
    rv = rv - alpha * qv
    niters, err = maxiters, float("nan")
    for it in range(2, maxiters + 1):
        zu, zv = _precond(P, precond, ru, rv, T, (zu, zv))
        azu, azv = _matvec(P, zu, zv)
        rho, delta = _gsum2(P, ru * zu, rv * zv, azu * zu, azv * zv)
        _halo(azu, par)
        _halo(azv, par)
        beta = rho / rho_old
        sigma = delta - beta * rho / alpha
        alpha = rho / sigma
        rho_old = rho
        if alpha != alpha:
            return xu, xv, err, -it
        du = zu + beta * du
        dv = zv + beta * dv
        qu = azu + beta * qu
        qv = azv + beta * qv
        xu = xu + alpha * du
        xv = xv + alpha * dv
        ru = ru - alpha * qu
        rv = rv - alpha * qv
        if it % ncheck == 0 or it == 5:
            zu, zv = _matvec(P, xu, xv)
            ru, rv = bu - zu, bv - zv
            err = np.sqrt(_gsum(P, ru * ru, rv * rv)) / l2_rhs
            if err < tol:
                niters = it
                break
            _halo(ru, par)
            _halo(rv, par)
    return xu, xv, err, niters


def _m3(iA, jA, kA):
    """indxA_3d(iA, jA, kA) - 1 for the standard map (1..27, iA fastest, then jA, then kA)."""
    return (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1)


def _matvec3(P, xu, xv):
    """matvec_multiply_structured_3d: over owned active columns, every level k, the couplings in the
    order kA, jA, iA; a coupling that leaves the arrays is skipped.  Arrays are (NY, NX, nz) and the
    blocks (NY, NX, nz, 27); the nodes are independent, so they are updated together."""
    par = P.par
    NY, NX, nz = xu.shape
    own = np.zeros((NY, NX), dtype=bool)
    own[par["staggered_jlo"] - 1:par["staggered_jhi"], par["staggered_ilo"] - 1:par["staggered_ihi"]] = True
    rows = (own & (P.active_vertex != 0))[:, :, None]
    J, I, K = np.meshgrid(np.arange(NY), np.arange(NX), np.arange(nz), indexing="ij")
    yu, yv = np.zeros_like(xu), np.zeros_like(xv)
    for kA in (-1, 0, 1):
        for jA in (-1, 0, 1):
            for iA in (-1, 0, 1):
                m = _m3(iA, jA, kA)
                jn, i_n, kn = J + jA, I + iA, K + kA
                ok = rows & (kn >= 0) & (kn < nz) & (i_n >= 0) & (i_n < NX) & (jn >= 0) & (jn < NY)
                jc, ic, kc = np.clip(jn, 0, NY - 1), np.clip(i_n, 0, NX - 1), np.clip(kn, 0, nz - 1)
                x1, x2 = xu[jc, ic, kc], xv[jc, ic, kc]
                nu = (yu + P.Auu[..., m] * x1) + P.Auv[..., m] * x2
                nv = (yv + P.Avu[..., m] * x1) + P.Avv[..., m] * x2
                yu = np.where(ok, nu, yu)
                yv = np.where(ok, nv, yv)
    return yu, yv


def _gsum3(P, a1, a2):
    """Sequential sum over owned vertices j, i, then levels k: local_sum + arr1 + arr2."""
    par = P.par
    l1, l2 = a1.tolist(), a2.tolist()
    s = 0.0
    for j in range(par["staggered_jlo"], par["staggered_jhi"] + 1):
        for i in range(par["staggered_ilo"], par["staggered_ihi"] + 1):
            c1, c2 = l1[j - 1][i - 1], l2[j - 1][i - 1]
            for k in range(len(c1)):
                s = (s + c1[k]) + c2[k]
    return np.float64(s)


def _sia(P, A, r, z):
    """easy_sia_solver with the SIA matrix of setup_preconditioner_sia_3d (the column couplings
    (0,0,-1), (0,0,0), (0,0,1) of A): tridiag_solver on every active column (halo included); z
    keeps its values on inactive columns.  Vectorized over columns, sequential over levels."""
    nz = r.shape[2]
    sb, dg, sp = A[..., _m3(0, 0, -1)], A[..., _m3(0, 0, 0)], A[..., _m3(0, 0, 1)]
    act = P.active_vertex != 0
    soln = np.zeros_like(r)
    gamma = np.zeros_like(r)
    beta = dg[:, :, 0].copy()
    with np.errstate(divide="ignore", invalid="ignore"):  # a zero pivot gives the IEEE result, as in Fortran
        soln[:, :, 0] = r[:, :, 0] / np.where(act, beta, 1.0)
        for k in range(1, nz):
            gamma[:, :, k] = sp[:, :, k - 1] / np.where(act, beta, 1.0)
            beta = dg[:, :, k] - sb[:, :, k] * gamma[:, :, k]
            soln[:, :, k] = (r[:, :, k] - sb[:, :, k] * soln[:, :, k - 1]) / np.where(act, beta, 1.0)
        for k in range(nz - 2, -1, -1):
            soln[:, :, k] = soln[:, :, k] - gamma[:, :, k + 1] * soln[:, :, k + 1]
    out = z.copy()
    out[act] = soln[act]
    return out


def _precond3(P, precond, ru, rv, zu, zv, T=None):
    if precond == 0:
        return ru.copy(), rv.copy()
    if precond in (3, 4):  # tridiag_solver_local_3d (:4524-4655) / _global_3d (:4662-4913)
        su, sv = _tri_solve_2d(P, T, _line_rhs_3d(ru), _line_rhs_3d(rv), glob=precond == 4)
        _halo(su, P.par)
        _halo(sv, P.par)
        zu, zv = _sia(P, P.Auu, ru, zu), _sia(P, P.Avv, rv, zv)
        return zu + su[:, :, None], zv + sv[:, :, None]
    if precond == 1:
        adu, adv = P.Auu[..., _m3(0, 0, 0)], P.Avv[..., _m3(0, 0, 0)]
        return (np.divide(ru, adu, out=np.zeros_like(ru), where=adu != 0.0),
                np.divide(rv, adv, out=np.zeros_like(rv), where=adv != 0.0))
    return _sia(P, P.Auu, ru, zu), _sia(P, P.Avv, rv, zv)


def pcg_chrongear_3d(P, precond, maxiters, ncheck=5, tol=1e-8, x0=None):
    """pcg_solver_chrongear_3d (:2632-3594) with precond 0-4, from x0 (default 0): the first pass
    (:3048-3290), then iterations 2.. (:3296-3581); returns (xu, xv, err, niters)."""
    par = P.par
    T = (_tri_setup_2d(P, _vsum_planes(P, P.Auu, precond == 4), _vsum_planes(P, P.Avv, precond == 4),
                       glob=precond == 4) if precond in (3, 4) else None)
    bu, bv = P.bu.astype(np.float64), P.bv.astype(np.float64)
    if x0 is None:
        xu, xv = np.zeros_like(bu), np.zeros_like(bv)
    else:
        xu, xv = np.array(x0[0], dtype=np.float64, copy=True), np.array(x0[1], dtype=np.float64, copy=True)
    du, dv = np.zeros_like(bu), np.zeros_like(bv)
    qu, qv = np.zeros_like(bu), np.zeros_like(bv)
    l2_rhs = np.sqrt(_gsum3(P, bu * bu, bv * bv))
    _halo(xu, par)
    _halo(xv, par)
    zu, zv = _matvec3(P, xu, xv)
    ru, rv = bu - zu, bv - zv
    _halo(ru, par)
    _halo(rv, par)
    zu, zv = _precond3(P, precond, ru, rv, zu, zv, T)
    w1u, w1v = ru * zu, rv * zv
    du, dv = zu.copy(), zv.copy()
    qu, qv = _matvec3(P, du, dv)
    rho_old, sigma = _gsum3(P, w1u, w1v), _gsum3(P, du * qu, dv * qv)
    _halo(qu, par)
    _halo(qv, par)
    alpha = rho_old / sigma
    if alpha != alpha:  # 'solver has failed, alpha = NaN', GM_FATAL
        return xu, xv, float("nan"), -1
    xu = xu + alpha * du
    xv = xv + alpha * dv
    ru = ru - alpha * qu
    rv = rv - alpha * qv
    niters, err = maxiters, float("nan")
    for it in range(2, maxiters + 1):
        zu, zv = _precond3(P, precond, ru, rv, zu, zv, T)
        azu, azv = _matvec3(P, zu, zv)
        rho, delta = _gsum3(P, ru * zu, rv * zv), _gsum3(P, azu * zu, azv * zv)
        _halo(azu, par)
        _halo(azv, par)
        beta = rho / rho_old
        sigma = delta - beta * rho / alpha
        alpha = rho / sigma
        rho_old = rho
        if alpha != alpha:
            return xu, xv, err, -it
        du = zu + beta * du
        dv = zv + beta * dv
        qu = azu + beta * qu
        qv = azv + beta * qv
        xu = xu + alpha * du
        xv = xv + alpha * dv
        ru = ru - alpha * qu
        rv = rv - alpha * qv
        if it % ncheck == 0 or it == 5:
            zu, zv = _matvec3(P, xu, xv)
            ru, rv = bu - zu, bv - zv
            err = np.sqrt(_gsum3(P, ru * ru, rv * rv)) / l2_rhs
            if err < tol:
                niters = it
                break
            _halo(ru, par)
            _halo(rv, par)
    return xu, xv, err, niters


def _run(solver, P, precond, maxiters):
    """A restated solve; a zero pivot in the line setup (GM_FATAL) comes back as niters = -1."""
    try:
        return solver(P, precond, maxiters)
    except ZeroDivisionError:
        return None, None, float("nan"), -1


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
    if st != 0:  # the reference stops with GM_FATAL (a NaN alpha); so must the restatement
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precond", [0, 1, 3, 4])
@pytest.mark.parametrize("maxiters", [1, 4, 12, 600])
def test_second_restatement_chrongear_2d(name, make, precond, maxiters):
    """pcg_solver_chrongear_2d: bit-identical x, err and niters with the oracle's reference-order solve."""
    P = make()
    xu, xv, err, nit = _run(pcg_chrongear_2d, P, precond, maxiters)
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, precond, tol=1e-8, maxiters=maxiters,
                                        summode=oracle.SUM_SEQ)
    if st != 0:  # the reference stops with GM_FATAL (a NaN alpha); so must the restatement
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


def pcg_standard_3d(P, precond, maxiters, ncheck=5, tol=1e-8, x0=None):
    """pcg_solver_standard_3d (:827-1537) with precond 0-4, from x0 (default 0; the loop
    :1169-1524); returns (xu, xv, err, niters), niters < 0 where the reference stops with
    GM_FATAL."""
    par = P.par
    T = (_tri_setup_2d(P, _vsum_planes(P, P.Auu, precond == 4), _vsum_planes(P, P.Avv, precond == 4),
                       glob=precond == 4) if precond in (3, 4) else None)
    bu, bv = P.bu.astype(np.float64), P.bv.astype(np.float64)
    if x0 is None:
        xu, xv = np.zeros_like(bu), np.zeros_like(bv)
    else:
        xu, xv = np.array(x0[0], dtype=np.float64, copy=True), np.array(x0[1], dtype=np.float64, copy=True)
    _halo(xu, par)
    _halo(xv, par)
    zu, zv = _matvec3(P, xu, xv)
    ru, rv = bu - zu, bv - zv
    niters, eta0, err = maxiters, 1.0, float("nan")
    du, dv = np.zeros_like(bu), np.zeros_like(bv)
    zu, zv = np.zeros_like(bu), np.zeros_like(bv)
    l2_rhs = np.sqrt(_gsum3(P, bu * bu, bv * bv))
    for it in range(1, maxiters + 1):
        zu, zv = _precond3(P, precond, ru, rv, zu, zv, T)
        eta1 = _gsum3(P, ru * zu, rv * zv)
        if eta1 != eta1:
            return xu, xv, err, -it
        beta = eta1 / eta0
        du = zu + beta * du
        dv = zv + beta * dv
        _halo(du, par)
        _halo(dv, par)
        qu, qv = _matvec3(P, du, dv)
        eta0 = eta1
        eta2 = _gsum3(P, du * qu, dv * qv)
        alpha = eta1 / eta2
        if alpha != alpha:
            return xu, xv, err, -it
        xu = xu + alpha * du
        xv = xv + alpha * dv
        ru = ru - alpha * qu
        rv = rv - alpha * qv
        if it % ncheck == 0 or it == 5:
            _halo(xu, par)
            _halo(xv, par)
            zu, zv = _matvec3(P, xu, xv)
            ru, rv = bu - zu, bv - zv
            err = np.sqrt(_gsum3(P, ru * ru, rv * rv)) / l2_rhs
            if err < tol:
                niters = it
                break
    return xu, xv, err, niters


def _no_ice_edge_coefficients():
    """A no_ice slab whose last owned row and column keep nonzero couplings (a matrix that was not
    halo-updated before the solve): the global line preconditioner's halo update of its summed
    planes then zeroes owned entries, which the local form does not."""
    P = problems.slab_3d(seed=3, boundary_ice=True, bc="no_ice", sliding=False)
    ihi, jhi = P.par["staggered_ihi"], P.par["staggered_jhi"]
    for name in ("Auu", "Auv", "Avu", "Avv"):
        A = getattr(P, name)
        A[:, ihi - 1] = A[:, ihi - 2]
        A[jhi - 1, :] = A[jhi - 2, :]
    return P


CASES3 = [
    ("slab-periodic-sliding", lambda: problems.slab_3d(seed=1)),
    ("slab-periodic-boundary-ice", lambda: problems.slab_3d(seed=3, boundary_ice=True, sliding=False)),
    ("slab-outflow-boundary-ice", lambda: problems.slab_3d(seed=4, boundary_ice=True, bc="outflow", sliding=False)),
    ("dome", lambda: asm.dome()),
    ("slab-no-ice-edge-coefficients", _no_ice_edge_coefficients),
]


@pytest.mark.parametrize("name,make", CASES3, ids=[c[0] for c in CASES3])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("maxiters", [1, 4, 12, 400])
def test_second_restatement_chrongear_3d(name, make, precond, maxiters):
    """pcg_solver_chrongear_3d: bit-identical x, err and niters with the oracle's reference-order solve."""
    P = make()
    xu, xv, err, nit = _run(pcg_chrongear_3d, P, precond, maxiters)
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, precond, tol=1e-8, maxiters=maxiters,
                                        summode=oracle.SUM_SEQ)
    if st != 0:  # the reference stops with GM_FATAL (a NaN alpha); so must the restatement
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


@pytest.mark.parametrize("name,make", CASES3, ids=[c[0] for c in CASES3])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("maxiters", [1, 4, 12, 400])
def test_second_restatement_standard_3d(name, make, precond, maxiters):
    """pcg_solver_standard_3d (the dome with the diagonal preconditioner is the reference's own CPU
    configuration): bit-identical x, err and niters with the oracle's reference-order solve."""
    P = make()
    xu, xv, err, nit = _run(pcg_standard_3d, P, precond, maxiters)
    st, ou, ov, oerr, onit = oracle.pcg("standard", P, precond, tol=1e-8, maxiters=maxiters,
                                        summode=oracle.SUM_SEQ)
    if st != 0:  # the reference stops with GM_FATAL (a NaN eta1 or alpha); so must the restatement
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precond", [0, 3, 4])
@pytest.mark.parametrize("maxiters", [3, 12, 400])
def test_second_restatement_standard_2d_lines(name, make, precond, maxiters):
    """pcg_solver_standard_2d with the tridiagonal line preconditioners (3 local, 4 global)."""
    P = make()
    try:
        xu, xv, err, nit = pcg_standard_2d_diag(P, maxiters, precond=precond)
    except ZeroDivisionError:
        xu = xv = None
        err, nit = float("nan"), -1
    st, ou, ov, oerr, onit = oracle.pcg("standard", P, precond, tol=1e-8, maxiters=maxiters,
                                        summode=oracle.SUM_SEQ)
    if st != 0:
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


# ---------------------------------------------------------------------------------------------
# the residual steps of the Picard loop around the solve
# ---------------------------------------------------------------------------------------------
def residual_vector(P, u, v):
    """compute_residual_vector_2d/_3d (glissade_velo_higher.F90:9502-9689, 9693-9894): A u - b on the
    owned active vertices (the matvec's statements and order), 0 elsewhere; L2_norm over them, and
    L2_norm_relative = L2_norm / |b| over the same vertices (0 for a zero b)."""
    is3d = P.kind == "3d"
    mv, gs = (_matvec3, _gsum3) if is3d else (_matvec, _gsum)
    yu, yv = mv(P, u, v)
    par = P.par
    own = np.zeros(P.active_vertex.shape, dtype=bool)
    own[par["staggered_jlo"] - 1:par["staggered_jhi"], par["staggered_ilo"] - 1:par["staggered_ihi"]] = True
    live = own & (P.active_vertex != 0)
    if is3d:
        live = np.broadcast_to(live[:, :, None], yu.shape)
    ru = np.where(live, yu - P.bu, 0.0)
    rv = np.where(live, yv - P.bv, 0.0)
    l2 = math.sqrt(gs(P, np.where(live, ru * ru, 0.0), np.where(live, rv * rv, 0.0)))
    l2b = math.sqrt(gs(P, np.where(live, P.bu * P.bu, 0.0), np.where(live, P.bv * P.bv, 0.0)))
    return ru, rv, l2, (l2 / l2b if l2b > 0.0 else 0.0)


def residual_velocity(P, which, u, v, us, vs):
    """compute_residual_velocity_2d/_3d (:10188-10310, :10314-10446): the largest relative speed change
    over the owned vertices, in 3D without the bed level for HO_RESID_MAXU_NO_UBAS (1); the mean
    for HO_RESID_MEANU (2); otherwise every level."""
    par = P.par
    is3d = P.kind == "3d"
    nz = u.shape[2] if is3d else 1
    kmax = nz - 1 if (is3d and which in (1, 2)) else nz
    res, count = 0.0, 0
    lu, lv, lus, lvs = u.tolist(), v.tolist(), us.tolist(), vs.tolist()
    for j in range(par["staggered_jlo"], par["staggered_jhi"] + 1):
        for i in range(par["staggered_ilo"], par["staggered_ihi"] + 1):
            for k in range(kmax):
                g = (lambda a: a[j - 1][i - 1][k]) if is3d else (lambda a: a[j - 1][i - 1])
                speed = math.sqrt(g(lu) * g(lu) + g(lv) * g(lv))
                if speed != 0.0:
                    old = math.sqrt(g(lus) * g(lus) + g(lvs) * g(lvs))
                    diff = abs((old - speed) / speed)
                    if which == 2:
                        count += 1
                        res = res + diff
                    elif diff > res:
                        res = diff
    if which == 2 and count > 0:
        res = res / count
    return res


RESID_CASES = CASES + [c for c in CASES3 if c[0] != "slab-no-ice-edge-coefficients"]


@pytest.mark.parametrize("name,make", RESID_CASES, ids=[c[0] for c in RESID_CASES])
def test_second_restatement_residuals(name, make):
    """The residual vector, its norms and the velocity residuals: bit-identical with the oracle."""
    P = make()
    rng = np.random.default_rng(11)
    u, v = rng.standard_normal(P.bu.shape) * 50.0, rng.standard_normal(P.bv.shape) * 50.0
    us, vs = u * (1.0 + 0.01 * rng.standard_normal(u.shape)), v * (1.0 + 0.01 * rng.standard_normal(v.shape))
    u[tuple(ix[:3] for ix in np.nonzero(np.ones(u.shape, dtype=bool)))] = 0.0  # a few zero speeds
    v[tuple(ix[:3] for ix in np.nonzero(np.ones(v.shape, dtype=bool)))] = 0.0
    ru, rv, l2, l2r = residual_vector(P, u, v)
    ou, ov, ol2, ol2r = oracle.residual_vector(P, u, v, summode=oracle.SUM_SEQ)
    np.testing.assert_array_equal(ru, ou)
    np.testing.assert_array_equal(rv, ov)
    assert l2 == ol2 and l2r == ol2r
    for which in (0, 1, 2):
        assert residual_velocity(P, which, u, v, us, vs) == \
            oracle.residual_velocity(P, which, u, v, us, vs, summode=oracle.SUM_SEQ)


# ---------------------------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, SSA (glissade_velo_higher.F90:4961-5378)
# ---------------------------------------------------------------------------------------------
_RSQRT3 = 1.0 / math.sqrt(3.0)
_XQP = (-_RSQRT3, _RSQRT3, _RSQRT3, -_RSQRT3)  # quadrature points in the reference square (:528-538)
_YQP = (-_RSQRT3, -_RSQRT3, _RSQRT3, _RSQRT3)
_ISHIFT = ((0, 1, 1, 0), (-1, 0, 0, -1), (-1, 0, 0, -1), (0, 1, 1, 0))  # rows 1-4, columns 1-4 (:461-468)
_JSHIFT = ((0, 0, 1, 1), (0, 0, 1, 1), (-1, -1, 0, 0), (-1, -1, 0, 0))  # (:474-481)


def _ref_square(p):
    """phi_2d, dphi_dxr_2d, dphi_dyr_2d at quadrature point p (:555-575)."""
    x, y = _XQP[p], _YQP[p]
    phi = ((1.0 - x) * (1.0 - y) / 4.0, (1.0 + x) * (1.0 - y) / 4.0, (1.0 + x) * (1.0 + y) / 4.0,
           (1.0 - x) * (1.0 + y) / 4.0)
    dxr = (-(1.0 - y) / 4.0, (1.0 - y) / 4.0, (1.0 + y) / 4.0, -(1.0 + y) / 4.0)
    dyr = (-(1.0 - x) / 4.0, -(1.0 + x) / 4.0, (1.0 + x) / 4.0, (1.0 - x) / 4.0)
    return phi, dxr, dyr


def assemble_ssa_2d(nx, ny, nz, sigma, active_cell, xv, yv, uvel, vvel, stagthck, flwafact, whichefvs,
                    efvs_constant, effstrain_min, n_glen, nhalo=2):
    """The SSA branch: glissade_vertical_average of the flow factor (glissade_grid_operators.F90:
    1882-1946), then per active cell of the reference's loop (nhalo+1 .. n-nhalo+1) and quadrature
    point get_basis_function_derivatives_2d (:6319-6504), compute_effective_viscosity (:7285-7470),
    the thickness at the point and compute_element_matrix (:8001-8123), the cell's viscosity, and
    element_to_global_matrix_2d (:8127-8196).  Arrays as the oracle's: vertex fields (ny-1, nx-1),
    cell fields (ny, nx[, nz-1]), blocks (9, ny-1, nx-1)."""
    vol0 = 1.0e9
    p_eff = (1.0 - n_glen) / n_glen
    effstrain_ff = 500.0 / 31536000.0 / 200.0e3 * 31536000.0  # velo_scale / len_scale * scyr
    ff2 = np.zeros((ny, nx))
    for j in range(ny):
        for i in range(nx):
            acc = 0.0
            for k in range(nz - 1):
                acc = acc + float(flwafact[j, i, k]) * (float(sigma[k + 1]) - float(sigma[k]))
            ff2[j, i] = acc
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    efvs_out = np.zeros((ny, nx, nz - 1))
    for j in range(nhalo + 1, ny - nhalo + 2):
        for i in range(nhalo + 1, nx - nhalo + 2):
            if not active_cell[j - 1, i - 1]:
                continue
            verts = [(i + _ISHIFT[2][n], j + _JSHIFT[2][n]) for n in range(4)]  # node n's vertex (1-based)
            x = [float(xv[jv - 1, iv - 1]) for iv, jv in verts]
            y = [float(yv[jv - 1, iv - 1]) for iv, jv in verts]
            u = [float(uvel[jv - 1, iv - 1]) for iv, jv in verts]
            v = [float(vvel[jv - 1, iv - 1]) for iv, jv in verts]
            h = [float(stagthck[jv - 1, iv - 1]) for iv, jv in verts]
            K = [[[0.0] * 4 for _ in range(4)] for _ in range(4)]  # Kuu, Kuv, Kvu, Kvv [nr][nc]
            evq = [0.0] * 4
            for p in range(4):
                phi, dxr, dyr = _ref_square(p)
                j11 = j12 = j21 = j22 = 0.0
                for n in range(4):
                    j11 = j11 + dxr[n] * x[n]
                    j12 = j12 + dxr[n] * y[n]
                    j21 = j21 + dyr[n] * x[n]
                    j22 = j22 + dyr[n] * y[n]
                det = j11 * j22 - j12 * j21
                if not abs(det) > 0.0:
                    raise ZeroDivisionError("Jacobian matrix is singular")
                i11, i12, i21, i22 = j22 / det, -j12 / det, -j21 / det, j11 / det
                dx = [(0.0 + i11 * dxr[n]) + i12 * dyr[n] for n in range(4)]
                dy = [(0.0 + i21 * dxr[n]) + i22 * dyr[n] for n in range(4)]
                if whichefvs == 0:
                    ev = efvs_constant
                elif whichefvs == 1:
                    ev = float(ff2[j - 1, i - 1]) * effstrain_ff ** p_eff
                else:
                    dudx = dudy = dvdx = dvdy = 0.0
                    for n in range(4):
                        dudx = dudx + dx[n] * u[n]
                        dudy = dudy + dy[n] * u[n]
                        dvdx = dvdx + dx[n] * v[n]
                        dvdy = dvdy + dy[n] * v[n]
                    sh = dvdx + dudy
                    esq = effstrain_min * effstrain_min + \
                        (((dudx * dudx + dvdy * dvdy) + dudx * dvdy) + 0.25 * (sh * sh))
                    ev = float(ff2[j - 1, i - 1]) * esq ** (p_eff / 2.0)
                evq[p] = ev
                hq = 0.0
                for n in range(4):
                    hq = hq + phi[n] * h[n]
                fac = (hq * ev) * 1.0 * det / vol0
                for nc in range(4):
                    for nr in range(4):
                        K[0][nr][nc] = K[0][nr][nc] + fac * (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc])
                        K[1][nr][nc] = K[1][nr][nc] + fac * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc])
                        K[2][nr][nc] = K[2][nr][nc] + fac * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc])
                        K[3][nr][nc] = K[3][nr][nc] + fac * (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc])
            acc = 0.0
            for p in range(4):
                acc = acc + evq[p]
            efvs_out[j - 1, i - 1, :] = acc / 4
            for nr in range(4):
                iv, jv = i + _ISHIFT[2][nr], j + _JSHIFT[2][nr]
                for nc in range(4):
                    m = _m(_ISHIFT[nr][nc], _JSHIFT[nr][nc])
                    for b in range(4):
                        A[b][m, jv - 1, iv - 1] = float(A[b][m, jv - 1, iv - 1]) + K[b][nr][nc]
    return efvs_out, A


def _ssa_inputs(seed, velocity):
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=seed)
    rng = np.random.default_rng(seed + 50)
    shape = (g["ny"] - 1, g["nx"] - 1)
    u = 40.0 * rng.standard_normal(shape) if velocity else np.zeros(shape)
    v = 40.0 * rng.standard_normal(shape) if velocity else np.zeros(shape)
    ff = 0.5 * 1.0e-16 ** (-1.0 / 3.0) * (1.0 + 0.2 * rng.random((g["ny"], g["nx"], g["nz"] - 1)))
    return g, u, v, ff


@pytest.mark.parametrize("whichefvs", [0, 1, 2])
@pytest.mark.parametrize("seed,velocity", [(31, False), (32, True), (33, True)])
def test_second_restatement_ssa_assembly(whichefvs, seed, velocity):
    """assemble_stiffness_matrix_2d (SSA): every coefficient and the cell viscosities bit-identical
    with the oracle, for constant, flow-factor and nonlinear (Glen) viscosity."""
    g, u, v, ff = _ssa_inputs(seed, velocity)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    args = (nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v, g["stagthck"], ff)
    kw = dict(whichefvs=whichefvs, efvs_constant=2.5e6, effstrain_min=1.0e-8, n_glen=3.0)
    st, oefvs, *oA = oracle.assemble_stiffness_2d(*args, **kw)
    assert st == 0
    efvs, A = assemble_ssa_2d(*args, whichefvs, 2.5e6, 1.0e-8, 3.0)
    np.testing.assert_array_equal(efvs, oefvs)
    for got, want in zip(A, oA):
        np.testing.assert_array_equal(got, want)


# ---------------------------------------------------------------------------------------------
# assemble_stiffness_matrix_3d (glissade_velo_higher.F90:5382-5643)
# ---------------------------------------------------------------------------------------------
_XQ3 = (-_RSQRT3, _RSQRT3, _RSQRT3, -_RSQRT3, -_RSQRT3, _RSQRT3, _RSQRT3, -_RSQRT3)  # (:314-338)
_YQ3 = (-_RSQRT3, -_RSQRT3, _RSQRT3, _RSQRT3, -_RSQRT3, -_RSQRT3, _RSQRT3, _RSQRT3)
_ZQ3 = (-_RSQRT3,) * 4 + (_RSQRT3,) * 4
_I1, _I2 = (0, 1, 1, 0, 0, 1, 1, 0), (-1, 0, 0, -1, -1, 0, 0, -1)  # ishift rows (:461-468)
_J1, _J3 = (0, 0, 1, 1, 0, 0, 1, 1), (-1, -1, 0, 0, -1, -1, 0, 0)  # jshift rows (:474-481)
_K1, _K5 = (0, 0, 0, 0, -1, -1, -1, -1), (1, 1, 1, 1, 0, 0, 0, 0)  # kshift rows (:486-493)
_ISH3 = (_I1, _I2, _I2, _I1, _I1, _I2, _I2, _I1)
_JSH3 = (_J1, _J1, _J3, _J3, _J1, _J1, _J3, _J3)
_KSH3 = (_K1, _K1, _K1, _K1, _K5, _K5, _K5, _K5)


def _ref_cube(p):
    """dphi_dxr_3d, dphi_dyr_3d, dphi_dzr_3d at quadrature point p (:355-391)."""
    x, y, z = _XQ3[p], _YQ3[p], _ZQ3[p]
    dxr = (-(1.0 - y) * (1.0 - z) / 8.0, (1.0 - y) * (1.0 - z) / 8.0, (1.0 + y) * (1.0 - z) / 8.0,
           -(1.0 + y) * (1.0 - z) / 8.0, -(1.0 - y) * (1.0 + z) / 8.0, (1.0 - y) * (1.0 + z) / 8.0,
           (1.0 + y) * (1.0 + z) / 8.0, -(1.0 + y) * (1.0 + z) / 8.0)
    dyr = (-(1.0 - x) * (1.0 - z) / 8.0, -(1.0 + x) * (1.0 - z) / 8.0, (1.0 + x) * (1.0 - z) / 8.0,
           (1.0 - x) * (1.0 - z) / 8.0, -(1.0 - x) * (1.0 + z) / 8.0, -(1.0 + x) * (1.0 + z) / 8.0,
           (1.0 + x) * (1.0 + z) / 8.0, (1.0 - x) * (1.0 + z) / 8.0)
    dzr = (-(1.0 - x) * (1.0 - y) / 8.0, -(1.0 + x) * (1.0 - y) / 8.0, -(1.0 + x) * (1.0 + y) / 8.0,
           -(1.0 - x) * (1.0 + y) / 8.0, (1.0 - x) * (1.0 - y) / 8.0, (1.0 + x) * (1.0 - y) / 8.0,
           (1.0 + x) * (1.0 + y) / 8.0, (1.0 - x) * (1.0 + y) / 8.0)
    return dxr, dyr, dzr


def assemble_3d(nx, ny, nz, sigma, active_cell, xv, yv, uvel, vvel, stagusrf, stagthck, flwafact, whichapprox,
                whichefvs, efvs_constant, effstrain_min, n_glen, nhalo=2):
    """Per active cell of the reference's loop and layer k: the element's nodes (ishift/jshift/
    kshift row 7: nodes 1-4 on level k+1, 5-8 on level k), per quadrature point
    get_basis_function_derivatives_3d (:6508-6732: Jacobian, cofactors, detJ, Jinv = cofactor^T /
    detJ), compute_effective_viscosity (:7285-7470, the SIA / SSA / 3D branches) and
    compute_element_matrix (:8001-8123), the layer's mean viscosity, element_to_global_matrix_3d
    (:8200-8268).  Arrays as the oracle's."""
    vol0 = 1.0e9
    p_eff = (1.0 - n_glen) / n_glen
    effstrain_ff = 500.0 / 31536000.0 / 200.0e3 * 31536000.0
    A = [np.zeros((ny - 1, nx - 1, nz, 27)) for _ in range(4)]
    efvs_out = np.zeros((ny, nx, nz - 1))
    cubes = [_ref_cube(p) for p in range(8)]
    for j in range(nhalo + 1, ny - nhalo + 2):
        for i in range(nhalo + 1, nx - nhalo + 2):
            if not active_cell[j - 1, i - 1]:
                continue
            for k in range(1, nz):
                nodes = [(i + _ISH3[6][n], j + _JSH3[6][n], k + _KSH3[6][n]) for n in range(8)]
                x = [float(xv[jn - 1, in_ - 1]) for in_, jn, kn in nodes]
                y = [float(yv[jn - 1, in_ - 1]) for in_, jn, kn in nodes]
                z = [float(stagusrf[jn - 1, in_ - 1]) - float(sigma[kn - 1]) * float(stagthck[jn - 1, in_ - 1])
                     for in_, jn, kn in nodes]
                u = [float(uvel[jn - 1, in_ - 1, kn - 1]) for in_, jn, kn in nodes]
                v = [float(vvel[jn - 1, in_ - 1, kn - 1]) for in_, jn, kn in nodes]
                ff = float(flwafact[j - 1, i - 1, k - 1])
                K = [[[0.0] * 8 for _ in range(8)] for _ in range(4)]
                evq = [0.0] * 8
                for p in range(8):
                    dxr, dyr, dzr = cubes[p]
                    J = [[0.0] * 3 for _ in range(3)]
                    for n in range(8):
                        for r, d in enumerate((dxr, dyr, dzr)):
                            J[r][0] = J[r][0] + d[n] * x[n]
                            J[r][1] = J[r][1] + d[n] * y[n]
                            J[r][2] = J[r][2] + d[n] * z[n]
                    c = [[J[1][1] * J[2][2] - J[1][2] * J[2][1], -(J[1][0] * J[2][2] - J[1][2] * J[2][0]),
                          J[1][0] * J[2][1] - J[1][1] * J[2][0]],
                         [-(J[0][1] * J[2][2] - J[0][2] * J[2][1]), J[0][0] * J[2][2] - J[0][2] * J[2][0],
                          -(J[0][0] * J[2][1] - J[0][1] * J[2][0])],
                         [J[0][1] * J[1][2] - J[0][2] * J[1][1], -(J[0][0] * J[1][2] - J[0][2] * J[1][0]),
                          J[0][0] * J[1][1] - J[0][1] * J[1][0]]]
                    det = (J[0][0] * c[0][0] + J[0][1] * c[0][1]) + J[0][2] * c[0][2]
                    if not abs(det) > 0.0:
                        raise ZeroDivisionError("Jacobian matrix is singular")
                    Ji = [[c[col][row] / det for col in range(3)] for row in range(3)]
                    dx = [(Ji[0][0] * dxr[n] + Ji[0][1] * dyr[n]) + Ji[0][2] * dzr[n] for n in range(8)]
                    dy = [(Ji[1][0] * dxr[n] + Ji[1][1] * dyr[n]) + Ji[1][2] * dzr[n] for n in range(8)]
                    dz = [(Ji[2][0] * dxr[n] + Ji[2][1] * dyr[n]) + Ji[2][2] * dzr[n] for n in range(8)]
                    if whichefvs == 0:
                        ev = efvs_constant
                    elif whichefvs == 1:
                        ev = ff * effstrain_ff ** p_eff
                    else:
                        dudx = dudy = dudz = dvdx = dvdy = dvdz = 0.0
                        for n in range(8):
                            if whichapprox == 0:
                                dudz = dudz + dz[n] * u[n]
                                dvdz = dvdz + dz[n] * v[n]
                            else:
                                dudx = dudx + dx[n] * u[n]
                                dudy = dudy + dy[n] * u[n]
                                dvdx = dvdx + dx[n] * v[n]
                                dvdy = dvdy + dy[n] * v[n]
                                if whichapprox != 1:
                                    dudz = dudz + dz[n] * u[n]
                                    dvdz = dvdz + dz[n] * v[n]
                        em2 = effstrain_min * effstrain_min
                        sh = dvdx + dudy
                        if whichapprox == 0:
                            esq = em2 + 0.25 * (dudz * dudz + dvdz * dvdz)
                        elif whichapprox == 1:
                            esq = em2 + (((dudx * dudx + dvdy * dvdy) + dudx * dvdy) + 0.25 * (sh * sh))
                        else:
                            esq = (em2 + (((dudx * dudx + dvdy * dvdy) + dudx * dvdy) + 0.25 * (sh * sh))) + \
                                0.25 * (dudz * dudz + dvdz * dvdz)
                        ev = ff * esq ** (p_eff / 2.0)
                    evq[p] = ev
                    fac = ev * 1.0 * det / vol0
                    for nc in range(8):
                        for nr in range(8):
                            if whichapprox == 0:
                                t = fac * (dz[nr] * dz[nc])
                                K[0][nr][nc] = K[0][nr][nc] + t
                                K[3][nr][nc] = K[3][nr][nc] + t
                                continue
                            if whichapprox == 1:
                                kuu = 4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc]
                                kvv = 4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc]
                            else:
                                kuu = (4.0 * dx[nr] * dx[nc] + dy[nr] * dy[nc]) + dz[nr] * dz[nc]
                                kvv = (4.0 * dy[nr] * dy[nc] + dx[nr] * dx[nc]) + dz[nr] * dz[nc]
                            K[0][nr][nc] = K[0][nr][nc] + fac * kuu
                            K[1][nr][nc] = K[1][nr][nc] + fac * (2.0 * dx[nr] * dy[nc] + dy[nr] * dx[nc])
                            K[2][nr][nc] = K[2][nr][nc] + fac * (2.0 * dy[nr] * dx[nc] + dx[nr] * dy[nc])
                            K[3][nr][nc] = K[3][nr][nc] + fac * kvv
                acc = 0.0
                for p in range(8):
                    acc = acc + evq[p]
                efvs_out[j - 1, i - 1, k - 1] = acc / 8
                for nr in range(8):
                    ir, jr, kr = nodes[nr]
                    for nc in range(8):
                        m = _m3(_ISH3[nr][nc], _JSH3[nr][nc], _KSH3[nr][nc])
                        for b in range(4):
                            A[b][jr - 1, ir - 1, kr - 1, m] = float(A[b][jr - 1, ir - 1, kr - 1, m]) + K[b][nr][nc]
    return efvs_out, A


@pytest.mark.parametrize("whichapprox", [0, 1, 2])
@pytest.mark.parametrize("whichefvs", [0, 1, 2])
@pytest.mark.parametrize("seed,velocity", [(41, False), (42, True)])
def test_second_restatement_3d_assembly(whichapprox, whichefvs, seed, velocity):
    """assemble_stiffness_matrix_3d (SIA, SSA and Blatter-Pattyn element matrices; constant,
    flow-factor and Glen viscosity): every coefficient and layer viscosity bit-identical with the
    oracle."""
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=seed)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed + 60)
    shape = (ny - 1, nx - 1, nz)
    u = 40.0 * rng.standard_normal(shape) if velocity else np.zeros(shape)
    v = 40.0 * rng.standard_normal(shape) if velocity else np.zeros(shape)
    ff = 0.5 * 1.0e-16 ** (-1.0 / 3.0) * (1.0 + 0.2 * rng.random((ny, nx, nz - 1)))
    args = (nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v, g["stagusrf"], g["stagthck"], ff)
    st, oefvs, *oA = oracle.assemble_stiffness_3d(*args, whichapprox=whichapprox, whichefvs=whichefvs,
                                                  efvs_constant=2.5e6, effstrain_min=1.0e-8, n_glen=3.0)
    assert st == 0
    efvs, A = assemble_3d(*args, whichapprox, whichefvs, 2.5e6, 1.0e-8, 3.0)
    np.testing.assert_array_equal(efvs, oefvs)
    for got, want in zip(A, oA):
        np.testing.assert_array_equal(got, want)


def _phi3(p):
    x, y, z = _XQ3[p], _YQ3[p], _ZQ3[p]
    return ((1.0 - x) * (1.0 - y) * (1.0 - z) / 8.0, (1.0 + x) * (1.0 - y) * (1.0 - z) / 8.0,
            (1.0 + x) * (1.0 + y) * (1.0 - z) / 8.0, (1.0 - x) * (1.0 + y) * (1.0 - z) / 8.0,
            (1.0 - x) * (1.0 - y) * (1.0 + z) / 8.0, (1.0 + x) * (1.0 - y) * (1.0 + z) / 8.0,
            (1.0 + x) * (1.0 + y) * (1.0 + z) / 8.0, (1.0 - x) * (1.0 + y) * (1.0 + z) / 8.0)


def load_vector_standard(nx, ny, nz, sigma, active_cell, xv, yv, stagusrf, stagthck, dsx, dsy, nhalo=2):
    """load_vector_gravity, standard finite-element form (glissade_velo_higher.F90:4341-4449): per
    element and quadrature point the surface gradient interpolated at the point, and each node's
    -rhoi*grav*wqp*detJ/vol0*ds*phi added in node order (rhoi = 910, grav = 9.81)."""
    vol0, rhoi, grav = 1.0e9, 910.0, 9.81
    lu, lv = np.zeros((ny - 1, nx - 1, nz)), np.zeros((ny - 1, nx - 1, nz))
    for j in range(nhalo + 1, ny - nhalo + 2):
        for i in range(nhalo + 1, nx - nhalo + 2):
            if not active_cell[j - 1, i - 1]:
                continue
            for k in range(1, nz):
                nodes = [(i + _ISH3[6][n], j + _JSH3[6][n], k + _KSH3[6][n]) for n in range(8)]
                x = [float(xv[jn - 1, in_ - 1]) for in_, jn, kn in nodes]
                y = [float(yv[jn - 1, in_ - 1]) for in_, jn, kn in nodes]
                z = [float(stagusrf[jn - 1, in_ - 1]) - float(sigma[kn - 1]) * float(stagthck[jn - 1, in_ - 1])
                     for in_, jn, kn in nodes]
                sx = [float(dsx[jn - 1, in_ - 1]) for in_, jn, kn in nodes]
                sy = [float(dsy[jn - 1, in_ - 1]) for in_, jn, kn in nodes]
                for p in range(8):
                    dxr, dyr, dzr = _ref_cube(p)
                    J = [[0.0] * 3 for _ in range(3)]
                    for n in range(8):
                        for r, d in enumerate((dxr, dyr, dzr)):
                            J[r][0] = J[r][0] + d[n] * x[n]
                            J[r][1] = J[r][1] + d[n] * y[n]
                            J[r][2] = J[r][2] + d[n] * z[n]
                    c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1]
                    c01 = -(J[1][0] * J[2][2] - J[1][2] * J[2][0])
                    c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0]
                    det = (J[0][0] * c00 + J[0][1] * c01) + J[0][2] * c02
                    phi = _phi3(p)
                    qx = qy = 0.0
                    for n in range(8):
                        qx = qx + phi[n] * sx[n]
                        qy = qy + phi[n] * sy[n]
                    for n in range(8):
                        in_, jn, kn = nodes[n]
                        lu[jn - 1, in_ - 1, kn - 1] = float(lu[jn - 1, in_ - 1, kn - 1]) - \
                            rhoi * grav * 1.0 * det / vol0 * qx * phi[n]
                        lv[jn - 1, in_ - 1, kn - 1] = float(lv[jn - 1, in_ - 1, kn - 1]) - \
                            rhoi * grav * 1.0 * det / vol0 * qy * phi[n]
    return lu, lv


def test_second_restatement_load_vector_standard():
    """load_vector_gravity, standard form: bit-identical with the oracle on a rough surface."""
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=44)
    nx, ny, nz, dx = g["nx"], g["ny"], g["nz"], g["dx"]
    rng = np.random.default_rng(9)
    sx, sy = 0.01 * rng.standard_normal((ny - 1, nx - 1)), 0.01 * rng.standard_normal((ny - 1, nx - 1))
    sig = g["sigma"]
    stagw = np.concatenate([[0.0], 0.5 * (sig[:-1] + sig[1:]), [1.0]])
    st, ou, ov = oracle.load_vector_gravity(nx, ny, nz, sig, stagw, dx, dx, g["ac"], g["av"], g["xVertex"],
                                            g["yVertex"], g["stagusrf"], g["stagthck"], sx, sy, 0)
    assert st == 0
    lu, lv = load_vector_standard(nx, ny, nz, sig, g["ac"], g["xVertex"], g["yVertex"], g["stagusrf"],
                                  g["stagthck"], sx, sy)
    assert np.count_nonzero(lu) > 0
    np.testing.assert_array_equal(lu, ou)
    np.testing.assert_array_equal(lv, ov)


def dirichlet_3d(nx, ny, nz, active_vertex, umask, vmask, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv, nhalo=2):
    """dirichlet_boundary_conditions_3d (glissade_velo_higher.F90:9305-9498), on copies, in the
    reference's order: vertices j = nhalo..ny-nhalo+1, i = nhalo..nx-nhalo+1, levels k; a u-prescribed
    node sets b, a unit diagonal (and zero uv, vu diagonals), zeroes its u row and moves each
    neighbour's coupling to it into that neighbour's b (kA, jA, iA order); then the same for v."""
    A = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Auv, Avu, Avv)]
    b = [np.array(bu, dtype=np.float64, copy=True), np.array(bv, dtype=np.float64, copy=True)]
    NX, NY = nx - 1, ny - 1
    masks = (umask, vmask)
    vel = (uvel, vvel)
    c0 = _m3(0, 0, 0)
    for j in range(nhalo, ny - nhalo + 2):
        for i in range(nhalo, nx - nhalo + 2):
            if not active_vertex[j - 1, i - 1]:
                continue
            for k in range(1, nz + 1):
                for comp in (0, 1):  # 0: u prescribed, 1: v prescribed
                    if masks[comp][j - 1, i - 1, k - 1] != 1:
                        continue
                    val = float(vel[comp][j - 1, i - 1, k - 1])
                    b[comp][j - 1, i - 1, k - 1] = val
                    for kA in (-1, 0, 1):
                        for jA in (-1, 0, 1):
                            for iA in (-1, 0, 1):
                                kn, jn, in_ = k + kA, j + jA, i + iA
                                if not (1 <= kn <= nz and 1 <= in_ <= NX and 1 <= jn <= NY):
                                    continue
                                if iA == 0 and jA == 0 and kA == 0:
                                    if comp == 0:
                                        A[0][j - 1, i - 1, k - 1, c0] = 1.0
                                        A[1][j - 1, i - 1, k - 1, c0] = 0.0
                                        A[2][j - 1, i - 1, k - 1, c0] = 0.0
                                    else:
                                        A[1][j - 1, i - 1, k - 1, c0] = 0.0
                                        A[2][j - 1, i - 1, k - 1, c0] = 0.0
                                        A[3][j - 1, i - 1, k - 1, c0] = 1.0
                                    continue
                                m = _m3(iA, jA, kA)
                                row = (0, 1) if comp == 0 else (2, 3)  # this node's row blocks
                                A[row[0]][j - 1, i - 1, k - 1, m] = 0.0
                                A[row[1]][j - 1, i - 1, k - 1, m] = 0.0
                                mt = _m3(-iA, -jA, -kA)
                                n = (jn - 1, in_ - 1, kn - 1)
                                # the neighbour's u row (block uu or uv) and v row (vu or vv) coupling
                                # to this node's prescribed component
                                bu_blk, bv_blk = (0, 2) if comp == 0 else (1, 3)
                                if umask[n] != 1:
                                    b[0][n] = float(b[0][n]) - float(A[bu_blk][n + (mt,)]) * val
                                    A[bu_blk][n + (mt,)] = 0.0
                                if vmask[n] != 1:
                                    b[1][n] = float(b[1][n]) - float(A[bv_blk][n + (mt,)]) * val
                                    A[bv_blk][n + (mt,)] = 0.0
    return (*A, *b)


@pytest.mark.parametrize("seed", [51, 52])
def test_second_restatement_dirichlet_3d(seed):
    """dirichlet_boundary_conditions_3d with random u-only, v-only and u+v prescribed nodes and
    nonzero prescribed values: every coefficient and b bit-identical with the oracle."""
    P = problems.slab_3d(seed=seed, boundary_ice=True, sliding=False)
    rng = np.random.default_rng(seed)
    shape = P.bu.shape
    um = (rng.random(shape) < 0.15).astype(np.int32)
    vm = (rng.random(shape) < 0.15).astype(np.int32)
    um[:, :, -1] = 1  # the no-slip bed
    vm[:, :, -1] = 1
    uv, vv = rng.standard_normal(shape) * 10.0, rng.standard_normal(shape) * 10.0
    args = (P.nx, P.ny, P.nz, P.active_vertex, um, vm, uv, vv, P.Auu, P.Auv, P.Avu, P.Avv, P.bu, P.bv)
    want = oracle.dirichlet_3d(*args)
    got = dirichlet_3d(*args)
    for g_, w in zip(got, want):
        np.testing.assert_array_equal(g_, w)


def basal_standard_3d(nx, ny, nz, active_cell, xv, yv, beta, lsrf, Auu, Avv, nhalo=2):
    """basal_sliding_bc_3d, standard finite-element form (glissade_velo_higher.F90:8953-9129): lsrf
    staggered to the vertices (glissade_stagger, all four cells, glissade_grid_operators.F90:69-157),
    per active cell and quadrature point the curved area factor (get_area_scale_factor_curved_2d
    :6736-6827), beta at the point, the 4x4 element matrix and its scatter into the bed layer's
    horizontal couplings, point by point."""
    vol0 = 1.0e9
    A = [np.array(Auu, dtype=np.float64, copy=True), np.array(Avv, dtype=np.float64, copy=True)]
    sl = np.zeros((ny - 1, nx - 1))
    for j in range(1, ny):
        for i in range(1, nx):
            sl[j - 1, i - 1] = (((float(lsrf[j, i - 1]) + float(lsrf[j, i])) + float(lsrf[j - 1, i - 1])) +
                                float(lsrf[j - 1, i])) / 4.0
    for j in range(nhalo + 1, ny - nhalo + 2):
        for i in range(nhalo + 1, nx - nhalo + 2):
            if not active_cell[j - 1, i - 1]:
                continue
            verts = ((i - 1, j - 1), (i, j - 1), (i, j), (i - 1, j))
            x = [float(xv[jv - 1, iv - 1]) for iv, jv in verts]
            y = [float(yv[jv - 1, iv - 1]) for iv, jv in verts]
            z = [float(sl[jv - 1, iv - 1]) for iv, jv in verts]
            bb = [float(beta[jv - 1, iv - 1]) for iv, jv in verts]
            for p in range(4):
                phi, dxr, dyr = _ref_square(p)
                j11 = j12 = j13 = j21 = j22 = j23 = 0.0
                for n in range(4):
                    j11 = j11 + dxr[n] * x[n]
                    j12 = j12 + dxr[n] * y[n]
                    j13 = j13 + dxr[n] * z[n]
                    j21 = j21 + dyr[n] * x[n]
                    j22 = j22 + dyr[n] * y[n]
                    j23 = j23 + dyr[n] * z[n]
                t1 = j11 * j22 - j12 * j21
                t2 = -(j11 * j23 - j13 * j21)
                t3 = j12 * j23 - j13 * j22
                det = math.sqrt((t1 * t1 + t2 * t2) + t3 * t3)
                bq = 0.0
                for n in range(4):
                    bq = bq + phi[n] * bb[n]
                K = [[0.0] * 4 for _ in range(4)]
                for nc in range(4):
                    for nr in range(4):
                        K[nr][nc] = K[nr][nc] + bq * 1.0 * det / vol0 * phi[nr] * phi[nc]
                for nr in range(4):
                    iv, jv = i + _ISHIFT[2][nr], j + _JSHIFT[2][nr]
                    for nc in range(4):
                        m = _m3(_ISHIFT[nr][nc], _JSHIFT[nr][nc], 0)
                        for a in A:
                            a[jv - 1, iv - 1, nz - 1, m] = float(a[jv - 1, iv - 1, nz - 1, m]) + K[nr][nc]
    return A[0], A[1]


@pytest.mark.parametrize("seed", [61, 62])
def test_second_restatement_basal_standard_3d(seed):
    """The standard (curved) basal friction term: bit-identical bed-layer couplings with the oracle."""
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=seed)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed)
    beta = np.exp(np.log(1.0e3) + rng.standard_normal((ny - 1, nx - 1)))
    lsrf = g["usrf"] - g["thck"] + 20.0 * rng.random((ny, nx))
    P = problems.slab_3d(seed=seed, ewn=nx - 4, nsn=ny - 4, nz=nz, sliding=False)
    st, ou, ov = oracle.basal_standard(True, nx, ny, nz, g["ac"], g["xVertex"], g["yVertex"], beta, lsrf, P.Auu, P.Avv)
    assert st == 0
    gu, gv = basal_standard_3d(nx, ny, nz, g["ac"], g["xVertex"], g["yVertex"], beta, lsrf, P.Auu, P.Avv)
    assert not np.array_equal(gu, P.Auu)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gv, ov)


def dirichlet_2d(nx, ny, active_vertex, umask, vmask, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv, nhalo=2):
    """dirichlet_boundary_conditions_2d (glissade_velo_higher.F90:9133-9301), on copies: the offsets
    (jA, iA) outermost, then the vertices; a u-prescribed vertex sets b and its uu, uv and vu
    diagonals to 1, a v-prescribed one its uv, vu diagonals to 0 and vv to 1; off the diagonal the
    vertex's row couplings are zeroed and each neighbour's coupling to it moves into that
    neighbour's b."""
    A = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Auv, Avu, Avv)]
    b = [np.array(bu, dtype=np.float64, copy=True), np.array(bv, dtype=np.float64, copy=True)]
    NX, NY = nx - 1, ny - 1
    c0 = _m(0, 0)
    for jA in (-1, 0, 1):
        for iA in (-1, 0, 1):
            m, mm = _m(iA, jA), _m(-iA, -jA)
            for j in range(nhalo, ny - nhalo + 2):
                for i in range(nhalo, nx - nhalo + 2):
                    if not active_vertex[j - 1, i - 1]:
                        continue
                    inb = 1 <= i + iA <= NX and 1 <= j + jA <= NY
                    n = (j + jA - 1, i + iA - 1)
                    if umask[j - 1, i - 1] == 1:
                        val = float(uvel[j - 1, i - 1])
                        b[0][j - 1, i - 1] = val
                        if inb:
                            if iA == 0 and jA == 0:
                                A[0][c0, j - 1, i - 1] = 1.0
                                A[1][c0, j - 1, i - 1] = 1.0
                                A[2][c0, j - 1, i - 1] = 1.0
                            else:
                                A[0][m, j - 1, i - 1] = 0.0
                                A[1][m, j - 1, i - 1] = 0.0
                                if umask[n] != 1:
                                    b[0][n] = float(b[0][n]) - float(A[0][(mm,) + n]) * val
                                    A[0][(mm,) + n] = 0.0
                                if vmask[n] != 1:
                                    b[1][n] = float(b[1][n]) - float(A[2][(mm,) + n]) * val
                                    A[2][(mm,) + n] = 0.0
                    if vmask[j - 1, i - 1] == 1:
                        val = float(vvel[j - 1, i - 1])
                        b[1][j - 1, i - 1] = val
                        if inb:
                            if iA == 0 and jA == 0:
                                A[1][c0, j - 1, i - 1] = 0.0
                                A[2][c0, j - 1, i - 1] = 0.0
                                A[3][c0, j - 1, i - 1] = 1.0
                            else:
                                A[2][m, j - 1, i - 1] = 0.0
                                A[3][m, j - 1, i - 1] = 0.0
                                if umask[n] != 1:
                                    b[0][n] = float(b[0][n]) - float(A[1][(mm,) + n]) * val
                                    A[1][(mm,) + n] = 0.0
                                if vmask[n] != 1:
                                    b[1][n] = float(b[1][n]) - float(A[3][(mm,) + n]) * val
                                    A[3][(mm,) + n] = 0.0
    return (*A, *b)


@pytest.mark.parametrize("seed", [71, 72])
def test_second_restatement_dirichlet_2d(seed):
    """dirichlet_boundary_conditions_2d with u-only, v-only and u+v prescribed vertices and nonzero
    values: every coefficient and b bit-identical with the oracle."""
    P = problems.slab_2d(seed=seed, boundary_ice=True)
    rng = np.random.default_rng(seed)
    shape = P.bu.shape
    um = (rng.random(shape) < 0.2).astype(np.int32)
    vm = (rng.random(shape) < 0.2).astype(np.int32)
    uv, vv = rng.standard_normal(shape) * 10.0, rng.standard_normal(shape) * 10.0
    args = (P.nx, P.ny, P.active_vertex, um, vm, uv, vv, P.Auu, P.Auv, P.Avu, P.Avv, P.bu, P.bv)
    want = oracle.dirichlet_2d(*args)
    got = dirichlet_2d(*args)
    for g_, w in zip(got, want):
        np.testing.assert_array_equal(g_, w)


def _stagger(var):
    """glissade_stagger with stagger_margin 0 (glissade_grid_operators.F90:69-157): each vertex the
    mean of its four cells, summed (i,j+1), (i+1,j+1), (i,j), (i+1,j)."""
    ny, nx = var.shape
    s = np.zeros((ny - 1, nx - 1))
    for j in range(1, ny):
        for i in range(1, nx):
            s[j - 1, i - 1] = (((float(var[j, i - 1]) + float(var[j, i])) + float(var[j - 1, i - 1])) +
                               float(var[j - 1, i])) / 4.0
    return s


def _slope_gradients(field, dx, dy):
    """glissade_slope_angle's gradient on an (nx, ny) field (glissade_grid_operators.F90:1264-1410):
    glissade_gradient with gradient_margin 1 and the default all-ones mask (:309-468; every edge it
    reads is in the mask, so each component is the mean of its two edge differences), then
    glissade_unstagger with stagger_margin 0 (:226-305) back to the field's points, zero on the
    outer ring.  Returns (dz_dx, dz_dy), both field-shaped."""
    ny, nx = field.shape
    gx = np.zeros((ny - 1, nx - 1))
    gy = np.zeros((ny - 1, nx - 1))
    f = lambda i, j: float(field[j - 1, i - 1])
    for j in range(1, ny):
        for i in range(1, nx):
            north = (f(i + 1, j + 1) - f(i, j + 1)) / dx
            south = (f(i + 1, j) - f(i, j)) / dx
            gx[j - 1, i - 1] = (north + south) / 2.0
            east = (f(i + 1, j + 1) - f(i + 1, j)) / dy
            west = (f(i, j + 1) - f(i, j)) / dy
            gy[j - 1, i - 1] = (east + west) / 2.0
    out = []
    for g in (gx, gy):
        u = np.zeros((ny, nx))
        for j in range(2, ny):
            for i in range(2, nx):
                u[j - 1, i - 1] = (((float(g[j - 1, i - 1]) + float(g[j - 1, i - 2])) + float(g[j - 2, i - 1])) +
                                   float(g[j - 2, i - 2])) / 4.0
        out.append(u)
    return out[0], out[1]


def basal_local_3d(nx, ny, nz, dx, dy, active_vertex, beta, lsrf, Auu, Avv):
    """basal_sliding_bc_3d with HO_ASSEMBLE_BETA_LOCAL (glissade_velo_higher.F90:8921-8951): theta =
    atan(sqrt(dz_dx**2 + dz_dy**2)) of the staggered lower surface (glissade_slope_angle called on the
    (nx-1, ny-1) grid), then at active vertices the bed diagonal of Auu and Avv += dx*dy/vol0 *
    beta / cos(theta).  Returns (Auu, Avv, theta)."""
    vol0 = 1.0e9
    A = [np.array(Auu, dtype=np.float64, copy=True), np.array(Avv, dtype=np.float64, copy=True)]
    ddx, ddy = _slope_gradients(_stagger(lsrf), dx, dy)
    theta = np.zeros((ny - 1, nx - 1))
    for j in range(ny - 1):
        for i in range(nx - 1):
            slope = math.sqrt(float(ddx[j, i]) ** 2 + float(ddy[j, i]) ** 2)
            theta[j, i] = math.atan(slope) if slope >= 0.0 else 0.0
    c = _m3(0, 0, 0)
    for j in range(ny - 1):
        for i in range(nx - 1):
            if active_vertex[j, i]:
                for a in A:
                    a[j, i, nz - 1, c] = float(a[j, i, nz - 1, c]) + dx * dy / vol0 * float(beta[j, i]) / \
                        math.cos(float(theta[j, i]))
    return A[0], A[1], theta


def basal_local_2d_diva(nx, ny, dx, dy, active_vertex, beta_eff_x, beta_eff_y, lsrf, Auu, Avv):
    """basal_sliding_bc_2d_diva with HO_ASSEMBLE_BETA_LOCAL (glissade_velo_higher.F90:8641-8680): the
    directional slope angles theta_x = atan(|dz_dx|), theta_y = atan(|dz_dy|) of the staggered lower
    surface, then at active vertices Auu(0,0) += (dx*dy/vol0)*beta_eff_x/cos(theta_x) and
    Avv(0,0) += (dx*dy/vol0)*beta_eff_y/cos(theta_y).  Blocks (9, ny-1, nx-1)."""
    vol0 = 1.0e9
    A = [np.array(Auu, dtype=np.float64, copy=True), np.array(Avv, dtype=np.float64, copy=True)]
    ddx, ddy = _slope_gradients(_stagger(lsrf), dx, dy)
    c = _m(0, 0)
    for j in range(ny - 1):
        for i in range(nx - 1):
            if not active_vertex[j, i]:
                continue
            tx = math.atan(abs(float(ddx[j, i])))
            ty = math.atan(abs(float(ddy[j, i])))
            A[0][c, j, i] = float(A[0][c, j, i]) + (dx * dy / vol0) * float(beta_eff_x[j, i]) / math.cos(tx)
            A[1][c, j, i] = float(A[1][c, j, i]) + (dx * dy / vol0) * float(beta_eff_y[j, i]) / math.cos(ty)
    return A[0], A[1]


def basal_local_2d(nx, ny, dx, dy, active_vertex, beta, Auu, Avv):
    """basal_sliding_bc_2d with HO_ASSEMBLE_BETA_LOCAL (glissade_velo_higher.F90:8373-8391): at
    active vertices the diagonal of Auu and Avv += (dx*dy/vol0) * beta, no slope correction."""
    vol0 = 1.0e9
    A = [np.array(Auu, dtype=np.float64, copy=True), np.array(Avv, dtype=np.float64, copy=True)]
    c = _m(0, 0)
    for j in range(ny - 1):
        for i in range(nx - 1):
            if active_vertex[j, i]:
                inc = (dx * dy / vol0) * float(beta[j, i])
                for a in A:
                    a[c, j, i] = float(a[c, j, i]) + inc
    return A[0], A[1]


def _basal_local_inputs(seed, nx, ny):
    rng = np.random.default_rng(seed)
    # a rough lower surface: a tilted plane, a bump and noise, so every slope angle differs
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    lsrf = 300.0 - 40.0 * ii + 15.0 * jj + 200.0 * np.sin(0.7 * ii) * np.cos(0.5 * jj) + 30.0 * rng.random((ny, nx))
    av = rng.random((ny - 1, nx - 1)) < 0.8
    beta = np.exp(np.log(1.0e3) + rng.standard_normal((ny - 1, nx - 1)))
    return lsrf, av, beta


@pytest.mark.parametrize("seed", [81, 82])
def test_second_restatement_basal_local_3d(seed):
    """The local basal friction term (CISM's default assembly of beta): the slope angle and the bed
    diagonals bit-identical with the oracle, on a grid with unequal dx and dy."""
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=seed)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    lsrf, av, beta = _basal_local_inputs(seed, nx, ny)
    P = problems.slab_3d(seed=seed, ewn=nx - 4, nsn=ny - 4, nz=nz, sliding=False)
    dx, dy = 1000.0, 1350.0
    ou, ov, ot = oracle.basal_local_3d(nx, ny, nz, dx, dy, av, beta, lsrf, P.Auu, P.Avv)
    gu, gv, gt = basal_local_3d(nx, ny, nz, dx, dy, av, beta, lsrf, P.Auu, P.Avv)
    assert np.count_nonzero(gt) > (nx - 3) * (ny - 3) // 2 and not np.array_equal(gu, P.Auu)
    np.testing.assert_array_equal(gt, ot)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gv, ov)


@pytest.mark.parametrize("seed", [83, 84])
def test_second_restatement_basal_local_2d(seed):
    """The local basal terms of the 2D systems: SSA/L1L2 (beta alone) and DIVA (beta_eff_x and
    beta_eff_y over the directional slope angles), bit-identical with the oracle."""
    P = problems.slab_2d(seed=seed, boundary_ice=True)
    nx, ny = P.nx, P.ny
    lsrf, av, beta = _basal_local_inputs(seed, nx, ny)
    bey = beta * np.exp(0.3 * np.random.default_rng(seed + 1).standard_normal(beta.shape))
    dx, dy = 2000.0, 1500.0
    ou, ov = oracle.basal_local_2d(nx, ny, dx, dy, av, beta, P.Auu, P.Avv)
    gu, gv = basal_local_2d(nx, ny, dx, dy, av, beta, P.Auu, P.Avv)
    assert not np.array_equal(gu, P.Auu)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gv, ov)
    zc = np.zeros((ny, nx), dtype=np.int32)
    zv = np.zeros((ny - 1, nx - 1))
    ou, ov = oracle.basal_diva(nx, ny, dx, dy, zc, av, beta, bey, lsrf, zv, zv, 1, P.Auu, P.Avv)
    gu, gv = basal_local_2d_diva(nx, ny, dx, dy, av, beta, bey, lsrf, P.Auu, P.Avv)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gv, ov)


# ---------------------------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, L1L2 and DIVA (glissade_velo_higher.F90:4961-5378)
# ---------------------------------------------------------------------------------------------
_RHOI, _GRAV = 910.0, 9.81  # glimmer_physcon.F90:67, :69


def _efvs_l1l2(whichefvs, efvs_constant, effstrain_min, n_glen, nz, sigma, phi, dx, dy, u, v, h, dsdx, dsdy, flwa,
               flwafact):
    """compute_effective_viscosity_L1L2 (:7474-7726) at one quadrature point: the layer viscosities
    from the cubic for tau_parallel, with tau_perp from the surface slope and the depth."""
    p_eff = (1.0 - n_glen) / n_glen
    if whichefvs == 0:
        return [efvs_constant] * (nz - 1)
    if whichefvs == 1:
        eff = 500.0 / 31536000.0 / 200.0e3 * 31536000.0
        return [float(flwafact[k]) * eff ** p_eff for k in range(nz - 1)]
    dudx = dudy = dvdx = dvdy = dsx = dsy = thck = 0.0
    for n in range(4):
        dudx = dudx + dx[n] * u[n]
        dudy = dudy + dy[n] * u[n]
        dvdx = dvdx + dx[n] * v[n]
        dvdy = dvdy + dy[n] * v[n]
        dsx = dsx + phi[n] * dsdx[n]
        dsy = dsy + phi[n] * dsdy[n]
        thck = thck + phi[n] * h[n]
    sh = dvdx + dudy
    esq = (((effstrain_min * effstrain_min + dudx * dudx) + dvdy * dvdy) + dudx * dvdy) + 0.25 * (sh * sh)
    eff = math.sqrt(esq)
    out = []
    for k in range(nz - 1):
        depth = thck * float(sigma[k + 1])
        grads = math.sqrt(dsx * dsx + dsy * dsy)
        tperp = ((_RHOI * _GRAV) * depth) * grads
        a = tperp * tperp
        b = -eff / float(flwa[k])
        c = math.sqrt((b * b) / 4.0 + ((a * a) * a) / 27.0)
        root_a = math.pow(-b / 2.0 + c, 1.0 / 3.0)
        if ((a * a) * a) / 27.0 > 1.0e-6 * ((b * b) / 4.0):
            root_b = -math.pow(b / 2.0 + c, 1.0 / 3.0)
        else:
            root_b = -a / (3.0 * math.pow(abs(b), 1.0 / 3.0))
        tpar = root_a + root_b
        if abs(n_glen - 1.0) < 1.0e-10:
            out.append(1.0 / (2.0 * float(flwa[k])))
        elif abs(n_glen - 3.0) < 1.0e-10:
            out.append(1.0 / ((2.0 * float(flwa[k])) * (tpar * tpar + tperp * tperp)))
        else:
            raise ValueError("Invalid value of n_glen for L1L2 solver")
    return out


def _efvs_diva(whichefvs, efvs_constant, effstrain_min, n_glen, nz, stagsigma, phi, dx, dy, u, v, bx, by, sfx, sfy,
               flwafact, old):
    """compute_effective_viscosity_diva (:7730-7997), the iterative form (cubic = .false.): the
    vertical shear of each layer from the basal traction over the layer's previous viscosity."""
    p_eff = (1.0 - n_glen) / n_glen
    if whichefvs == 0:
        return [efvs_constant] * (nz - 1)
    if whichefvs == 1:
        eff = 500.0 / 31536000.0 / 200.0e3 * 31536000.0
        return [float(flwafact[k]) * eff ** p_eff for k in range(nz - 1)]
    dudx = dudy = dvdx = dvdy = taux = tauy = 0.0
    for n in range(4):
        dudx = dudx + dx[n] * u[n]
        dudy = dudy + dy[n] * u[n]
        dvdx = dvdx + dx[n] * v[n]
        dvdy = dvdy + dy[n] * v[n]
        taux = taux + phi[n] * bx[n]
        tauy = tauy + phi[n] * by[n]
    out = list(old)
    for k in range(nz - 1):
        if out[k] == 0.0:
            out[k] = float(flwafact[k]) * effstrain_min ** p_eff
        dudz = taux * float(stagsigma[k]) / (out[k] * sfx)
        dvdz = tauy * float(stagsigma[k]) / (out[k] * sfy)
        sh = dvdx + dudy
        esq = (((((effstrain_min * effstrain_min + dudx * dudx) + dvdy * dvdy) + dudx * dvdy) + 0.25 * (sh * sh)) +
               (0.25 * (dudz * dudz)) * sfx) + (0.25 * (dvdz * dvdz)) * sfy
        out[k] = float(flwafact[k]) * esq ** (p_eff / 2.0)
    return out


def _integrals_diva(nz, sigma, thck, eqp):
    """compute_integrals_diva (:5649-5775): omega_k at each level, the mean over the points of the
    integral of depth/efvs from the level to the surface, and omega, its layer-midpoint integral."""
    okp = [[0.0] * nz for _ in range(4)]
    for p in range(4):
        for k in range(nz - 2, -1, -1):
            depth = 0.5 * (float(sigma[k]) + float(sigma[k + 1]))
            dz = (float(sigma[k + 1]) - float(sigma[k])) * thck
            okp[p][k] = okp[p][k + 1] + depth / eqp[p][k] * dz
    ok = []
    for k in range(nz):
        acc = 0.0
        for p in range(4):
            acc = acc + okp[p][k]
        ok.append(acc / 4)
    om = 0.0
    for k in range(nz - 1):
        om = om + 0.5 * (ok[k] + ok[k + 1]) * (float(sigma[k + 1]) - float(sigma[k]))
    return ok, om


def assemble_layered_2d(approx, nx, ny, nz, sigma, active_cell, xv, yv, uvel, vvel, stagthck, flwafact, whichefvs,
                        efvs_constant, effstrain_min, n_glen, l1l2=None, diva=None, nhalo=2):
    """The L1L2 and DIVA branches: per active cell and quadrature point the basis derivatives, the
    layer viscosities, their sigma-weighted average times the thickness at the point into the
    element matrix of the Blatter-Pattyn form with zero vertical derivatives (compute_element_matrix
    :8001-8123), the cell's viscosity (the mean over the points), for DIVA the integrals, and
    element_to_global_matrix_2d.  l1l2 = (dusrf_dx, dusrf_dy, flwa); diva = (stagsigma, thck,
    btractx, btracty, dsfx, dsfy, efvs_qp_3d)."""
    vol0 = 1.0e9
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    efvs_out = np.zeros((ny, nx, nz - 1))
    if diva is not None:
        stagsigma, thck, btx, bty, dsfx, dsfy, eq_in = diva
        eq3 = np.array(eq_in, dtype=np.float64, copy=True)
        omega_k = np.zeros((ny, nx, nz))
        omega = np.zeros((ny, nx))
    for j in range(nhalo + 1, ny - nhalo + 2):
        for i in range(nhalo + 1, nx - nhalo + 2):
            if not active_cell[j - 1, i - 1]:
                continue
            verts = [(i + _ISHIFT[2][n], j + _JSHIFT[2][n]) for n in range(4)]
            pick = lambda f: [float(f[jv - 1, iv - 1]) for iv, jv in verts]
            x, y, u, v, h = pick(xv), pick(yv), pick(uvel), pick(vvel), pick(stagthck)
            if l1l2 is not None:
                dsdx, dsdy = pick(l1l2[0]), pick(l1l2[1])
            else:
                bx, by = pick(btx), pick(bty)
            K = [[[0.0] * 4 for _ in range(4)] for _ in range(4)]
            eqp = [None] * 4
            for p in range(4):
                phi, dxr, dyr = _ref_square(p)
                j11 = j12 = j21 = j22 = 0.0
                for n in range(4):
                    j11 = j11 + dxr[n] * x[n]
                    j12 = j12 + dxr[n] * y[n]
                    j21 = j21 + dyr[n] * x[n]
                    j22 = j22 + dyr[n] * y[n]
                det = j11 * j22 - j12 * j21
                if not abs(det) > 0.0:
                    raise ZeroDivisionError("Jacobian matrix is singular")
                i11, i12, i21, i22 = j22 / det, -j12 / det, -j21 / det, j11 / det
                ddx = [(0.0 + i11 * dxr[n]) + i12 * dyr[n] for n in range(4)]
                ddy = [(0.0 + i21 * dxr[n]) + i22 * dyr[n] for n in range(4)]
                if approx == "l1l2":
                    eqp[p] = _efvs_l1l2(whichefvs, efvs_constant, effstrain_min, n_glen, nz, sigma, phi, ddx, ddy, u,
                                        v, h, dsdx, dsdy, l1l2[2][j - 1, i - 1], flwafact[j - 1, i - 1])
                else:
                    old = [float(eq3[j - 1, i - 1, p, k]) for k in range(nz - 1)]
                    eqp[p] = _efvs_diva(whichefvs, efvs_constant, effstrain_min, n_glen, nz, stagsigma, phi, ddx, ddy,
                                        u, v, bx, by, float(dsfx[j - 1, i - 1]), float(dsfy[j - 1, i - 1]),
                                        flwafact[j - 1, i - 1], old)
                    eq3[j - 1, i - 1, p, :] = eqp[p]
                avg = 0.0
                for k in range(nz - 1):
                    avg = avg + eqp[p][k] * (float(sigma[k + 1]) - float(sigma[k]))
                hq = 0.0
                for n in range(4):
                    hq = hq + phi[n] * h[n]
                fac = (hq * avg) * 1.0 * det / vol0
                for nc in range(4):
                    for nr in range(4):
                        zz = 0.0 * 0.0
                        K[0][nr][nc] = K[0][nr][nc] + fac * ((4.0 * ddx[nr] * ddx[nc] + ddy[nr] * ddy[nc]) + zz)
                        K[1][nr][nc] = K[1][nr][nc] + fac * (2.0 * ddx[nr] * ddy[nc] + ddy[nr] * ddx[nc])
                        K[2][nr][nc] = K[2][nr][nc] + fac * (2.0 * ddy[nr] * ddx[nc] + ddx[nr] * ddy[nc])
                        K[3][nr][nc] = K[3][nr][nc] + fac * ((4.0 * ddy[nr] * ddy[nc] + ddx[nr] * ddx[nc]) + zz)
            if diva is not None:
                ok, om = _integrals_diva(nz, sigma, float(thck[j - 1, i - 1]), eqp)
                omega_k[j - 1, i - 1, :] = ok
                omega[j - 1, i - 1] = om
            for k in range(nz - 1):
                acc = 0.0
                for p in range(4):
                    acc = acc + eqp[p][k]
                efvs_out[j - 1, i - 1, k] = acc / 4
            for nr in range(4):
                iv, jv = i + _ISHIFT[2][nr], j + _JSHIFT[2][nr]
                for nc in range(4):
                    m = _m(_ISHIFT[nr][nc], _JSHIFT[nr][nc])
                    for b in range(4):
                        A[b][m, jv - 1, iv - 1] = float(A[b][m, jv - 1, iv - 1]) + K[b][nr][nc]
    if diva is not None:
        return efvs_out, eq3, omega_k, omega, A
    return efvs_out, A


@pytest.mark.parametrize("whichefvs", [0, 1, 2])
@pytest.mark.parametrize("seed,n_glen", [(41, 3.0), (42, 3.0), (43, 1.0)])
def test_second_restatement_l1l2_assembly(whichefvs, seed, n_glen):
    """assemble_stiffness_matrix_2d (L1L2): the layer viscosities of the tau_parallel cubic on a
    sloping surface and every coefficient, bit-identical with the oracle."""
    g, u, v, _ = _ssa_inputs(seed, True)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed + 7)
    dsdx = 0.02 * rng.standard_normal((ny - 1, nx - 1))
    dsdy = 0.02 * rng.standard_normal((ny - 1, nx - 1))
    dsdx[4:6, :] = 0.0  # the cells between two flat vertex rows take the cubic's first-order branch
    dsdy[4:6, :] = 0.0
    flwa = 1.0e-16 * (1.0 + rng.random((ny, nx, nz - 1)))
    ff = 0.5 * flwa ** (-1.0 / 3.0)
    st, oefvs, *oA = oracle.assemble_stiffness_2d_l1l2(nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u,
                                                       v, g["stagthck"], dsdx, dsdy, flwa, ff, whichefvs=whichefvs,
                                                       efvs_constant=2.5e6, effstrain_min=1.0e-8, n_glen=n_glen)
    assert st == 0
    efvs, A = assemble_layered_2d("l1l2", nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v,
                                  g["stagthck"], ff, whichefvs, 2.5e6, 1.0e-8, n_glen, l1l2=(dsdx, dsdy, flwa))
    assert np.count_nonzero(efvs) > 0
    np.testing.assert_array_equal(efvs, oefvs)
    for got, want in zip(A, oA):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("whichefvs", [0, 1, 2])
@pytest.mark.parametrize("seed,traction,first", [(44, 5.0e4, False), (45, 2.0e4, True), (46, 0.0, False)])
def test_second_restatement_diva_assembly(whichefvs, seed, traction, first):
    """assemble_stiffness_matrix_2d (DIVA): the point viscosities updated from the stored ones (or
    from the minimum strain rate on a first call, stored zeros), omega_k, omega, the cell
    viscosities and every coefficient, bit-identical with the oracle."""
    g, u, v, ff = _ssa_inputs(seed, True)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed + 9)
    sig = g["sigma"]
    stagsig = 0.5 * (sig[:-1] + sig[1:])
    bx = traction * (1.0 + rng.random((ny - 1, nx - 1)))
    by = -0.5 * traction * (1.0 + rng.random((ny - 1, nx - 1)))
    dsfx = 1.0 + 0.1 * rng.random((ny, nx))
    dsfy = 1.0 + 0.1 * rng.random((ny, nx))
    eq0 = np.zeros((ny, nx, 4, nz - 1)) if first else 2.0e6 * (1.0 + 0.3 * rng.random((ny, nx, 4, nz - 1)))
    o = oracle.assemble_stiffness_2d_diva(nx, ny, nz, sig, stagsig, g["ac"], g["xVertex"], g["yVertex"], u, v,
                                          g["stagthck"], g["thck"], bx, by, dsfx, dsfy, ff, eq0, whichefvs=whichefvs,
                                          efvs_constant=2.5e6, effstrain_min=1.0e-8, n_glen=3.0)
    assert o[0] == 0
    got = assemble_layered_2d("diva", nx, ny, nz, sig, g["ac"], g["xVertex"], g["yVertex"], u, v, g["stagthck"], ff,
                              whichefvs, 2.5e6, 1.0e-8, 3.0,
                              diva=(stagsig, g["thck"], bx, by, dsfx, dsfy, eq0))
    efvs, eq, ok, om, A = got
    assert np.count_nonzero(om) > 0
    for g_, w in zip((efvs, eq, ok, om, *A), o[1:]):
        np.testing.assert_array_equal(g_, w)


def basal_standard_2d(nx, ny, active_cell, xv, yv, beta_x, beta_y, Auu, Avv, lsrf=None, nhalo=2):
    """The standard finite-element basal terms of the 2D systems, on copies of the (9, ny-1, nx-1)
    blocks.  lsrf None: basal_sliding_bc_2d (glissade_velo_higher.F90:8393-8531), one beta, the
    flat Jacobian determinant of get_basis_function_derivatives_2d (:6319-6504) and Kvv = Kuu.
    lsrf given: basal_sliding_bc_2d_diva (:8682-8811), beta_eff_x into Auu and beta_eff_y into Avv
    with the area factor of the staggered lower surface (get_area_scale_factor_curved_2d
    :6736-6827)."""
    vol0 = 1.0e9
    A = [np.array(Auu, dtype=np.float64, copy=True), np.array(Avv, dtype=np.float64, copy=True)]
    sl = None if lsrf is None else _stagger(lsrf)
    for j in range(nhalo + 1, ny - nhalo + 2):
        for i in range(nhalo + 1, nx - nhalo + 2):
            if not active_cell[j - 1, i - 1]:
                continue
            verts = ((i - 1, j - 1), (i, j - 1), (i, j), (i - 1, j))
            pick = lambda f: [float(f[jv - 1, iv - 1]) for iv, jv in verts]
            x, y, bx, by = pick(xv), pick(yv), pick(beta_x), pick(beta_y)
            for p in range(4):
                phi, dxr, dyr = _ref_square(p)
                if sl is None:
                    j11 = j12 = j21 = j22 = 0.0
                    for n in range(4):
                        j11 = j11 + dxr[n] * x[n]
                        j12 = j12 + dxr[n] * y[n]
                        j21 = j21 + dyr[n] * x[n]
                        j22 = j22 + dyr[n] * y[n]
                    det = j11 * j22 - j12 * j21
                    if not abs(det) > 0.0:
                        raise ZeroDivisionError("Jacobian matrix is singular")
                else:
                    z = pick(sl)
                    j11 = j12 = j13 = j21 = j22 = j23 = 0.0
                    for n in range(4):
                        j11 = j11 + dxr[n] * x[n]
                        j12 = j12 + dxr[n] * y[n]
                        j13 = j13 + dxr[n] * z[n]
                        j21 = j21 + dyr[n] * x[n]
                        j22 = j22 + dyr[n] * y[n]
                        j23 = j23 + dyr[n] * z[n]
                    t1 = j11 * j22 - j12 * j21
                    t2 = -(j11 * j23 - j13 * j21)
                    t3 = j12 * j23 - j13 * j22
                    det = math.sqrt((t1 * t1 + t2 * t2) + t3 * t3)
                bqx = bqy = 0.0
                for n in range(4):
                    bqx = bqx + phi[n] * bx[n]
                    bqy = bqy + phi[n] * by[n]
                Ku = [[0.0] * 4 for _ in range(4)]
                Kv = [[0.0] * 4 for _ in range(4)]
                for nc in range(4):
                    for nr in range(4):
                        Ku[nr][nc] = Ku[nr][nc] + bqx * 1.0 * det / vol0 * phi[nr] * phi[nc]
                        Kv[nr][nc] = Kv[nr][nc] + bqy * 1.0 * det / vol0 * phi[nr] * phi[nc]
                if sl is None:
                    Kv = Ku
                for nr in range(4):
                    iv, jv = i + _ISHIFT[2][nr], j + _JSHIFT[2][nr]
                    for nc in range(4):
                        m = _m(_ISHIFT[nr][nc], _JSHIFT[nr][nc])
                        A[0][m, jv - 1, iv - 1] = float(A[0][m, jv - 1, iv - 1]) + Ku[nr][nc]
                        A[1][m, jv - 1, iv - 1] = float(A[1][m, jv - 1, iv - 1]) + Kv[nr][nc]
    return A[0], A[1]


@pytest.mark.parametrize("seed", [91, 92])
def test_second_restatement_basal_standard_2d(seed):
    """The standard basal terms of the SSA/L1L2 systems (one beta, flat element) and of DIVA
    (beta_eff_x, beta_eff_y, curved lower surface): every coefficient bit-identical with the oracle."""
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=seed)
    nx, ny = g["nx"], g["ny"]
    rng = np.random.default_rng(seed)
    shape = (ny - 1, nx - 1)
    beta = np.exp(np.log(1.0e3) + rng.standard_normal(shape))
    bey = beta * np.exp(0.3 * rng.standard_normal(shape))
    lsrf, _, _ = _basal_local_inputs(seed, nx, ny)
    Auu = rng.standard_normal((9,) + shape)
    Avv = rng.standard_normal((9,) + shape)
    st, ou, ov = oracle.basal_standard(False, nx, ny, 2, g["ac"], g["xVertex"], g["yVertex"], beta, None, Auu, Avv)
    assert st == 0
    gu, gv = basal_standard_2d(nx, ny, g["ac"], g["xVertex"], g["yVertex"], beta, beta, Auu, Avv)
    assert not np.array_equal(gu, Auu)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gv, ov)
    av = np.ones(shape, dtype=np.int32)
    ou, ov = oracle.basal_diva(nx, ny, 1.0, 1.0, g["ac"], av, beta, bey, lsrf, g["xVertex"], g["yVertex"], 0, Auu,
                               Avv)
    gu, gv = basal_standard_2d(nx, ny, g["ac"], g["xVertex"], g["yVertex"], beta, bey, Auu, Avv, lsrf=lsrf)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gv, ov)


# ---------------------------------------------------------------------------------------------
# The reproducible sum: cism_reprosum_calc / cism_reprosum_int (libglimmer/cism_reprosum_mod.F90)
# as parallel_reduce_reprosum calls it (parallel_mpi.F90:9637-9730): one field, no bounds given
# (the recompute path), validation off for the recompute, one task and one thread.
# ---------------------------------------------------------------------------------------------
_I8_DIGITS, _R8_DIGITS, _R8_MINEXP, _R8_MAXEXP = 63, 53, -1021, 1024


def _exponent(x):
    """Fortran exponent(): x = fraction * 2**exponent with |fraction| in [0.5, 1); 0 for 0."""
    return 0 if x == 0.0 else math.frexp(x)[1]


def _set_exponent(x, e):
    return math.ldexp(math.frexp(x)[0], e)


def _idiv(a, b):
    """Fortran integer division of a by b > 0: the quotient truncated toward zero."""
    q = abs(a) // b
    return q if a >= 0 else -q


def _isign(x):
    """sign(1_i8, x): +1 for x >= 0."""
    return -1 if x < 0 else 1


def reprosum(arr):
    arr = [float(v) for v in np.ravel(arr)]
    n = len(arr)
    # exponent extremes (cism_reprosum_mod.F90:820-867; one task, so the global ones are the same)
    tlmin, tlmax = _R8_MAXEXP, _R8_MINEXP
    for v in arr:
        if v != 0.0:
            e = _exponent(v)
            tlmin, tlmax = min(e, tlmin), max(e, tlmax)
    gmax = tlmax
    gmin = min(gmax, tlmin)
    max_nsummands = max(n // 1 + 1, 1 * 1)
    ams = _I8_DIGITS - (_exponent(float(max_nsummands)) + 1)  # arr_max_shift
    assert ams >= 2, "number of summands too large for integer vector algorithm"
    max_levels = 2 + (_R8_DIGITS + (gmax - gmin)) // ams
    extra_levels = (_I8_DIGITS - 1) // ams
    min_level = -(extra_levels - 1)
    radix_s = 2 ** ams
    lev = {il: 0 for il in range(min_level, max_levels + 1)}
    # the integer expansion of every summand (cism_reprosum_int, :1256-1370)
    for v in arr:
        if v == 0.0:
            continue
        e, frac = _exponent(v), math.frexp(v)[0]
        shift = ams - (gmax - e)
        if shift < 1:
            il = (1 + (gmax - e)) // ams
            shift = il * ams - (gmax - e)
            while shift < 1:
                shift += ams
                il += 1
        else:
            il = 1
        if il <= max_levels:
            rem = math.ldexp(frac, shift)
            k = int(rem)
            lev[il] += k
            rem = rem - k
            while rem != 0.0 and il < max_levels:
                il += 1
                rem = math.ldexp(rem, ams)
                k = int(rem)
                lev[il] += k
                rem = rem - k

    def carry(g):
        for il in range(max_levels, min_level, -1):
            if abs(g[il]) >= radix_s:
                q = _idiv(g[il], radix_s)
                g[il - 1] += q
                g[il] -= q * radix_s

    carry(lev)       # the thread's own normalisation (:1374-1387)
    g = dict(lev)    # the global level sums (one task) and their normalisation (:1564-1577)
    carry(g)
    il = min_level
    while g[il] == 0 and il < max_levels:
        il += 1
    sgn = -1 if g[il] < 0 else 1
    if il < max_levels:  # make every level's sign the leading one's (:1596-1645)
        for jl in range(il, max_levels):
            if _isign(g[jl]) != _isign(g[jl + 1]) or g[jl + 1] == 0:
                g[jl] -= sgn
                g[jl + 1] += sgn * radix_s
    if sgn < 0:
        for jl in range(il, max_levels + 1):
            g[jl] = -g[jl]
    carry(g)
    # conversion into pieces of 53 binary digits, added smallest first (:1653-1780)
    first = True
    shift = gmax - min_level * ams
    count = 0
    begin = min_level
    pieces = []
    while begin <= max_levels:
        tloc, tlev = 0, max_levels
        for il in range(begin, max_levels + 1):
            if first:
                if count == 0:
                    lx = _exponent(float(g[il])) if g[il] != 0 else 0
                else:
                    lx = ams
            else:
                lx = 0 if (il == begin and count != 0) else ams
            if count + lx >= _R8_DIGITS:
                tlev, tloc = il, (count + lx) - _R8_DIGITS
                break
            count += lx
        first = False
        if tloc == 0:
            trem = 0
        else:
            q = _idiv(g[tlev], 2 ** tloc) * 2 ** tloc
            trem = g[tlev] - q
            g[tlev] = q
        piece = 0.0
        for il in range(begin, tlev + 1):
            if g[il] != 0:
                x = float(g[il])
                cur = _exponent(x) + shift
                if cur >= _R8_MINEXP:
                    piece = piece + _set_exponent(x, cur)
                else:
                    piece = piece + math.ldexp(_set_exponent(x, cur - _R8_MINEXP), _R8_MINEXP)
            if il < tlev or tloc == 0:
                shift -= ams
        pieces.append(piece)
        if tloc == 0:
            count, begin = 0, tlev + 1
        else:
            count, begin = tloc, tlev
            g[tlev] = trem
    total = 0.0
    for piece in reversed(pieces):
        total = total + piece
    return sgn * total


def test_second_restatement_reprosum():
    """The reproducible sum, bit-identical with the oracle's on random arrays (normal values, wide
    exponent spreads reaching the subnormals, zeros and cancellation), on the near-tie case its
    conversion double-rounds, independent of the summands' order, and equal to the correctly
    rounded sum elsewhere."""
    rng = np.random.default_rng(21)
    cases = []
    for t in range(120):
        n = int(rng.integers(1, 400))
        if t % 4 == 0:
            a = rng.standard_normal(n)
        elif t % 4 == 1:
            a = rng.standard_normal(n) * np.exp(rng.uniform(-700, 700, n))
        elif t % 4 == 2:
            a = np.where(rng.random(n) < 0.5, 0.0, rng.standard_normal(n) * 1e7)
        else:
            b = rng.standard_normal(n // 2 + 1) * np.exp(rng.uniform(-40, 40, n // 2 + 1))
            a = np.concatenate([b, -b[: n // 2] * (1.0 + 2.0**-52)])  # heavy cancellation
        cases.append(a)
    cases += [np.array([1.0, 2.0**-53, 2.0**-106, -1e-40]), np.zeros(5), np.array([-3.5]),
              np.array([5e-324, -1e-320, 2.5e-310]), np.array([1.7e308, -1.6e308, 1e292])]
    for a in cases:
        got = reprosum(a)
        assert got == oracle.reprosum(a), a
        if a.size == 4 and a[1] == 2.0**-53:
            assert got == 1.0 and math.fsum(a) == 1.0 + 2.0**-52
        elif a.size > 5:
            assert got == math.fsum(a)
    b = cases[1]
    assert len({reprosum(rng.permutation(b)) for _ in range(5)}) == 1


def load_vector_local(nx, ny, nz, stagwbndsigma, dx, dy, active_vertex, stagthck, dsx, dsy):
    """load_vector_gravity, local form (glissade_velo_higher.F90:4311-4342): at every active vertex
    and level the driving stress over the node's share of the column, -rhoi*grav*dx*dy*dz/vol0 *
    ds, dz the thickness between the staggered level boundaries."""
    vol0, rhoi, grav = 1.0e9, 910.0, 9.81
    lu, lv = np.zeros((ny - 1, nx - 1, nz)), np.zeros((ny - 1, nx - 1, nz))
    for j in range(ny - 1):
        for i in range(nx - 1):
            if not active_vertex[j, i]:
                continue
            for k in range(1, nz + 1):
                dz = float(stagthck[j, i]) * (float(stagwbndsigma[k]) - float(stagwbndsigma[k - 1]))
                lu[j, i, k - 1] = float(lu[j, i, k - 1]) - rhoi * grav * dx * dy * dz / vol0 * float(dsx[j, i])
                lv[j, i, k - 1] = float(lv[j, i, k - 1]) - rhoi * grav * dx * dy * dz / vol0 * float(dsy[j, i])
    return lu, lv


def test_second_restatement_load_vector_local():
    """load_vector_gravity, local form: bit-identical with the oracle, unequal dx and dy."""
    from tests.test_oracle_assembly import geometry
    g = geometry(seed=45)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(10)
    sx, sy = 0.01 * rng.standard_normal((ny - 1, nx - 1)), 0.01 * rng.standard_normal((ny - 1, nx - 1))
    sig = g["sigma"]
    stagw = np.concatenate([[0.0], 0.5 * (sig[:-1] + sig[1:]), [1.0]])
    dx, dy = 1000.0, 1250.0
    st, ou, ov = oracle.load_vector_gravity(nx, ny, nz, sig, stagw, dx, dy, g["ac"], g["av"], g["xVertex"],
                                            g["yVertex"], g["stagusrf"], g["stagthck"], sx, sy, 1)
    assert st == 0
    lu, lv = load_vector_local(nx, ny, nz, stagw, dx, dy, g["av"], g["stagthck"], sx, sy)
    assert np.count_nonzero(lu) > 0
    np.testing.assert_array_equal(lu, ou)
    np.testing.assert_array_equal(lv, ov)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
def test_second_restatement_2d_from_x0(name, make, alg, precond):
    """Both 2D solvers from a random starting guess, with every preconditioner value, precond 2
    included (no branch taken: the standard solver breaks down at once on its zeroed z, the
    Chronopoulos-Gear solver iterates on z = A x0): bit-identical with the oracle."""
    P = make()
    x0 = problems.random_x0(P, seed=8, scale=10.0)
    try:
        with np.errstate(divide="ignore", invalid="ignore"):  # precond 2's first alpha is 0/0
            xu, xv, err, nit = (pcg_standard_2d_diag(P, 60, precond=precond, x0=x0) if alg == "standard" else
                                pcg_chrongear_2d(P, precond, 60, x0=x0))
    except ZeroDivisionError:
        xu = xv = None
        err, nit = float("nan"), -1
    st, ou, ov, oerr, onit = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=60, summode=oracle.SUM_SEQ, x0=x0)
    if st != 0:
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


CASES3_X0 = [c for c in CASES3 if c[0] != "dome"]  # the dome runs from zero above, at four counts


@pytest.mark.parametrize("name,make", CASES3_X0, ids=[c[0] for c in CASES3_X0])
@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
def test_second_restatement_3d_from_x0(name, make, alg, precond):
    """Both 3D solvers from a random starting guess (the GPU parity tests' form), with every
    preconditioner: bit-identical with the oracle through 40 iterations or the breakdown."""
    P = make()
    x0 = problems.random_x0(P, seed=7, scale=10.0)
    solver = pcg_standard_3d if alg == "standard" else pcg_chrongear_3d
    try:
        xu, xv, err, nit = solver(P, precond, 40, x0=x0)
    except ZeroDivisionError:
        xu = xv = None
        err, nit = float("nan"), -1
    st, ou, ov, oerr, onit = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=40, summode=oracle.SUM_SEQ, x0=x0)
    if st != 0:
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


def _solve_both(alg, P, precond, maxiters, x0):
    """One solve by this restatement and by the oracle (reference order); the restatement's
    breakdown (a NaN alpha or eta1, GM_FATAL in the reference) as niters < 0."""
    is3d = P.kind == "3d"
    with np.errstate(divide="ignore", invalid="ignore"):
        if alg == "standard":
            got = (pcg_standard_3d(P, precond, maxiters, x0=x0) if is3d else
                   pcg_standard_2d_diag(P, maxiters, precond=precond, x0=x0))
        else:
            got = (pcg_chrongear_3d(P, precond, maxiters, x0=x0) if is3d else
                   pcg_chrongear_2d(P, precond, maxiters, x0=x0))
    want = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=maxiters, summode=oracle.SUM_SEQ, x0=x0)
    return got, want


def _assert_same(got, want):
    xu, xv, err, nit = got
    st, ou, ov, oerr, onit = want
    if st != 0:
        assert nit < 0
        return
    assert nit == onit
    assert (err == oerr) or (math.isnan(err) and math.isnan(oerr))
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


EDGE = [("2d", lambda: problems.slab_2d(seed=1)), ("3d", lambda: problems.slab_3d(seed=5, sliding=False))]


@pytest.mark.parametrize("kind,make", EDGE, ids=[e[0] for e in EDGE])
@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 2, 3])
def test_second_restatement_zero_rhs(kind, make, alg, precond):
    """A zero right-hand side.  From x0 = 0 every sum is zero and the first alpha is 0/0: the
    reference stops with GM_FATAL, and so do both restatements.  From a nonzero x0, |b| = 0 makes
    every convergence check's err +inf (|r|/0), so the solve runs to maxiters: x, err and niters
    bit-identical with the oracle."""
    import dataclasses
    P = make()
    Z = dataclasses.replace(P, bu=np.zeros_like(P.bu), bv=np.zeros_like(P.bv))
    got, want = _solve_both(alg, Z, precond, 12, None)
    assert want[0] != 0 and got[3] < 0
    x0 = problems.random_x0(P, seed=9, scale=10.0)
    got, want = _solve_both(alg, Z, precond, 12, x0)
    _assert_same(got, want)
    if want[0] == 0:  # Chronopoulos-Gear 2D gives line-preconditioned solves 100 iterations,
        cap = 100 if (kind == "2d" and alg == "chrongear" and precond == 3) else 12  # whatever maxiters (:1728-1732)
        assert want[4] == cap and want[3] == float("inf")


@pytest.mark.parametrize("kind,make", EDGE, ids=[e[0] for e in EDGE])
@pytest.mark.parametrize("alg", ["standard", "chrongear"])
def test_second_restatement_no_active_vertices(kind, make, alg):
    """No active vertex: zero rows everywhere, so the matvec is zero.  With the diagonal
    preconditioner (zero diagonals: z = 0) the first alpha is 0/0; with none, z = r gives alpha =
    eta1/0 = +inf, x and r turn non-finite and the second iteration meets a NaN (eta1 in the
    standard solver, alpha in Chronopoulos-Gear).  Both restatements stop where the reference's
    GM_FATAL checks do, from zero and from a random x0."""
    import dataclasses
    P = make()
    Z = dataclasses.replace(P, active_vertex=np.zeros_like(P.active_vertex), Auu=np.zeros_like(P.Auu),
                            Auv=np.zeros_like(P.Auv), Avu=np.zeros_like(P.Avu), Avv=np.zeros_like(P.Avv))
    for x0 in (None, problems.random_x0(P, seed=9, scale=10.0)):
        for precond in (0, 1):
            got, want = _solve_both(alg, Z, precond, 12, x0)
            _assert_same(got, want)
