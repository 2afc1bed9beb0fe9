"""CPU oracle for the structured PCG solve -- TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/liboracle.so (built by oracle/Makefile), loop-for-loop C++
restatements of:
- pcg_oracle.cpp: libglissade/glissade_velo_higher_pcg.F90 and the one-rank semantics
  of libglimmer/parallel_mpi.F90's global sum (incl. reprosum) and staggered halo; the
  residual routines and the symmetry check of glissade_velo_higher.F90;
- assembly_oracle.cpp: the stiffness assembly (assemble_stiffness_matrix_3d/_2d) and
  the Dirichlet and local basal terms of glissade_velo_higher.F90.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline arm may use it, and only as
the checker or the timed CPU baseline.

Parity is unpinned against reference outputs (no Fortran compiler here and no
golden vectors in the reference); it is checked against mathematical known answers and,
bit for bit, against a second restatement of the solver path written separately in Python
(tests/test_oracle_restatement.py); see pcg_oracle.cpp's header.

Sum modes: SUM_SEQ (the reference's order), SUM_EXACT (exact, reproducible),
SUM_DDTREE (restatement of the GPU library's reduction tree), SUM_REPRO (restatement of
the reference's reprosum branch, cism_reprosum_mod.F90, as CISM calls it on one rank).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

SUM_SEQ, SUM_EXACT, SUM_DDTREE, SUM_REPRO = 0, 1, 2, 3

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class _Par(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "staggered_ilo", "staggered_ihi", "staggered_jlo", "staggered_jhi", "periodic_bc", "outflow_bc",
        "no_ice_bc", "reprosum", "tasks_row", "tasks_col")]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        d, i, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        P = ctypes.POINTER
        tail = [d, d, d, d, d, d, d, d, i, i, dbl, i, P(dbl), P(i), i, i, i, i]
        L.oracle_pcg_standard_3d.argtypes = [i, i, i, P(_Par), d, d, d] + tail
        L.oracle_pcg_chrongear_3d.argtypes = [i, i, i, P(_Par), d, d, d] + tail
        L.oracle_pcg_standard_2d.argtypes = [i, i, P(_Par), d, d] + tail
        L.oracle_pcg_chrongear_2d.argtypes = [i, i, P(_Par), d, d] + tail
        L.oracle_matvec_3d.argtypes = [i, i, i, P(_Par), d, d, d, d, d, d, d, d, d, d]
        L.oracle_matvec_2d.argtypes = [i, i, P(_Par), d, d, d, d, d, d, d, d, d, d]
        L.oracle_halo.argtypes = [i, i, i, P(_Par), d]
        L.oracle_global_sum.argtypes = [i, i, i, P(_Par), d, d, i]
        L.oracle_global_sum.restype = dbl
        L.oracle_easy_sia.argtypes = [i, i, i, d, d, d, d]
        L.oracle_precond_apply.argtypes = [i, i, i, i, P(_Par), d, d, d, d, d, i, d, d, d, d]
        L.oracle_compute_residual_vector.argtypes = [i, i, i, i, P(_Par), d, d, d, d, d, d, d, d, d, d, d, d,
                                                     P(dbl), P(dbl), i]
        L.oracle_compute_residual_velocity.argtypes = [i, i, i, i, i, P(_Par), d, d, d, d, i]
        L.oracle_compute_residual_velocity.restype = dbl
        L.oracle_exact_sum.argtypes = [d, ctypes.c_long]
        L.oracle_reprosum.argtypes = [d, ctypes.c_long]
        L.oracle_assemble_stiffness_3d.argtypes = [i, i, i, i, d, d, d, d, d, d, d, d, d, i, i, dbl, dbl, dbl,
                                                   d, d, d, d, d]
        L.oracle_assemble_stiffness_2d.argtypes = [i, i, i, i, d, d, d, d, d, d, d, d, i, dbl, dbl, dbl, d, d, d, d, d]
        L.oracle_dirichlet_3d.argtypes = [i, i, i, i, d, d, d, d, d, d, d, d, d, d, d]
        L.oracle_dirichlet_3d.restype = None
        L.oracle_basal_local_3d.argtypes = [i, i, i, dbl, dbl, d, d, d, d, d, d]
        L.oracle_basal_local_3d.restype = None
        L.oracle_dirichlet_2d.argtypes = [i, i, i, d, d, d, d, d, d, d, d, d, d, d]
        L.oracle_dirichlet_2d.restype = None
        L.oracle_basal_local_2d.argtypes = [i, i, dbl, dbl, d, d, d, d]
        L.oracle_basal_local_2d.restype = None
        L.oracle_basal_standard.argtypes = [i, i, i, i, i, d, d, d, d, d, d, d]
        L.oracle_assemble_stiffness_2d_diva.argtypes = [i, i, i, i] + [d] * 14 + [i, dbl, dbl, dbl] + [d] * 8
        L.oracle_basal_diva.argtypes = [i, i, i, dbl, dbl, d, d, d, d, d, d, d, i, d, d]
        L.oracle_basal_diva.restype = None
        L.oracle_assemble_stiffness_2d_l1l2.argtypes = [i, i, i, i] + [d] * 11 + [i, dbl, dbl, dbl] + [d] * 5
        L.oracle_load_vector_gravity.argtypes = [i, i, i, i, d, d, dbl, dbl, d, d, d, d, d, d, d, d, i, d, d]
        L.oracle_check_symmetry.argtypes = [i, i, i, i, P(_Par), d, d, d, d, d, d, P(dbl), P(ctypes.c_long)]
        L.oracle_reprosum.restype = dbl
        L.oracle_exact_sum.restype = dbl
        _lib = L
    return _lib


def _p(a):
    assert isinstance(a, np.ndarray) and (a.flags.c_contiguous or a.flags.f_contiguous)
    return ctypes.c_void_p(a.ctypes.data)


def _par(par: dict) -> _Par:
    return _Par(*(int(par[f]) for f, _ in _Par._fields_))


def indx3():
    return np.arange(1, 28, dtype=np.int32)


def indx2():
    return np.arange(1, 10, dtype=np.int32)


def pcg(alg: str, prob, precond: int, ncheck: int = 5, tol: float = 1e-8, maxiters: int = 200,
        summode: int = SUM_SEQ, x0=None):
    """Run one oracle solve on a cism_b200.assembly.Problem; returns (status, xu, xv, err, niters)."""
    L = lib()
    xu = np.array(prob.bu * 0.0 if x0 is None else x0[0], dtype=np.float64, copy=True)
    xv = np.array(prob.bv * 0.0 if x0 is None else x0[1], dtype=np.float64, copy=True)
    err = ctypes.c_double(0.0)
    nit = ctypes.c_int(0)
    par = _par(prob.par)
    i2 = indx2()
    i3 = indx3()
    common = [_p(prob.active_vertex), _p(prob.Auu), _p(prob.Auv), _p(prob.Avu), _p(prob.Avv), _p(prob.bu),
              _p(prob.bv), _p(xu), _p(xv), precond, ncheck, tol, maxiters, ctypes.byref(err), ctypes.byref(nit),
              1, 1, 0, summode]
    if prob.kind == "3d":
        f = L.oracle_pcg_standard_3d if alg == "standard" else L.oracle_pcg_chrongear_3d
        st = f(prob.nx, prob.ny, prob.nz, ctypes.byref(par), _p(i2), _p(i3), *common)
    else:
        f = L.oracle_pcg_standard_2d if alg == "standard" else L.oracle_pcg_chrongear_2d
        st = f(prob.nx, prob.ny, ctypes.byref(par), _p(i2), *common)
    return st, xu, xv, err.value, nit.value


def matvec(prob, xu, xv):
    L = lib()
    yu, yv = np.empty_like(xu), np.empty_like(xv)
    par = _par(prob.par)
    if prob.kind == "3d":
        L.oracle_matvec_3d(prob.nx, prob.ny, prob.nz, ctypes.byref(par), _p(indx3()), _p(prob.active_vertex),
                           _p(prob.Auu), _p(prob.Auv), _p(prob.Avu), _p(prob.Avv), _p(xu), _p(xv), _p(yu), _p(yv))
    else:
        L.oracle_matvec_2d(prob.nx, prob.ny, ctypes.byref(par), _p(indx2()), _p(prob.active_vertex),
                           _p(prob.Auu), _p(prob.Auv), _p(prob.Avu), _p(prob.Avv), _p(xu), _p(xv), _p(yu), _p(yv))
    return yu, yv


def halo(nx, ny, nz, par: dict, a: np.ndarray) -> np.ndarray:
    out = np.array(a, dtype=np.float64, copy=True)
    p = _par(par)
    lib().oracle_halo(nx, ny, nz, ctypes.byref(p), _p(out))
    return out


def global_sum(nx, ny, nz, par: dict, a1, a2, summode=SUM_SEQ) -> float:
    p = _par(par)
    return lib().oracle_global_sum(nx, ny, nz, ctypes.byref(p), _p(np.ascontiguousarray(a1)),
                                   _p(np.ascontiguousarray(a2)), summode)


def easy_sia(nx, ny, nz, active, M, b, x):
    out = np.array(x, dtype=np.float64, copy=True)
    lib().oracle_easy_sia(nx, ny, nz, _p(active), _p(np.ascontiguousarray(M)), _p(np.ascontiguousarray(b)),
                          _p(out))
    return out


def precond_apply(prob, precond: int, ru, rv, zu0=None, zv0=None):
    """z = PC(r) for one preconditioner of prob's matrix (setup + one apply); z starts from
    zu0/zv0 (default zero), which the SIA column solve keeps on inactive columns.
    Returns (status, zu, zv)."""
    is3d = prob.kind == "3d"
    zu = np.array(np.zeros_like(ru) if zu0 is None else zu0, dtype=np.float64, copy=True)
    zv = np.array(np.zeros_like(rv) if zv0 is None else zv0, dtype=np.float64, copy=True)
    par = _par(prob.par)
    st = lib().oracle_precond_apply(int(is3d), prob.nx, prob.ny, prob.nz if is3d else 1, ctypes.byref(par),
                                    _p(indx2()), _p(indx3()), _p(prob.active_vertex), _p(prob.Auu), _p(prob.Avv),
                                    precond, _p(np.ascontiguousarray(ru)), _p(np.ascontiguousarray(rv)), _p(zu),
                                    _p(zv))
    return st, zu, zv


def residual_vector(prob, uvel, vvel, summode: int = SUM_SEQ):
    """compute_residual_vector_{2d,3d} of prob's system at (uvel, vvel):
    (resid_u, resid_v, L2_norm, L2_norm_relative)."""
    is3d = prob.kind == "3d"
    ru, rv = np.empty_like(prob.bu), np.empty_like(prob.bv)
    l2, l2r = ctypes.c_double(0.0), ctypes.c_double(0.0)
    par = _par(prob.par)
    lib().oracle_compute_residual_vector(int(is3d), prob.nx, prob.ny, prob.nz if is3d else 1, ctypes.byref(par),
                                         _p(indx3() if is3d else indx2()), _p(prob.active_vertex), _p(prob.Auu),
                                         _p(prob.Auv), _p(prob.Avu), _p(prob.Avv), _p(prob.bu), _p(prob.bv),
                                         _p(np.ascontiguousarray(uvel)), _p(np.ascontiguousarray(vvel)), _p(ru),
                                         _p(rv), ctypes.byref(l2), ctypes.byref(l2r), summode)
    return ru, rv, l2.value, l2r.value


def residual_velocity(prob, whichresid: int, uvel, vvel, usav, vsav, summode: int = SUM_SEQ) -> float:
    """compute_residual_velocity_{2d,3d} on prob's grid."""
    is3d = prob.kind == "3d"
    par = _par(prob.par)
    arrs = [_p(np.ascontiguousarray(a, dtype=np.float64)) for a in (uvel, vvel, usav, vsav)]
    return lib().oracle_compute_residual_velocity(int(is3d), whichresid, prob.nx, prob.ny, prob.nz if is3d else 1,
                                                  ctypes.byref(par), *arrs, summode)


def check_symmetry(prob, Auu=None, Auv=None, Avu=None, Avv=None):
    """check_symmetry_assembled_matrix_{2d,3d} on prob's matrix (or the given blocks, prob's
    layout).  Returns (Auu, Auv, Avu, Avv, maxdiff, nwarn): copies of the blocks, with the 3D
    check's averages written in (the 2D check changes nothing), the largest asymmetry seen and
    the number of asymmetry warnings the reference prints."""
    is3d = prob.kind == "3d"
    blocks = [np.array(prob.Auu if Auu is None else Auu, dtype=np.float64, copy=True),
              np.array(prob.Auv if Auv is None else Auv, dtype=np.float64, copy=True),
              np.array(prob.Avu if Avu is None else Avu, dtype=np.float64, copy=True),
              np.array(prob.Avv if Avv is None else Avv, dtype=np.float64, copy=True)]
    md, nw = ctypes.c_double(0.0), ctypes.c_long(0)
    par = _par(prob.par)
    lib().oracle_check_symmetry(int(is3d), prob.nx, prob.ny, prob.nz if is3d else 1, ctypes.byref(par),
                                _p(indx3() if is3d else indx2()), _p(prob.active_vertex), *[_p(b) for b in blocks],
                                ctypes.byref(md), ctypes.byref(nw))
    return (*blocks, md.value, nw.value)


def assemble_stiffness_3d(nx, ny, nz, sigma, active_cell, xVertex, yVertex, uvel, vvel, stagusrf, stagthck,
                          flwafact, whichapprox=2, whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8,
                          n_glen=3.0, nhalo=2):
    """assemble_stiffness_matrix_3d (glissade_velo_higher.F90:5382-5643) on numpy arrays in
    the caller's layout as C-order arrays with reversed dimensions: active_cell (ny, nx),
    vertex fields (ny-1, nx-1), uvel/vvel (ny-1, nx-1, nz), flwafact (ny, nx, nz-1).
    Returns (status, efvs (ny, nx, nz-1), Auu, Auv, Avu, Avv (ny-1, nx-1, nz, 27))."""
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    efvs = np.zeros((ny, nx, nz - 1))
    A = [np.zeros((ny - 1, nx - 1, nz, 27)) for _ in range(4)]
    ins = [f64(sigma), np.ascontiguousarray(active_cell, dtype=np.int32), f64(xVertex), f64(yVertex), f64(uvel),
           f64(vvel), f64(stagusrf), f64(stagthck), f64(flwafact)]
    st = lib().oracle_assemble_stiffness_3d(nx, ny, nz, nhalo, *[_p(a) for a in ins], whichapprox, whichefvs,
                                            efvs_constant, effstrain_min, n_glen, _p(efvs), *[_p(a) for a in A])
    return (st, efvs, *A)


def assemble_stiffness_2d(nx, ny, nz, sigma, active_cell, xVertex, yVertex, uvel, vvel, stagthck, flwafact,
                          whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8, n_glen=3.0, nhalo=2):
    """assemble_stiffness_matrix_2d (glissade_velo_higher.F90:4961-5378), SSA: vertex fields
    (ny-1, nx-1), flwafact (ny, nx, nz-1).  Returns (status, efvs (ny, nx, nz-1), Auu, Auv,
    Avu, Avv (9, ny-1, nx-1))."""
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    efvs = np.zeros((ny, nx, nz - 1))
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    ins = [f64(sigma), np.ascontiguousarray(active_cell, dtype=np.int32), f64(xVertex), f64(yVertex), f64(uvel),
           f64(vvel), f64(stagthck), f64(flwafact)]
    st = lib().oracle_assemble_stiffness_2d(nx, ny, nz, nhalo, *[_p(a) for a in ins], whichefvs, efvs_constant,
                                            effstrain_min, n_glen, _p(efvs), *[_p(a) for a in A])
    return (st, efvs, *A)


def dirichlet_3d(nx, ny, nz, active_vertex, umask, vmask, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv, nhalo=2):
    """dirichlet_boundary_conditions_3d (glissade_velo_higher.F90:9305-9498) on copies:
    masks and velocities (ny-1, nx-1, nz), blocks (ny-1, nx-1, nz, 27).  Returns
    (Auu, Auv, Avu, Avv, bu, bv)."""
    out = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Auv, Avu, Avv, bu, bv)]
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    lib().oracle_dirichlet_3d(nx, ny, nz, nhalo, _p(i32(active_vertex)), _p(i32(umask)), _p(i32(vmask)),
                              _p(f64(uvel)), _p(f64(vvel)), *[_p(a) for a in out])
    return tuple(out)


def basal_local_3d(nx, ny, nz, dx, dy, active_vertex, beta, lsrf, Auu, Avv):
    """basal_sliding_bc_3d with HO_ASSEMBLE_BETA_LOCAL (glissade_velo_higher.F90:8815-9129) on
    copies of the blocks; returns (Auu, Avv, theta (ny-1, nx-1))."""
    out = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Avv)]
    theta = np.zeros((ny - 1, nx - 1))
    lib().oracle_basal_local_3d(nx, ny, nz, float(dx), float(dy),
                                _p(np.ascontiguousarray(active_vertex, dtype=np.int32)),
                                _p(np.ascontiguousarray(beta, dtype=np.float64)),
                                _p(np.ascontiguousarray(lsrf, dtype=np.float64)), _p(out[0]), _p(out[1]), _p(theta))
    return out[0], out[1], theta


def dirichlet_2d(nx, ny, active_vertex, umask, vmask, uvel, vvel, Auu, Auv, Avu, Avv, bu, bv, nhalo=2):
    """dirichlet_boundary_conditions_2d (glissade_velo_higher.F90:9133-9301) on copies: masks,
    velocities and b (ny-1, nx-1), blocks (9, ny-1, nx-1).  Returns (Auu, Auv, Avu, Avv, bu, bv)."""
    out = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Auv, Avu, Avv, bu, bv)]
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    lib().oracle_dirichlet_2d(nx, ny, nhalo, _p(i32(active_vertex)), _p(i32(umask)), _p(i32(vmask)), _p(f64(uvel)),
                              _p(f64(vvel)), *[_p(a) for a in out])
    return tuple(out)


def basal_local_2d(nx, ny, dx, dy, active_vertex, beta, Auu, Avv):
    """basal_sliding_bc_2d with HO_ASSEMBLE_BETA_LOCAL on copies; returns (Auu, Avv)."""
    out = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Avv)]
    lib().oracle_basal_local_2d(nx, ny, float(dx), float(dy), _p(np.ascontiguousarray(active_vertex, dtype=np.int32)),
                                _p(np.ascontiguousarray(beta, dtype=np.float64)), _p(out[0]), _p(out[1]))
    return out[0], out[1]


def basal_standard(is3d, nx, ny, nz, active_cell, xVertex, yVertex, beta, lsrf, Auu, Avv, nhalo=2):
    """basal_sliding_bc_3d / _2d, standard finite-element form (whichassemble_beta = 0), on copies
    of the blocks (3D (ny-1, nx-1, nz, 27), 2D (9, ny-1, nx-1)).  Returns (status, Auu, Avv)."""
    out = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Avv)]
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    st = lib().oracle_basal_standard(int(is3d), nx, ny, nz, nhalo, _p(np.ascontiguousarray(active_cell, dtype=np.int32)),
                                     _p(f64(xVertex)), _p(f64(yVertex)), _p(f64(beta)),
                                     _p(f64(np.zeros((ny, nx)) if lsrf is None else lsrf)), _p(out[0]), _p(out[1]))
    return st, out[0], out[1]


def assemble_stiffness_2d_diva(nx, ny, nz, sigma, stagsigma, active_cell, xVertex, yVertex, uvel, vvel, stagthck,
                               thck, btractx, btracty, dsfx, dsfy, flwafact, efvs_qp_3d, whichefvs=2,
                               efvs_constant=0.0, effstrain_min=1.0e-8, n_glen=3.0, nhalo=2):
    """assemble_stiffness_matrix_2d with HO_APPROX_DIVA: vertex fields (ny-1, nx-1), cell fields
    (ny, nx), flwafact (ny, nx, nz-1), efvs_qp_3d (ny, nx, 4, nz-1) (a copy is updated).
    Returns (status, efvs (ny, nx, nz-1), efvs_qp_3d, omega_k (ny, nx, nz), omega (ny, nx),
    Auu, Auv, Avu, Avv (9, ny-1, nx-1))."""
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    eq = np.array(efvs_qp_3d, dtype=np.float64, copy=True)
    efvs = np.zeros((ny, nx, nz - 1))
    ok = np.zeros((ny, nx, nz))
    om = np.zeros((ny, nx))
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    ins = [f64(sigma), f64(stagsigma), np.ascontiguousarray(active_cell, dtype=np.int32), f64(xVertex), f64(yVertex),
           f64(uvel), f64(vvel), f64(stagthck), f64(thck), f64(btractx), f64(btracty), f64(dsfx), f64(dsfy),
           f64(flwafact)]
    st = lib().oracle_assemble_stiffness_2d_diva(nx, ny, nz, nhalo, *[_p(a) for a in ins], whichefvs, efvs_constant,
                                                 effstrain_min, n_glen, _p(eq), _p(efvs), _p(ok), _p(om),
                                                 *[_p(a) for a in A])
    return (st, efvs, eq, ok, om, *A)


def basal_diva(nx, ny, dx, dy, active_cell, active_vertex, beta_eff_x, beta_eff_y, lsrf, xVertex, yVertex,
               whichassemble_beta, Auu, Avv, nhalo=2):
    """basal_sliding_bc_2d_diva (glissade_velo_higher.F90:8535-8811) on copies of the (9, ny-1,
    nx-1) blocks; returns (Auu, Avv)."""
    out = [np.array(a, dtype=np.float64, copy=True) for a in (Auu, Avv)]
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    lib().oracle_basal_diva(nx, ny, nhalo, float(dx), float(dy), _p(i32(active_cell)), _p(i32(active_vertex)),
                            _p(f64(beta_eff_x)), _p(f64(beta_eff_y)), _p(f64(lsrf)), _p(f64(xVertex)), _p(f64(yVertex)),
                            int(whichassemble_beta), _p(out[0]), _p(out[1]))
    return out[0], out[1]


def assemble_stiffness_2d_l1l2(nx, ny, nz, sigma, active_cell, xVertex, yVertex, uvel, vvel, stagthck, dusrf_dx,
                               dusrf_dy, flwa, flwafact, whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8,
                               n_glen=3.0, nhalo=2):
    """assemble_stiffness_matrix_2d with HO_APPROX_L1L2: vertex fields (ny-1, nx-1), flwa and
    flwafact (ny, nx, nz-1).  Returns (status, efvs (ny, nx, nz-1), Auu, Auv, Avu, Avv)."""
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    efvs = np.zeros((ny, nx, nz - 1))
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    ins = [f64(sigma), np.ascontiguousarray(active_cell, dtype=np.int32), f64(xVertex), f64(yVertex), f64(uvel),
           f64(vvel), f64(stagthck), f64(dusrf_dx), f64(dusrf_dy), f64(flwa), f64(flwafact)]
    st = lib().oracle_assemble_stiffness_2d_l1l2(nx, ny, nz, nhalo, *[_p(a) for a in ins], whichefvs, efvs_constant,
                                                 effstrain_min, n_glen, _p(efvs), *[_p(a) for a in A])
    return (st, efvs, *A)


def load_vector_gravity(nx, ny, nz, sigma, stagwbndsigma, dx, dy, active_cell, active_vertex, xVertex, yVertex,
                        stagusrf, stagthck, dusrf_dx, dusrf_dy, whichassemble_taud, nhalo=2):
    """load_vector_gravity (glissade_velo_higher.F90:4228-4449) from zero: vertex fields
    (ny-1, nx-1), stagwbndsigma (nz+1).  Returns (status, loadu, loadv (ny-1, nx-1, nz))."""
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    lu, lv = np.zeros((ny - 1, nx - 1, nz)), np.zeros((ny - 1, nx - 1, nz))
    st = lib().oracle_load_vector_gravity(nx, ny, nz, nhalo, _p(f64(sigma)), _p(f64(stagwbndsigma)), float(dx),
                                          float(dy), _p(i32(active_cell)), _p(i32(active_vertex)), _p(f64(xVertex)),
                                          _p(f64(yVertex)), _p(f64(stagusrf)), _p(f64(stagthck)), _p(f64(dusrf_dx)),
                                          _p(f64(dusrf_dy)), int(whichassemble_taud), _p(lu), _p(lv))
    return st, lu, lv


def reprosum(a) -> float:
    """The reference's reproducible sum (cism_reprosum_calc as CISM calls it, one rank)."""
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    return lib().oracle_reprosum(_p(a), a.size)


def exact_sum(a) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return lib().oracle_exact_sum(_p(a), a.size)
