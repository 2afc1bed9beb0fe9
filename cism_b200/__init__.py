"""B200-native structured PCG velocity solve for CISM's Glissade higher-order solver.

Python mirror of the reference solver interface
(libglissade/glissade_velo_higher_pcg.F90, public list :56-58).  Each function
calls the compiled sm_100a library ``_lib/libcismgpu.so`` through its C ABI
(include/cismgpu.h); there is no Python or CPU fallback: if the library or a
B200 is missing, the call raises.

Array arguments use the memory layout the Fortran caller passes.  Either give
arrays with the reference's dimensions in Fortran order, e.g. Auu of shape
(27, nz, nx-1, ny-1) with order='F', or the same memory as C-order arrays with the
dimensions reversed, e.g. shape (ny-1, nx-1, nz, 27).  xu and xv are updated in
place (intent(inout)), and (err, niters) is returned.  A nonzero library status
raises CismGpuError, which is where the reference calls
write_log(..., GM_FATAL).
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

__all__ = [
    "ParallelType", "CismGpuError", "load_library", "pcg_solver_standard_3d", "pcg_solver_chrongear_3d",
    "pcg_solver_standard_2d", "pcg_solver_chrongear_2d", "matvec_multiply_structured_3d",
    "matvec_multiply_structured_2d", "HO_PRECOND_NONE", "HO_PRECOND_DIAG", "HO_PRECOND_SIA",
    "HO_PRECOND_TRIDIAG_LOCAL", "HO_PRECOND_TRIDIAG_GLOBAL", "DeviceSolver", "solve_batch",
    "ALG_STANDARD", "ALG_CHRONGEAR", "ALG_MIXED_CHRONGEAR", "compute_residual_vector_3d",
    "compute_residual_vector_2d", "compute_residual_velocity_3d", "compute_residual_velocity_2d",
    "check_symmetry_assembled_matrix_3d", "check_symmetry_assembled_matrix_2d", "assemble_stiffness_matrix_3d",
    "assemble_stiffness_matrix_2d", "dirichlet_boundary_conditions_3d", "basal_sliding_bc_3d",
    "dirichlet_boundary_conditions_2d", "basal_sliding_bc_2d", "assemble_stiffness_matrix_2d_diva",
    "basal_sliding_bc_2d_diva", "assemble_stiffness_matrix_2d_l1l2", "load_vector_gravity",
]

ALG_STANDARD, ALG_CHRONGEAR, ALG_MIXED_CHRONGEAR = 0, 1, 2

# libglide/glide_types.F90:342-346
HO_PRECOND_NONE = 0
HO_PRECOND_DIAG = 1
HO_PRECOND_SIA = 2
HO_PRECOND_TRIDIAG_LOCAL = 3
HO_PRECOND_TRIDIAG_GLOBAL = 4

STATUS_NAMES = {
    0: "CISMGPU_OK", 1: "CISMGPU_EBREAKDOWN_ETA1", 2: "CISMGPU_EBREAKDOWN_ALPHA", 3: "CISMGPU_EUNSUPPORTED",
    4: "CISMGPU_EINVAL", 5: "CISMGPU_ECUDA", 6: "CISMGPU_ETIMEOUT", 7: "CISMGPU_ENOMEM", 8: "CISMGPU_ENODEV",
    9: "CISMGPU_EDIVZERO",
}

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcismgpu.so")


class CismGpuError(RuntimeError):
    """A nonzero status from the library (the reference's GM_FATAL cases and GPU errors)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class CParallel(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "staggered_ilo", "staggered_ihi", "staggered_jlo", "staggered_jhi", "periodic_bc", "outflow_bc",
        "no_ice_bc", "reprosum", "tasks_row", "tasks_col")]


class CRequest(ctypes.Structure):
    """cismgpu_request_t: one system for the serving loop."""
    _fields_ = [("dims", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("par", ctypes.POINTER(CParallel)), ("indxA", ctypes.c_void_p), ("active_vertex", ctypes.c_void_p),
                ("Auu", ctypes.c_void_p), ("Auv", ctypes.c_void_p), ("Avu", ctypes.c_void_p),
                ("Avv", ctypes.c_void_p), ("bu", ctypes.c_void_p), ("bv", ctypes.c_void_p),
                ("xu0", ctypes.c_void_p), ("xv0", ctypes.c_void_p), ("xu", ctypes.c_void_p), ("xv", ctypes.c_void_p),
                ("precond", ctypes.c_int), ("linear_solve_ncheck", ctypes.c_int), ("tolerance", ctypes.c_double),
                ("maxiters", ctypes.c_int)]


@dataclasses.dataclass
class ParallelType:
    """The fields of type(parallel_type) read on this path (libglimmer/parallel_mpi.F90:78-153)."""
    staggered_ilo: int
    staggered_ihi: int
    staggered_jlo: int
    staggered_jhi: int
    periodic_bc: bool = True
    outflow_bc: bool = False
    no_ice_bc: bool = False
    reprosum: bool = False
    tasks_row: int = 1
    tasks_col: int = 1

    @classmethod
    def from_dict(cls, d: dict) -> "ParallelType":
        return cls(**{f.name: d[f.name] for f in dataclasses.fields(cls) if f.name in d})

    def to_c(self) -> CParallel:
        return CParallel(*(int(getattr(self, f.name)) for f in dataclasses.fields(self)))


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libcismgpu.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with cism_b200.build.build() (no CPU fallback exists)")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    d, i32, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    par = P(CParallel)
    common_tail = [d, d, d, d, d, d, d, d, i32, i32, dbl, i32, P(dbl), P(i32), i32, i32, i32]
    lib.cismgpu_pcg_standard_3d.argtypes = [i32, i32, i32, par, d, d, d] + common_tail
    lib.cismgpu_pcg_chrongear_3d.argtypes = [i32, i32, i32, par, d, d, d] + common_tail
    lib.cismgpu_pcg_standard_2d.argtypes = [i32, i32, par, d, d] + common_tail
    lib.cismgpu_pcg_chrongear_2d.argtypes = [i32, i32, par, d, d] + common_tail
    for f in ("cismgpu_pcg_standard_3d", "cismgpu_pcg_chrongear_3d", "cismgpu_pcg_standard_2d",
              "cismgpu_pcg_chrongear_2d"):
        getattr(lib, f).restype = ctypes.c_int
    lib.cismgpu_matvec_structured_3d.argtypes = [i32, i32, i32, par, d, d, d, d, d, d, d, d, d, d]
    lib.cismgpu_matvec_structured_3d.restype = ctypes.c_int
    lib.cismgpu_matvec_structured_2d.argtypes = [i32, i32, par, d, d, d, d, d, d, d, d, d, d]
    lib.cismgpu_matvec_structured_2d.restype = ctypes.c_int
    vp = ctypes.c_void_p
    lib.cismgpu_solver_create.argtypes = [P(vp), i32, i32, i32, i32, par, d, d, d, d, d, d, d, d, d, d, vp]
    lib.cismgpu_solver_create.restype = ctypes.c_int
    lib.cismgpu_solver_solve.argtypes = [vp, i32, i32, i32, dbl, i32, P(dbl), P(i32)]
    lib.cismgpu_solver_solve.restype = ctypes.c_int
    lib.cismgpu_solver_solve_batch.argtypes = [P(vp), i32, i32, i32, i32, dbl, i32, P(dbl), P(i32), P(i32), vp]
    lib.cismgpu_solver_solve_batch.restype = ctypes.c_int
    lib.cismgpu_batch_create.argtypes = [P(vp), P(vp), i32, i32, i32, dbl, i32, vp]
    lib.cismgpu_batch_create.restype = ctypes.c_int
    lib.cismgpu_batch_run.argtypes = [vp]
    lib.cismgpu_batch_run.restype = ctypes.c_int
    lib.cismgpu_batch_wait.argtypes = [vp, P(dbl), P(i32), P(i32)]
    lib.cismgpu_batch_wait.restype = ctypes.c_int
    lib.cismgpu_batch_destroy.argtypes = [vp]
    lib.cismgpu_batch_destroy.restype = ctypes.c_int
    lib.cismgpu_server_create.argtypes = [P(vp), ctypes.c_size_t, i32]
    lib.cismgpu_server_create.restype = ctypes.c_int
    lib.cismgpu_server_submit.argtypes = [vp, P(CRequest), P(ctypes.c_longlong)]
    lib.cismgpu_server_submit.restype = ctypes.c_int
    lib.cismgpu_server_poll.argtypes = [vp, ctypes.c_longlong, P(i32), P(dbl), P(i32), P(i32), P(dbl), P(dbl)]
    lib.cismgpu_server_poll.restype = ctypes.c_int
    lib.cismgpu_server_drain.argtypes = [vp]
    lib.cismgpu_server_drain.restype = ctypes.c_int
    lib.cismgpu_server_stats.argtypes = [vp, P(ctypes.c_longlong), P(ctypes.c_size_t), P(i32), P(i32)]
    lib.cismgpu_server_stats.restype = ctypes.c_int
    lib.cismgpu_server_launch_stats.argtypes = [vp, P(ctypes.c_longlong), P(ctypes.c_longlong)]
    lib.cismgpu_server_launch_stats.restype = ctypes.c_int
    lib.cismgpu_server_destroy.argtypes = [vp]
    lib.cismgpu_server_destroy.restype = ctypes.c_int
    lib.cismgpu_solver_get_x.argtypes = [vp, d, d]
    lib.cismgpu_solver_get_x.restype = ctypes.c_int
    lib.cismgpu_solver_profile.argtypes = [vp, i32]
    lib.cismgpu_solver_profile.restype = ctypes.c_int
    lib.cismgpu_solver_profile_read.argtypes = [vp, P(dbl), P(i32), P(dbl)]
    lib.cismgpu_solver_profile_read.restype = ctypes.c_int
    lib.cismgpu_solver_device_bytes.argtypes = [vp]
    lib.cismgpu_solver_device_bytes.restype = ctypes.c_size_t
    lib.cismgpu_solver_destroy.argtypes = [vp]
    lib.cismgpu_solver_destroy.restype = ctypes.c_int
    lib.cismgpu_global_sum_stagger.argtypes = [i32, i32, i32, par, d, d, P(dbl)]
    lib.cismgpu_global_sum_stagger.restype = ctypes.c_int
    lib.cismgpu_global_sum_stagger_noalloc.argtypes = [i32, i32, i32, par, vp, vp, vp, vp]
    lib.cismgpu_global_sum_stagger_noalloc.restype = ctypes.c_int
    lib.cismgpu_compute_residual_vector_3d.argtypes = [i32, i32, i32, par, d, d, d, d, d, d, d, d, d, d, d, d,
                                                       P(dbl), P(dbl)]
    lib.cismgpu_compute_residual_vector_2d.argtypes = [i32, i32, par, d, d, d, d, d, d, d, d, d, d, d, d,
                                                       P(dbl), P(dbl)]
    lib.cismgpu_compute_residual_velocity_3d.argtypes = [i32, i32, i32, i32, par, d, d, d, d, P(dbl)]
    lib.cismgpu_compute_residual_velocity_2d.argtypes = [i32, i32, i32, par, d, d, d, d, P(dbl)]
    lib.cismgpu_solver_set_system.argtypes = [vp, d, d, d, d, d, d, i32]
    lib.cismgpu_solver_residual_vector.argtypes = [vp, d, d, P(dbl), P(dbl)]
    lib.cismgpu_solver_residual_velocity.argtypes = [vp, i32, P(dbl)]
    lib.cismgpu_solver_save.argtypes = [vp]
    lib.cismgpu_solver_restore.argtypes = [vp]
    i64 = ctypes.c_longlong
    lib.cismgpu_check_symmetry_assembled_matrix_3d.argtypes = [i32, i32, i32, par, d, d, d, d, d, d, P(dbl), P(i64)]
    lib.cismgpu_check_symmetry_assembled_matrix_2d.argtypes = [i32, i32, par, d, d, d, d, d, d, P(dbl), P(i64)]
    lib.cismgpu_solver_check_symmetry.argtypes = [vp, P(dbl), P(i64)]
    lib.cismgpu_assemble_stiffness_matrix_3d.argtypes = [i32, i32, i32, i32, d, d, d, d, d, d, d, d, d, i32, i32,
                                                         dbl, dbl, dbl, d, d, d, d, d, d]
    lib.cismgpu_solver_assemble_stiffness_3d.argtypes = [vp, i32, d, d, d, d, d, d, d, d, d, i32, i32, dbl, dbl,
                                                         dbl, d]
    lib.cismgpu_assemble_stiffness_matrix_2d.argtypes = [i32, i32, i32, i32, d, d, d, d, d, d, d, d, i32, dbl, dbl,
                                                         dbl, d, d, d, d, d, d]
    lib.cismgpu_solver_assemble_stiffness_2d.argtypes = [vp, i32, i32, d, d, d, d, d, d, d, d, i32, dbl, dbl, dbl, d]
    lib.cismgpu_dirichlet_boundary_conditions_3d.argtypes = [i32, i32, i32, i32, d, d, d, d, d, d, d, d, d, d, d, d]
    lib.cismgpu_basal_sliding_bc_3d.argtypes = [i32, i32, i32, i32, dbl, dbl, d, d, d, d, d, d, i32, d, d, d]
    lib.cismgpu_solver_assemble_system_3d.argtypes = [vp, i32, dbl, dbl, d, d, d, d, d, d, d, d, i32, i32, dbl, dbl,
                                                      dbl, d, d, i32, d, d, d, d, d]
    lib.cismgpu_assemble_stiffness_matrix_2d_diva.argtypes = [i32, i32, i32, i32] + [d] * 14 + [i32, dbl, dbl, dbl] + \
        [d] * 9
    lib.cismgpu_solver_assemble_stiffness_2d_diva.argtypes = [vp, i32, i32] + [d] * 14 + [i32, dbl, dbl, dbl] + [d] * 4
    lib.cismgpu_basal_sliding_bc_2d_diva.argtypes = [i32, i32, i32, dbl, dbl, d, d, d, d, d, d, d, i32, d, d, d]
    lib.cismgpu_load_vector_gravity.argtypes = [i32, i32, i32, i32, d, d, dbl, dbl, d, d, d, d, d, d, d, d, i32, d, d]
    lib.cismgpu_assemble_stiffness_matrix_2d_l1l2.argtypes = [i32, i32, i32, i32] + [d] * 11 + \
        [i32, dbl, dbl, dbl] + [d] * 6
    lib.cismgpu_solver_assemble_system_2d_diva.argtypes = [vp, i32, i32, dbl, dbl] + [d] * 13 + \
        [i32, dbl, dbl, dbl, d, d, d, i32] + [d] * 7
    lib.cismgpu_dirichlet_boundary_conditions_2d.argtypes = [i32, i32, i32, d, d, d, d, d, d, d, d, d, d, d, d]
    lib.cismgpu_basal_sliding_bc_2d.argtypes = [i32, i32, i32, dbl, dbl, d, d, d, d, d, i32, d, d, d]
    lib.cismgpu_solver_assemble_system_2d.argtypes = [vp, i32, i32, dbl, dbl, d, d, d, d, d, d, d, i32, dbl, dbl, dbl,
                                                      d, i32, d, d, d, d, d]
    for f in ("cismgpu_compute_residual_vector_3d", "cismgpu_compute_residual_vector_2d",
              "cismgpu_compute_residual_velocity_3d", "cismgpu_compute_residual_velocity_2d",
              "cismgpu_solver_set_system", "cismgpu_solver_residual_vector", "cismgpu_solver_residual_velocity",
              "cismgpu_solver_save", "cismgpu_solver_restore", "cismgpu_check_symmetry_assembled_matrix_3d",
              "cismgpu_check_symmetry_assembled_matrix_2d", "cismgpu_solver_check_symmetry",
              "cismgpu_assemble_stiffness_matrix_3d", "cismgpu_solver_assemble_stiffness_3d",
              "cismgpu_assemble_stiffness_matrix_2d", "cismgpu_solver_assemble_stiffness_2d",
              "cismgpu_dirichlet_boundary_conditions_3d", "cismgpu_basal_sliding_bc_3d",
              "cismgpu_solver_assemble_system_3d", "cismgpu_dirichlet_boundary_conditions_2d",
              "cismgpu_basal_sliding_bc_2d", "cismgpu_solver_assemble_system_2d",
              "cismgpu_assemble_stiffness_matrix_2d_diva", "cismgpu_solver_assemble_stiffness_2d_diva",
              "cismgpu_basal_sliding_bc_2d_diva", "cismgpu_solver_assemble_system_2d_diva",
              "cismgpu_assemble_stiffness_matrix_2d_l1l2", "cismgpu_load_vector_gravity"):
        getattr(lib, f).restype = ctypes.c_int
    lib.cismgpu_set_oneshot_algorithm.argtypes = [i32]
    lib.cismgpu_set_oneshot_algorithm.restype = ctypes.c_int
    lib.cismgpu_set_sum_order.argtypes = [i32]
    lib.cismgpu_set_sum_order.restype = ctypes.c_int
    lib.cismgpu_set_mixed_layout.argtypes = [i32]
    lib.cismgpu_set_mixed_layout.restype = ctypes.c_int
    lib.cismgpu_solver_mixed_layout.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    lib.cismgpu_solver_mixed_layout.restype = ctypes.c_int
    lib.cismgpu_tile_table.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.cismgpu_tile_table.restype = ctypes.c_size_t
    lib.cismgpu_test_set_device_waits.argtypes = [ctypes.c_longlong, ctypes.c_uint]
    lib.cismgpu_test_set_device_waits.restype = ctypes.c_int
    lib.cismgpu_last_error.restype = ctypes.c_char_p
    lib.cismgpu_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _ptr(a: np.ndarray, dtype, n: int, writable: bool = False):
    if not isinstance(a, np.ndarray) or a.dtype != dtype:
        raise TypeError(f"expected a numpy array of {np.dtype(dtype).name}")
    if a.size != n:
        raise ValueError(f"array has {a.size} elements, expected {n}")
    if not (a.flags.c_contiguous or a.flags.f_contiguous):
        raise ValueError("array must be contiguous in the caller's layout")
    if writable and not a.flags.writeable:
        raise ValueError("output array is read-only")
    return ctypes.c_void_p(a.ctypes.data)


def _par(parallel) -> CParallel:
    if isinstance(parallel, ParallelType):
        return parallel.to_c()
    if isinstance(parallel, dict):
        return ParallelType.from_dict(parallel).to_c()
    raise TypeError("parallel must be a ParallelType or dict")


def _check(lib, status: int):
    if status != 0:
        raise CismGpuError(status, lib.cismgpu_last_error().decode())


def _solve(fname: str, is3d: bool, nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv,
           bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest, jtest, rtest):
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    nvec = nv * (nz if is3d else 1)
    nblk = nvec * (27 if is3d else 9)
    err = ctypes.c_double(0.0)
    niters = ctypes.c_int(0)
    par = _par(parallel)
    i2 = _ptr(np.ascontiguousarray(indxA_2d, dtype=np.int32), np.int32, 9)
    head = [nx, ny] + ([nz] if is3d else []) + [ctypes.byref(par), i2]
    if is3d:
        head.append(_ptr(np.ascontiguousarray(indxA_3d, dtype=np.int32), np.int32, 27))
    args = head + [
        _ptr(active_vertex, np.int32, nv),
        _ptr(Auu, np.float64, nblk), _ptr(Auv, np.float64, nblk), _ptr(Avu, np.float64, nblk),
        _ptr(Avv, np.float64, nblk), _ptr(bu, np.float64, nvec), _ptr(bv, np.float64, nvec),
        _ptr(xu, np.float64, nvec, True), _ptr(xv, np.float64, nvec, True),
        int(precond), int(linear_solve_ncheck), float(tolerance), int(maxiters), ctypes.byref(err),
        ctypes.byref(niters), int(itest), int(jtest), int(rtest)]
    _check(lib, getattr(lib, fname)(*args))
    return err.value, niters.value


def parallel_global_sum_stagger(nx, ny, nz, parallel, arr1, arr2) -> float:
    """Mirrors parallel_global_sum_stagger(arr1, parallel, arr2) (libglimmer/parallel_mpi.F90:6537-6794)
    on one rank: the sum over owned vertices of arr1 + arr2 (nz = 1 for 2D fields)."""
    lib = load_library()
    n = (nx - 1) * (ny - 1) * nz
    out = ctypes.c_double(0.0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_global_sum_stagger(nx, ny, nz, ctypes.byref(par), _ptr(arr1, np.float64, n),
                                               _ptr(arr2, np.float64, n), ctypes.byref(out)))
    return out.value


NOALLOC_MAX_COLUMNS = 4194304  # CISMGPU_NOALLOC_MAX_COLUMNS


def parallel_global_sum_stagger_noalloc(nx, ny, nz, parallel, arr1_dev: int, arr2_dev: int, sum_dev: int,
                                        stream: int = 0) -> None:
    """The owned-vertex sum of parallel_global_sum_stagger for callers that cannot let the
    library allocate device memory: arr1_dev, arr2_dev and sum_dev are device addresses (e.g. a
    torch tensor's data_ptr()), the kernel is enqueued on `stream` (a cudaStream_t as an int, 0 for
    the default stream) and writes the sum to sum_dev without synchronizing.  The scratch is a fixed
    array inside the library, shared by every call on a device, so calls that overlap on the GPU race;
    grids with more than NOALLOC_MAX_COLUMNS vertex columns are rejected."""
    lib = load_library()
    par = _par(parallel)
    _check(lib, lib.cismgpu_global_sum_stagger_noalloc(nx, ny, nz, ctypes.byref(par), ctypes.c_void_p(arr1_dev),
                                                       ctypes.c_void_p(arr2_dev), ctypes.c_void_p(sum_dev),
                                                       ctypes.c_void_p(stream)))


SUM_TREE, SUM_SEQUENTIAL = 0, 1  # CISMGPU_SUM_*


def set_sum_order(order: int = SUM_TREE) -> int:
    """Order of the FP64 solvers' and the global-sum calls' sums when parallel%reprosum is off:
    SUM_TREE (the library's fixed tree, default) or SUM_SEQUENTIAL (the reference's own
    sequential order, parallel_mpi.F90:6770, bit for bit; slower).  Process-wide; returns
    the previous setting."""
    return int(load_library().cismgpu_set_sum_order(int(order)))


class sum_order:
    """Context manager: `with sum_order(SUM_SEQUENTIAL): ...` restores the previous order on exit."""

    def __init__(self, order: int):
        self.order = order
        self.prev = None

    def __enter__(self):
        self.prev = set_sum_order(self.order)
        return self

    def __exit__(self, *exc):
        set_sum_order(self.prev)
        return False


def tile_table() -> list:
    """The mixed solver's tile-height table: one 'key height [# timings]' string per key."""
    lib = load_library()
    n = int(lib.cismgpu_tile_table(None, 0))
    buf = ctypes.create_string_buffer(n)
    lib.cismgpu_tile_table(buf, n)
    return [ln for ln in buf.value.decode().split("\n") if ln]


MIXED_LAYOUT_AUTO, MIXED_LAYOUT_FULL = 0, 1  # CISMGPU_MIXED_LAYOUT_*


def set_mixed_layout(layout: int = MIXED_LAYOUT_AUTO) -> int:
    """Matrix layout of the mixed solver's copies: MIXED_LAYOUT_AUTO stores an exactly symmetric 3D
    matrix as its symmetric half (bit-identical results, about half the matrix bytes);
    MIXED_LAYOUT_FULL keeps every coupling.  Read when a handle builds its copies; returns the
    previous setting."""
    return int(load_library().cismgpu_set_mixed_layout(int(layout)))


def debug_set_device_waits(wait_cycles: int = 0, withhold_step: int = 0) -> None:
    """Test hook of the mixed kernels' bounded waits: wait bound in SM cycles (0: the default,
    about 1 s) and a step whose record tile 0 of every solve does not publish (0: none), so the
    waits for it run out and the launch ends with CISMGPU_ETIMEOUT.  (0, 0) restores normal
    operation."""
    lib = load_library()
    _check(lib, lib.cismgpu_test_set_device_waits(int(wait_cycles), int(withhold_step)))


def set_oneshot_algorithm(algorithm: int = -1) -> int:
    """Select the algorithm of the reference-signature calls (-1: the one each call names, FP64)."""
    return int(load_library().cismgpu_set_oneshot_algorithm(int(algorithm)))


def pcg_solver_standard_3d(nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                           xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest=1, jtest=1, rtest=0):
    """Mirrors pcg_solver_standard_3d (glissade_velo_higher_pcg.F90:827-1537)."""
    return _solve("cismgpu_pcg_standard_3d", True, nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, Auu,
                  Auv, Avu, Avv, bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest, jtest,
                  rtest)


def pcg_solver_chrongear_3d(nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                            xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest=1, jtest=1, rtest=0):
    """Mirrors pcg_solver_chrongear_3d (glissade_velo_higher_pcg.F90:2632-3594)."""
    return _solve("cismgpu_pcg_chrongear_3d", True, nx, ny, nz, parallel, indxA_2d, indxA_3d, active_vertex, Auu,
                  Auv, Avu, Avv, bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest, jtest,
                  rtest)


def pcg_solver_standard_2d(nx, ny, parallel, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond,
                           linear_solve_ncheck, tolerance, maxiters, itest=1, jtest=1, rtest=0):
    """Mirrors pcg_solver_standard_2d (glissade_velo_higher_pcg.F90:67-823)."""
    return _solve("cismgpu_pcg_standard_2d", False, nx, ny, 1, parallel, indxA_2d, None, active_vertex, Auu, Auv,
                  Avu, Avv, bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest, jtest, rtest)


def pcg_solver_chrongear_2d(nx, ny, parallel, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond,
                            linear_solve_ncheck, tolerance, maxiters, itest=1, jtest=1, rtest=0):
    """Mirrors pcg_solver_chrongear_2d (glissade_velo_higher_pcg.F90:1541-2628)."""
    return _solve("cismgpu_pcg_chrongear_2d", False, nx, ny, 1, parallel, indxA_2d, None, active_vertex, Auu, Auv,
                  Avu, Avv, bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, itest, jtest, rtest)


def matvec_multiply_structured_3d(nx, ny, nz, parallel, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, xu, xv):
    """Mirrors matvec_multiply_structured_3d (glissade_velo_higher_pcg.F90:5528-5652); returns (yu, yv)."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    nvec, nblk = nv * nz, nv * nz * 27
    yu, yv = np.empty_like(xu), np.empty_like(xv)
    par = _par(parallel)
    _check(lib, lib.cismgpu_matvec_structured_3d(
        nx, ny, nz, ctypes.byref(par), _ptr(np.ascontiguousarray(indxA_3d, dtype=np.int32), np.int32, 27),
        _ptr(active_vertex, np.int32, nv), _ptr(Auu, np.float64, nblk), _ptr(Auv, np.float64, nblk),
        _ptr(Avu, np.float64, nblk), _ptr(Avv, np.float64, nblk), _ptr(xu, np.float64, nvec),
        _ptr(xv, np.float64, nvec), _ptr(yu, np.float64, nvec, True), _ptr(yv, np.float64, nvec, True)))
    return yu, yv


def matvec_multiply_structured_2d(nx, ny, parallel, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, xu, xv):
    """Mirrors matvec_multiply_structured_2d (glissade_velo_higher_pcg.F90:5656-5773); returns (yu, yv)."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    yu, yv = np.empty_like(xu), np.empty_like(xv)
    par = _par(parallel)
    _check(lib, lib.cismgpu_matvec_structured_2d(
        nx, ny, ctypes.byref(par), _ptr(np.ascontiguousarray(indxA_2d, dtype=np.int32), np.int32, 9),
        _ptr(active_vertex, np.int32, nv), _ptr(Auu, np.float64, nv * 9), _ptr(Auv, np.float64, nv * 9),
        _ptr(Avu, np.float64, nv * 9), _ptr(Avv, np.float64, nv * 9), _ptr(xu, np.float64, nv),
        _ptr(xv, np.float64, nv), _ptr(yu, np.float64, nv, True), _ptr(yv, np.float64, nv, True)))
    return yu, yv


def compute_residual_vector_3d(nx, ny, nz, parallel, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu, bv, uvel,
                               vvel):
    """Mirrors compute_residual_vector_3d (glissade_velo_higher.F90:9693-9894);
    returns (resid_u, resid_v, L2_norm, L2_norm_relative)."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    nvec, nblk = nv * nz, nv * nz * 27
    ru, rv = np.empty_like(bu), np.empty_like(bv)
    l2, l2r = ctypes.c_double(0.0), ctypes.c_double(0.0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_compute_residual_vector_3d(
        nx, ny, nz, ctypes.byref(par), _ptr(np.ascontiguousarray(indxA_3d, dtype=np.int32), np.int32, 27),
        _ptr(active_vertex, np.int32, nv), _ptr(Auu, np.float64, nblk), _ptr(Auv, np.float64, nblk),
        _ptr(Avu, np.float64, nblk), _ptr(Avv, np.float64, nblk), _ptr(bu, np.float64, nvec),
        _ptr(bv, np.float64, nvec), _ptr(uvel, np.float64, nvec), _ptr(vvel, np.float64, nvec),
        _ptr(ru, np.float64, nvec, True), _ptr(rv, np.float64, nvec, True), ctypes.byref(l2), ctypes.byref(l2r)))
    return ru, rv, l2.value, l2r.value


def compute_residual_vector_2d(nx, ny, parallel, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, bu, bv, uvel, vvel):
    """Mirrors compute_residual_vector_2d (glissade_velo_higher.F90:9502-9689);
    returns (resid_u, resid_v, L2_norm, L2_norm_relative)."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    ru, rv = np.empty_like(bu), np.empty_like(bv)
    l2, l2r = ctypes.c_double(0.0), ctypes.c_double(0.0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_compute_residual_vector_2d(
        nx, ny, ctypes.byref(par), _ptr(np.ascontiguousarray(indxA_2d, dtype=np.int32), np.int32, 9),
        _ptr(active_vertex, np.int32, nv), _ptr(Auu, np.float64, nv * 9), _ptr(Auv, np.float64, nv * 9),
        _ptr(Avu, np.float64, nv * 9), _ptr(Avv, np.float64, nv * 9), _ptr(bu, np.float64, nv),
        _ptr(bv, np.float64, nv), _ptr(uvel, np.float64, nv), _ptr(vvel, np.float64, nv),
        _ptr(ru, np.float64, nv, True), _ptr(rv, np.float64, nv, True), ctypes.byref(l2), ctypes.byref(l2r)))
    return ru, rv, l2.value, l2r.value


def compute_residual_velocity_3d(whichresid, nx, ny, nz, parallel, uvel, vvel, usav, vsav) -> float:
    """Mirrors compute_residual_velocity_3d (glissade_velo_higher.F90:10314-10446)."""
    lib = load_library()
    n = (nx - 1) * (ny - 1) * nz
    out = ctypes.c_double(0.0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_compute_residual_velocity_3d(
        int(whichresid), nx, ny, nz, ctypes.byref(par), _ptr(uvel, np.float64, n), _ptr(vvel, np.float64, n),
        _ptr(usav, np.float64, n), _ptr(vsav, np.float64, n), ctypes.byref(out)))
    return out.value


def compute_residual_velocity_2d(whichresid, nx, ny, parallel, uvel, vvel, usav, vsav) -> float:
    """Mirrors compute_residual_velocity_2d (glissade_velo_higher.F90:10188-10310)."""
    lib = load_library()
    n = (nx - 1) * (ny - 1)
    out = ctypes.c_double(0.0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_compute_residual_velocity_2d(
        int(whichresid), nx, ny, ctypes.byref(par), _ptr(uvel, np.float64, n), _ptr(vvel, np.float64, n),
        _ptr(usav, np.float64, n), _ptr(vsav, np.float64, n), ctypes.byref(out)))
    return out.value


def check_symmetry_assembled_matrix_3d(nx, ny, nz, parallel, indxA_3d, active_vertex, Auu, Auv, Avu, Avv):
    """Mirrors check_symmetry_assembled_matrix_3d (glissade_velo_higher.F90:10854-11117): the
    nearly symmetric pairs of the four blocks are averaged in place (the arrays must be
    writable float64 in the caller's layout).  Returns (maxdiff, nwarn): the largest asymmetry
    met and the number of asymmetry warnings the reference logs."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    nblk = nv * nz * 27
    md, nw = ctypes.c_double(0.0), ctypes.c_longlong(0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_check_symmetry_assembled_matrix_3d(
        nx, ny, nz, ctypes.byref(par), _ptr(np.ascontiguousarray(indxA_3d, dtype=np.int32), np.int32, 27),
        _ptr(active_vertex, np.int32, nv), _ptr(Auu, np.float64, nblk, True), _ptr(Auv, np.float64, nblk, True),
        _ptr(Avu, np.float64, nblk, True), _ptr(Avv, np.float64, nblk, True), ctypes.byref(md), ctypes.byref(nw)))
    return md.value, nw.value


def check_symmetry_assembled_matrix_2d(nx, ny, parallel, indxA_2d, active_vertex, Auu, Auv, Avu, Avv):
    """Mirrors check_symmetry_assembled_matrix_2d (glissade_velo_higher.F90:10648-10850), which
    only reports: returns (maxdiff, nwarn) and leaves the blocks unchanged."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    md, nw = ctypes.c_double(0.0), ctypes.c_longlong(0)
    par = _par(parallel)
    _check(lib, lib.cismgpu_check_symmetry_assembled_matrix_2d(
        nx, ny, ctypes.byref(par), _ptr(np.ascontiguousarray(indxA_2d, dtype=np.int32), np.int32, 9),
        _ptr(active_vertex, np.int32, nv), _ptr(Auu, np.float64, nv * 9), _ptr(Auv, np.float64, nv * 9),
        _ptr(Avu, np.float64, nv * 9), _ptr(Avv, np.float64, nv * 9), ctypes.byref(md), ctypes.byref(nw)))
    return md.value, nw.value


def _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagusrf, stagthck, flwafact):
    nv = (nx - 1) * (ny - 1)
    return [_ptr(np.ascontiguousarray(sigma, dtype=np.float64), np.float64, nz),
            _ptr(np.ascontiguousarray(active_cell, dtype=np.int32), np.int32, nx * ny),
            _ptr(xVertex, np.float64, nv), _ptr(yVertex, np.float64, nv)], \
        [_ptr(stagusrf, np.float64, nv), _ptr(stagthck, np.float64, nv),
         _ptr(flwafact, np.float64, (nz - 1) * nx * ny)]


def assemble_stiffness_matrix_3d(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel, vvel, stagusrf,
                                 stagthck, flwafact, whichapprox=2, whichefvs=2, efvs_constant=0.0,
                                 effstrain_min=1.0e-8, n_glen=3.0, indxA_3d=None):
    """Mirrors assemble_stiffness_matrix_3d (glissade_velo_higher.F90:5382-5643) on the GPU.
    Arrays in the caller's layout (C-order numpy with reversed dimensions): active_cell
    (ny, nx), vertex fields (ny-1, nx-1), uvel/vvel (ny-1, nx-1, nz), flwafact (ny, nx, nz-1).
    Returns (efvs (ny, nx, nz-1), Auu, Auv, Avu, Avv (ny-1, nx-1, nz, 27))."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 28, dtype=np.int32) if indxA_3d is None else np.ascontiguousarray(indxA_3d, dtype=np.int32)
    efvs = np.zeros((ny, nx, nz - 1))
    A = [np.zeros((ny - 1, nx - 1, nz, 27)) for _ in range(4)]
    head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagusrf, stagthck, flwafact)
    _check(lib, lib.cismgpu_assemble_stiffness_matrix_3d(
        nx, ny, nz, int(nhalo), *head, _ptr(uvel, np.float64, nv * nz), _ptr(vvel, np.float64, nv * nz), *tail,
        int(whichapprox), int(whichefvs), float(efvs_constant), float(effstrain_min), float(n_glen),
        _ptr(indx, np.int32, 27), _ptr(efvs, np.float64, efvs.size, True), *[_ptr(a, np.float64, a.size, True) for a in A]))
    return (efvs, *A)


def assemble_stiffness_matrix_2d(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel_2d, vvel_2d,
                                 stagthck, flwafact, whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8,
                                 n_glen=3.0, indxA_2d=None):
    """Mirrors assemble_stiffness_matrix_2d (glissade_velo_higher.F90:4961-5378), SSA, on the
    GPU.  Vertex fields (ny-1, nx-1), active_cell (ny, nx), flwafact (ny, nx, nz-1).
    Returns (efvs (ny, nx, nz-1), Auu, Auv, Avu, Avv (9, ny-1, nx-1))."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 10, dtype=np.int32) if indxA_2d is None else np.ascontiguousarray(indxA_2d, dtype=np.int32)
    efvs = np.zeros((ny, nx, nz - 1))
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagthck, stagthck, flwafact)
    _check(lib, lib.cismgpu_assemble_stiffness_matrix_2d(
        nx, ny, nz, int(nhalo), *head, _ptr(uvel_2d, np.float64, nv), _ptr(vvel_2d, np.float64, nv), tail[1],
        tail[2], int(whichefvs), float(efvs_constant), float(effstrain_min), float(n_glen), _ptr(indx, np.int32, 9),
        _ptr(efvs, np.float64, efvs.size, True), *[_ptr(a, np.float64, a.size, True) for a in A]))
    return (efvs, *A)


def dirichlet_boundary_conditions_3d(nx, ny, nz, nhalo, active_vertex, umask, vmask, uvel, vvel, Auu, Auv, Avu, Avv,
                                     bu, bv, indxA_3d=None):
    """Mirrors dirichlet_boundary_conditions_3d (glissade_velo_higher.F90:9305-9498) on the GPU;
    the blocks and b (writable float64, caller's layout) are modified in place."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    n = nv * nz
    indx = np.arange(1, 28, dtype=np.int32) if indxA_3d is None else np.ascontiguousarray(indxA_3d, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    _check(lib, lib.cismgpu_dirichlet_boundary_conditions_3d(
        nx, ny, nz, int(nhalo), _ptr(i32(active_vertex), np.int32, nv), _ptr(i32(umask), np.int32, n),
        _ptr(i32(vmask), np.int32, n), _ptr(uvel, np.float64, n), _ptr(vvel, np.float64, n), _ptr(indx, np.int32, 27),
        *[_ptr(a, np.float64, 27 * n, True) for a in (Auu, Auv, Avu, Avv)], _ptr(bu, np.float64, n, True),
        _ptr(bv, np.float64, n, True)))


def basal_sliding_bc_3d(nx, ny, nz, nhalo, dx, dy, active_cell, active_vertex, beta, lsrf, xVertex, yVertex, Auu,
                        Avv, whichassemble_beta=1, indxA_3d=None):
    """Mirrors basal_sliding_bc_3d (glissade_velo_higher.F90:8815-9129) on the GPU (1: local,
    0: standard form): the bed level of the full Auu and Avv blocks is increased in place."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 28, dtype=np.int32) if indxA_3d is None else np.ascontiguousarray(indxA_3d, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    _check(lib, lib.cismgpu_basal_sliding_bc_3d(
        nx, ny, nz, int(nhalo), float(dx), float(dy), _ptr(i32(active_cell), np.int32, nx * ny),
        _ptr(i32(active_vertex), np.int32, nv), _ptr(beta, np.float64, nv), _ptr(lsrf, np.float64, nx * ny),
        _ptr(xVertex, np.float64, nv), _ptr(yVertex, np.float64, nv), int(whichassemble_beta), _ptr(indx, np.int32, 27),
        _ptr(Auu, np.float64, 27 * nv * nz, True), _ptr(Avv, np.float64, 27 * nv * nz, True)))


def _diva_inputs(nx, ny, nz, stagsigma, stagthck, thck, btractx, btracty, dsfx, dsfy):
    nv, nc = (nx - 1) * (ny - 1), nx * ny
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    return [_ptr(f64(stagsigma), np.float64, nz - 1)], [_ptr(stagthck, np.float64, nv), _ptr(f64(thck), np.float64, nc),
                                                       _ptr(btractx, np.float64, nv), _ptr(btracty, np.float64, nv),
                                                       _ptr(f64(dsfx), np.float64, nc), _ptr(f64(dsfy), np.float64, nc)]


def assemble_stiffness_matrix_2d_diva(nx, ny, nz, nhalo, sigma, stagsigma, active_cell, xVertex, yVertex, uvel_2d,
                                      vvel_2d, stagthck, thck, btractx, btracty, dsfx, dsfy, flwafact, efvs_qp_3d,
                                      whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8, n_glen=3.0,
                                      indxA_2d=None):
    """Mirrors assemble_stiffness_matrix_2d with HO_APPROX_DIVA (glissade_velo_higher.F90:4961-5378)
    on the GPU.  efvs_qp_3d (ny, nx, 4, nz-1), writable float64, is the state, updated in place.
    Returns (efvs (ny, nx, nz-1), omega_k (ny, nx, nz), omega (ny, nx), Auu, Auv, Avu, Avv)."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 10, dtype=np.int32) if indxA_2d is None else np.ascontiguousarray(indxA_2d, dtype=np.int32)
    efvs = np.zeros((ny, nx, nz - 1))
    ok = np.zeros((ny, nx, nz))
    om = np.zeros((ny, nx))
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagthck, stagthck, flwafact)
    ss, dv = _diva_inputs(nx, ny, nz, stagsigma, stagthck, thck, btractx, btracty, dsfx, dsfy)
    _check(lib, lib.cismgpu_assemble_stiffness_matrix_2d_diva(
        nx, ny, nz, int(nhalo), head[0], *ss, head[1], head[2], head[3], _ptr(uvel_2d, np.float64, nv),
        _ptr(vvel_2d, np.float64, nv), *dv, tail[2], int(whichefvs), float(efvs_constant), float(effstrain_min),
        float(n_glen), _ptr(indx, np.int32, 9), _ptr(efvs_qp_3d, np.float64, (nz - 1) * 4 * nx * ny, True),
        _ptr(efvs, np.float64, efvs.size, True), _ptr(ok, np.float64, ok.size, True), _ptr(om, np.float64, om.size, True),
        *[_ptr(a, np.float64, a.size, True) for a in A]))
    return (efvs, ok, om, *A)


def assemble_stiffness_matrix_2d_l1l2(nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel_2d, vvel_2d,
                                      stagthck, dusrf_dx, dusrf_dy, flwa, flwafact, whichefvs=2, efvs_constant=0.0,
                                      effstrain_min=1.0e-8, n_glen=3.0, indxA_2d=None):
    """Mirrors assemble_stiffness_matrix_2d with HO_APPROX_L1L2 (glissade_velo_higher.F90:4961-5378)
    on the GPU.  Returns (efvs (ny, nx, nz-1), Auu, Auv, Avu, Avv (9, ny-1, nx-1))."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 10, dtype=np.int32) if indxA_2d is None else np.ascontiguousarray(indxA_2d, dtype=np.int32)
    efvs = np.zeros((ny, nx, nz - 1))
    A = [np.zeros((9, ny - 1, nx - 1)) for _ in range(4)]
    head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagthck, stagthck, flwafact)
    _check(lib, lib.cismgpu_assemble_stiffness_matrix_2d_l1l2(
        nx, ny, nz, int(nhalo), *head, _ptr(uvel_2d, np.float64, nv), _ptr(vvel_2d, np.float64, nv), tail[1],
        _ptr(dusrf_dx, np.float64, nv), _ptr(dusrf_dy, np.float64, nv),
        _ptr(np.ascontiguousarray(flwa, dtype=np.float64), np.float64, (nz - 1) * nx * ny), tail[2], int(whichefvs),
        float(efvs_constant), float(effstrain_min), float(n_glen), _ptr(indx, np.int32, 9),
        _ptr(efvs, np.float64, efvs.size, True), *[_ptr(a, np.float64, a.size, True) for a in A]))
    return (efvs, *A)


def load_vector_gravity(nx, ny, nz, nhalo, sigma, stagwbndsigma, dx, dy, active_cell, active_vertex, xVertex,
                        yVertex, stagusrf, stagthck, dusrf_dx, dusrf_dy, whichassemble_taud=1):
    """Mirrors load_vector_gravity (glissade_velo_higher.F90:4228-4449) on the GPU from zero loads;
    returns (loadu, loadv) of shape (ny-1, nx-1, nz)."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    lu, lv = np.zeros((ny - 1, nx - 1, nz)), np.zeros((ny - 1, nx - 1, nz))
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    _check(lib, lib.cismgpu_load_vector_gravity(
        nx, ny, nz, int(nhalo), _ptr(f64(sigma), np.float64, nz), _ptr(f64(stagwbndsigma), np.float64, nz + 1),
        float(dx), float(dy), _ptr(i32(active_cell), np.int32, nx * ny), _ptr(i32(active_vertex), np.int32, nv),
        _ptr(xVertex, np.float64, nv), _ptr(yVertex, np.float64, nv), _ptr(stagusrf, np.float64, nv),
        _ptr(stagthck, np.float64, nv), _ptr(dusrf_dx, np.float64, nv), _ptr(dusrf_dy, np.float64, nv),
        int(whichassemble_taud), _ptr(lu, np.float64, lu.size, True), _ptr(lv, np.float64, lv.size, True)))
    return lu, lv


def basal_sliding_bc_2d_diva(nx, ny, nhalo, dx, dy, active_cell, active_vertex, beta_eff_x, beta_eff_y, lsrf,
                             xVertex, yVertex, Auu, Avv, whichassemble_beta=1, indxA_2d=None):
    """Mirrors basal_sliding_bc_2d_diva (glissade_velo_higher.F90:8535-8811) on the GPU, in place
    on the (9, ny-1, nx-1) blocks."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 10, dtype=np.int32) if indxA_2d is None else np.ascontiguousarray(indxA_2d, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    _check(lib, lib.cismgpu_basal_sliding_bc_2d_diva(
        nx, ny, int(nhalo), float(dx), float(dy), _ptr(i32(active_cell), np.int32, nx * ny),
        _ptr(i32(active_vertex), np.int32, nv), _ptr(beta_eff_x, np.float64, nv), _ptr(beta_eff_y, np.float64, nv),
        _ptr(np.ascontiguousarray(lsrf, dtype=np.float64), np.float64, nx * ny), _ptr(xVertex, np.float64, nv),
        _ptr(yVertex, np.float64, nv), int(whichassemble_beta), _ptr(indx, np.int32, 9),
        _ptr(Auu, np.float64, 9 * nv, True), _ptr(Avv, np.float64, 9 * nv, True)))


def dirichlet_boundary_conditions_2d(nx, ny, nhalo, active_vertex, umask, vmask, uvel, vvel, Auu, Auv, Avu, Avv,
                                     bu, bv, indxA_2d=None):
    """Mirrors dirichlet_boundary_conditions_2d (glissade_velo_higher.F90:9133-9301) on the GPU,
    in place on the (9, ny-1, nx-1) blocks and b."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 10, dtype=np.int32) if indxA_2d is None else np.ascontiguousarray(indxA_2d, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    _check(lib, lib.cismgpu_dirichlet_boundary_conditions_2d(
        nx, ny, int(nhalo), _ptr(i32(active_vertex), np.int32, nv), _ptr(i32(umask), np.int32, nv),
        _ptr(i32(vmask), np.int32, nv), _ptr(uvel, np.float64, nv), _ptr(vvel, np.float64, nv), _ptr(indx, np.int32, 9),
        *[_ptr(a, np.float64, 9 * nv, True) for a in (Auu, Auv, Avu, Avv)], _ptr(bu, np.float64, nv, True),
        _ptr(bv, np.float64, nv, True)))


def basal_sliding_bc_2d(nx, ny, nhalo, dx, dy, active_cell, active_vertex, beta, xVertex, yVertex, Auu, Avv,
                        whichassemble_beta=1, indxA_2d=None):
    """Mirrors basal_sliding_bc_2d (glissade_velo_higher.F90:8281-8531) on the GPU (1: local,
    0: standard form), in place."""
    lib = load_library()
    nv = (nx - 1) * (ny - 1)
    indx = np.arange(1, 10, dtype=np.int32) if indxA_2d is None else np.ascontiguousarray(indxA_2d, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    _check(lib, lib.cismgpu_basal_sliding_bc_2d(
        nx, ny, int(nhalo), float(dx), float(dy), _ptr(i32(active_cell), np.int32, nx * ny),
        _ptr(i32(active_vertex), np.int32, nv), _ptr(beta, np.float64, nv), _ptr(xVertex, np.float64, nv),
        _ptr(yVertex, np.float64, nv), int(whichassemble_beta), _ptr(indx, np.int32, 9),
        _ptr(Auu, np.float64, 9 * nv, True), _ptr(Avv, np.float64, 9 * nv, True)))


class DeviceSolver:
    """A device-resident linear system (cismgpu_solver_create): A, b and x0 live in HBM.

    ``problem`` is a cism_b200.assembly.Problem (or any object with the same fields).
    ``stream`` is a CUDA stream handle (int) or None for a private stream.
    """

    def __init__(self, problem, x0=None, stream=None):
        lib = load_library()
        self._lib = lib
        P = problem
        self.problem = P
        is3d = P.kind == "3d"
        nv = (P.nx - 1) * (P.ny - 1)
        nvec = nv * (P.nz if is3d else 1)
        nblk = nvec * (27 if is3d else 9)
        indx = np.arange(1, 28 if is3d else 10, dtype=np.int32)
        self._keep = [indx]
        par = _par(P.par)
        self._par = par
        h = ctypes.c_void_p()
        xu0 = xv0 = None
        if x0 is not None:
            xu0, xv0 = _ptr(x0[0], np.float64, nvec), _ptr(x0[1], np.float64, nvec)
            self._keep += [x0]
        st = lib.cismgpu_solver_create(
            ctypes.byref(h), 3 if is3d else 2, P.nx, P.ny, P.nz if is3d else 1, ctypes.byref(par),
            _ptr(indx, np.int32, indx.size), _ptr(P.active_vertex, np.int32, nv), _ptr(P.Auu, np.float64, nblk),
            _ptr(P.Auv, np.float64, nblk), _ptr(P.Avu, np.float64, nblk), _ptr(P.Avv, np.float64, nblk),
            _ptr(P.bu, np.float64, nvec), _ptr(P.bv, np.float64, nvec), xu0, xv0,
            ctypes.c_void_p(stream) if stream else None)
        _check(lib, st)
        self.handle = h
        self._shape = P.bu.shape

    def solve(self, algorithm=ALG_CHRONGEAR, precond=HO_PRECOND_DIAG, ncheck=5, tol=1e-8, maxiters=200):
        """Returns (err, niters); raises CismGpuError on a nonzero status."""
        err = ctypes.c_double(0.0)
        nit = ctypes.c_int(0)
        _check(self._lib, self._lib.cismgpu_solver_solve(self.handle, algorithm, precond, ncheck, tol, maxiters,
                                                          ctypes.byref(err), ctypes.byref(nit)))
        return err.value, nit.value

    def set_system(self, Auu, Auv, Avu, Avv, bu, bv, x0_from_solution=True):
        """New coefficients and right-hand side (same geometry and active vertices) for the next
        Picard iteration; with x0_from_solution the next solve starts from the last solution,
        which stays on the device."""
        P = self.problem
        is3d = P.kind == "3d"
        nv = (P.nx - 1) * (P.ny - 1)
        nvec = nv * (P.nz if is3d else 1)
        nblk = nvec * (27 if is3d else 9)
        _check(self._lib, self._lib.cismgpu_solver_set_system(
            self.handle, _ptr(Auu, np.float64, nblk), _ptr(Auv, np.float64, nblk), _ptr(Avu, np.float64, nblk),
            _ptr(Avv, np.float64, nblk), _ptr(bu, np.float64, nvec), _ptr(bv, np.float64, nvec),
            1 if x0_from_solution else 0))

    def residual_vector(self, arrays=True):
        """compute_residual_vector of the current velocity with the current system:
        (resid_u, resid_v, L2_norm, L2_norm_relative); resid arrays are None with arrays=False."""
        l2, l2r = ctypes.c_double(0.0), ctypes.c_double(0.0)
        ru = rv = None
        pu = pv = None
        if arrays:
            ru, rv = np.empty(self._shape), np.empty(self._shape)
            pu, pv = ctypes.c_void_p(ru.ctypes.data), ctypes.c_void_p(rv.ctypes.data)
        _check(self._lib, self._lib.cismgpu_solver_residual_vector(self.handle, pu, pv, ctypes.byref(l2),
                                                                   ctypes.byref(l2r)))
        return ru, rv, l2.value, l2r.value

    def check_symmetry(self):
        """check_symmetry_assembled_matrix on the resident blocks (3D: the averages go into the
        device copy the next solve uses); returns (maxdiff, nwarn)."""
        md, nw = ctypes.c_double(0.0), ctypes.c_longlong(0)
        _check(self._lib, self._lib.cismgpu_solver_check_symmetry(self.handle, ctypes.byref(md), ctypes.byref(nw)))
        return md.value, nw.value

    def assemble_stiffness(self, nhalo, sigma, active_cell, xVertex, yVertex, stagusrf, stagthck, flwafact,
                           uvel=None, vvel=None, whichapprox=2, whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8,
                           n_glen=3.0):
        """assemble_stiffness_matrix_3d (3D handles) or _2d (SSA, 2D handles; stagusrf unused)
        into the resident blocks; uvel = vvel = None uses the handle's current velocity.
        Returns efvs (ny, nx, nz-1)."""
        P = self.problem
        is3d = P.kind == "3d"
        nx, ny = P.nx, P.ny
        nz = P.nz if is3d else len(sigma)  # 2D: the sigma levels of flwafact
        nv = (nx - 1) * (ny - 1)
        nvel = nv * (nz if is3d else 1)
        efvs = np.zeros((ny, nx, nz - 1))
        head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagusrf, stagthck, flwafact)
        pu = None if uvel is None else _ptr(uvel, np.float64, nvel)
        pv = None if vvel is None else _ptr(vvel, np.float64, nvel)
        pe = _ptr(efvs, np.float64, efvs.size, True)
        if is3d:
            st = self._lib.cismgpu_solver_assemble_stiffness_3d(
                self.handle, int(nhalo), *head, pu, pv, *tail, int(whichapprox), int(whichefvs), float(efvs_constant),
                float(effstrain_min), float(n_glen), pe)
        else:
            st = self._lib.cismgpu_solver_assemble_stiffness_2d(
                self.handle, nz, int(nhalo), *head, pu, pv, tail[1], tail[2], int(whichefvs), float(efvs_constant),
                float(effstrain_min), float(n_glen), pe)
        _check(self._lib, st)
        return efvs

    def assemble_system(self, nhalo, dx, dy, sigma, active_cell, active_vertex, xVertex, yVertex, stagusrf,
                        stagthck, flwafact, loadu, loadv, beta=None, lsrf=None, umask=None, vmask=None,
                        whichapprox=2, whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8, n_glen=3.0,
                        whichassemble_beta=1):
        """One Picard iteration's system on the device (cismgpu_solver_assemble_system_3d / _2d):
        stiffness from the current velocity, local basal term, b = load, Dirichlet conditions,
        staggered halo.  2D handles: stagusrf and lsrf unused, masks (ny-1, nx-1).  Returns efvs
        (ny, nx, nz-1)."""
        P = self.problem
        if P.kind != "3d":
            return self._assemble_system_2d(nhalo, dx, dy, sigma, active_cell, active_vertex, xVertex, yVertex,
                                            stagthck, flwafact, loadu, loadv, beta, umask, vmask, whichefvs,
                                            efvs_constant, effstrain_min, n_glen, whichassemble_beta)
        nx, ny, nz = P.nx, P.ny, P.nz
        nv = (nx - 1) * (ny - 1)
        efvs = np.zeros((ny, nx, nz - 1))
        head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagusrf, stagthck, flwafact)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        keep = [i32(active_vertex)] + ([i32(umask), i32(vmask)] if umask is not None else [])
        pm = (_ptr(keep[1], np.int32, nv * nz), _ptr(keep[2], np.int32, nv * nz)) if umask is not None else (None, None)
        pb = (_ptr(beta, np.float64, nv), _ptr(lsrf, np.float64, nx * ny)) if beta is not None else (None, None)
        _check(self._lib, self._lib.cismgpu_solver_assemble_system_3d(
            self.handle, int(nhalo), float(dx), float(dy), head[0], head[1], _ptr(keep[0], np.int32, nv), head[2],
            head[3], *tail, int(whichapprox), int(whichefvs), float(efvs_constant), float(effstrain_min),
            float(n_glen), *pb, int(whichassemble_beta), _ptr(loadu, np.float64, nv * nz),
            _ptr(loadv, np.float64, nv * nz), *pm,
            _ptr(efvs, np.float64, efvs.size, True)))
        return efvs

    def _assemble_system_2d(self, nhalo, dx, dy, sigma, active_cell, active_vertex, xVertex, yVertex, stagthck,
                            flwafact, loadu, loadv, beta, umask, vmask, whichefvs, efvs_constant, effstrain_min,
                            n_glen, whichassemble_beta=1):
        P = self.problem
        nx, ny, nz = P.nx, P.ny, len(sigma)
        nv = (nx - 1) * (ny - 1)
        efvs = np.zeros((ny, nx, nz - 1))
        head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagthck, stagthck, flwafact)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        keep = [i32(active_vertex)] + ([i32(umask), i32(vmask)] if umask is not None else [])
        pm = (_ptr(keep[1], np.int32, nv), _ptr(keep[2], np.int32, nv)) if umask is not None else (None, None)
        pb = _ptr(beta, np.float64, nv) if beta is not None else None
        _check(self._lib, self._lib.cismgpu_solver_assemble_system_2d(
            self.handle, nz, int(nhalo), float(dx), float(dy), head[0], head[1], _ptr(keep[0], np.int32, nv), head[2],
            head[3], tail[1], tail[2], int(whichefvs), float(efvs_constant), float(effstrain_min), float(n_glen), pb,
            int(whichassemble_beta), _ptr(loadu, np.float64, nv), _ptr(loadv, np.float64, nv), *pm,
            _ptr(efvs, np.float64, efvs.size, True)))
        return efvs

    def assemble_stiffness_diva(self, nz, nhalo, sigma, stagsigma, active_cell, xVertex, yVertex, stagthck, thck,
                                btractx, btracty, dsfx, dsfy, flwafact, uvel=None, vvel=None, efvs_qp_3d=None,
                                whichefvs=2, efvs_constant=0.0, effstrain_min=1.0e-8, n_glen=3.0):
        """The DIVA assembly into this 2D handle (cismgpu_solver_assemble_stiffness_2d_diva); the
        layer viscosities stay on the device between calls.  Returns (efvs, omega_k, omega)."""
        P = self.problem
        nx, ny = P.nx, P.ny
        nv = (nx - 1) * (ny - 1)
        efvs = np.zeros((ny, nx, nz - 1))
        ok = np.zeros((ny, nx, nz))
        om = np.zeros((ny, nx))
        head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagthck, stagthck, flwafact)
        ss, dv = _diva_inputs(nx, ny, nz, stagsigma, stagthck, thck, btractx, btracty, dsfx, dsfy)
        pu = None if uvel is None else _ptr(uvel, np.float64, nv)
        pv = None if vvel is None else _ptr(vvel, np.float64, nv)
        pe = None if efvs_qp_3d is None else _ptr(np.ascontiguousarray(efvs_qp_3d, dtype=np.float64), np.float64,
                                                  (nz - 1) * 4 * nx * ny)
        _check(self._lib, self._lib.cismgpu_solver_assemble_stiffness_2d_diva(
            self.handle, nz, int(nhalo), head[0], *ss, head[1], head[2], head[3], pu, pv, *dv, tail[2], int(whichefvs),
            float(efvs_constant), float(effstrain_min), float(n_glen), pe, _ptr(efvs, np.float64, efvs.size, True),
            _ptr(ok, np.float64, ok.size, True), _ptr(om, np.float64, om.size, True)))
        return efvs, ok, om

    def assemble_system_diva(self, nz, nhalo, dx, dy, sigma, stagsigma, active_cell, active_vertex, xVertex, yVertex,
                             stagthck, thck, btractx, btracty, dsfx, dsfy, flwafact, loadu, loadv, beta_eff_x=None,
                             beta_eff_y=None, lsrf=None, umask=None, vmask=None, whichassemble_beta=1, whichefvs=2,
                             efvs_constant=0.0, effstrain_min=1.0e-8, n_glen=3.0):
        """One Picard iteration's DIVA system on this 2D handle; returns (efvs, omega_k, omega)."""
        P = self.problem
        nx, ny = P.nx, P.ny
        nv = (nx - 1) * (ny - 1)
        efvs = np.zeros((ny, nx, nz - 1))
        ok = np.zeros((ny, nx, nz))
        om = np.zeros((ny, nx))
        head, tail = _assembly_inputs(nx, ny, nz, sigma, active_cell, xVertex, yVertex, stagthck, stagthck, flwafact)
        ss, dv = _diva_inputs(nx, ny, nz, stagsigma, stagthck, thck, btractx, btracty, dsfx, dsfy)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        keep = [i32(active_vertex)] + ([i32(umask), i32(vmask)] if umask is not None else [])
        pm = (_ptr(keep[1], np.int32, nv), _ptr(keep[2], np.int32, nv)) if umask is not None else (None, None)
        if beta_eff_x is not None:
            lk = np.ascontiguousarray(lsrf, dtype=np.float64)
            keep.append(lk)
            pb = (_ptr(beta_eff_x, np.float64, nv), _ptr(beta_eff_y, np.float64, nv), _ptr(lk, np.float64, nx * ny))
        else:
            pb = (None, None, None)
        _check(self._lib, self._lib.cismgpu_solver_assemble_system_2d_diva(
            self.handle, nz, int(nhalo), float(dx), float(dy), head[0], *ss, head[1], _ptr(keep[0], np.int32, nv),
            head[2], head[3], *dv, tail[2], int(whichefvs), float(efvs_constant), float(effstrain_min), float(n_glen),
            *pb, int(whichassemble_beta), _ptr(loadu, np.float64, nv), _ptr(loadv, np.float64, nv), *pm,
            _ptr(efvs, np.float64, efvs.size, True), _ptr(ok, np.float64, ok.size, True),
            _ptr(om, np.float64, om.size, True)))
        return efvs, ok, om

    def save(self):
        """Accelerated Picard's saved state: the current velocity and A (not b) on the device."""
        _check(self._lib, self._lib.cismgpu_solver_save(self.handle))

    def restore(self):
        """Back to the saved velocity and A; the velocity becomes the next solve's initial guess."""
        _check(self._lib, self._lib.cismgpu_solver_restore(self.handle))

    def residual_velocity(self, whichresid=1):
        """compute_residual_velocity between the last solution and the guess it started from."""
        out = ctypes.c_double(0.0)
        _check(self._lib, self._lib.cismgpu_solver_residual_velocity(self.handle, int(whichresid),
                                                                     ctypes.byref(out)))
        return out.value

    def x(self):
        xu = np.empty(self._shape)
        xv = np.empty(self._shape)
        _check(self._lib, self._lib.cismgpu_solver_get_x(self.handle, ctypes.c_void_p(xu.ctypes.data),
                                                         ctypes.c_void_p(xv.ctypes.data)))
        return xu, xv

    def mixed_symmetric_half(self) -> bool:
        """True if the mixed copies of this handle hold the symmetric half of the matrix."""
        v = ctypes.c_int(0)
        _check(self._lib, self._lib.cismgpu_solver_mixed_layout(self.handle, ctypes.byref(v)))
        return bool(v.value)

    def x_into(self, xu, xv):
        """The current solution into caller arrays (e.g. pinned host buffers) of the problem's shape."""
        n = int(np.prod(self._shape))
        _check(self._lib, self._lib.cismgpu_solver_get_x(self.handle, _ptr(xu, np.float64, n, True),
                                                         _ptr(xv, np.float64, n, True)))

    def profile(self, enable=True):
        _check(self._lib, self._lib.cismgpu_solver_profile(self.handle, int(enable)))

    def profile_read(self):
        ms, n, by = ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
        _check(self._lib, self._lib.cismgpu_solver_profile_read(self.handle, ctypes.byref(ms), ctypes.byref(n),
                                                                ctypes.byref(by)))
        return ms.value, n.value, by.value

    def device_bytes(self) -> int:
        return int(self._lib.cismgpu_solver_device_bytes(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self._lib.cismgpu_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch(solvers, algorithm=ALG_MIXED_CHRONGEAR, precond=HO_PRECOND_DIAG, ncheck=5, tol=1e-8, maxiters=200,
                stream=None):
    """One persistent launch over many DeviceSolvers; returns (errs, niters, statuses) arrays."""
    lib = load_library()
    n = len(solvers)
    hs = (ctypes.c_void_p * n)(*[s.handle for s in solvers])
    errs = (ctypes.c_double * n)()
    nits = (ctypes.c_int * n)()
    sts = (ctypes.c_int * n)()
    rc = lib.cismgpu_solver_solve_batch(hs, n, algorithm, precond, ncheck, tol, maxiters, errs, nits, sts,
                                        ctypes.c_void_p(stream) if stream else None)
    statuses = np.array(list(sts), dtype=np.int32)
    if rc != 0 and not np.any(statuses):
        _check(lib, rc)
    return np.array(list(errs)), np.array(list(nits), dtype=np.int32), statuses


class GraphBatch:
    """A batched mixed-precision solve over DeviceSolvers captured in a CUDA graph
    (cismgpu_batch_create): run() replays it asynchronously, wait() returns
    (errs, niters, statuses).  The members are locked until close()."""

    def __init__(self, solvers, precond=HO_PRECOND_DIAG, ncheck=5, tol=1e-8, maxiters=200, stream=None):
        lib = load_library()
        self._lib = lib
        self.solvers = list(solvers)
        n = len(self.solvers)
        self.n = n
        hs = (ctypes.c_void_p * n)(*[s.handle for s in self.solvers])
        h = ctypes.c_void_p()
        _check(lib, lib.cismgpu_batch_create(ctypes.byref(h), hs, n, precond, ncheck, tol, maxiters,
                                             ctypes.c_void_p(stream) if stream else None))
        self.handle = h.value

    def run(self):
        _check(self._lib, self._lib.cismgpu_batch_run(self.handle))

    def wait(self):
        n = self.n
        errs, nits, sts = (ctypes.c_double * n)(), (ctypes.c_int * n)(), (ctypes.c_int * n)()
        rc = self._lib.cismgpu_batch_wait(self.handle, errs, nits, sts)
        statuses = np.array(list(sts), dtype=np.int32)
        if rc != 0 and not np.any(statuses):
            _check(self._lib, rc)
        return np.array(list(errs)), np.array(list(nits), dtype=np.int32), statuses

    def close(self):
        if self.handle:
            self._lib.cismgpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The continuous-batching serving loop (cismgpu_server_*): submit() queues a system and
    returns its id at once; the library's server thread admits it within the HBM budget,
    solves it alongside whatever else is running, and writes the solution into the arrays
    returned by result()."""

    def __init__(self, hbm_budget_bytes=150 * 10**9, epoch_steps=64):
        lib = load_library()
        self._lib = lib
        h = ctypes.c_void_p()
        _check(lib, lib.cismgpu_server_create(ctypes.byref(h), int(hbm_budget_bytes), int(epoch_steps)))
        self.handle = h.value
        self._keep = {}

    def submit(self, problem, precond=HO_PRECOND_DIAG, ncheck=5, tol=1e-8, maxiters=20000, x0=None) -> int:
        P = problem
        is3d = P.kind == "3d"
        nv = (P.nx - 1) * (P.ny - 1)
        nvec = nv * (P.nz if is3d else 1)
        nblk = nvec * (27 if is3d else 9)
        indx = np.arange(1, 28 if is3d else 10, dtype=np.int32)
        par = _par(P.par)
        xu = np.zeros_like(P.bu)
        xv = np.zeros_like(P.bv)
        keep = [P, indx, par, xu, xv]
        rq = CRequest(3 if is3d else 2, P.nx, P.ny, P.nz if is3d else 1, ctypes.pointer(par),
                      _ptr(indx, np.int32, indx.size), _ptr(P.active_vertex, np.int32, nv),
                      _ptr(P.Auu, np.float64, nblk), _ptr(P.Auv, np.float64, nblk), _ptr(P.Avu, np.float64, nblk),
                      _ptr(P.Avv, np.float64, nblk), _ptr(P.bu, np.float64, nvec), _ptr(P.bv, np.float64, nvec),
                      None, None, _ptr(xu, np.float64, nvec, True), _ptr(xv, np.float64, nvec, True),
                      precond, ncheck, tol, maxiters)
        if x0 is not None:
            rq.xu0 = _ptr(x0[0], np.float64, nvec)
            rq.xv0 = _ptr(x0[1], np.float64, nvec)
            keep.append(x0)
        rid = ctypes.c_longlong()
        _check(self._lib, self._lib.cismgpu_server_submit(self.handle, ctypes.byref(rq), ctypes.byref(rid)))
        self._keep[rid.value] = keep
        return rid.value

    def poll(self, rid):
        """dict(done, err, niters, status, latency_ms, queue_ms)."""
        d, e, n, st, lat, q = (ctypes.c_int(), ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double(),
                               ctypes.c_double())
        _check(self._lib, self._lib.cismgpu_server_poll(self.handle, rid, d, e, n, st, lat, q))
        return {"done": bool(d.value), "err": e.value, "niters": n.value, "status": st.value,
                "latency_ms": lat.value, "queue_ms": q.value}

    def result(self, rid):
        """(xu, xv, poll dict) of a finished request."""
        info = self.poll(rid)
        if not info["done"]:
            raise RuntimeError(f"request {rid} is not done")
        keep = self._keep[rid]
        return keep[3], keep[4], info

    def drain(self):
        _check(self._lib, self._lib.cismgpu_server_drain(self.handle))

    def launch_stats(self):
        """(kernel launches, launches that held 2D and 3D requests together)."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        _check(self._lib, self._lib.cismgpu_server_launch_stats(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def stats(self):
        ep, by, ac, qu = ctypes.c_longlong(), ctypes.c_size_t(), ctypes.c_int(), ctypes.c_int()
        _check(self._lib, self._lib.cismgpu_server_stats(self.handle, ep, by, ac, qu))
        return {"epochs": ep.value, "bytes_in_use": by.value, "active": ac.value, "queued": qu.value}

    def close(self):
        if getattr(self, "handle", None):
            self._lib.cismgpu_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

