"""Parity of the B200 library against the CPU oracle, called through the C ABI.

Bars, all on the same seeded inputs:
  * bit-exact (x including halo entries, err, niters, status) against the oracle run
    with its restatement of the device reduction tree (oracle.SUM_DDTREE): every
    matvec, preconditioner, halo and vector statement is an exact restatement;
  * bit-exact against the reference's own sequential summation order (oracle.SUM_SEQ)
    when the library sums in that order too (cismgpu_set_sum_order(CISMGPU_SUM_SEQUENTIAL)):
    the dome at standard/Chronopoulos-Gear x precond 0/1/2 and slabs with ice on the
    boundary, through convergence;
  * with the default tree order, against SUM_SEQ: the SIA-preconditioned dome agrees
    within 1e-10 relative through convergence; diag/none trajectories are sensitive to
    the summation order, so there both sides converge (err < tol) and x agrees within 1e-6.
"""
import math

import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests import problems

pytestmark = pytest.mark.gpu


def gpu_solve(alg, P, precond, ncheck=5, tol=1e-8, maxiters=200, x0=None):
    xu = np.zeros_like(P.bu) if x0 is None else x0[0].copy()
    xv = np.zeros_like(P.bv) if x0 is None else x0[1].copy()
    try:
        if P.kind == "3d":
            f = cg.pcg_solver_standard_3d if alg == "standard" else cg.pcg_solver_chrongear_3d
            err, nit = f(P.nx, P.ny, P.nz, P.par, asm.indxA_2d(), asm.indxA_3d(), P.active_vertex, P.Auu, P.Auv,
                         P.Avu, P.Avv, P.bu, P.bv, xu, xv, precond, ncheck, tol, maxiters)
        else:
            f = cg.pcg_solver_standard_2d if alg == "standard" else cg.pcg_solver_chrongear_2d
            err, nit = f(P.nx, P.ny, P.par, asm.indxA_2d(), P.active_vertex, P.Auu, P.Auv, P.Avu, P.Avv, P.bu,
                         P.bv, xu, xv, precond, ncheck, tol, maxiters)
        st = 0
    except cg.CismGpuError as e:
        st, err, nit = e.status, float("nan"), -1
    return st, xu, xv, err, nit


def rel(a, b):
    num = np.linalg.norm(np.concatenate([(a[0] - b[0]).ravel(), (a[1] - b[1]).ravel()]))
    den = np.linalg.norm(np.concatenate([b[0].ravel(), b[1].ravel()]))
    return num / den


def assert_bitexact(g, o):
    assert g[0] == o[0], ("status", g[0], o[0])
    if g[0] != 0:
        return
    np.testing.assert_array_equal(g[1], o[1])
    np.testing.assert_array_equal(g[2], o[2])
    assert g[4] == o[4], ("niters", g[4], o[4])
    assert (math.isnan(g[3]) and math.isnan(o[3])) or g[3] == o[3], ("err", g[3], o[3])


CASES_3D = [
    ("interior-periodic", dict(seed=1)),
    ("boundary-periodic", dict(seed=2, boundary_ice=True, bc="periodic")),
    ("boundary-outflow", dict(seed=3, boundary_ice=True, bc="outflow")),
    ("boundary-noice", dict(seed=4, boundary_ice=True, bc="no_ice")),
    ("noslip", dict(seed=5, sliding=False)),
]


@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("case", CASES_3D, ids=[c[0] for c in CASES_3D])
def test_3d_bitexact_vs_device_tree_oracle(gpu_lib, alg, precond, case):
    P = problems.slab_3d(**case[1])
    x0 = problems.random_x0(P, seed=7, scale=10.0)
    o = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=300, summode=oracle.SUM_DDTREE, x0=x0)
    g = gpu_solve(alg, P, precond, tol=1e-8, maxiters=300, x0=x0)
    assert_bitexact(g, o)


@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [3, 4])
def test_3d_lines_noice_edge_coefficients(gpu_lib, alg, precond):
    """A no_ice system whose last owned row and column keep nonzero couplings: the global line
    preconditioner's halo update of its summed planes zeroes those owned entries (the local form
    keeps them), bit-exact against the oracle through 12 iterations or the breakdown."""
    from tests.test_oracle_restatement import _no_ice_edge_coefficients
    P = _no_ice_edge_coefficients()
    o = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=12, summode=oracle.SUM_DDTREE)
    g = gpu_solve(alg, P, precond, tol=1e-8, maxiters=12)
    assert_bitexact(g, o)


CASES_2D = [
    ("interior-periodic", dict(seed=1)),
    ("boundary-periodic", dict(seed=2, boundary_ice=True, bc="periodic")),
    ("boundary-outflow", dict(seed=3, boundary_ice=True, bc="outflow")),
    ("boundary-noice", dict(seed=4, boundary_ice=True, bc="no_ice")),
]


@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("case", CASES_2D, ids=[c[0] for c in CASES_2D])
def test_2d_bitexact_vs_device_tree_oracle(gpu_lib, alg, precond, case):
    # precond 2 in 2D takes no branch in the reference (z unchanged): reproduced, not rejected;
    # with 3/4 Chronopoulos-Gear stops at 100 iterations on both sides (:1704-1732)
    P = problems.slab_2d(**case[1])
    x0 = problems.random_x0(P, seed=8, scale=10.0)
    o = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=400, summode=oracle.SUM_DDTREE, x0=x0)
    g = gpu_solve(alg, P, precond, tol=1e-8, maxiters=400, x0=x0)
    assert_bitexact(g, o)


@pytest.mark.parametrize("alg,precond", [("standard", 1), ("chrongear", 2), ("standard", 2), ("chrongear", 1)])
def test_dome_vs_reference_order(gpu_lib, alg, precond):
    """The 31x31x11 dome (the reference's CPU case) against the reference summation order."""
    P = asm.dome()
    seq = oracle.pcg(alg, P, precond, maxiters=400, summode=oracle.SUM_SEQ)
    tree = oracle.pcg(alg, P, precond, maxiters=400, summode=oracle.SUM_DDTREE)
    g = gpu_solve(alg, P, precond, maxiters=400)
    assert_bitexact(g, tree)
    assert g[0] == seq[0] == 0
    assert g[3] < 1e-8 and seq[3] < 1e-8
    bound = 1e-10 if precond == 2 else 1e-6
    assert rel(g[1:3], seq[1:3]) < bound


SEQ_DOME = [("standard", 1), ("chrongear", 1), ("standard", 0), ("chrongear", 0), ("standard", 2),
            ("chrongear", 2)]


@pytest.mark.parametrize("alg,precond", SEQ_DOME, ids=[f"{a}-{p}" for a, p in SEQ_DOME])
def test_dome_bitexact_reference_order(gpu_lib, alg, precond):
    """The 31x31x11 dome (the reference's CPU case: standard PCG + diagonal precond) with the
    library summing in the reference's sequential order: x (halo included), err, niters and
    status identical to the oracle's SUM_SEQ run, the reference's own one-rank arithmetic,
    through convergence."""
    P = asm.dome()
    seq = oracle.pcg(alg, P, precond, maxiters=400, summode=oracle.SUM_SEQ)
    with cg.sum_order(cg.SUM_SEQUENTIAL):
        g = gpu_solve(alg, P, precond, maxiters=400)
    assert seq[0] == 0 and seq[3] < 1e-8
    assert_bitexact(g, seq)
    # the default order again afterwards: the tree's result
    assert_bitexact(gpu_solve(alg, P, precond, maxiters=400),
                    oracle.pcg(alg, P, precond, maxiters=400, summode=oracle.SUM_DDTREE))


SEQ_SLABS = [("3d", "boundary-periodic", dict(seed=2, boundary_ice=True, bc="periodic")),
             ("3d", "noslip", dict(seed=5, sliding=False)),
             ("2d", "interior-periodic", dict(seed=1)),
             ("2d", "boundary-outflow", dict(seed=3, boundary_ice=True, bc="outflow")),
             ("2d", "boundary-noice", dict(seed=4, boundary_ice=True, bc="no_ice"))]


@pytest.mark.parametrize("alg", ["standard", "chrongear"])
@pytest.mark.parametrize("precond", [1, 3])
@pytest.mark.parametrize("case", SEQ_SLABS, ids=[f"{c[0]}-{c[1]}" for c in SEQ_SLABS])
def test_slab_bitexact_reference_order(gpu_lib, alg, precond, case):
    """3D and 2D slabs with ice on the periodic / outflow / no_ice boundary, diagonal and local
    tridiagonal preconditioners, random x0: bit-exact against oracle SUM_SEQ in the sequential
    sum order."""
    kind, _, kw = case
    P = problems.slab_3d(**kw) if kind == "3d" else problems.slab_2d(**kw)
    x0 = problems.random_x0(P, seed=11, scale=10.0)
    o = oracle.pcg(alg, P, precond, tol=1e-8, maxiters=400, summode=oracle.SUM_SEQ, x0=x0)
    with cg.sum_order(cg.SUM_SEQUENTIAL):
        g = gpu_solve(alg, P, precond, tol=1e-8, maxiters=400, x0=x0)
    assert_bitexact(g, o)


def test_reference_order_nan_breakdown(gpu_lib):
    """A zero right-hand side breaks down with alpha = NaN in the sequential order too."""
    Z = problems.slab_3d(seed=2)
    Z.bu[:] = 0.0
    Z.bv[:] = 0.0
    with cg.sum_order(cg.SUM_SEQUENTIAL):
        assert gpu_solve("standard", Z, 1)[0] == oracle.pcg("standard", Z, 1)[0] == 2
        assert gpu_solve("chrongear", Z, 2)[0] == oracle.pcg("chrongear", Z, 2)[0] == 2


def test_dome_trajectory_vs_reference_order(gpu_lib):
    """At a fixed iteration count early in the solve, the diag-preconditioned trajectory
    agrees with the reference order to 1e-10."""
    P = asm.dome()
    for n in (5, 20, 50):
        seq = oracle.pcg("standard", P, 1, tol=0.0, maxiters=n, summode=oracle.SUM_SEQ)
        g = gpu_solve("standard", P, 1, tol=0.0, maxiters=n)
        assert g[4] == n and rel(g[1:3], seq[1:3]) < 1e-10


def test_matvec_3d_bitexact(gpu_lib):
    P = problems.slab_3d(seed=9, boundary_ice=True, bc="periodic")
    rng = np.random.default_rng(3)
    xu, xv = rng.standard_normal(P.bu.shape), rng.standard_normal(P.bv.shape)
    yu, yv = cg.matvec_multiply_structured_3d(P.nx, P.ny, P.nz, P.par, asm.indxA_3d(), P.active_vertex, P.Auu,
                                              P.Auv, P.Avu, P.Avv, xu, xv)
    eu, ev = oracle.matvec(P, xu, xv)
    np.testing.assert_array_equal(yu, eu)
    np.testing.assert_array_equal(yv, ev)


def test_matvec_2d_bitexact(gpu_lib):
    P = problems.slab_2d(seed=9, boundary_ice=True, bc="outflow")
    rng = np.random.default_rng(4)
    xu, xv = rng.standard_normal(P.bu.shape), rng.standard_normal(P.bv.shape)
    yu, yv = cg.matvec_multiply_structured_2d(P.nx, P.ny, P.par, asm.indxA_2d(), P.active_vertex, P.Auu, P.Auv,
                                              P.Avu, P.Avv, xu, xv)
    eu, ev = oracle.matvec(P, xu, xv)
    np.testing.assert_array_equal(yu, eu)
    np.testing.assert_array_equal(yv, ev)


def test_error_statuses(gpu_lib):
    P = problems.slab_3d(seed=2)
    Q = problems.slab_3d(seed=2)
    Q.par = dict(Q.par, tasks_col=2)
    assert gpu_solve("standard", Q, 1)[0] == 3
    Z = problems.slab_3d(seed=2)
    Z.bu[:] = 0.0
    Z.bv[:] = 0.0
    assert gpu_solve("standard", Z, 1)[0] == oracle.pcg("standard", Z, 1)[0] == 2
    assert gpu_solve("chrongear", Z, 2)[0] == oracle.pcg("chrongear", Z, 2)[0] == 2
    assert gpu_solve("standard", P, 1, ncheck=0)[0] == 4


def test_tridiag_zero_pivot(gpu_lib):
    """A zero pivot in the line factorization: CISMGPU_EDIVZERO (GM_FATAL in the reference,
    :4339, :4380), x unchanged; the global form's reverse-recurrence check (:4475, :4492)
    fails precond 4 only."""
    P = problems.slab_2d(seed=23)
    p = P.par
    j, a, b = p["staggered_jlo"] - 1, p["staggered_ilo"] - 1, p["staggered_ihi"] - 1
    P.Auu[4, j, a], P.Auu[5, j, a] = 1.0, 1.0
    P.Auu[3, j, a + 1], P.Auu[4, j, a + 1] = 2.0, 2.0
    x0 = problems.random_x0(P, seed=3, scale=1.0)
    for alg, pc in (("standard", 3), ("chrongear", 4)):
        st, xu, xv, err, nit = gpu_solve(alg, P, pc, maxiters=3, x0=x0)
        assert st == 9 == oracle.pcg(alg, P, pc, maxiters=3)[0]
        np.testing.assert_array_equal(xu, x0[0])
        np.testing.assert_array_equal(xv, x0[1])
    Q = problems.slab_2d(seed=23)
    Q.Auu[3, j, b], Q.Auu[4, j, b] = 1.0, 1.0
    Q.Auu[5, j, b - 1], Q.Auu[4, j, b - 1] = 3.0, 3.0
    for pc in (3, 4):
        g = gpu_solve("standard", Q, pc, maxiters=3)
        o = oracle.pcg("standard", Q, pc, maxiters=3, summode=oracle.SUM_DDTREE)
        assert (g[0] == 9) == (pc == 4)
        assert_bitexact(g, o)


def test_no_check_leaves_err_nan(gpu_lib):
    P = problems.slab_3d(seed=2)
    st, xu, xv, err, nit = gpu_solve("standard", P, 1, ncheck=10, maxiters=3)
    assert st == 0 and nit == 3 and math.isnan(err)


def test_golden_dense_solutions(gpu_lib):
    import os
    data = np.load(os.path.join(os.path.dirname(__file__), "golden", "dense_kat.npz"))
    from tests.test_oracle_kat import owned_active_mask
    for name in ("slab3d", "slab2d"):
        P = problems.slab_3d(seed=21, nz=4, symmetrize=False) if name == "slab3d" else problems.slab_2d(seed=22)
        m = owned_active_mask(P)
        for alg in ("standard", "chrongear"):
            st, xu, xv, err, nit = gpu_solve(alg, P, 1, tol=1e-10, maxiters=10000)
            assert st == 0 and err < 1e-10
            xs_u, xs_v = data[f"{name}_xu"], data[f"{name}_xv"]
            r = np.linalg.norm(np.concatenate([(xu - xs_u)[m], (xv - xs_v)[m]])) / \
                np.linalg.norm(np.concatenate([xs_u[m], xs_v[m]]))
            assert r < float(data[f"{name}_bound"])


def test_repeated_calls_reuse_workspace(gpu_lib):
    """Same call twice (as the Picard loop does) and a size change in between give identical results."""
    P = problems.slab_3d(seed=6)
    a = gpu_solve("chrongear", P, 2)
    Q = problems.slab_2d(seed=6)
    gpu_solve("chrongear", Q, 1)
    b = gpu_solve("chrongear", P, 2)
    assert_bitexact(a, b)


@pytest.mark.parametrize("nz,bc", [(11, "periodic"), (1, "outflow"), (7, "no_ice")])
def test_global_sum_stagger(gpu_lib, nz, bc):
    """parallel_global_sum_stagger: bit-identical to the oracle's restatement of the device tree,
    equal to the exact sum, and within rounding of the reference's sequential order."""
    nx, ny = 37, 29
    par = asm.default_par(nx, ny, bc)
    rng = np.random.default_rng(nz)
    a1 = rng.standard_normal((ny - 1, nx - 1, nz)) * np.exp(rng.uniform(-20, 20, (ny - 1, nx - 1, nz)))
    a2 = rng.standard_normal((ny - 1, nx - 1, nz))
    g = cg.parallel_global_sum_stagger(nx, ny, nz, par, a1, a2)
    assert g == oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_DDTREE)
    assert g == oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_EXACT)
    seq = oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_SEQ)
    assert abs(g - seq) <= 1e-12 * np.sum(np.abs(a1 + a2))


@pytest.mark.parametrize("nz,bc", [(11, "periodic"), (1, "outflow"), (7, "no_ice"), (21, "periodic")])
def test_global_sum_reference_order(gpu_lib, nz, bc):
    """parallel_global_sum_stagger in the sequential sum order: bit-identical to the reference's
    loop (oracle SUM_SEQ), on a grid larger than one staging chunk; the no-allocation entry
    point gives the same bits on device buffers."""
    torch = pytest.importorskip("torch")
    nx, ny = 53, 41
    par = asm.default_par(nx, ny, bc)
    rng = np.random.default_rng(100 + nz)
    a1 = rng.standard_normal((ny - 1, nx - 1, nz)) * np.exp(rng.uniform(-20, 20, (ny - 1, nx - 1, nz)))
    a2 = rng.standard_normal((ny - 1, nx - 1, nz))
    seq = oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_SEQ)
    with cg.sum_order(cg.SUM_SEQUENTIAL):
        g = cg.parallel_global_sum_stagger(nx, ny, nz, par, a1, a2)
        dev = torch.device("cuda:0")
        t1, t2 = torch.from_numpy(a1).to(dev), torch.from_numpy(a2).to(dev)
        out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        cg.parallel_global_sum_stagger_noalloc(nx, ny, nz, par, t1.data_ptr(), t2.data_ptr(), out.data_ptr(),
                                               torch.cuda.current_stream(dev).cuda_stream)
        torch.cuda.synchronize(dev)
    assert g == seq
    assert float(out.cpu()[0]) == seq
    assert cg.parallel_global_sum_stagger(nx, ny, nz, par, a1, a2) == \
        oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_DDTREE)


def test_global_sum_multitask_rejected(gpu_lib):
    nx, ny = 37, 29
    par = dict(asm.default_par(nx, ny, "periodic"), tasks_row=2)
    a = np.ones((ny - 1, nx - 1, 1))
    with pytest.raises(cg.CismGpuError) as e:
        cg.parallel_global_sum_stagger(nx, ny, 1, par, a, a)
    assert e.value.status == 3


@pytest.mark.parametrize("nz,bc,spread", [(11, "periodic", 20), (1, "outflow", 600), (7, "no_ice", 300)])
def test_global_sum_reprosum(gpu_lib, nz, bc, spread):
    """parallel_global_sum_stagger with parallel%reprosum: the reference's integer-vector sum
    (cism_reprosum_calc as CISM calls it), bit-identical to the oracle's restatement, also for
    exponent spreads of hundreds of binades, zeros, and a near-tie the reference double-rounds."""
    nx, ny = 37, 29
    par = dict(asm.default_par(nx, ny, bc), reprosum=1)
    rng = np.random.default_rng(nz + spread)
    a1 = rng.standard_normal((ny - 1, nx - 1, nz)) * np.exp(rng.uniform(-spread, spread, (ny - 1, nx - 1, nz)))
    a2 = np.where(rng.random((ny - 1, nx - 1, nz)) < 0.3, 0.0, rng.standard_normal((ny - 1, nx - 1, nz)))
    g = cg.parallel_global_sum_stagger(nx, ny, nz, par, a1, a2)
    assert g == oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_REPRO)
    # a near-tie: 1 + 2^-53 + 2^-106 - 1e-40 on four owned vertices, zeros elsewhere
    z1, z2 = np.zeros_like(a1), np.zeros_like(a2)
    j, i = par["staggered_jlo"] - 1, par["staggered_ilo"] - 1
    z1[j, i, 0], z1[j, i + 1, 0], z1[j + 1, i, 0], z1[j + 1, i + 1, 0] = 1.0, 2.0**-53, 2.0**-106, -1e-40
    t = cg.parallel_global_sum_stagger(nx, ny, nz, par, z1, z2)
    assert t == oracle.global_sum(nx, ny, nz, par, z1, z2, oracle.SUM_REPRO) == 1.0


def test_global_sum_reprosum_nonfinite(gpu_lib):
    """One-shot reproducible sum with non-finite owned summands: the IEEE sum of those summands
    (NaN for NaN or for +Inf and -Inf together, else the infinity), as the solvers' sums."""
    nx, ny, nz = 37, 29, 3
    par = dict(asm.default_par(nx, ny, "periodic"), reprosum=1)
    rng = np.random.default_rng(5)
    a1 = rng.standard_normal((ny - 1, nx - 1, nz))
    a2 = rng.standard_normal((ny - 1, nx - 1, nz))
    j, i = par["staggered_jlo"] - 1, par["staggered_ilo"] - 1
    b1 = a1.copy()
    b1[j, i, 0] = np.inf
    assert cg.parallel_global_sum_stagger(nx, ny, nz, par, b1, a2) == np.inf
    b1[j + 1, i, 1] = -np.inf
    assert math.isnan(cg.parallel_global_sum_stagger(nx, ny, nz, par, b1, a2))
    c1 = a1.copy()
    c1[j, i + 2, 2] = np.nan
    c2 = a2.copy()
    c2[j + 2, i, 0] = -np.inf
    assert math.isnan(cg.parallel_global_sum_stagger(nx, ny, nz, par, c1, c2))
    d2 = a2.copy()
    d2[j, i, 0] = -np.inf
    assert cg.parallel_global_sum_stagger(nx, ny, nz, par, a1, d2) == -np.inf
    # halo summands do not count: a NaN outside the owned range leaves the finite sum
    e1 = a1.copy()
    e1[0, 0, 0] = np.nan
    assert cg.parallel_global_sum_stagger(nx, ny, nz, par, e1, a2) == \
        oracle.global_sum(nx, ny, nz, par, a1, a2, oracle.SUM_REPRO)
