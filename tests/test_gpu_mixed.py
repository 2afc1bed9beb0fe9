"""Mixed-precision persistent Chronopoulos-Gear (FP32 recurrences, FP64 x, FP64 residual
replacement) and its batched form.  Every result is checked against the FP64 oracle:
the FP64 true relative residual must reach the tolerance, and x must agree with the
oracle's FP64 solution within the accuracy a 1e-8 residual implies (bound in each test).
"""
import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests import problems

pytestmark = pytest.mark.gpu


def rel(a, b, P=None):
    """Relative difference on the owned, active entries (the unknowns).  Halo entries of x
    are not part of the solution: the mixed path leaves them at halo(x0), which is what the
    reference leaves with the diagonal or SIA preconditioner and inactive halo vertices; with
    no preconditioner the reference also adds periodic copies there."""
    if P is not None:
        from tests.test_oracle_kat import owned_active_mask
        m = owned_active_mask(P)
        a, b = (a[0][m], a[1][m]), (b[0][m], b[1][m])
    num = np.linalg.norm(np.concatenate([(a[0] - b[0]).ravel(), (a[1] - b[1]).ravel()]))
    den = np.linalg.norm(np.concatenate([b[0].ravel(), b[1].ravel()]))
    return num / den


def true_residual(P, xu, xv):
    yu, yv = oracle.matvec(P, oracle.halo(P.nx, P.ny, P.nz, P.par, xu), oracle.halo(P.nx, P.ny, P.nz, P.par, xv))
    p = P.par
    sl = (slice(p["staggered_jlo"] - 1, p["staggered_jhi"]), slice(p["staggered_ilo"] - 1, p["staggered_ihi"]))
    ru, rv = (P.bu - yu)[sl], (P.bv - yv)[sl]
    return np.sqrt(np.sum(ru * ru) + np.sum(rv * rv)) / np.sqrt(np.sum(P.bu[sl] ** 2) + np.sum(P.bv[sl] ** 2))


CASES = [
    ("dome-sia", lambda: asm.dome(), 2, 1e-7),
    ("dome-diag", lambda: asm.dome(), 1, 1e-6),
    ("slab3d-noslip-diag", lambda: problems.slab_3d(seed=5, sliding=False), 1, 1e-6),
    ("slab3d-sliding-sia", lambda: problems.slab_3d(seed=1, ewn=20, nsn=17), 2, 1e-5),
    ("ssa2d-diag", lambda: asm.ssa_random(ewn=61, nsn=57, seed=3), 1, 1e-5),
    ("ssa2d-none", lambda: problems.slab_2d(seed=1), 0, 1e-5),
]


@pytest.mark.parametrize("name,make,precond,xbound", CASES, ids=[c[0] for c in CASES])
def test_mixed_reaches_fp64_tolerance(gpu_lib, name, make, precond, xbound):
    P = make()
    S = cg.DeviceSolver(P)
    err, nit = S.solve(cg.ALG_MIXED_CHRONGEAR, precond, 5, 1e-8, 5000)
    xu, xv = S.x()
    assert err < 1e-8
    assert true_residual(P, xu, xv) < 1.5e-8        # independent FP64 residual on the CPU
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, precond, tol=1e-8, maxiters=5000)
    assert st == 0 and oerr < 1e-8
    assert rel((xu, xv), (ou, ov), P) < xbound
    # the FP64 reference algorithm needs about as many iterations; without a preconditioner the
    # small ill-conditioned 2D slab is sensitive to FP32 rounding, which moves with the tile height
    # the tuner picks (310-390 iterations measured against 150 in FP64)
    assert nit <= (3.0 if precond == 0 else 2.0) * onit + 10


def test_mixed_is_deterministic(gpu_lib):
    P = asm.ssa_random(ewn=61, nsn=57, seed=4)
    S = cg.DeviceSolver(P)
    a = S.solve(cg.ALG_MIXED_CHRONGEAR, 1, 5, 1e-8, 5000), S.x()
    b = S.solve(cg.ALG_MIXED_CHRONGEAR, 1, 5, 1e-8, 5000), S.x()
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1][0], b[1][0])
    np.testing.assert_array_equal(a[1][1], b[1][1])


def batch_alone(S, precond, maxiters):
    """A system solved alone by the batched kernel (same tile height as in any batch)."""
    errs, nits, sts = cg.solve_batch([S], cg.ALG_MIXED_CHRONGEAR, precond, 5, 1e-8, maxiters)
    assert sts[0] == 0
    return errs[0], nits[0], S.x()


def test_batch_equals_alone(gpu_lib):
    """Uneven 3D solves in one dynamic persistent launch give bit-identical results to each
    system batched alone, and agree with the single-solve kernel within the solve tolerance."""
    probs = [problems.slab_3d(seed=s, ewn=8 + 5 * s, nsn=9 + 3 * s, nz=5 + (s % 3)) for s in range(5)]
    solvers = [cg.DeviceSolver(P) for P in probs]
    alone = [batch_alone(S, 2, 3000) for S in solvers]
    for S, P in zip(solvers, probs):
        S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 3000)
        assert rel(S.x(), alone[solvers.index(S)][2], P) < 1e-6
    errs, nits, sts = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 3000)
    assert not np.any(sts)
    for t, S in enumerate(solvers):
        xu, xv = S.x()
        assert errs[t] == alone[t][0] and nits[t] == alone[t][1]
        np.testing.assert_array_equal(xu, alone[t][2][0])
        np.testing.assert_array_equal(xv, alone[t][2][1])
        assert errs[t] < 1e-8


def test_batch_mixed_2d_sizes(gpu_lib):
    probs = [asm.ssa_random(ewn=40 + 9 * s, nsn=33 + 7 * s, seed=10 + s) for s in range(4)]
    solvers = [cg.DeviceSolver(P) for P in probs]
    errs, nits, sts = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, 1, 5, 1e-8, 5000)
    assert not np.any(sts) and np.all(errs < 1e-8)
    for t, P in enumerate(probs):
        st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, 1, tol=1e-8, maxiters=5000)
        assert rel(solvers[t].x(), (ou, ov), P) < 1e-5


def test_handle_fp64_matches_oneshot(gpu_lib):
    """The device-resident handle runs the same FP64 kernels as the one-shot C-ABI call."""
    P = asm.dome()
    S = cg.DeviceSolver(P)
    e, n = S.solve(cg.ALG_CHRONGEAR, 2, 5, 1e-8, 200)
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, 2, summode=oracle.SUM_DDTREE)
    xu, xv = S.x()
    assert e == oerr and n == onit
    np.testing.assert_array_equal(xu, ou)
    np.testing.assert_array_equal(xv, ov)


def test_mixed_boundary_conditions(gpu_lib):
    for bc in ("outflow", "no_ice"):
        P = problems.slab_3d(seed=3, boundary_ice=True, bc=bc, sliding=False)
        st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, 1, tol=1e-8, maxiters=3000)
        S = cg.DeviceSolver(P)
        try:
            err, nit = S.solve(cg.ALG_MIXED_CHRONGEAR, 1, 5, 1e-8, 3000)
        except cg.CismGpuError as e:
            err = None
        if st == 0 and oerr < 1e-8:
            assert err is not None and err < 1e-8
            assert rel(S.x(), (ou, ov), P) < 1e-5


def test_mixed_rejects_unsupported(gpu_lib):
    P = problems.slab_2d(seed=1)
    S = cg.DeviceSolver(P)
    with pytest.raises(cg.CismGpuError) as e:
        S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 100)  # SIA in 2D
    assert e.value.status == 3


def test_graph_batch_replays_bit_identical(gpu_lib):
    """A CUDA-graph batch (sliding 3D members, each with its own log-normal friction) gives the
    same bits as solving each member alone, on every replay."""
    probs = [asm.batch_member(n, seed=s, nz=7) for s, n in enumerate((20, 27, 33, 24))]
    solvers = [cg.DeviceSolver(P) for P in probs]
    alone = [batch_alone(S, 2, 3000) for S in solvers]
    B = cg.GraphBatch(solvers, precond=2, ncheck=5, tol=1e-8, maxiters=3000)
    try:
        with pytest.raises(cg.CismGpuError) as e:  # members belong to the batch until it is closed
            solvers[1].solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 3000)
        assert e.value.status == 4
        for rep in range(2):
            B.run()
            errs, nits, sts = B.wait()
            assert not np.any(sts)
            for t, S in enumerate(solvers):
                assert errs[t] == alone[t][0] and nits[t] == alone[t][1] and errs[t] < 1e-8
                xu, xv = S.x()
                np.testing.assert_array_equal(xu, alone[t][2][0])
                np.testing.assert_array_equal(xv, alone[t][2][1])
    finally:
        B.close()


def test_batch_more_tiles_than_ctas(gpu_lib):
    """Thousands of tiles over a few hundred CTAs (blocked tile order with padding): every
    member bit-identical to its solve alone, and within tolerance of the FP64 oracle."""
    probs = [asm.ssa_random(ewn=90 + 7 * (s % 5), nsn=80 + 5 * (s % 3), seed=30 + s) for s in range(24)]
    solvers = [cg.DeviceSolver(P) for P in probs]
    errs, nits, sts = cg.solve_batch(solvers, cg.ALG_MIXED_CHRONGEAR, 1, 5, 1e-8, 5000)
    assert not np.any(sts) and np.all(errs < 1e-8)
    xb = [S.x() for S in solvers]
    for t in (0, 7, 23):
        e, n, (xu, xv) = batch_alone(solvers[t], 1, 5000)
        assert e == errs[t] and n == nits[t]
        np.testing.assert_array_equal(xu, xb[t][0])
        np.testing.assert_array_equal(xv, xb[t][1])
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", probs[3], 1, tol=1e-8, maxiters=5000)
    assert rel(xb[3], (ou, ov), probs[3]) < 1e-5


@pytest.mark.parametrize("maxiters", [5, 7, 10])
def test_mixed_stops_with_updated_x(gpu_lib, maxiters):
    """A solve that stops at maxiters returns niters = maxiters.  When the last iteration is a
    check iteration (5, 10), err is the FP64 residual of the returned x, so the update whose
    writes are deferred past the check has been applied; both kernels agree."""
    P = asm.dome()
    S = cg.DeviceSolver(P)
    err, nit = S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-14, maxiters)
    xu, xv = S.x()
    assert nit == maxiters and np.all(np.isfinite(xu)) and np.all(np.isfinite(xv))
    errs, nits, sts = cg.solve_batch([S], cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-14, maxiters)
    bu, bv = S.x()
    assert sts[0] == 0 and nits[0] == maxiters
    if maxiters % 5 == 0:
        assert abs(true_residual(P, xu, xv) - err) <= 1e-9 * err
        assert abs(true_residual(P, bu, bv) - errs[0]) <= 1e-9 * errs[0]


# (name, problem, precond, stored as the symmetric half): the boundary-ice periodic slab takes its
# halo rows from the far side, so pairs across the periodic seam stay unequal (the reference's check
# warns about them instead of averaging) and the matrix keeps the full layout
LAYOUT_CASES = [
    ("dome", lambda: asm.dome(), 2, True),
    ("member-sliding", lambda: asm.batch_member(37, seed=9, nz=11), 2, True),
    ("slab-noslip-diag", lambda: problems.slab_3d(seed=5, sliding=False), 1, True),
    ("slab-periodic-boundary", lambda: problems.slab_3d(seed=6, boundary_ice=True, bc="periodic", sliding=False), 1,
     False),
]


def _mixed(P, precond, layout, batch=False):
    prev = cg.set_mixed_layout(layout)
    try:
        S = cg.DeviceSolver(P)
        try:
            if batch:
                errs, nits, sts = cg.solve_batch([S], cg.ALG_MIXED_CHRONGEAR, precond, 5, 1e-8, 4000)
                assert sts[0] == 0
                e, n = errs[0], nits[0]
            else:
                e, n = S.solve(cg.ALG_MIXED_CHRONGEAR, precond, 5, 1e-8, 4000)
            return e, n, S.x(), S.mixed_symmetric_half()
        finally:
            S.close()
    finally:
        cg.set_mixed_layout(prev)


@pytest.mark.parametrize("batch", [False, True], ids=["single", "batched"])
@pytest.mark.parametrize("name,make,precond,sym", LAYOUT_CASES, ids=[c[0] for c in LAYOUT_CASES])
def test_symmetric_half_layout_bit_identical(gpu_lib, name, make, precond, sym, batch):
    """An exactly symmetric 3D matrix (the reference symmetrizes every 3D system before its
    solve) is stored as its symmetric half; the kernels read a lower coupling from its transpose
    partner, which holds the same number, so err, niters and x equal the full layout's bit for
    bit, in the single-solve and in the batched kernel."""
    P = make()
    half = _mixed(P, precond, cg.MIXED_LAYOUT_AUTO, batch)
    full = _mixed(P, precond, cg.MIXED_LAYOUT_FULL, batch)
    assert half[3] is sym and full[3] is False
    assert half[0] == full[0] and half[1] == full[1] and half[0] < 1e-8
    np.testing.assert_array_equal(half[2][0], full[2][0])
    np.testing.assert_array_equal(half[2][1], full[2][1])
    assert true_residual(P, *half[2]) < 1.0001e-8


def test_asymmetric_matrix_keeps_full_layout(gpu_lib):
    """One lower coupling off its partner by a relative 1e-13 (below the reference check's
    averaging threshold, but not equal): the matrix keeps every coupling and still solves to the
    FP64 tolerance against the oracle."""
    P = asm.dome()
    p = P.par
    j, i, k = p["staggered_jlo"] + 12, p["staggered_ilo"] + 14, 4
    assert P.active_vertex[j, i]
    P.Auu[j, i, k, 4] *= 1.0 + 1e-13
    e, n, x, half = _mixed(P, 2, cg.MIXED_LAYOUT_AUTO)
    assert half is False and e < 1e-8
    assert true_residual(P, *x) < 1.0001e-8
    st, ou, ov, oerr, onit = oracle.pcg("chrongear", P, 2, tol=1e-8, maxiters=4000)
    assert rel(x, (ou, ov), P) < 1e-7


def test_tile_tuner_keeps_a_system_on_one_tiling(gpu_lib):
    """The tile tuner times candidate heights the first time it meets a system's key and keeps
    the winner: repeated solves of the system (and of a copy of it) give the same bits, and the
    table names the key with the height it chose."""
    P = asm.batch_member(45, seed=12, nz=9)
    S = cg.DeviceSolver(P)
    try:
        a = S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 4000), S.x()
        b = S.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 4000), S.x()
    finally:
        S.close()
    T = cg.DeviceSolver(P)
    try:
        c = T.solve(cg.ALG_MIXED_CHRONGEAR, 2, 5, 1e-8, 4000), T.x()
    finally:
        T.close()
    for r in (b, c):
        assert r[0] == a[0]
        np.testing.assert_array_equal(r[1][0], a[1][0])
        np.testing.assert_array_equal(r[1][1], a[1][1])
    table = cg.tile_table()
    keys = [ln.split()[0] for ln in table]
    assert any(k.startswith("solve:3d:nzm16:nz9:half:") for k in keys), table
