"""check_symmetry_assembled_matrix_{3d,2d} (glissade_velo_higher.F90:10648-11117) on the
device, through the C ABI: one-shot on the caller's arrays and on a device-resident handle.

Bar: bit-exact against the oracle's in-place restatement (blocks after the check, maxdiff and
the number of asymmetry warnings).  Inputs: assembled blocks with seeded perturbations, some
below the averaging tolerance (eps11 * |diag|) and some far above it, on interior and
boundary-ice grids (whose halo copies are not transposes and so warn by the thousand).
"""
import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests import problems

pytestmark = pytest.mark.gpu

BLOCKS = ("Auu", "Auv", "Avu", "Avv")
CASES = [
    ("3d-interior", lambda: problems.slab_3d(seed=51, symmetrize=False)),
    ("3d-periodic", lambda: problems.slab_3d(seed=52, boundary_ice=True, bc="periodic", symmetrize=False)),
    ("3d-outflow", lambda: problems.slab_3d(seed=53, boundary_ice=True, bc="outflow", symmetrize=False)),
    ("2d-interior", lambda: problems.slab_2d(seed=54)),
    ("2d-noice", lambda: problems.slab_2d(seed=55, boundary_ice=True, bc="no_ice")),
]


def perturbed(P, seed=9, frac=0.04):
    rng = np.random.default_rng(seed)
    for n in BLOCKS:
        A = getattr(P, n)
        sel = rng.random(A.shape) < frac
        scale = np.where(rng.random(A.shape) < 0.5, 1e-14, 1e-9)
        setattr(P, n, np.ascontiguousarray(np.where(sel, A * (1.0 + scale * rng.standard_normal(A.shape)), A)))
    return P


def gpu_check(P, blocks):
    if P.kind == "3d":
        return cg.check_symmetry_assembled_matrix_3d(P.nx, P.ny, P.nz, P.par, asm.indxA_3d(), P.active_vertex,
                                                     *blocks)
    return cg.check_symmetry_assembled_matrix_2d(P.nx, P.ny, P.par, asm.indxA_2d(), P.active_vertex, *blocks)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_check_symmetry_oneshot_bitexact(gpu_lib, case):
    P = perturbed(case[1]())
    want = oracle.check_symmetry(P)
    blocks = [np.array(getattr(P, n), copy=True) for n in BLOCKS]
    md, nw = gpu_check(P, blocks)
    assert md == want[4] and nw == want[5] and nw > 0
    for b, w in zip(blocks, want[:4]):
        np.testing.assert_array_equal(b, w)
    if P.kind == "3d":
        assert any(not np.array_equal(b, getattr(P, n)) for b, n in zip(blocks, BLOCKS))


def test_check_symmetry_oneshot_idempotent(gpu_lib):
    """An interior 3D system has only roundoff asymmetry: one pass averages it all, and a
    second pass finds nothing."""
    P = problems.slab_3d(seed=56, symmetrize=False)
    blocks = [np.array(getattr(P, n), copy=True) for n in BLOCKS]
    md, nw = gpu_check(P, blocks)
    assert md > 0.0 and nw == 0
    md2, nw2 = gpu_check(P, blocks)
    assert md2 == 0.0 and nw2 == 0


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[3]], ids=[CASES[i][0] for i in (0, 2, 3)])
def test_check_symmetry_on_handle(gpu_lib, case):
    """On a handle the check works on the resident canonical planes; the residual of the
    checked system then equals the oracle's residual of the oracle-checked blocks, bit for bit."""
    P = perturbed(case[1]())
    want = oracle.check_symmetry(P)
    x0 = problems.random_x0(P, seed=3, scale=20.0)
    s = cg.DeviceSolver(P, x0=x0)
    try:
        md, nw = s.check_symmetry()
        assert md == want[4] and nw == want[5]
        ru, rv, l2, l2r = s.residual_vector()
    finally:
        s.close()
    Q = case[1]()
    for n, w in zip(BLOCKS, want[:4]):
        setattr(Q, n, np.ascontiguousarray(w))
    o = oracle.residual_vector(Q, x0[0], x0[1], summode=oracle.SUM_DDTREE)
    np.testing.assert_array_equal(ru, o[0])
    np.testing.assert_array_equal(rv, o[1])
    assert l2 == o[2]


def test_check_symmetry_errors(gpu_lib):
    P = problems.slab_3d(seed=57, symmetrize=False)
    blocks = [np.array(getattr(P, n), copy=True) for n in BLOCKS]
    bad = np.array(asm.indxA_3d(), copy=True)
    bad[0] = 0
    with pytest.raises(cg.CismGpuError):
        cg.check_symmetry_assembled_matrix_3d(P.nx, P.ny, P.nz, P.par, bad, P.active_vertex, *blocks)
