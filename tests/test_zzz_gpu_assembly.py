"""The system assembly of a Picard iteration on the device, through the C ABI:
assemble_stiffness_matrix_3d / _2d (glissade_velo_higher.F90:5382-5643, :4961-5378), the
Dirichlet and local basal terms, and the whole 3D and 2D systems on a device-resident handle.
The file is named to be collected last, so that a failure here under -x leaves every other
GPU test's result in place.

Bars, against the oracle's restatement on the same inputs:
  - constant and flow-factor viscosity: bit-exact blocks and efvs (no pow on the device, or
    the host's pow);
  - nonlinear viscosity: the flow law's pow is CUDA's, not the host C library's (a few ulp
    apart), so efvs within 1e-14 relative and every coefficient within 1e-13 of its block's
    largest; the blocks are still exactly symmetric (each element's terms are shared by the
    pair in the same order);
  - a handle's assembly equals the one-shot assembly bit for bit, with the velocity given or
    taken from the last solution.
"""
import numpy as np
import pytest

import cism_b200 as cg
import oracle
from cism_b200 import assembly as asm
from tests.test_oracle_assembly import geometry

pytestmark = pytest.mark.gpu

BLOCKS = ("Auu", "Auv", "Avu", "Avv")


def inputs(g, seed=3, scale=40.0):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed)
    shape = (ny - 1, nx - 1, nz)
    u, v = scale * rng.standard_normal(shape), scale * rng.standard_normal(shape)
    ff = 0.5 * 1.0e-16 ** (-1.0 / 3.0) * (1.0 + 0.2 * rng.random((ny, nx, nz - 1)))
    return u, v, ff


def both(g, u, v, ff, **kw):
    args = (g["nx"], g["ny"], g["nz"])
    geo = (g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"])
    o = oracle.assemble_stiffness_3d(*args, *geo, u, v, g["stagusrf"], g["stagthck"], ff, **kw)
    assert o[0] == 0
    d = cg.assemble_stiffness_matrix_3d(*args, 2, *geo, u, v, g["stagusrf"], g["stagthck"], ff, **kw)
    return o[1:], d


@pytest.mark.parametrize("efvs_opt", [0, 1])
@pytest.mark.parametrize("approx", [2, 1, 0])
def test_assembly_bitexact_without_pow(gpu_lib, approx, efvs_opt):
    g = geometry(seed=21)
    u, v, ff = inputs(g)
    o, d = both(g, u, v, ff, whichapprox=approx, whichefvs=efvs_opt, efvs_constant=3.0e6)
    for a, b in zip(o, d):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("approx", [2, 1, 0])
def test_assembly_nonlinear_viscosity(gpu_lib, approx):
    g = geometry(seed=22)
    u, v, ff = inputs(g)
    o, d = both(g, u, v, ff, whichapprox=approx)
    act = g["ac"]
    rel = np.abs(d[0][act] - o[0][act]) / o[0][act]
    assert rel.max() <= 1e-14 and np.all(d[0][~act] == 0.0)
    for a, b in zip(o[1:], d[1:]):
        scale = max(np.abs(a).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-13 * scale
    P = asm.Problem("3d", g["nx"], g["ny"], g["nz"], *d[1:], np.zeros_like(u), np.zeros_like(u),
                    g["av"].astype(np.int32), asm.default_par(g["nx"], g["ny"]))
    r = oracle.check_symmetry(P)
    assert r[4] == 0.0 and r[5] == 0


def test_assembly_permuted_index_map(gpu_lib):
    """The blocks come back in the caller's layout through its indxA_3d map."""
    g = geometry(seed=23)
    u, v, ff = inputs(g)
    perm = np.random.default_rng(5).permutation(27).astype(np.int32) + 1
    args = (g["nx"], g["ny"], g["nz"], 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"], u, v,
            g["stagusrf"], g["stagthck"], ff)
    base = cg.assemble_stiffness_matrix_3d(*args, whichefvs=0, efvs_constant=1.0e6)
    got = cg.assemble_stiffness_matrix_3d(*args, whichefvs=0, efvs_constant=1.0e6, indxA_3d=perm)
    for a, b in zip(base[1:], got[1:]):
        for c in range(27):
            np.testing.assert_array_equal(b[..., perm[c] - 1], a[..., c])


def _slab_problem(g):
    """A solvable system on the same grid: the first-Picard slab the solver tests use."""
    return asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"],
                              beta=asm.lognormal_beta((g["ny"] - 1, g["nx"] - 1), 7))


def test_assembly_on_handle(gpu_lib):
    """Into a handle: the resident blocks are the one-shot blocks (checked through the
    residual of the assembled system), with the velocity given and from the last solution."""
    g = geometry(seed=24)
    u, v, ff = inputs(g, scale=10.0)
    P = _slab_problem(g)
    geo = (2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"], g["stagusrf"], g["stagthck"], ff)
    s = cg.DeviceSolver(P, x0=(u, v))
    try:
        s.solve(cg.ALG_CHRONGEAR, cg.HO_PRECOND_DIAG, 5, 1e-6, 50)  # the slab's own, well-posed system
        xs = s.x()
        efvs_x = s.assemble_stiffness(*geo)                 # velocity: the solution, on the device
        efvs_h = s.assemble_stiffness(*geo, uvel=u, vvel=v)  # velocity from the host
        ru, rv, l2, _ = s.residual_vector()                 # A(u, v) xs - b
    finally:
        s.close()
    d = cg.assemble_stiffness_matrix_3d(g["nx"], g["ny"], g["nz"], 2, g["sigma"], g["ac"].astype(np.int32),
                                        g["xVertex"], g["yVertex"], u, v, g["stagusrf"], g["stagthck"], ff)
    np.testing.assert_array_equal(efvs_h, d[0])
    Q = _slab_problem(g)
    for n, a in zip(BLOCKS, d[1:]):
        setattr(Q, n, a)
    want = cg.compute_residual_vector_3d(Q.nx, Q.ny, Q.nz, Q.par, asm.indxA_3d(), Q.active_vertex, Q.Auu, Q.Auv,
                                         Q.Avu, Q.Avv, Q.bu, Q.bv, xs[0], xs[1])
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert l2 == want[2]
    dx = cg.assemble_stiffness_matrix_3d(g["nx"], g["ny"], g["nz"], 2, g["sigma"], g["ac"].astype(np.int32),
                                         g["xVertex"], g["yVertex"], xs[0], xs[1], g["stagusrf"], g["stagthck"], ff)
    np.testing.assert_array_equal(efvs_x, dx[0])


def test_assembly_errors(gpu_lib):
    g = geometry(seed=25)
    u, v, ff = inputs(g)
    args = [g["nx"], g["ny"], g["nz"], 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"], u, v,
            g["stagusrf"], g["stagthck"], ff]
    bad = list(args)
    bad[3] = 1  # nhalo < 2: element vertices outside the arrays
    with pytest.raises(cg.CismGpuError):
        cg.assemble_stiffness_matrix_3d(*bad)
    flat = list(args)
    flat[10] = np.zeros_like(g["stagusrf"])  # every node at z = 0: the Jacobian's z column is zero
    flat[11] = np.zeros_like(g["stagthck"])
    with pytest.raises(cg.CismGpuError):
        cg.assemble_stiffness_matrix_3d(*flat)


# ---------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, SSA (:4961-5378)
# ---------------------------------------------------------------------------

def both2(g, u, v, ff, **kw):
    args = (g["nx"], g["ny"], g["nz"])
    geo = (g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"])
    o = oracle.assemble_stiffness_2d(*args, *geo, u, v, g["stagthck"], ff, **kw)
    assert o[0] == 0
    d = cg.assemble_stiffness_matrix_2d(*args, 2, *geo, u, v, g["stagthck"], ff, **kw)
    return o[1:], d


def inputs2(g, seed=4, scale=40.0):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed)
    u, v = scale * rng.standard_normal((ny - 1, nx - 1)), scale * rng.standard_normal((ny - 1, nx - 1))
    ff = 0.5 * 1.0e-16 ** (-1.0 / 3.0) * (1.0 + 0.2 * rng.random((ny, nx, nz - 1)))
    return u, v, ff


@pytest.mark.parametrize("efvs_opt", [0, 1])
def test_ssa_assembly_bitexact_without_pow(gpu_lib, efvs_opt):
    g = geometry(seed=41, nz=6)
    u, v, ff = inputs2(g)
    o, d = both2(g, u, v, ff, whichefvs=efvs_opt, efvs_constant=2.0e6)
    for a, b in zip(o, d):
        np.testing.assert_array_equal(a, b)


def test_ssa_assembly_nonlinear_viscosity(gpu_lib):
    g = geometry(seed=42, nz=6)
    u, v, ff = inputs2(g)
    o, d = both2(g, u, v, ff)
    act = g["ac"]
    assert (np.abs(d[0][act] - o[0][act]) / o[0][act]).max() <= 1e-14 and np.all(d[0][~act] == 0.0)
    for a, b in zip(o[1:], d[1:]):
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    shape = (g["ny"] - 1, g["nx"] - 1)
    P = asm.Problem("2d", g["nx"], g["ny"], 1, *d[1:], np.zeros(shape), np.zeros(shape), g["av"].astype(np.int32),
                    asm.default_par(g["nx"], g["ny"]))
    r = oracle.check_symmetry(P)
    assert r[4] == 0.0 and r[5] == 0


def test_ssa_assembly_on_handle(gpu_lib):
    """A 2D handle: assembly from the host velocity and from the last solution equals the
    one-shot assembly (efvs bit for bit; the blocks through the residual)."""
    g = geometry(seed=43, nz=6)
    u, v, ff = inputs2(g, scale=10.0)
    P = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], asm.lognormal_beta((g["ny"] - 1, g["nx"] - 1), 8))
    geo = (2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"], g["stagthck"], g["stagthck"], ff)
    s = cg.DeviceSolver(P, x0=(u, v))
    try:
        s.solve(cg.ALG_CHRONGEAR, cg.HO_PRECOND_DIAG, 5, 1e-6, 50)
        xs = s.x()
        efvs_x = s.assemble_stiffness(*geo)
        efvs_h = s.assemble_stiffness(*geo, uvel=u, vvel=v)
        ru, rv, l2, _ = s.residual_vector()
    finally:
        s.close()
    args = (g["nx"], g["ny"], g["nz"], 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"], g["yVertex"])
    d = cg.assemble_stiffness_matrix_2d(*args, u, v, g["stagthck"], ff)
    np.testing.assert_array_equal(efvs_h, d[0])
    Q = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], asm.lognormal_beta((g["ny"] - 1, g["nx"] - 1), 8))
    for n, a in zip(BLOCKS, d[1:]):
        setattr(Q, n, a)
    want = cg.compute_residual_vector_2d(Q.nx, Q.ny, Q.par, asm.indxA_2d(), Q.active_vertex, Q.Auu, Q.Auv, Q.Avu,
                                         Q.Avv, Q.bu, Q.bv, xs[0], xs[1])
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert l2 == want[2]
    dx = cg.assemble_stiffness_matrix_2d(*args, xs[0], xs[1], g["stagthck"], ff)
    np.testing.assert_array_equal(efvs_x, dx[0])


# ---------------------------------------------------------------------------
# Boundary terms and the whole 3D system of one Picard iteration (:2829-2904)
# ---------------------------------------------------------------------------

def _masks(g, seed=9):
    from tests.test_oracle_bc import no_slip_mask
    rng = np.random.default_rng(seed)
    m = no_slip_mask(g)
    um, vm = m.copy(), m.copy()
    um[rng.random(um.shape) < 0.05] = 1
    vm[rng.random(vm.shape) < 0.05] = 1
    return um, vm


def test_dirichlet_bitexact(gpu_lib):
    g = geometry(seed=61)
    S = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], stiffness_only=True)
    um, vm = _masks(g)
    rng = np.random.default_rng(2)
    x = (rng.standard_normal(S.bu.shape), rng.standard_normal(S.bv.shape))
    want = oracle.dirichlet_3d(g["nx"], g["ny"], g["nz"], g["av"], um, vm, x[0], x[1], S.Auu, S.Auv, S.Avu, S.Avv,
                               S.bu, S.bv)
    got = [np.array(a, copy=True) for a in (S.Auu, S.Auv, S.Avu, S.Avv, S.bu, S.bv)]
    cg.dirichlet_boundary_conditions_3d(g["nx"], g["ny"], g["nz"], 2, g["av"], um, vm, x[0], x[1], *got)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_basal_local(gpu_lib):
    """atan and cos are CUDA's: the bed diagonals within 1e-15 of their size, the rest exact."""
    g = geometry(seed=62)
    S = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], stiffness_only=True)
    lsrf = g["usrf"] - g["thck"] + 5.0 * np.random.default_rng(3).random(g["thck"].shape)
    beta = asm.lognormal_beta((g["ny"] - 1, g["nx"] - 1), 5)
    wu, wv, _ = oracle.basal_local_3d(g["nx"], g["ny"], g["nz"], g["dx"], g["dx"], g["av"], beta, lsrf, S.Auu, S.Avv)
    Auu, Avv = np.array(S.Auu, copy=True), np.array(S.Avv, copy=True)
    cg.basal_sliding_bc_3d(g["nx"], g["ny"], g["nz"], 2, g["dx"], g["dx"], g["ac"], g["av"], beta, lsrf, g["xVertex"],
                           g["yVertex"], Auu, Avv)
    for a, b in ((Auu, wu), (Avv, wv)):
        d = np.abs(a - b)
        assert d[..., g["nz"] - 1, 13].max() <= 1e-15 * np.abs(b[..., g["nz"] - 1, 13]).max()
        d[..., g["nz"] - 1, 13] = 0.0
        assert np.all(d == 0.0)


@pytest.mark.parametrize("bed", ["beta", "no-slip"])
def test_system_on_handle(gpu_lib, bed):
    """cismgpu_solver_assemble_system_3d equals the one-shot calls in the reference's sequence
    (stiffness, basal term, b = load, Dirichlet, staggered halo) bit for bit, seen through the
    residual of the resident system; against the oracle's sequence within the pow/atan/cos bar."""
    g = geometry(seed=63)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    P = _slab_problem(g)
    u, v, ff = inputs(g, scale=10.0)
    lsrf = g["usrf"] - g["thck"]
    beta = asm.lognormal_beta((ny - 1, nx - 1), 7) if bed == "beta" else None
    um, vm = _masks(g) if bed == "no-slip" else (None, None)
    load = (np.array(P.bu, copy=True), np.array(P.bv, copy=True))
    geo = (g["sigma"], g["ac"].astype(np.int32), g["av"].astype(np.int32), g["xVertex"], g["yVertex"], g["stagusrf"],
           g["stagthck"], ff)
    s = cg.DeviceSolver(P, x0=(u, v))
    try:
        efvs_h = s.assemble_system(2, g["dx"], g["dx"], *geo, load[0], load[1], beta=beta, lsrf=lsrf, umask=um,
                                   vmask=vm)
        ru, rv, l2, _ = s.residual_vector()
    finally:
        s.close()
    # the same sequence through the one-shot calls
    efvs, *A = cg.assemble_stiffness_matrix_3d(nx, ny, nz, 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"],
                                               g["yVertex"], u, v, g["stagusrf"], g["stagthck"], ff)
    np.testing.assert_array_equal(efvs_h, efvs)
    bu, bv = np.array(load[0], copy=True), np.array(load[1], copy=True)
    if beta is not None:
        cg.basal_sliding_bc_3d(nx, ny, nz, 2, g["dx"], g["dx"], g["ac"], g["av"], beta, lsrf, g["xVertex"],
                               g["yVertex"], A[0], A[3])
    if um is not None:
        cg.dirichlet_boundary_conditions_3d(nx, ny, nz, 2, g["av"], um, vm, u, v, *A, bu, bv)
    Q = _slab_problem(g)
    from tests import problems
    for n, a in zip(BLOCKS, A):
        setattr(Q, n, a)
    Q.bu, Q.bv = bu, bv
    Q = problems.halo_blocks_3d(Q)
    want = cg.compute_residual_vector_3d(nx, ny, nz, Q.par, asm.indxA_3d(), Q.active_vertex, Q.Auu, Q.Auv, Q.Avu,
                                         Q.Avv, Q.bu, Q.bv, u, v)
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert l2 == want[2]


def test_dirichlet_2d_and_basal_2d_bitexact(gpu_lib):
    g = geometry(seed=71)
    nx, ny = g["nx"], g["ny"]
    S = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], np.zeros((ny - 1, nx - 1)), stiffness_only=True)
    rng = np.random.default_rng(71)
    um = (rng.random(S.bu.shape) < 0.15).astype(np.int32)
    vm = (rng.random(S.bu.shape) < 0.15).astype(np.int32)
    x = (rng.standard_normal(S.bu.shape), rng.standard_normal(S.bv.shape))
    want = oracle.dirichlet_2d(nx, ny, g["av"], um, vm, x[0], x[1], S.Auu, S.Auv, S.Avu, S.Avv, S.bu, S.bv)
    got = [np.array(a, copy=True) for a in (S.Auu, S.Auv, S.Avu, S.Avv, S.bu, S.bv)]
    cg.dirichlet_boundary_conditions_2d(nx, ny, 2, g["av"], um, vm, x[0], x[1], *got)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    beta = asm.lognormal_beta((ny - 1, nx - 1), 6)
    wu, wv = oracle.basal_local_2d(nx, ny, g["dx"], g["dx"], g["av"], beta, S.Auu, S.Avv)
    Auu, Avv = np.array(S.Auu, copy=True), np.array(S.Avv, copy=True)
    cg.basal_sliding_bc_2d(nx, ny, 2, g["dx"], g["dx"], g["ac"], g["av"], beta, g["xVertex"], g["yVertex"], Auu, Avv)
    np.testing.assert_array_equal(Auu, wu)
    np.testing.assert_array_equal(Avv, wv)


def test_system_2d_on_handle(gpu_lib):
    """cismgpu_solver_assemble_system_2d equals the one-shot sequence bit for bit (residual)."""
    g = geometry(seed=73, nz=6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    P = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], asm.lognormal_beta((ny - 1, nx - 1), 8))
    u, v, ff = inputs2(g, scale=10.0)
    beta = asm.lognormal_beta((ny - 1, nx - 1), 9)
    rng = np.random.default_rng(3)
    um = (rng.random(P.bu.shape) < 0.1).astype(np.int32)
    load = (np.array(P.bu, copy=True), np.array(P.bv, copy=True))
    s = cg.DeviceSolver(P, x0=(u, v))
    try:
        efvs_h = s.assemble_system(2, g["dx"], g["dx"], g["sigma"], g["ac"].astype(np.int32), g["av"].astype(np.int32),
                                   g["xVertex"], g["yVertex"], g["stagthck"], g["stagthck"], ff, load[0], load[1],
                                   beta=beta, umask=um, vmask=um)
        ru, rv, l2, _ = s.residual_vector()
    finally:
        s.close()
    efvs, *A = cg.assemble_stiffness_matrix_2d(nx, ny, nz, 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"],
                                               g["yVertex"], u, v, g["stagthck"], ff)
    np.testing.assert_array_equal(efvs_h, efvs)
    bu, bv = np.array(load[0], copy=True), np.array(load[1], copy=True)
    cg.basal_sliding_bc_2d(nx, ny, 2, g["dx"], g["dx"], g["ac"], g["av"], beta, g["xVertex"], g["yVertex"], A[0], A[3])
    cg.dirichlet_boundary_conditions_2d(nx, ny, 2, g["av"], um, um, u, v, *A, bu, bv)
    from tests import problems
    Q = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], asm.lognormal_beta((ny - 1, nx - 1), 8))
    for n, a in zip(BLOCKS, A):
        setattr(Q, n, a)
    Q.bu, Q.bv = bu, bv
    Q = problems.halo_blocks_2d(Q)
    want = cg.compute_residual_vector_2d(nx, ny, Q.par, asm.indxA_2d(), Q.active_vertex, Q.Auu, Q.Auv, Q.Avu, Q.Avv,
                                         Q.bu, Q.bv, u, v)
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert l2 == want[2]


@pytest.mark.parametrize("kind", ["3d", "2d"])
def test_basal_standard_bitexact(gpu_lib, kind):
    """The standard finite-element basal form: only IEEE operations (sqrt included), so the
    blocks equal the oracle's bit for bit, also on top of an assembled stiffness."""
    g = geometry(seed=64)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    lsrf = g["usrf"] - g["thck"] + 5.0 * np.random.default_rng(4).random(g["thck"].shape)
    beta = asm.lognormal_beta((ny - 1, nx - 1), 6)
    if kind == "3d":
        S = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], nz, stiffness_only=True)
    else:
        S = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], np.zeros((ny - 1, nx - 1)),
                                stiffness_only=True)
    st, wu, wv = oracle.basal_standard(kind == "3d", nx, ny, nz, g["ac"], g["xVertex"], g["yVertex"], beta,
                                       lsrf if kind == "3d" else None, S.Auu, S.Avv)
    assert st == 0
    Auu, Avv = np.array(S.Auu, copy=True), np.array(S.Avv, copy=True)
    if kind == "3d":
        cg.basal_sliding_bc_3d(nx, ny, nz, 2, g["dx"], g["dx"], g["ac"], g["av"], beta, lsrf, g["xVertex"],
                               g["yVertex"], Auu, Avv, whichassemble_beta=0)
    else:
        cg.basal_sliding_bc_2d(nx, ny, 2, g["dx"], g["dx"], g["ac"], g["av"], beta, g["xVertex"], g["yVertex"], Auu,
                               Avv, whichassemble_beta=0)
    np.testing.assert_array_equal(Auu, wu)
    np.testing.assert_array_equal(Avv, wv)


# ---------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, DIVA branch
# ---------------------------------------------------------------------------

def _diva_case(seed=37, nz=5, traction=4.0e4):
    from tests.test_oracle_assembly import diva_inputs
    g = geometry(seed=seed, nz=nz)
    nx, ny = g["nx"], g["ny"]
    rng = np.random.default_rng(seed)
    u, v = 20 * rng.standard_normal((ny - 1, nx - 1)), 20 * rng.standard_normal((ny - 1, nx - 1))
    ff = 0.5 * 1e-16 ** (-1 / 3) * (1 + 0.3 * rng.random((ny, nx, nz - 1)))
    return g, u, v, ff, diva_inputs(g, 2, traction)


def _diva_gpu(g, u, v, ff, extra, eq, **kw):
    stagsig, bx, by, dsfx, dsfy = extra
    return cg.assemble_stiffness_matrix_2d_diva(g["nx"], g["ny"], g["nz"], 2, g["sigma"], stagsig,
                                                g["ac"].astype(np.int32), g["xVertex"], g["yVertex"], u, v,
                                                g["stagthck"], g["thck"], bx, by, dsfx, dsfy, ff, eq, **kw)


def _diva_oracle(g, u, v, ff, extra, eq, **kw):
    stagsig, bx, by, dsfx, dsfy = extra
    o = oracle.assemble_stiffness_2d_diva(g["nx"], g["ny"], g["nz"], g["sigma"], stagsig, g["ac"], g["xVertex"],
                                          g["yVertex"], u, v, g["stagthck"], g["thck"], bx, by, dsfx, dsfy, ff, eq, **kw)
    assert o[0] == 0
    return o[1:]


def test_diva_constant_viscosity_bitexact(gpu_lib):
    g, u, v, ff, extra = _diva_case()
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    eq = np.zeros((ny, nx, 4, nz - 1))
    efvs, eq_o, ok_o, om_o, *Ao = _diva_oracle(g, u, v, ff, extra, eq, whichefvs=0, efvs_constant=2.0e6)
    d = _diva_gpu(g, u, v, ff, extra, eq, whichefvs=0, efvs_constant=2.0e6)
    np.testing.assert_array_equal(eq, eq_o)
    for a, b in zip(d, (efvs, ok_o, om_o, *Ao)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("start", ["zero", "previous"])
def test_diva_nonlinear(gpu_lib, start):
    """The layer viscosities within 1e-14 (pow is CUDA's), the blocks within 1e-13 of their
    largest, the integrals within 1e-13; from a zero state (the first Picard iteration) and
    from a previous one."""
    g, u, v, ff, extra = _diva_case(seed=38)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(1)
    eq = np.zeros((ny, nx, 4, nz - 1)) if start == "zero" else 1e6 * (1 + rng.random((ny, nx, 4, nz - 1)))
    eq_gpu = np.array(eq, copy=True)
    efvs, eq_o, ok_o, om_o, *Ao = _diva_oracle(g, u, v, ff, extra, eq)
    efvs_d, ok_d, om_d, *Ad = _diva_gpu(g, u, v, ff, extra, eq_gpu)
    act = g["ac"]
    assert np.abs(eq_gpu - eq_o).max() <= 1e-14 * np.abs(eq_o).max()
    assert np.all(eq_gpu[~act] == eq[~act])
    assert np.abs(efvs_d - efvs).max() <= 1e-14 * np.abs(efvs).max()
    assert np.abs(ok_d - ok_o).max() <= 1e-13 * np.abs(ok_o).max()
    assert np.abs(om_d - om_o).max() <= 1e-13 * np.abs(om_o).max()
    for a, b in zip(Ad, Ao):
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_diva_state_on_handle(gpu_lib):
    """Two DIVA assemblies in a row on a handle, the layer viscosities kept on the device, equal
    the one-shot calls carrying the state on the host, bit for bit."""
    g, u, v, ff, extra = _diva_case(seed=39)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    stagsig, bx, by, dsfx, dsfy = extra
    P = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], asm.lognormal_beta((ny - 1, nx - 1), 8))
    s = cg.DeviceSolver(P, x0=(u, v))
    out_h = []
    try:
        for it in range(2):
            out_h.append(s.assemble_stiffness_diva(nz, 2, g["sigma"], stagsig, g["ac"].astype(np.int32), g["xVertex"],
                                                   g["yVertex"], g["stagthck"], g["thck"], bx, by, dsfx, dsfy, ff,
                                                   uvel=u * (1 + it), vvel=v * (1 + it)))
        ru, rv, l2, _ = s.residual_vector()
    finally:
        s.close()
    eq = np.zeros((ny, nx, 4, nz - 1))
    for it in range(2):
        d = _diva_gpu(g, u * (1 + it), v * (1 + it), ff, extra, eq)
        for a, b in zip(out_h[it], d[:3]):
            np.testing.assert_array_equal(a, b)
    Q = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], asm.lognormal_beta((ny - 1, nx - 1), 8))
    for n, a in zip(BLOCKS, d[3:]):
        setattr(Q, n, a)
    want = cg.compute_residual_vector_2d(nx, ny, Q.par, asm.indxA_2d(), Q.active_vertex, Q.Auu, Q.Auv, Q.Avu, Q.Avv,
                                         Q.bu, Q.bv, u, v)
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])


@pytest.mark.parametrize("mode", [1, 0])
def test_basal_diva(gpu_lib, mode):
    """basal_sliding_bc_2d_diva: the standard form bit-exact; the local form's diagonals within
    1e-15 of their size (atan and cos are CUDA's), the rest exact."""
    g = geometry(seed=65)
    nx, ny, dx = g["nx"], g["ny"], g["dx"]
    S = asm.assemble_ssa_2d(g["thck"], g["usrf"], dx, dx, np.zeros((ny - 1, nx - 1)), stiffness_only=True)
    lsrf = g["usrf"] - g["thck"] + 5.0 * np.random.default_rng(4).random(g["thck"].shape)
    bex, bey = asm.lognormal_beta((ny - 1, nx - 1), 6), asm.lognormal_beta((ny - 1, nx - 1), 7)
    wu, wv = oracle.basal_diva(nx, ny, dx, dx, g["ac"], g["av"], bex, bey, lsrf, g["xVertex"], g["yVertex"], mode,
                               S.Auu, S.Avv)
    Auu, Avv = np.array(S.Auu, copy=True), np.array(S.Avv, copy=True)
    cg.basal_sliding_bc_2d_diva(nx, ny, 2, dx, dx, g["ac"], g["av"], bex, bey, lsrf, g["xVertex"], g["yVertex"], Auu, Avv,
                                whichassemble_beta=mode)
    if mode == 0:
        np.testing.assert_array_equal(Auu, wu)
        np.testing.assert_array_equal(Avv, wv)
    else:
        for a, b in ((Auu, wu), (Avv, wv)):
            d = np.abs(a - b)
            assert d[4].max() <= 1e-15 * np.abs(b[4]).max()
            d[4] = 0.0
            assert np.all(d == 0.0)


def test_diva_system_on_handle(gpu_lib):
    """cismgpu_solver_assemble_system_2d_diva equals the one-shot sequence (DIVA stiffness, DIVA
    basal term, b = load, Dirichlet, staggered halo) bit for bit, through the residual."""
    g, u, v, ff, extra = _diva_case(seed=40)
    nx, ny, nz, dx = g["nx"], g["ny"], g["nz"], g["dx"]
    stagsig, bx, by, dsfx, dsfy = extra
    P = asm.assemble_ssa_2d(g["thck"], g["usrf"], dx, dx, asm.lognormal_beta((ny - 1, nx - 1), 8))
    bex, bey = asm.lognormal_beta((ny - 1, nx - 1), 6), asm.lognormal_beta((ny - 1, nx - 1), 7)
    lsrf = g["usrf"] - g["thck"]
    um = (np.random.default_rng(3).random(P.bu.shape) < 0.1).astype(np.int32)
    load = (np.array(P.bu, copy=True), np.array(P.bv, copy=True))
    s = cg.DeviceSolver(P, x0=(u, v))
    try:
        eh = s.assemble_system_diva(nz, 2, dx, dx, g["sigma"], stagsig, g["ac"].astype(np.int32),
                                    g["av"].astype(np.int32), g["xVertex"], g["yVertex"], g["stagthck"], g["thck"], bx,
                                    by, dsfx, dsfy, ff, load[0], load[1], beta_eff_x=bex, beta_eff_y=bey, lsrf=lsrf,
                                    umask=um, vmask=um)
        ru, rv, l2, _ = s.residual_vector()
    finally:
        s.close()
    eq = np.zeros((ny, nx, 4, nz - 1))
    efvs, ok, om, *A = _diva_gpu(g, u, v, ff, extra, eq)
    for a, b in zip(eh, (efvs, ok, om)):
        np.testing.assert_array_equal(a, b)
    bu, bv = np.array(load[0], copy=True), np.array(load[1], copy=True)
    cg.basal_sliding_bc_2d_diva(nx, ny, 2, dx, dx, g["ac"], g["av"], bex, bey, lsrf, g["xVertex"], g["yVertex"], A[0],
                                A[3])
    cg.dirichlet_boundary_conditions_2d(nx, ny, 2, g["av"], um, um, u, v, *A, bu, bv)
    from tests import problems
    Q = asm.assemble_ssa_2d(g["thck"], g["usrf"], dx, dx, asm.lognormal_beta((ny - 1, nx - 1), 8))
    for n, a in zip(BLOCKS, A):
        setattr(Q, n, a)
    Q.bu, Q.bv = bu, bv
    Q = problems.halo_blocks_2d(Q)
    want = cg.compute_residual_vector_2d(nx, ny, Q.par, asm.indxA_2d(), Q.active_vertex, Q.Auu, Q.Auv, Q.Avu, Q.Avv,
                                         Q.bu, Q.bv, u, v)
    np.testing.assert_array_equal(ru, want[0])
    np.testing.assert_array_equal(rv, want[1])
    assert l2 == want[2]


# ---------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, L1L2 branch
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n_glen", [3.0, 1.0])
def test_l1l2(gpu_lib, n_glen):
    """n = 1 bit-exact (no pow); n = 3 within the pow bar: efvs 1e-14, blocks 1e-13."""
    g = geometry(seed=93, nz=5)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(3)
    u, v = 30 * rng.standard_normal((ny - 1, nx - 1)), 30 * rng.standard_normal((ny - 1, nx - 1))
    dsdx, dsdy = 0.01 * rng.standard_normal((ny - 1, nx - 1)), 0.01 * rng.standard_normal((ny - 1, nx - 1))
    flwa = 1e-16 * (1 + rng.random((ny, nx, nz - 1)))
    ff = 0.5 * flwa ** (-1 / 3)
    st, eo, *Ao = oracle.assemble_stiffness_2d_l1l2(nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v,
                                                     g["stagthck"], dsdx, dsdy, flwa, ff, n_glen=n_glen)
    assert st == 0
    e, *Ad = cg.assemble_stiffness_matrix_2d_l1l2(nx, ny, nz, 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"],
                                                  g["yVertex"], u, v, g["stagthck"], dsdx, dsdy, flwa, ff,
                                                  n_glen=n_glen)
    if n_glen == 1.0:
        np.testing.assert_array_equal(e, eo)
        for a, b in zip(Ad, Ao):
            np.testing.assert_array_equal(a, b)
    else:
        assert np.abs(e - eo).max() <= 1e-14 * np.abs(eo).max()
        for a, b in zip(Ad, Ao):
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    with pytest.raises(cg.CismGpuError):
        cg.assemble_stiffness_matrix_2d_l1l2(nx, ny, nz, 2, g["sigma"], g["ac"].astype(np.int32), g["xVertex"],
                                             g["yVertex"], u, v, g["stagthck"], dsdx, dsdy, flwa, ff, n_glen=2.0)


@pytest.mark.parametrize("taud", [1, 0])
def test_load_vector_gravity_bitexact(gpu_lib, taud):
    from tests.test_oracle_bc import load_geometry
    g = load_geometry()
    nx, ny, nz, dx = g["nx"], g["ny"], g["nz"], g["dx"]
    rng = np.random.default_rng(5)
    sx, sy = 0.01 * rng.standard_normal((ny - 1, nx - 1)), 0.01 * rng.standard_normal((ny - 1, nx - 1))
    args = (nx, ny, nz)
    st, wu, wv = oracle.load_vector_gravity(*args, g["sigma"], g["stagw"], dx, dx, g["ac"], g["av"], g["xVertex"],
                                            g["yVertex"], g["stagusrf"], g["stagthck"], sx, sy, taud)
    assert st == 0
    lu, lv = cg.load_vector_gravity(*args, 2, g["sigma"], g["stagw"], dx, dx, g["ac"], g["av"], g["xVertex"],
                                    g["yVertex"], g["stagusrf"], g["stagthck"], sx, sy, whichassemble_taud=taud)
    np.testing.assert_array_equal(lu, wu)
    np.testing.assert_array_equal(lv, wv)
