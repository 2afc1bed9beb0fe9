"""Known-answer tests of the oracle's restatements of the boundary terms of the 3D system:
dirichlet_boundary_conditions_3d (glissade_velo_higher.F90:9305-9498) and the local form of
basal_sliding_bc_3d (:8815-9129, with glissade_stagger, glissade_gradient, glissade_unstagger
and glissade_slope_angle of glissade_grid_operators.F90).

Dirichlet: with the no-slip mask and a zero bed velocity the result is the package's numpy
no-slip assembly bit for bit; with prescribed nonzero values the modified system has, at
every other row, the residual of the original system for any velocity that takes those
values, and a zero residual at the prescribed rows.  Basal: theta against a numpy
restatement of the grid operators in the same operation order, and the bed diagonal increment.
"""
from __future__ import annotations

import numpy as np

import oracle
from cism_b200 import assembly as asm
from tests.test_oracle_assembly import geometry

BLOCKS = ("Auu", "Auv", "Avu", "Avv")


def no_slip_mask(g):
    """The vertices assemble_bp_3d treats as no-slip bed nodes (level nz)."""
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    av = g["av"]
    vmask = np.zeros_like(av)
    vmask[1:ny - 1, 1:nx - 1] = av[1:ny - 1, 1:nx - 1]
    m = np.zeros((ny - 1, nx - 1, nz), dtype=np.int32)
    m[:, :, nz - 1] = vmask
    return m


def test_dirichlet_no_slip_matches_numpy_assembly():
    g = geometry(seed=51)
    S = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], stiffness_only=True)
    W = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"])  # no-slip bed
    m = no_slip_mask(g)
    z = np.zeros_like(S.bu)
    out = oracle.dirichlet_3d(g["nx"], g["ny"], g["nz"], g["av"], m, m, z, z, S.Auu, S.Auv, S.Avu, S.Avv, S.bu, S.bv)
    for got, want in zip(out, (W.Auu, W.Auv, W.Avu, W.Avv, W.bu, W.bv)):
        np.testing.assert_array_equal(got, want)


def test_dirichlet_prescribed_values_keep_the_residual():
    g = geometry(seed=52)
    S = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], stiffness_only=True)
    rng = np.random.default_rng(9)
    m = no_slip_mask(g)
    um = m.copy()
    vm = m.copy()
    um[rng.random(um.shape) < 0.05] = 1  # extra prescribed nodes, u and v apart
    vm[rng.random(vm.shape) < 0.05] = 1
    um[~g["av"].astype(bool)] = 0
    vm[~g["av"].astype(bool)] = 0
    x = (rng.standard_normal(S.bu.shape), rng.standard_normal(S.bv.shape))
    out = oracle.dirichlet_3d(g["nx"], g["ny"], g["nz"], g["av"], um, vm, x[0], x[1], S.Auu, S.Auv, S.Avu, S.Avv,
                              S.bu, S.bv)
    P0, P1 = S, asm.Problem("3d", S.nx, S.ny, S.nz, *out, S.active_vertex, S.par)
    r0 = [a - b for a, b in zip(oracle.matvec(P0, *x), (S.bu, S.bv))]
    r1 = [a - b for a, b in zip(oracle.matvec(P1, *x), out[4:])]
    p = S.par
    own = np.zeros(S.bu.shape, dtype=bool)
    own[p["staggered_jlo"] - 1:p["staggered_jhi"], p["staggered_ilo"] - 1:p["staggered_ihi"], :] = True
    act = own & S.active_vertex.astype(bool)[..., None]
    # A node prescribed in one component only also loses the diagonal coupling to it in the
    # other component's row (Auv(0) / Avu(0) zeroed, :9355-9358, :9426-9429) without a move to
    # the right-hand side, so those rows are left out of the comparison.
    for mask, other, a, b in ((um, vm, r0[0], r1[0]), (vm, um, r0[1], r1[1])):
        fixed = act & (mask == 1)
        free = act & (mask != 1) & (other != 1)
        assert np.all(b[fixed] == 0.0)
        scale = np.abs(a[free]).max()
        assert np.abs(a[free] - b[free]).max() <= 1e-9 * scale
    assert np.any(um == 1) and np.any(vm == 1)


def numpy_theta(lsrf, dx, dy):
    """glissade_stagger, glissade_gradient (every edge), glissade_unstagger, atan: the same
    operations in the same order as the reference, vectorized."""
    s = (lsrf[1:, :-1] + lsrf[1:, 1:] + lsrf[:-1, :-1] + lsrf[:-1, 1:]) / 4.0  # (NY, NX)
    north = (s[1:, 1:] - s[1:, :-1]) / dx
    south = (s[:-1, 1:] - s[:-1, :-1]) / dx
    gx = (north + south) / 2.0
    east = (s[1:, 1:] - s[:-1, 1:]) / dy
    west = (s[1:, :-1] - s[:-1, :-1]) / dy
    gy = (east + west) / 2.0
    ddx = np.zeros_like(s)
    ddy = np.zeros_like(s)
    ddx[1:-1, 1:-1] = (gx[1:, 1:] + gx[1:, :-1] + gx[:-1, 1:] + gx[:-1, :-1]) / 4.0
    ddy[1:-1, 1:-1] = (gy[1:, 1:] + gy[1:, :-1] + gy[:-1, 1:] + gy[:-1, :-1]) / 4.0
    return np.arctan(np.sqrt(ddx * ddx + ddy * ddy))


def test_basal_local_theta_and_diagonal():
    g = geometry(seed=53)
    S = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], stiffness_only=True)
    lsrf = g["usrf"] - g["thck"] + 5.0 * np.random.default_rng(3).random(g["thck"].shape)
    beta = asm.lognormal_beta((g["ny"] - 1, g["nx"] - 1), 5)
    Auu, Avv, theta = oracle.basal_local_3d(g["nx"], g["ny"], g["nz"], g["dx"], g["dx"], g["av"], beta, lsrf, S.Auu,
                                            S.Avv)
    want = numpy_theta(lsrf, g["dx"], g["dx"])
    assert np.abs(theta - want).max() <= 1e-15 * max(np.abs(want).max(), 1e-300)
    assert np.all(theta[0, :] == 0.0) and np.all(theta[:, -1] == 0.0) and theta.max() > 0.0
    add = np.where(g["av"].astype(bool), g["dx"] * g["dx"] / 1.0e9 * beta / np.cos(theta), 0.0)
    nz = g["nz"]
    want_diag = S.Auu[..., nz - 1, 13] + add
    assert np.abs(Auu[..., nz - 1, 13] - want_diag).max() <= 1e-15 * np.abs(want_diag).max()
    d = Auu - S.Auu
    d[..., nz - 1, 13] = 0.0
    assert np.all(d == 0.0)  # nothing else changes
    np.testing.assert_array_equal(Auu[..., g["nz"] - 1, 13] - S.Auu[..., g["nz"] - 1, 13],
                                  Avv[..., g["nz"] - 1, 13] - S.Avv[..., g["nz"] - 1, 13])
