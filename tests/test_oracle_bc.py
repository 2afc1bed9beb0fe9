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
    W = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], symmetrize=False)  # no-slip bed
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


# ---------------------------------------------------------------------------
# 2D: dirichlet_boundary_conditions_2d (:9133-9301), basal_sliding_bc_2d local (:8281-8531)
# ---------------------------------------------------------------------------

def _ssa(g):
    return asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], np.zeros((g["ny"] - 1, g["nx"] - 1)),
                               stiffness_only=True)


def test_dirichlet_2d_prescribed_values_keep_the_residual():
    g = geometry(seed=54)
    S = _ssa(g)
    rng = np.random.default_rng(10)
    m = (rng.random(S.bu.shape) < 0.1).astype(np.int32) * g["av"].astype(np.int32)
    x = (rng.standard_normal(S.bu.shape), rng.standard_normal(S.bv.shape))
    out = oracle.dirichlet_2d(g["nx"], g["ny"], g["av"], m, m, x[0], x[1], S.Auu, S.Auv, S.Avu, S.Avv, S.bu, S.bv)
    P1 = asm.Problem("2d", S.nx, S.ny, 1, *out, S.active_vertex, S.par)
    r0 = [a - b for a, b in zip(oracle.matvec(S, *x), (S.bu, S.bv))]
    r1 = [a - b for a, b in zip(oracle.matvec(P1, *x), out[4:])]
    p = S.par
    own = np.zeros(S.bu.shape, dtype=bool)
    own[p["staggered_jlo"] - 1:p["staggered_jhi"], p["staggered_ilo"] - 1:p["staggered_ihi"]] = True
    act = own & S.active_vertex.astype(bool)
    for a, b in zip(r0, r1):
        assert np.all(b[act & (m == 1)] == 0.0)
        free = act & (m != 1)
        assert np.abs(a[free] - b[free]).max() <= 1e-9 * np.abs(a[free]).max()
    assert np.any(m[act] == 1)


def test_dirichlet_2d_diagonals():
    """A u-only prescribed vertex gets unit Auu, Auv and Avu diagonals, a v-only one zero Auv
    and Avu and a unit Avv; with both, Auu = Avv = 1 and Auv = Avu = 0."""
    g = geometry(seed=55)
    S = _ssa(g)
    av = g["av"].astype(bool)
    J, I = np.nonzero(av[2:-2, 2:-2])
    pts = [(J[n] + 2, I[n] + 2) for n in (0, len(J) // 2, len(J) - 1)]
    um = np.zeros(S.bu.shape, np.int32)
    vm = np.zeros(S.bu.shape, np.int32)
    (ju, iu), (jv, iv), (jb, ib) = pts
    um[ju, iu] = 1
    vm[jv, iv] = 1
    um[jb, ib] = vm[jb, ib] = 1
    z = np.zeros(S.bu.shape)
    Auu, Auv, Avu, Avv, bu, bv = oracle.dirichlet_2d(g["nx"], g["ny"], g["av"], um, vm, z, z, S.Auu, S.Auv, S.Avu,
                                                     S.Avv, S.bu, S.bv)
    assert (Auu[4, ju, iu], Auv[4, ju, iu], Avu[4, ju, iu]) == (1.0, 1.0, 1.0)
    assert Avv[4, ju, iu] == S.Avv[4, ju, iu]
    assert (Auv[4, jv, iv], Avu[4, jv, iv], Avv[4, jv, iv]) == (0.0, 0.0, 1.0)
    assert (Auu[4, jb, ib], Auv[4, jb, ib], Avu[4, jb, ib], Avv[4, jb, ib]) == (1.0, 0.0, 0.0, 1.0)
    for m in range(9):
        if m != 4:
            assert Auu[m, ju, iu] == Auv[m, ju, iu] == 0.0
            assert Avu[m, jv, iv] == Avv[m, jv, iv] == 0.0


def test_basal_local_2d():
    g = geometry(seed=56)
    S = _ssa(g)
    beta = asm.lognormal_beta((g["ny"] - 1, g["nx"] - 1), 6)
    Auu, Avv = oracle.basal_local_2d(g["nx"], g["ny"], g["dx"], g["dx"], g["av"], beta, S.Auu, S.Avv)
    inc = np.where(g["av"].astype(bool), (g["dx"] * g["dx"] / 1.0e9) * beta, 0.0)
    np.testing.assert_array_equal(Auu[4], S.Auu[4] + inc)
    np.testing.assert_array_equal(Avv[4], S.Avv[4] + inc)
    np.testing.assert_array_equal(np.delete(Auu, 4, axis=0), np.delete(S.Auu, 4, axis=0))


# ---------------------------------------------------------------------------
# basal_sliding_bc_3d / _2d, standard finite-element form
# ---------------------------------------------------------------------------

def test_basal_standard_integrates_beta_over_the_bed():
    """Summed over all coefficients, the basal matrices integrate beta over the bed: with a
    constant beta and a planar lower surface z = a x + b y, each active cell adds
    beta * dx*dy * sqrt(1 + a^2 + b^2) / vol0 in 3D (the curved area factor) and
    beta * dx*dy / vol0 in 2D; Auu and Avv get the same increments; row sums split each cell's
    share over its 4 vertices."""
    g = geometry(seed=57)
    nx, ny, nz, dx = g["nx"], g["ny"], g["nz"], g["dx"]
    a, b = 0.02, -0.01
    xc = (np.arange(nx) - 0.5) * dx  # cell centres, so the staggered surface is a x + b y at vertices
    yc = (np.arange(ny) - 0.5) * dx
    lsrf = a * xc[None, :] + b * yc[:, None]
    beta = np.full((ny - 1, nx - 1), 250.0)
    ncell = int(np.count_nonzero(g["ac"][2:ny - 1, 2:nx - 1]))
    z3 = np.zeros((ny - 1, nx - 1, nz, 27))  # zero blocks: the increments alone
    st, d, dv = oracle.basal_standard(True, nx, ny, nz, g["ac"], g["xVertex"], g["yVertex"], beta, lsrf, z3, z3)
    assert st == 0
    np.testing.assert_array_equal(d, dv)
    want = 250.0 * dx * dx * np.sqrt(1 + a * a + b * b) / 1.0e9 * ncell
    assert abs(d.sum() - want) <= 1e-12 * want
    assert np.all(d[..., :nz - 1, :] == 0.0) and np.all(d[..., nz - 1, :9] == 0.0) and np.all(d[..., nz - 1, 18:] == 0.0)
    z2 = np.zeros((9, ny - 1, nx - 1))
    st, d2, _ = oracle.basal_standard(False, nx, ny, 1, g["ac"], g["xVertex"], g["yVertex"], beta, None, z2, z2)
    assert st == 0
    want2 = 250.0 * dx * dx / 1.0e9 * ncell
    assert abs(d2.sum() - want2) <= 1e-12 * want2
    # a flat bed cell splits its integral 4/9, 2/9, 2/9, 1/9 (the bilinear mass matrix): the
    # diagonal of a vertex inside the ice gets 4 cells x 4/9 x (beta dx dy / 4 / vol0) ... here
    # just the ratio of the 2D diagonal to the row sum at such a vertex
    full = g["ac"][:-1, :-1] & g["ac"][:-1, 1:] & g["ac"][1:, :-1] & g["ac"][1:, 1:]
    J, I = np.nonzero(full)
    j, i = J[len(J) // 2], I[len(I) // 2]
    assert abs(d2[4, j, i] / d2[:, j, i].sum() - 4.0 / 9.0) <= 1e-12


# ---------------------------------------------------------------------------
# basal_sliding_bc_2d_diva (:8535-8811)
# ---------------------------------------------------------------------------

def numpy_slope_xy(lsrf, dx, dy):
    """dz/dx and dz/dy of glissade_slope_angle on the staggered lower surface (the chain of
    numpy_theta without the final atan of the length)."""
    s = (lsrf[1:, :-1] + lsrf[1:, 1:] + lsrf[:-1, :-1] + lsrf[:-1, 1:]) / 4.0
    gx = ((s[1:, 1:] - s[1:, :-1]) / dx + (s[:-1, 1:] - s[:-1, :-1]) / dx) / 2.0
    gy = ((s[1:, 1:] - s[:-1, 1:]) / dy + (s[1:, :-1] - s[:-1, :-1]) / dy) / 2.0
    ddx = np.zeros_like(s)
    ddy = np.zeros_like(s)
    ddx[1:-1, 1:-1] = (gx[1:, 1:] + gx[1:, :-1] + gx[:-1, 1:] + gx[:-1, :-1]) / 4.0
    ddy[1:-1, 1:-1] = (gy[1:, 1:] + gy[1:, :-1] + gy[:-1, 1:] + gy[:-1, :-1]) / 4.0
    return ddx, ddy


def test_basal_diva_local():
    g = geometry(seed=58)
    nx, ny, dx = g["nx"], g["ny"], g["dx"]
    z2 = np.zeros((9, ny - 1, nx - 1))
    lsrf = g["usrf"] - g["thck"] + 5.0 * np.random.default_rng(2).random(g["thck"].shape)
    bex, bey = asm.lognormal_beta((ny - 1, nx - 1), 3), asm.lognormal_beta((ny - 1, nx - 1), 4)
    Auu, Avv = oracle.basal_diva(nx, ny, dx, dx, g["ac"], g["av"], bex, bey, lsrf, g["xVertex"], g["yVertex"], 1, z2, z2)
    ddx, ddy = numpy_slope_xy(lsrf, dx, dx)
    av = g["av"].astype(bool)
    wu = np.where(av, (dx * dx / 1.0e9) * bex / np.cos(np.arctan(np.abs(ddx))), 0.0)
    wv = np.where(av, (dx * dx / 1.0e9) * bey / np.cos(np.arctan(np.abs(ddy))), 0.0)
    assert np.abs(Auu[4] - wu).max() <= 1e-15 * np.abs(wu).max()
    assert np.abs(Avv[4] - wv).max() <= 1e-15 * np.abs(wv).max()
    assert np.all(np.delete(Auu, 4, axis=0) == 0.0) and np.all(np.delete(Avv, 4, axis=0) == 0.0)


def test_basal_diva_standard_integrates_over_the_bed():
    g = geometry(seed=59)
    nx, ny, dx = g["nx"], g["ny"], g["dx"]
    a, b = -0.015, 0.02
    xc = (np.arange(nx) - 0.5) * dx
    yc = (np.arange(ny) - 0.5) * dx
    lsrf = a * xc[None, :] + b * yc[:, None]
    z2 = np.zeros((9, ny - 1, nx - 1))
    bex, bey = np.full((ny - 1, nx - 1), 200.0), np.full((ny - 1, nx - 1), 300.0)
    Auu, Avv = oracle.basal_diva(nx, ny, dx, dx, g["ac"], g["av"], bex, bey, lsrf, g["xVertex"], g["yVertex"], 0, z2, z2)
    ncell = int(np.count_nonzero(g["ac"][2:ny - 1, 2:nx - 1]))
    area = dx * dx * np.sqrt(1 + a * a + b * b) / 1.0e9 * ncell
    assert abs(Auu.sum() - 200.0 * area) <= 1e-12 * 200.0 * area
    assert abs(Avv.sum() - 300.0 * area) <= 1e-12 * 300.0 * area


# ---------------------------------------------------------------------------
# load_vector_gravity (:4228-4449)
# ---------------------------------------------------------------------------

def load_geometry(H0=900.0, a=-0.01, b=0.004, nz=5, seed=60):
    g = geometry(seed=seed, nz=nz)
    nx, ny, dx = g["nx"], g["ny"], g["dx"]
    ice = g["thck"] > 0.0
    thck = np.where(ice, H0, 0.0)
    xc = (np.arange(nx) - 0.5) * dx
    yc = (np.arange(ny) - 0.5) * dx
    usrf = 2000.0 + a * xc[None, :] + b * yc[:, None]
    ac, av = asm.active_masks(thck)
    sig = g["sigma"]
    stagw = np.concatenate([[0.0], 0.5 * (sig[:-1] + sig[1:]), [1.0]])
    return dict(g, thck=thck, ac=ac, av=av, stagusrf=asm.stagger(usrf, thck > 1.0),
                stagthck=asm.stagger(thck, thck > 1.0), stagw=stagw, H0=H0, a=a, b=b)


def test_load_local_is_the_column_formula():
    g = load_geometry()
    nx, ny, nz, dx = g["nx"], g["ny"], g["nz"], g["dx"]
    rng = np.random.default_rng(5)
    sx, sy = 0.01 * rng.standard_normal((ny - 1, nx - 1)), 0.01 * rng.standard_normal((ny - 1, nx - 1))
    st, lu, lv = oracle.load_vector_gravity(nx, ny, nz, g["sigma"], g["stagw"], dx, dx, g["ac"], g["av"], g["xVertex"],
                                            g["yVertex"], g["stagusrf"], g["stagthck"], sx, sy, 1)
    assert st == 0
    dz = g["stagthck"][..., None] * np.diff(g["stagw"])[None, None, :]
    av = g["av"].astype(bool)[..., None]
    np.testing.assert_array_equal(lu, np.where(av, 0.0 - 910.0 * 9.81 * dx * dx * dz / 1.0e9 * sx[..., None], 0.0))
    np.testing.assert_array_equal(lv, np.where(av, 0.0 - 910.0 * 9.81 * dx * dx * dz / 1.0e9 * sy[..., None], 0.0))


def test_load_standard_integrates_the_driving_stress():
    """Constant thickness H0 and a constant surface gradient: summed over all nodes, the
    standard load is -rhoi*g*(ds/dx)*(ice volume)/vol0, the volume being dx*dy*H0 per active cell
    (the 2x2x2 Gauss rule integrates the trilinear Jacobian exactly)."""
    g = load_geometry()
    nx, ny, nz, dx = g["nx"], g["ny"], g["nz"], g["dx"]
    sx, sy = np.full((ny - 1, nx - 1), g["a"]), np.full((ny - 1, nx - 1), g["b"])
    st, lu, lv = oracle.load_vector_gravity(nx, ny, nz, g["sigma"], g["stagw"], dx, dx, g["ac"], g["av"], g["xVertex"],
                                            g["yVertex"], g["stagusrf"], g["stagthck"], sx, sy, 0)
    assert st == 0
    ncell = int(np.count_nonzero(g["ac"][2:ny - 1, 2:nx - 1]))
    vol = ncell * dx * dx * g["H0"]
    for load, s in ((lu, g["a"]), (lv, g["b"])):
        want = -910.0 * 9.81 * s * vol / 1.0e9
        assert abs(load.sum() - want) <= 1e-11 * abs(want)
