"""Known-answer tests of the oracle's restatement of assemble_stiffness_matrix_3d
(libglissade/glissade_velo_higher.F90:5382-5643).

Checks against independent mathematics and against the package's vectorized numpy
assembly (a different summation order, so agreement is to roundoff):
  - at u = 0 the blocks equal the numpy first-Picard assembly to 1e-12 of the largest entry;
  - the element-by-element scatter makes A exactly symmetric (the symmetry check finds 0);
  - a velocity linear in x, y and z has constant strain rates on trilinear elements, so
    every element's viscosity equals the flow law evaluated at those rates;
  - constant viscosity: a uniform velocity is in the null space of each interior row;
  - efvs constant and flow-factor options.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from cism_b200 import assembly as asm

N_GLEN = 3.0


def geometry(ewn=9, nsn=8, nz=5, seed=0, dx=2000.0):
    """Cell fields of a sloping slab with a notch (as the solver tests use) and the inputs
    assemble_stiffness_matrix_3d takes."""
    rng = np.random.default_rng(seed)
    nx, ny = ewn + 4, nsn + 4
    H = 800.0 + 400.0 * rng.random((ny, nx))
    x = (np.arange(nx) + 0.5) * dx
    usrf = 2000.0 - x[None, :] * 0.01 + 30.0 * rng.random((ny, nx))
    ice = np.zeros((ny, nx), dtype=bool)
    ice[3:ny - 3, 3:nx - 3] = True
    ice[3:5, 3:5] = False
    thck = np.where(ice, H, 0.0)
    usrf = np.where(ice, usrf, usrf - H)
    ac, av = asm.active_masks(thck)
    g = dict(nx=nx, ny=ny, nz=nz, dx=dx, thck=thck, usrf=usrf, ac=ac, av=av,
             sigma=asm.glide_sigma(nz),
             xVertex=np.broadcast_to(np.arange(nx - 1) * dx, (ny - 1, nx - 1)).copy(),
             yVertex=np.broadcast_to((np.arange(ny - 1) * dx)[:, None], (ny - 1, nx - 1)).copy(),
             stagusrf=asm.stagger(usrf, thck > 1.0), stagthck=asm.stagger(thck, thck > 1.0))
    return g


def run(g, uvel=None, vvel=None, flwa=1.0e-16, **kw):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    shape = (ny - 1, nx - 1, nz)
    u = np.zeros(shape) if uvel is None else uvel
    v = np.zeros(shape) if vvel is None else vvel
    flwafact = np.full((ny, nx, nz - 1), 0.5 * flwa ** (-1.0 / N_GLEN))
    st, efvs, Auu, Auv, Avu, Avv = oracle.assemble_stiffness_3d(
        nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v, g["stagusrf"], g["stagthck"], flwafact,
        **kw)
    assert st == 0
    return efvs, Auu, Auv, Avu, Avv


def test_first_picard_matches_numpy_assembly():
    g = geometry(seed=1)
    efvs, *A = run(g)
    P = asm.assemble_bp_3d(g["thck"], g["usrf"], g["dx"], g["dx"], g["nz"], stiffness_only=True)
    scale = max(np.abs(P.Auu).max(), np.abs(P.Avv).max())
    for got, want in zip(A, (P.Auu, P.Auv, P.Avu, P.Avv)):
        assert np.abs(got - want).max() <= 1e-12 * scale
    e0 = asm.first_picard_efvs(1.0e-16)
    act = g["ac"]
    assert np.all(np.abs(efvs[act] - e0) <= 1e-14 * e0) and np.all(efvs[~act] == 0.0)


def test_scatter_is_exactly_symmetric():
    """Each element matrix is symmetric bit for bit and every entry sums its elements in the
    same order as its transpose partner: the assembled blocks are exactly symmetric."""
    g = geometry(seed=2)
    rng = np.random.default_rng(3)
    shape = (g["ny"] - 1, g["nx"] - 1, g["nz"])
    efvs, *A = run(g, 50.0 * rng.standard_normal(shape), 50.0 * rng.standard_normal(shape))
    P = asm.Problem("3d", g["nx"], g["ny"], g["nz"], *A, np.zeros(shape), np.zeros(shape),
                    g["av"].astype(np.int32), asm.default_par(g["nx"], g["ny"]))
    r = oracle.check_symmetry(P)
    assert r[4] == 0.0 and r[5] == 0
    assert np.abs(A[0]).max() > 0.0


@pytest.mark.parametrize("approx", [2, 1, 0])
def test_linear_velocity_gives_the_flow_law_viscosity(approx):
    """u = a.x, v = b.x (x = (x, y, z) of each node): trilinear elements reproduce linear
    fields, so the strain rates at every quadrature point are (a, b)."""
    g = geometry(seed=4)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    X = np.broadcast_to(g["xVertex"][..., None], (ny - 1, nx - 1, nz))
    Y = np.broadcast_to(g["yVertex"][..., None], (ny - 1, nx - 1, nz))
    Z = g["stagusrf"][..., None] - g["sigma"][None, None, :] * g["stagthck"][..., None]
    a = (3.0e-3, -1.0e-3, 2.0e-2)
    b = (1.5e-3, 2.5e-3, -1.0e-2)
    u = a[0] * X + a[1] * Y + a[2] * Z
    v = b[0] * X + b[1] * Y + b[2] * Z
    flwa = 1.0e-16
    efvs, *A = run(g, u, v, flwa=flwa, whichapprox=approx)
    emin = 1.0e-8
    if approx == 0:
        sq = emin ** 2 + 0.25 * (a[2] ** 2 + b[2] ** 2)
    else:
        sq = emin ** 2 + (a[0] ** 2 + b[1] ** 2 + a[0] * b[1] + 0.25 * (b[0] + a[1]) ** 2)
        if approx == 2:
            sq += 0.25 * (a[2] ** 2 + b[2] ** 2)
    want = 0.5 * flwa ** (-1.0 / N_GLEN) * sq ** ((1.0 - N_GLEN) / N_GLEN / 2.0)
    act = g["ac"]
    assert np.all(np.abs(efvs[act] - want) <= 1e-12 * want)
    if approx == 0:  # SIA: only vertical derivatives, no coupling blocks
        assert np.all(A[1] == 0.0) and np.all(A[2] == 0.0)


def test_constant_viscosity_null_space():
    """With a constant viscosity, a uniform velocity (u = 1, v = 0) gives zero stress: every
    row whose 8 surrounding elements all exist sums to zero (to roundoff)."""
    g = geometry(seed=5)
    efvs, Auu, Auv, Avu, Avv = run(g, whichefvs=0, efvs_constant=1.0e6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    ac = g["ac"]
    full = ac[:-1, :-1] & ac[:-1, 1:] & ac[1:, :-1] & ac[1:, 1:]  # vertex with 4 active cells around
    rows_u = Auu.sum(axis=-1)
    rows_v = Avu.sum(axis=-1)
    scale = np.abs(Auu).max()
    inner = np.zeros((ny - 1, nx - 1, nz), dtype=bool)
    inner[full, :] = True
    assert np.abs(rows_u[inner]).max() <= 1e-12 * scale
    assert np.abs(rows_v[inner]).max() <= 1e-12 * scale
    assert np.all(efvs[ac] == 1.0e6)


def test_flowfact_viscosity():
    """whichefvs = 1: efvs = flwafact * (velo_scale / len_scale * scyr)^((1-n)/n)."""
    g = geometry(seed=6)
    flwa = 2.0e-17
    efvs, *A = run(g, flwa=flwa, whichefvs=1)
    scyr = 31536000.0
    eff = (500.0 / scyr) / 200.0e3 * scyr
    want = 0.5 * flwa ** (-1.0 / N_GLEN) * math.pow(eff, (1.0 - N_GLEN) / N_GLEN)
    assert np.all(efvs[g["ac"]] == want)


def test_singular_and_halo_errors():
    g = geometry(seed=7)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    shape = (ny - 1, nx - 1, nz)
    ff = np.ones((ny, nx, nz - 1))
    st = oracle.assemble_stiffness_3d(nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], np.zeros(shape),
                                      np.zeros(shape), g["stagusrf"], g["stagthck"], ff, nhalo=1)[0]
    assert st == 2
    flat = np.zeros_like(g["stagthck"])  # every node at z = 0: the Jacobian's z column is zero
    st = oracle.assemble_stiffness_3d(nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], np.zeros(shape),
                                      np.zeros(shape), flat, flat, ff)[0]
    assert st == 1


# ---------------------------------------------------------------------------
# assemble_stiffness_matrix_2d (:4961-5378), SSA
# ---------------------------------------------------------------------------

def run2(g, uvel=None, vvel=None, flwa=1.0e-16, ff=None, **kw):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    shape = (ny - 1, nx - 1)
    u = np.zeros(shape) if uvel is None else uvel
    v = np.zeros(shape) if vvel is None else vvel
    if ff is None:
        ff = np.full((ny, nx, nz - 1), 0.5 * flwa ** (-1.0 / N_GLEN))
    st, efvs, *A = oracle.assemble_stiffness_2d(nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v,
                                                g["stagthck"], ff, **kw)
    assert st == 0
    return efvs, A


def test_ssa_first_picard_matches_numpy_assembly():
    g = geometry(seed=31)
    efvs, A = run2(g)
    P = asm.assemble_ssa_2d(g["thck"], g["usrf"], g["dx"], g["dx"], np.zeros((g["ny"] - 1, g["nx"] - 1)),
                            stiffness_only=True)
    scale = max(np.abs(P.Auu).max(), np.abs(P.Avv).max())
    for got, want in zip(A, (P.Auu, P.Auv, P.Avu, P.Avv)):
        assert np.abs(got - want).max() <= 1e-13 * scale
    e0 = asm.first_picard_efvs(1.0e-16)
    act = g["ac"]
    assert np.all(np.abs(efvs[act] - e0) <= 1e-14 * e0) and np.all(efvs[~act] == 0.0)


def test_ssa_scatter_is_exactly_symmetric():
    g = geometry(seed=32)
    rng = np.random.default_rng(4)
    shape = (g["ny"] - 1, g["nx"] - 1)
    efvs, A = run2(g, 50.0 * rng.standard_normal(shape), 50.0 * rng.standard_normal(shape))
    P = asm.Problem("2d", g["nx"], g["ny"], 1, *A, np.zeros(shape), np.zeros(shape), g["av"].astype(np.int32),
                    asm.default_par(g["nx"], g["ny"]))
    r = oracle.check_symmetry(P)
    assert r[4] == 0.0 and r[5] == 0 and np.abs(A[0]).max() > 0.0


def test_ssa_linear_velocity_and_layer_averaged_flow_factor():
    """u, v linear in x and y: constant SSA strain rates, so efvs = the flow law at those rates
    with the layer average of flwafact (weights sigma(k+1) - sigma(k)), the same in every layer."""
    g = geometry(seed=33, nz=6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    a, b = (2.0e-3, -1.5e-3), (0.5e-3, 3.0e-3)
    u = a[0] * g["xVertex"] + a[1] * g["yVertex"]
    v = b[0] * g["xVertex"] + b[1] * g["yVertex"]
    rng = np.random.default_rng(6)
    layer = 0.5 * 1.0e-16 ** (-1.0 / N_GLEN) * (1.0 + 0.5 * rng.random(nz - 1))
    ff = np.broadcast_to(layer, (ny, nx, nz - 1)).copy()
    efvs, A = run2(g, u, v, ff=ff)
    ff2 = float(np.sum(layer * np.diff(g["sigma"])))
    sq = 1.0e-16 + (a[0] ** 2 + b[1] ** 2 + a[0] * b[1] + 0.25 * (b[0] + a[1]) ** 2)
    want = ff2 * sq ** ((1.0 - N_GLEN) / N_GLEN / 2.0)
    act = g["ac"]
    assert np.all(np.abs(efvs[act] - want) <= 1e-12 * want)
    assert np.all(efvs[act] == efvs[act][:, :1])  # every layer the same


def test_ssa_constant_viscosity_null_space():
    g = geometry(seed=34)
    efvs, (Auu, Auv, Avu, Avv) = run2(g, whichefvs=0, efvs_constant=1.0e6)
    ac = g["ac"]
    full = ac[:-1, :-1] & ac[:-1, 1:] & ac[1:, :-1] & ac[1:, 1:]
    scale = np.abs(Auu).max()
    assert np.abs(Auu.sum(axis=0)[full]).max() <= 1e-12 * scale
    assert np.abs(Avu.sum(axis=0)[full]).max() <= 1e-12 * scale


# ---------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, DIVA branch (compute_effective_viscosity_diva :7730-7997,
# compute_integrals_diva :5649-5775)
# ---------------------------------------------------------------------------

def diva_inputs(g, seed=0, traction=0.0):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(seed)
    sig = g["sigma"]
    stagsig = 0.5 * (sig[:-1] + sig[1:])
    bx = np.full((ny - 1, nx - 1), traction)
    by = np.full((ny - 1, nx - 1), -0.5 * traction)
    dsf = 1.0 + 0.1 * rng.random((ny, nx))
    return stagsig, bx, by, dsf, dsf[::-1].copy()


def run_diva(g, u, v, ff, eq, traction=0.0, seed=0, **kw):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    stagsig, bx, by, dsfx, dsfy = diva_inputs(g, seed, traction)
    out = oracle.assemble_stiffness_2d_diva(nx, ny, nz, g["sigma"], stagsig, g["ac"], g["xVertex"], g["yVertex"], u, v,
                                            g["stagthck"], g["thck"], bx, by, dsfx, dsfy, ff, eq, **kw)
    assert out[0] == 0
    return out[1:], (stagsig, bx, by, dsfx, dsfy)


def test_diva_without_traction_is_the_ssa_system():
    """With zero basal traction the vertical shear terms vanish; with one flow factor in all
    layers DIVA's layer-averaged viscosity is the SSA's (to roundoff)."""
    g = geometry(seed=35, nz=6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(7)
    u, v = 30 * rng.standard_normal((ny - 1, nx - 1)), 30 * rng.standard_normal((ny - 1, nx - 1))
    ff = np.full((ny, nx, nz - 1), 0.5 * 1e-16 ** (-1 / 3))
    (efvs, eq, ok, om, *A), _ = run_diva(g, u, v, ff, np.zeros((ny, nx, 4, nz - 1)))
    e2, A2 = run2(g, u, v, ff=ff)
    for a, b in zip(A, A2):
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    act = g["ac"]
    assert np.abs(efvs[act] - e2[act]).max() <= 1e-13 * np.abs(e2[act]).max()
    assert np.all(eq[~act] == 0.0) and np.all(eq[act] > 0.0)


def test_diva_layer_viscosity_and_integrals():
    """Linear velocity and uniform traction: each layer's new viscosity is the flow law at the
    strain rates plus the vertical shear from the traction and the previous viscosity; omega_k
    and omega are the integrals of compute_integrals_diva."""
    g = geometry(seed=36, nz=6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    a, b = (2.0e-3, -1.0e-3), (0.5e-3, 2.5e-3)
    u = a[0] * g["xVertex"] + a[1] * g["yVertex"]
    v = b[0] * g["xVertex"] + b[1] * g["yVertex"]
    rng = np.random.default_rng(8)
    layer = 0.5 * 1e-16 ** (-1 / 3) * (1 + 0.5 * rng.random(nz - 1))
    ff = np.broadcast_to(layer, (ny, nx, nz - 1)).copy()
    eq0 = np.broadcast_to(2.0e6 * (1 + 0.3 * rng.random(nz - 1)), (ny, nx, 4, nz - 1)).copy()
    T = 5.0e4
    (efvs, eq, ok, om, *A), (stagsig, bx, by, dsfx, dsfy) = run_diva(g, u, v, ff, eq0, traction=T, seed=3)
    act = g["ac"]
    J, I = np.nonzero(act)
    for j, i in list(zip(J, I))[:: max(1, len(J) // 7)]:
        sx, sy = dsfx[j, i], dsfy[j, i]
        du_dz = T * stagsig / (eq0[j, i, 0] * sx)
        dv_dz = -0.5 * T * stagsig / (eq0[j, i, 0] * sy)
        sq = (1e-16 + a[0] ** 2 + b[1] ** 2 + a[0] * b[1] + 0.25 * (b[0] + a[1]) ** 2 + 0.25 * du_dz ** 2 * sx
              + 0.25 * dv_dz ** 2 * sy)
        want = layer * sq ** ((1 - 3.0) / 3.0 / 2.0)
        for p in range(4):
            assert np.abs(eq[j, i, p] - want).max() <= 1e-12 * want.max()
        sig = g["sigma"]
        depth = 0.5 * (sig[:-1] + sig[1:])
        dz = np.diff(sig) * g["thck"][j, i]
        okp = np.zeros((4, nz))
        for p in range(4):
            for k in range(nz - 2, -1, -1):
                okp[p, k] = okp[p, k + 1] + depth[k] / eq[j, i, p, k] * dz[k]
        want_ok = okp.sum(axis=0) / 4
        assert np.abs(ok[j, i] - want_ok).max() <= 1e-13 * want_ok.max()
        want_om = np.sum(0.5 * (want_ok[:-1] + want_ok[1:]) * np.diff(sig))
        assert abs(om[j, i] - want_om) <= 1e-13 * want_om
        np.testing.assert_allclose(efvs[j, i], eq[j, i].mean(axis=0), rtol=1e-14)
    assert np.all(ok[~act] == 0.0) and np.all(om[~act] == 0.0)


# ---------------------------------------------------------------------------
# assemble_stiffness_matrix_2d, L1L2 branch (compute_effective_viscosity_L1L2 :7474-7726)
# ---------------------------------------------------------------------------

def run_l1l2(g, u, v, dsdx, dsdy, flwa, n_glen=3.0, **kw):
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    ff = 0.5 * flwa ** (-1.0 / 3.0)
    return oracle.assemble_stiffness_2d_l1l2(nx, ny, nz, g["sigma"], g["ac"], g["xVertex"], g["yVertex"], u, v,
                                             g["stagthck"], dsdx, dsdy, flwa, ff, n_glen=n_glen, **kw)


def test_l1l2_flat_surface_is_glen():
    """With a flat surface tau_perp = 0, the cubic gives tau_parallel = (effstrain/A)^(1/3) and
    efvs = 1/(2 A tau_parallel^2), Glen's viscosity 0.5 A^(-1/3) effstrain^(-2/3)."""
    g = geometry(seed=91, nz=6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    a, b = (2.0e-3, -1.0e-3), (0.5e-3, 2.5e-3)
    u = a[0] * g["xVertex"] + a[1] * g["yVertex"]
    v = b[0] * g["xVertex"] + b[1] * g["yVertex"]
    layer = 1e-16 * (1 + np.random.default_rng(2).random(nz - 1))
    flwa = np.broadcast_to(layer, (ny, nx, nz - 1)).copy()
    z = np.zeros((ny - 1, nx - 1))
    st, efvs, *A = run_l1l2(g, u, v, z, z, flwa)
    assert st == 0
    eff = np.sqrt(1e-16 + a[0] ** 2 + b[1] ** 2 + a[0] * b[1] + 0.25 * (b[0] + a[1]) ** 2)
    want = 0.5 * layer ** (-1.0 / 3.0) * eff ** (-2.0 / 3.0)
    act = g["ac"]
    assert np.abs(efvs[act] - want).max() <= 1e-12 * want.max()


def test_l1l2_linear_rheology_and_errors():
    """n = 1: efvs = 1/(2A) in every layer whatever the flow; another n is the reference's
    GM_FATAL (status 3)."""
    g = geometry(seed=92, nz=6)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    rng = np.random.default_rng(3)
    u, v = rng.standard_normal((ny - 1, nx - 1)), rng.standard_normal((ny - 1, nx - 1))
    dsdx, dsdy = 0.01 * rng.standard_normal((ny - 1, nx - 1)), 0.01 * rng.standard_normal((ny - 1, nx - 1))
    flwa = 1e-16 * (1 + rng.random((ny, nx, nz - 1)))
    st, efvs, *A = run_l1l2(g, u, v, dsdx, dsdy, flwa, n_glen=1.0)
    assert st == 0
    act = g["ac"]
    np.testing.assert_array_equal(efvs[act], (1.0 / (2.0 * flwa))[act])
    assert run_l1l2(g, u, v, dsdx, dsdy, flwa, n_glen=2.0)[0] == 3
    st, efvs3, *A3 = run_l1l2(g, u, v, dsdx, dsdy, flwa)  # n = 3 with a sloping surface: below Glen's
    assert st == 0 and np.all(efvs3[act] > 0.0)
    P = asm.Problem("2d", nx, ny, 1, *A3, np.zeros_like(u), np.zeros_like(u), g["av"].astype(np.int32),
                    asm.default_par(nx, ny))
    r = oracle.check_symmetry(P)
    assert r[4] == 0.0 and r[5] == 0
