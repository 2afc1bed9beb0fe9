"""Host-side first-Picard assembly of the Glissade velocity system.

The linear solve this package accelerates is fed by matrix assembly that stays
on the host (glissade_velo_higher_solve, libglissade/glissade_velo_higher.F90
:662-3918).  This module restates that assembly for the first Picard iteration
(u = 0, so the effective strain rate is effstrain_min and the viscosity is
uniform per element) to build realistic solver inputs:

  get_vertex_geometry            glissade_velo_higher.F90:4052-4224
  glide sigma levels             libglide/glide_setup.F90:290-295, 369-376
  assemble_stiffness_matrix_3d   glissade_velo_higher.F90:5382-5643
  assemble_stiffness_matrix_2d   glissade_velo_higher.F90:4961-5378 (SSA branch)
  get_basis_function_derivatives_3d/2d   :6508-6732 / :6319-6504
  compute_effective_viscosity    :7285-7470 (nonlinear, u = 0)
  compute_element_matrix         :8001-8123 (BP and SSA forms)
  element_to_global_matrix_3d/2d :8200-8268 / :8127-8196
  load_vector_gravity (local)    :4228-4264
  basal_sliding_bc (beta local)  :8815-8873
  dirichlet_boundary_conditions_3d :9305-9498 (no-slip bed, u = 0)

Arrays are returned in the memory layout the Fortran caller passes, held as
C-order numpy arrays with reversed dimensions:
  3D blocks A(27,nz,nx-1,ny-1)  -> shape (ny-1, nx-1, nz, 27)
  3D vectors b(nz,nx-1,ny-1)    -> shape (ny-1, nx-1, nz)
  2D blocks A(nx-1,ny-1,9)      -> shape (9, ny-1, nx-1)
  2D vectors b(nx-1,ny-1)       -> shape (ny-1, nx-1)
  active_vertex(nx-1,ny-1)      -> int32 shape (ny-1, nx-1)
The coefficient index m is the reference's indxA_3d(iA,jA,kA) = 1 + (iA+1) +
3(jA+1) + 9(kA+1) (glissade_velo_higher.F90:608-626), 0-based here.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

NHALO = 2
RHOI = 910.0        # glimmer_physcon.F90:67
GRAV = 9.81         # glimmer_physcon.F90:69
VOL0 = 1.0e9        # glissade_velo_higher.F90:1254
N_GLEN = 3.0        # glimmer_physcon.F90:87
EFFSTRAIN_MIN = 1.0e-8  # glide_types.F90:2567
RSQRT3 = 1.0 / math.sqrt(3.0)

# element node offsets relative to cell (i,j) and layer k: ishift(7,:), jshift(7,:), kshift(7,:)
ISH3 = np.array([-1, 0, 0, -1, -1, 0, 0, -1])
JSH3 = np.array([-1, -1, 0, 0, -1, -1, 0, 0])
KSH3 = np.array([1, 1, 1, 1, 0, 0, 0, 0])
ISH2 = ISH3[:4]
JSH2 = JSH3[:4]


def indxA_3d() -> np.ndarray:
    """indxA_3d(-1:1,-1:1,-1:1) as 27 int32 in Fortran order (iA fastest)."""
    return np.arange(1, 28, dtype=np.int32)


def indxA_2d() -> np.ndarray:
    """indxA_2d(-1:1,-1:1) as 9 int32 in Fortran order (iA fastest)."""
    return np.arange(1, 10, dtype=np.int32)


def glide_sigma(nz: int) -> np.ndarray:
    """Glide sigma levels (glide_setup.F90:290-295, 374)."""
    x = np.arange(nz, dtype=np.float64) / (nz - 1)
    n = 2.0
    return (1.0 - (x + 1.0) ** (-n)) / (1.0 - 2.0 ** (-n))


def _quad3():
    pts = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1),
           (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
    xq = np.array([p[0] for p in pts], dtype=np.float64) * RSQRT3
    yq = np.array([p[1] for p in pts], dtype=np.float64) * RSQRT3
    zq = np.array([p[2] for p in pts], dtype=np.float64) * RSQRT3
    sx = np.array([-1, 1, 1, -1, -1, 1, 1, -1], dtype=np.float64)
    sy = np.array([-1, -1, 1, 1, -1, -1, 1, 1], dtype=np.float64)
    sz = np.array([-1, -1, -1, -1, 1, 1, 1, 1], dtype=np.float64)
    # derivatives of the trilinear basis w.r.t. reference coords, (qp, node, 3)
    d = np.empty((8, 8, 3))
    for p in range(8):
        d[p, :, 0] = sx * (1 + sy * yq[p]) * (1 + sz * zq[p]) / 8.0
        d[p, :, 1] = sy * (1 + sx * xq[p]) * (1 + sz * zq[p]) / 8.0
        d[p, :, 2] = sz * (1 + sx * xq[p]) * (1 + sy * yq[p]) / 8.0
    return d


def _quad2():
    pts = [(-1, -1), (1, -1), (1, 1), (-1, 1)]
    xq = np.array([p[0] for p in pts], dtype=np.float64) * RSQRT3
    yq = np.array([p[1] for p in pts], dtype=np.float64) * RSQRT3
    sx = np.array([-1, 1, 1, -1], dtype=np.float64)
    sy = np.array([-1, -1, 1, 1], dtype=np.float64)
    phi = np.empty((4, 4))
    d = np.empty((4, 4, 2))
    for p in range(4):
        phi[p] = (1 + sx * xq[p]) * (1 + sy * yq[p]) / 4.0
        d[p, :, 0] = sx * (1 + sy * yq[p]) / 4.0
        d[p, :, 1] = sy * (1 + sx * xq[p]) / 4.0
    return phi, d


DPHIR3 = _quad3()
PHI2, DPHIR2 = _quad2()


def stagger(field: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """Average a cell field (ny, nx) to vertices (ny-1, nx-1) over the ice cells among the four."""
    f = np.where(mask, field, 0.0)
    w = mask.astype(np.float64)
    s = f[:-1, :-1] + f[:-1, 1:] + f[1:, :-1] + f[1:, 1:]
    c = w[:-1, :-1] + w[:-1, 1:] + w[1:, :-1] + w[1:, 1:]
    return np.where(c > 0, s / np.maximum(c, 1.0), 0.0)


def vertex_gradient(field: np.ndarray, dx: float, dy: float):
    """Centered gradient of a cell field at vertices (glissade_centered_gradient form)."""
    dfdx = ((field[:-1, 1:] + field[1:, 1:]) - (field[:-1, :-1] + field[1:, :-1])) / (2.0 * dx)
    dfdy = ((field[1:, :-1] + field[1:, 1:]) - (field[:-1, :-1] + field[:-1, 1:])) / (2.0 * dy)
    return dfdx, dfdy


def active_masks(thck: np.ndarray, thklim: float = 1.0):
    """active_cell over cells nhalo+1..n-nhalo+1 (1-based) with ice, and active_vertex (:4152-4182)."""
    ny, nx = thck.shape
    ice = thck > thklim
    ac = np.zeros_like(ice)
    ac[NHALO:ny - NHALO + 1, NHALO:nx - NHALO + 1] = ice[NHALO:ny - NHALO + 1, NHALO:nx - NHALO + 1]
    av = ac[:-1, :-1] | ac[:-1, 1:] | ac[1:, :-1] | ac[1:, 1:]
    return ac, av


@dataclasses.dataclass
class Problem:
    """One linear system in the reference caller's layout."""
    kind: str                 # "3d" or "2d"
    nx: int                   # cells including halo
    ny: int
    nz: int                   # 1 for 2D
    Auu: np.ndarray
    Auv: np.ndarray
    Avu: np.ndarray
    Avv: np.ndarray
    bu: np.ndarray
    bv: np.ndarray
    active_vertex: np.ndarray
    par: dict
    name: str = ""

    @property
    def nvert_active_owned(self) -> int:
        p = self.par
        a = self.active_vertex[p["staggered_jlo"] - 1:p["staggered_jhi"], p["staggered_ilo"] - 1:p["staggered_ihi"]]
        return int(np.count_nonzero(a))

    @property
    def n_unknowns(self) -> int:
        return 2 * self.nz * self.nvert_active_owned

    def x0(self):
        return np.zeros_like(self.bu), np.zeros_like(self.bv)


def default_par(nx: int, ny: int, bc: str = "periodic", reprosum: bool = False) -> dict:
    """Fields of parallel_type on one rank (parallel_mpi.F90:2640-2653)."""
    lo = NHALO if bc == "outflow" else NHALO + 1
    return dict(staggered_ilo=lo, staggered_ihi=nx - 2, staggered_jlo=lo, staggered_jhi=ny - 2,
                periodic_bc=int(bc in ("periodic", "no_penetration")), outflow_bc=int(bc == "outflow"),
                no_ice_bc=int(bc == "no_ice"), reprosum=int(reprosum), tasks_row=1, tasks_col=1)


def first_picard_efvs(flwa: float) -> float:
    """Viscosity at u = 0: flwafact * (effstrain_min^2)^(p/2), p = (1-n)/n (:7411-7464)."""
    flwafact = 0.5 * flwa ** (-1.0 / N_GLEN)
    p_effstr = (1.0 - N_GLEN) / N_GLEN
    return flwafact * (EFFSTRAIN_MIN ** 2) ** (p_effstr / 2.0)


def assemble_bp_3d(thck, usrf, dx, dy, nz, flwa=1.0e-16, beta=None, bc="periodic", name="",
                   chunk=40000, stiffness_only=False, symmetrize=True) -> Problem:
    """Blatter-Pattyn 3D system for the first Picard iteration.

    thck, usrf: cell fields (ny, nx) including the 2-cell halo.
    beta: vertex field (ny-1, nx-1) in Pa yr/m for 'beta local' sliding, or None for a
          no-slip bed (Dirichlet u = v = 0 at k = nz, which_ho_babc = 4).
    stiffness_only: return the assembled stiffness blocks before any basal condition.
    symmetrize: finish with the reference's pre-solve symmetry check (symmetrize_3d), as
          glissade_velo_higher_solve does; the element sums here run in another order than the
          reference's scatter, which leaves transpose pairs a rounding apart.
    """
    ny, nx = thck.shape
    NX, NY = nx - 1, ny - 1
    ac, av = active_masks(thck)
    stagthck = stagger(thck, thck > 1.0)
    stagusrf = stagger(usrf, thck > 1.0)
    sigma = glide_sigma(nz)
    efvs = first_picard_efvs(flwa)
    xv = np.arange(NX, dtype=np.float64) * dx
    yv = np.arange(NY, dtype=np.float64) * dy

    A = np.zeros((4, NY, NX, nz, 27))  # uu, uv, vu, vv
    Af = A.reshape(4, -1)               # flat views for the element scatter
    cj, ci = np.nonzero(ac)
    # elements: every active cell x every layer
    ecj = np.repeat(cj, nz - 1)
    eci = np.repeat(ci, nz - 1)
    ek = np.tile(np.arange(nz - 1), len(cj))
    for s in range(0, len(ek), chunk):
        sl = slice(s, s + chunk)
        vj = ecj[sl, None] + JSH3[None, :]     # (E, 8) vertex indices (0-based)
        vi = eci[sl, None] + ISH3[None, :]
        kk = ek[sl, None] + KSH3[None, :]      # 0-based levels
        X = xv[vi]
        Y = yv[vj]
        Z = stagusrf[vj, vi] - sigma[kk] * stagthck[vj, vi]
        coords = np.stack([X, Y, Z], axis=-1)  # (E, 8, 3)
        jac = np.einsum("pna,enb->epab", DPHIR3, coords)
        det = np.linalg.det(jac)
        if np.any(np.abs(det) <= 0.0):
            raise ValueError("degenerate element (singular Jacobian)")
        jinv = np.linalg.inv(jac)
        dphi = np.einsum("epba,pna->epnb", jinv, DPHIR3)  # (E, qp, node, xyz)
        f = efvs * 1.0 * det / VOL0                       # efvs * wqp * detJ / vol0
        dx_, dy_, dz_ = dphi[..., 0], dphi[..., 1], dphi[..., 2]
        Kxx = np.einsum("ep,epr,epc->erc", f, dx_, dx_)
        Kyy = np.einsum("ep,epr,epc->erc", f, dy_, dy_)
        Kzz = np.einsum("ep,epr,epc->erc", f, dz_, dz_)
        Kxy = np.einsum("ep,epr,epc->erc", f, dx_, dy_)
        Kyx = np.einsum("ep,epr,epc->erc", f, dy_, dx_)
        Kuu = Kxx * 4 + Kyy + Kzz
        Kvv = Kyy * 4 + Kxx + Kzz
        Kuv = Kxy * 2 + Kyx
        Kvu = Kyx * 2 + Kxy
        node = ((vj * NX + vi) * nz + kk) * 27                 # flat (j, i, k, m=0) offsets, (E, 8)
        for nr in range(8):
            base = node[:, nr]
            for nc in range(8):
                iA = ISH3[nc] - ISH3[nr]
                jA = JSH3[nc] - JSH3[nr]
                kA = KSH3[nc] - KSH3[nr]
                fi = base + ((iA + 1) + 3 * (jA + 1) + 9 * (kA + 1))  # unique within the chunk
                Af[0][fi] += Kuu[:, nr, nc]
                Af[1][fi] += Kuv[:, nr, nc]
                Af[2][fi] += Kvu[:, nr, nc]
                Af[3][fi] += Kvv[:, nr, nc]

    # load vector, local driving stress (:4243-4262)
    dsdx, dsdy = vertex_gradient(usrf, dx, dy)
    wb = np.zeros(nz + 1)
    wb[nz] = 1.0
    wb[1:nz] = 0.5 * (sigma[:-1] + sigma[1:])
    dzk = stagthck[:, :, None] * (wb[1:] - wb[:-1])[None, None, :]
    bu = np.where(av[:, :, None], -RHOI * GRAV * dx * dy * dzk / VOL0 * dsdx[:, :, None], 0.0)
    bv = np.where(av[:, :, None], -RHOI * GRAV * dx * dy * dzk / VOL0 * dsdy[:, :, None], 0.0)

    m0 = 13
    if stiffness_only:
        pass
    elif beta is not None:
        lsrf = usrf - thck
        staglsrf = stagger(lsrf, np.ones_like(thck, dtype=bool))
        gx, gy = np.gradient(staglsrf, dy, dx)
        theta = np.arctan(np.sqrt(gx * gx + gy * gy))
        add = np.where(av, dx * dy / VOL0 * beta / np.cos(theta), 0.0)
        A[0, :, :, nz - 1, m0] += add
        A[3, :, :, nz - 1, m0] += add
    else:
        # no-slip bed: Dirichlet rows at k = nz for active vertices in nhalo..n-nhalo+1
        dmask = np.zeros((NY, NX, nz), dtype=bool)
        vmask = np.zeros_like(av)
        vmask[NHALO - 1:ny - NHALO + 1, NHALO - 1:nx - NHALO + 1] = av[NHALO - 1:ny - NHALO + 1,
                                                                       NHALO - 1:nx - NHALO + 1]
        dmask[:, :, nz - 1] = vmask
        # zero the Dirichlet columns in every row whose neighbor (iA,jA,kA) is a Dirichlet node
        pad = np.zeros((NY + 2, NX + 2, nz + 2), dtype=bool)
        pad[1:-1, 1:-1, 1:-1] = dmask
        for kA in (-1, 0, 1):
            for jA in (-1, 0, 1):
                for iA in (-1, 0, 1):
                    m = (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1)
                    nb = pad[1 + jA:NY + 1 + jA, 1 + iA:NX + 1 + iA, 1 + kA:nz + 1 + kA]
                    A[:, nb, m] = 0.0
        # Dirichlet rows become identity rows
        A[:, dmask, :] = 0.0
        A[0, dmask, m0] = 1.0
        A[3, dmask, m0] = 1.0
        bu[dmask] = 0.0
        bv[dmask] = 0.0

    par = default_par(nx, ny, bc)
    if symmetrize and not stiffness_only:
        symmetrize_3d(A, av, par)
    return Problem("3d", nx, ny, nz, np.ascontiguousarray(A[0]), np.ascontiguousarray(A[1]),
                   np.ascontiguousarray(A[2]), np.ascontiguousarray(A[3]), bu, bv,
                   av.astype(np.int32), par, name)


def symmetrize_3d(A, active, par, eps11=1.0e-11):
    """The averaging of check_symmetry_assembled_matrix_3d (glissade_velo_higher.F90:10854-11117),
    which glissade_velo_higher_solve applies to every assembled 3D system before the solve
    (:2923-2931; check_symmetry = .true., :197): every coupling of an owned active row and its
    transpose partner (Auu with Auu, Auv with Avu, Avu with Auv, Avv with Avv, at the neighbour
    node and the opposite offset) that differ by less than eps11 times the row's diagonal (Auu's
    for the Auu and Auv entries, Avv's for the Avu and Avv entries) both become 0.5*(val1 + val2).
    A pair is visited from both of its rows when both are owned and active; each coefficient
    belongs to one pair, so the in-place loop's result does not depend on its order and the
    pairs are averaged here all at once.  A: (4, NY, NX, nz, 27) of uu, uv, vu, vv, in place."""
    _, NY, NX, nz, _ = A.shape
    own = np.zeros((NY, NX), dtype=bool)
    jl, jh, il, ih = par["staggered_jlo"] - 1, par["staggered_jhi"], par["staggered_ilo"] - 1, par["staggered_ihi"]
    own[jl:jh, il:ih] = active[jl:jh, il:ih] != 0
    orig = A.copy()
    diag = (np.abs(orig[0][..., 13]), np.abs(orig[3][..., 13]))  # Auu, Avv diagonals (NY, NX, nz)
    # (block at R, block at the partner, diagonal tested at R, diagonal tested at the partner)
    groups = ((0, 0, 0, 0), (1, 2, 0, 1), (2, 1, 1, 0), (3, 3, 1, 1))
    for c in range(27):
        iA, jA, kA = c % 3 - 1, (c // 3) % 3 - 1, c // 9 - 1
        cp = 26 - c
        rj = slice(max(0, -jA), NY - max(0, jA))
        ri = slice(max(0, -iA), NX - max(0, iA))
        rk = slice(max(0, -kA), nz - max(0, kA))
        nj = slice(rj.start + jA, rj.stop + jA)
        ni = slice(ri.start + iA, ri.stop + iA)
        nk = slice(rk.start + kA, rk.stop + kA)
        ownR = own[rj, ri][:, :, None]
        ownN = own[nj, ni][:, :, None]
        for bR, bN, dR, dN in groups:
            v1 = orig[bR][rj, ri, rk, c]
            v2 = orig[bN][nj, ni, nk, cp]
            diff = np.abs(v1 - v2)
            hit = (ownR & (diff < eps11 * diag[dR][rj, ri, rk])) | (ownN & (diff < eps11 * diag[dN][nj, ni, nk]))
            avg = 0.5 * (v1 + v2)
            A[bR][rj, ri, rk, c] = np.where(hit, avg, A[bR][rj, ri, rk, c])
            A[bN][nj, ni, nk, cp] = np.where(hit, avg, A[bN][nj, ni, nk, cp])


def assemble_ssa_2d(thck, usrf, dx, dy, beta, flwa=1.0e-16, bc="periodic", name="",
                    stiffness_only=False) -> Problem:
    """SSA 2D system (9-point blocks) for the first Picard iteration, beta-local sliding.
    stiffness_only: the assembled stiffness blocks without the basal term."""
    ny, nx = thck.shape
    NX, NY = nx - 1, ny - 1
    ac, av = active_masks(thck)
    stagthck = stagger(thck, thck > 1.0)
    efvs = first_picard_efvs(flwa)
    xv = np.arange(NX, dtype=np.float64) * dx
    yv = np.arange(NY, dtype=np.float64) * dy
    A = np.zeros((4, 9, NY, NX))
    cj, ci = np.nonzero(ac)
    vj = cj[:, None] + JSH2[None, :]
    vi = ci[:, None] + ISH2[None, :]
    coords = np.stack([xv[vi], yv[vj]], axis=-1)   # (E,4,2)
    jac = np.einsum("pna,enb->epab", DPHIR2, coords)
    det = np.linalg.det(jac)
    jinv = np.linalg.inv(jac)
    dphi = np.einsum("epba,pna->epnb", jinv, DPHIR2)
    h_qp = np.einsum("pn,en->ep", PHI2, stagthck[vj, vi])
    f = h_qp * efvs * 1.0 * det / VOL0
    dx_, dy_ = dphi[..., 0], dphi[..., 1]
    Kuu = 4 * np.einsum("ep,epr,epc->erc", f, dx_, dx_) + np.einsum("ep,epr,epc->erc", f, dy_, dy_)
    Kvv = 4 * np.einsum("ep,epr,epc->erc", f, dy_, dy_) + np.einsum("ep,epr,epc->erc", f, dx_, dx_)
    Kuv = 2 * np.einsum("ep,epr,epc->erc", f, dx_, dy_) + np.einsum("ep,epr,epc->erc", f, dy_, dx_)
    Kvu = 2 * np.einsum("ep,epr,epc->erc", f, dy_, dx_) + np.einsum("ep,epr,epc->erc", f, dx_, dy_)
    for nr in range(4):
        rj, ri = vj[:, nr], vi[:, nr]
        for nc in range(4):
            m = (ISH2[nc] - ISH2[nr] + 1) + 3 * (JSH2[nc] - JSH2[nr] + 1)
            A[0, m, rj, ri] += Kuu[:, nr, nc]
            A[1, m, rj, ri] += Kuv[:, nr, nc]
            A[2, m, rj, ri] += Kvu[:, nr, nc]
            A[3, m, rj, ri] += Kvv[:, nr, nc]
    lsrf = usrf - thck
    staglsrf = stagger(lsrf, np.ones_like(thck, dtype=bool))
    gx, gy = np.gradient(staglsrf, dy, dx)
    theta = np.arctan(np.sqrt(gx * gx + gy * gy))
    add = np.where(av, dx * dy / VOL0 * beta / np.cos(theta), 0.0)
    if not stiffness_only:
        A[0, 4] += add
        A[3, 4] += add
    dsdx, dsdy = vertex_gradient(usrf, dx, dy)
    bu = np.where(av, -RHOI * GRAV * dx * dy * stagthck / VOL0 * dsdx, 0.0)
    bv = np.where(av, -RHOI * GRAV * dx * dy * stagthck / VOL0 * dsdy, 0.0)
    par = default_par(nx, ny, bc)
    return Problem("2d", nx, ny, 1, np.ascontiguousarray(A[0]), np.ascontiguousarray(A[1]),
                   np.ascontiguousarray(A[2]), np.ascontiguousarray(A[3]), bu, bv,
                   av.astype(np.int32), par, name)


# ---------------------------------------------------------------------------
# Geometries named by the benchmark configurations (synthetic, seeded)
# ---------------------------------------------------------------------------

def smooth_field(shape, corr_cells: float, rng: np.random.Generator) -> np.ndarray:
    """Unit-variance Gaussian random field with a Gaussian correlation of corr_cells cells."""
    w = rng.standard_normal(shape)
    ky = np.fft.fftfreq(shape[0])[:, None]
    kx = np.fft.fftfreq(shape[1])[None, :]
    filt = np.exp(-2.0 * (math.pi * corr_cells) ** 2 * (kx * kx + ky * ky))
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def _ice_interior(ny, nx):
    """Cells that may hold ice: the owned cells minus their outermost ring."""
    m = np.zeros((ny, nx), dtype=bool)
    m[NHALO + 1:ny - NHALO - 1, NHALO + 1:nx - NHALO - 1] = True
    return m


def dome(ewn=31, nsn=31, nz=11, dx=2000.0, H0=1000.0, R=25000.0, name="dome", symmetrize=True) -> Problem:
    """Parabolic dome H = H0 sqrt(1 - r^2/R^2) on a flat bed, no-slip bed (benchmark cfg 1)."""
    nx, ny = ewn + 2 * NHALO, nsn + 2 * NHALO
    # owned cells are 3..nx-2 (1-based); cell centres at (i - 0.5) dx in vertex coordinates
    ci = (np.arange(nx) + 0.5) * dx
    cj = (np.arange(ny) + 0.5) * dx
    xc = 0.5 * (ci[NHALO] + ci[nx - NHALO - 1])
    yc = 0.5 * (cj[NHALO] + cj[ny - NHALO - 1])
    X, Y = np.meshgrid(ci - xc, cj - yc)
    r2 = (X * X + Y * Y) / (R * R)
    thck = np.where(r2 < 1.0, H0 * np.sqrt(np.maximum(1.0 - r2, 0.0)), 0.0)
    thck = np.where(_ice_interior(ny, nx), thck, 0.0)
    usrf = thck.copy()
    return assemble_bp_3d(thck, usrf, dx, dx, nz, flwa=1.0e-16, beta=None, name=name, symmetrize=symmetrize)


def ice_stream(ewn=201, nsn=201, nz=11, dx=2000.0, H=1500.0, slope_deg=0.5, rough=0.05, seed=3,
               beta=None, name="ice_stream", symmetrize=True) -> Problem:
    """Slab ice stream: surface and bed slope slope_deg in x, seeded bed roughness of rough*H."""
    rng = np.random.default_rng(seed)
    nx, ny = ewn + 2 * NHALO, nsn + 2 * NHALO
    x = (np.arange(nx) + 0.5) * dx
    usrf0 = 3000.0 - x * math.tan(math.radians(slope_deg))
    bump = rough * H * smooth_field((ny, nx), 4.0, rng)
    topg = usrf0[None, :] - H + bump
    usrf = np.broadcast_to(usrf0[None, :], (ny, nx)).copy()
    thck = np.where(_ice_interior(ny, nx), usrf - topg, 0.0)
    usrf = np.where(thck > 0, usrf, topg)
    return assemble_bp_3d(thck, usrf, dx, dx, nz, flwa=1.0e-16, beta=beta, name=name, symmetrize=symmetrize)


def ssa_random(ewn=401, nsn=401, dx=1000.0, seed=7, corr_km=20.0, name="ssa") -> Problem:
    """2D SSA: thickness a smooth seeded random field in 500..2000 m, log-normal beta (cfg 2)."""
    rng = np.random.default_rng(seed)
    nx, ny = ewn + 2 * NHALO, nsn + 2 * NHALO
    f = smooth_field((ny, nx), corr_km * 1000.0 / dx, rng)
    f = (f - f.min()) / max(f.max() - f.min(), 1e-30)
    thck = 500.0 + 1500.0 * f
    thck = np.where(_ice_interior(ny, nx), thck, 0.0)
    usrf = thck.copy()
    beta = np.exp(math.log(1.0e3) + 1.0 * rng.standard_normal((ny - 1, nx - 1)))
    return assemble_ssa_2d(thck, usrf, dx, dx, beta, name=name)


def lognormal_beta(shape, seed, mu=math.log(1.0e3), sd=1.0):
    rng = np.random.default_rng(seed)
    return np.exp(mu + sd * rng.standard_normal(shape))


def batch_member(n, seed, nz=11, dx=2000.0, symmetrize=True) -> Problem:
    """One member of the batched 3D workload: an n x n x nz ice stream (seeded bed roughness)
    sliding on its own seeded log-normal basal friction field (mu = ln 1e3 Pa yr/m, sigma = 1)."""
    shape = (n + 2 * NHALO - 1, n + 2 * NHALO - 1)
    return ice_stream(ewn=n, nsn=n, nz=nz, dx=dx, seed=seed, beta=lognormal_beta(shape, 1000 + seed),
                      name=f"member{seed}_{n}", symmetrize=symmetrize)


def batch_sizes(count=64, seed=11, lo=64, hi=256):
    """Seeded horizontal sizes, uniform on lo..hi vertices per side."""
    return [int(v) for v in np.random.default_rng(seed).integers(lo, hi + 1, count)]

