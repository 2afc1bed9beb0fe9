"""Small seeded solver inputs for the parity tests.

Physical cases come from cism_b200.assembly (first-Picard BP / SSA assembly).
Boundary cases put ice on every cell the assembly loop visits
(glissade_velo_higher.F90:5457-5458, cells nhalo+1..n-nhalo+1), so halo vertices
are active, and then apply the caller's staggered halo update to the matrix
blocks and the right-hand side, as glissade_velo_higher_solve does before the
solve (glissade_velo_higher.F90:2893-2898).
"""
from __future__ import annotations

import numpy as np

from cism_b200 import assembly as asm
import oracle


def halo_blocks_3d(P):
    """Apply the staggered halo to each (m, k) plane of the 3D blocks and to b."""
    NY, NX, nz = P.bu.shape
    for name in ("Auu", "Auv", "Avu", "Avv"):
        A = getattr(P, name)  # (NY, NX, nz, 27) == Fortran (27, nz, NX, NY)
        flat = np.ascontiguousarray(A).reshape(NY, NX, nz * 27)
        setattr(P, name, oracle.halo(P.nx, P.ny, nz * 27, P.par, flat).reshape(NY, NX, nz, 27))
    P.bu = oracle.halo(P.nx, P.ny, nz, P.par, P.bu)
    P.bv = oracle.halo(P.nx, P.ny, nz, P.par, P.bv)
    return P


def halo_blocks_2d(P):
    for name in ("Auu", "Auv", "Avu", "Avv"):
        A = getattr(P, name)  # (9, NY, NX)
        out = np.empty_like(A)
        for m in range(9):
            out[m] = oracle.halo(P.nx, P.ny, 1, P.par, np.ascontiguousarray(A[m]))
        setattr(P, name, out)
    P.bu = oracle.halo(P.nx, P.ny, 1, P.par, P.bu)
    P.bv = oracle.halo(P.nx, P.ny, 1, P.par, P.bv)
    return P


def slab_3d(ewn=9, nsn=8, nz=5, seed=0, bc="periodic", boundary_ice=False, sliding=True, dx=2000.0,
            symmetrize=True):
    """A small 3D slab; with boundary_ice the matrix halo is filled as the reference's staggered halo
    update does, and (symmetrize) the reference's pre-solve symmetry check runs last, in the
    reference's order (glissade_velo_higher.F90:2893-2931)."""
    rng = np.random.default_rng(seed)
    nx, ny = ewn + 4, nsn + 4
    H = 800.0 + 400.0 * rng.random((ny, nx))
    x = (np.arange(nx) + 0.5) * dx
    usrf = 2000.0 - x[None, :] * 0.01 + 30.0 * rng.random((ny, nx))
    ice = np.zeros((ny, nx), dtype=bool)
    if boundary_ice:
        ice[2:ny - 1, 2:nx - 1] = True
    else:
        ice[3:ny - 3, 3:nx - 3] = True
        ice[3:5, 3:5] = False  # a notch so that some owned vertices are inactive
    thck = np.where(ice, H, 0.0)
    usrf = np.where(ice, usrf, usrf - H)
    beta = asm.lognormal_beta((ny - 1, nx - 1), seed + 100) if sliding else None
    P = asm.assemble_bp_3d(thck, usrf, dx, dx, nz, beta=beta, bc=bc, name=f"slab3d-{bc}-{seed}",
                           symmetrize=symmetrize and not boundary_ice)
    if boundary_ice:
        P = halo_blocks_3d(P)
        if symmetrize:
            A = np.stack([P.Auu, P.Auv, P.Avu, P.Avv])
            asm.symmetrize_3d(A, P.active_vertex, P.par)
            P.Auu, P.Auv, P.Avu, P.Avv = (np.ascontiguousarray(a) for a in A)
    return P


def slab_2d(ewn=11, nsn=10, seed=0, bc="periodic", boundary_ice=False, dx=1000.0):
    rng = np.random.default_rng(seed)
    nx, ny = ewn + 4, nsn + 4
    H = 500.0 + 1500.0 * rng.random((ny, nx))
    ice = np.zeros((ny, nx), dtype=bool)
    if boundary_ice:
        ice[2:ny - 1, 2:nx - 1] = True
    else:
        ice[3:ny - 3, 3:nx - 3] = True
        ice[-5:-3, -5:-3] = False
    thck = np.where(ice, H, 0.0)
    usrf = thck.copy()
    beta = asm.lognormal_beta((ny - 1, nx - 1), seed + 200)
    P = asm.assemble_ssa_2d(thck, usrf, dx, dx, beta, bc=bc, name=f"slab2d-{bc}-{seed}")
    if boundary_ice:
        P = halo_blocks_2d(P)
    return P


def random_x0(P, seed=1, scale=1.0):
    rng = np.random.default_rng(seed)
    return (scale * rng.standard_normal(P.bu.shape), scale * rng.standard_normal(P.bv.shape))
