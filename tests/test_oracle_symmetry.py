"""Known-answer tests of the oracle's restatement of check_symmetry_assembled_matrix_{3d,2d}
(libglissade/glissade_velo_higher.F90:10648-11117).

The oracle follows the reference's loops in order, averaging in place.  These tests check it
against hand-computed cases and against a second restatement that works pair by pair: every
coefficient has exactly one transpose partner, each pair is visited from at most two rows
(with that row's diagonal in the tolerance), and the in-place loop then averages the pair when
either visit's tolerance test passes; a visit warns when the values still differ when it comes
and its own test fails.  That pairwise form is the one a parallel device pass can compute.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np
import pytest

import oracle
from tests import problems

EPS11 = 1.0e-11  # libglimmer/glimmer_paramets.F90:77
BLOCKS = ("Auu", "Auv", "Avu", "Avv")


def _owned_rows(P):
    p = P.par
    for j in range(p["staggered_jlo"] - 1, p["staggered_jhi"]):
        for i in range(p["staggered_ilo"] - 1, p["staggered_ihi"]):
            if P.active_vertex[j, i]:
                yield j, i


def _visits_3d(P, A):
    """Visits of the 3D check: (order, pair key, (block, index) of val1, of val2, diag).
    Blocks are numpy (NY, NX, nz, 27) == Fortran (27, nz, NX, NY); m = 13 is the diagonal."""
    NY, NX, nz = P.bu.shape
    out = []
    for j, i in _owned_rows(P):
        for k in range(nz):
            for ps in (0, 1):
                diag = A["Auu" if ps == 0 else "Avv"][j, i, k, 13]
                for jA in (-1, 0, 1):
                    for iA in (-1, 0, 1):
                        for kA in (-1, 0, 1):
                            if not (0 <= k + kA < nz and 0 <= i + iA < NX and 0 <= j + jA < NY):
                                continue
                            m = (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1)
                            a, b = (j, i, k, m), (j + jA, i + iA, k + kA, 26 - m)
                            order = (j, i, k, ps, jA, iA, kA)
                            if ps == 0:
                                out.append((order + (0,), ("uu",) + min(a, b) + max(a, b), ("Auu", a), ("Auu", b),
                                            diag))
                                out.append((order + (1,), ("x",) + a + b, ("Auv", a), ("Avu", b), diag))
                            else:
                                out.append((order + (0,), ("vv",) + min(a, b) + max(a, b), ("Avv", a), ("Avv", b),
                                            diag))
                                out.append((order + (1,), ("x",) + b + a, ("Avu", a), ("Auv", b), diag))
    return out


def pairwise_3d(P, A):
    """The 3D check pair by pair; returns (blocks after the check, maxdiff, nwarn)."""
    A = {n: np.array(A[n], copy=True) for n in BLOCKS}
    orig = {n: np.array(A[n], copy=True) for n in BLOCKS}
    pairs = defaultdict(list)
    for v in _visits_3d(P, orig):
        pairs[v[1]].append(v)
    maxdiff, nwarn = 0.0, 0
    for vis in pairs.values():
        vis.sort(key=lambda v: v[0])
        _, _, (n1, a), (n2, b), _ = vis[0]
        x, y = orig[n1][a], orig[n2][b]
        if x == y:
            continue
        d = abs(y - x)
        maxdiff = max(maxdiff, d)
        fixed = False
        for v in vis:
            if fixed:
                break
            if d < EPS11 * abs(v[4]):
                fixed = True
            else:
                nwarn += 1
        if fixed:
            avg = 0.5 * (x + y)
            for v in vis:
                A[v[2][0]][v[2][1]] = avg
                A[v[3][0]][v[3][1]] = avg
    return A, maxdiff, nwarn


def _blocks(P):
    return {n: np.array(getattr(P, n), copy=True) for n in BLOCKS}


def _check(P, A):
    r = oracle.check_symmetry(P, *(A[n] for n in BLOCKS))
    return dict(zip(BLOCKS, r[:4])), r[4], r[5]


def _symmetrized(P):
    """P's blocks after one 3D check of an interior-ice slab: every pair averaged, none warned."""
    A, md, nw = _check(P, _blocks(P))
    assert nw == 0 and md > 0.0  # the assembly leaves roundoff asymmetry
    A2, md2, nw2 = _check(P, A)
    assert md2 == 0.0 and nw2 == 0 and all(np.array_equal(A[n], A2[n]) for n in BLOCKS)  # idempotent
    return A


def test_symmetry_3d_known_answers():
    P = problems.slab_3d(seed=41, symmetrize=False)
    S = _symmetrized(P)
    J, I = (P.par["staggered_jlo"] + 1, P.par["staggered_ilo"] + 2)  # an owned active interior row
    assert P.active_vertex[J, I] and P.active_vertex[J, I + 1]
    k = 2
    # (1) Auu(iA=+1) of row (J, I, k) raised below eps11 * diag: the pair is averaged
    A = {n: np.array(S[n], copy=True) for n in BLOCKS}
    m = 2 + 3 * 1 + 9 * 1  # (iA, jA, kA) = (1, 0, 0)
    s = A["Auu"][J, I, k, m]
    assert s == A["Auu"][J, I + 1, k, 26 - m]
    delta = 0.25 * EPS11 * min(abs(A["Auu"][J, I, k, 13]), abs(A["Auu"][J, I + 1, k, 13]))
    A["Auu"][J, I, k, m] = s + delta
    got, md, nw = _check(P, A)
    avg = 0.5 * ((s + delta) + s)
    assert md == abs(s - (s + delta)) and nw == 0
    assert got["Auu"][J, I, k, m] == avg and got["Auu"][J, I + 1, k, 26 - m] == avg
    # (2) Auv(iA=+1) raised far above tolerance: both rows warn, nothing changes
    A = {n: np.array(S[n], copy=True) for n in BLOCKS}
    A["Auv"][J, I, k, m] += 1.0e-3 * abs(A["Auu"][J, I, k, 13])
    got, md, nw = _check(P, A)
    assert nw == 2 and md == abs(A["Avu"][J, I + 1, k, 26 - m] - A["Auv"][J, I, k, m])
    assert all(np.array_equal(got[n], A[n]) for n in BLOCKS)
    # (3) one visit passes, the other fails (the later row's Avv diagonal made tiny): averaged;
    # the earlier row (J, I) passes first, so the later visit sees equal values and is silent
    A = {n: np.array(S[n], copy=True) for n in BLOCKS}
    A["Avv"][J, I + 1, k, 13] *= 1.0e-9
    v = A["Avv"][J, I, k, m]
    A["Avv"][J, I, k, m] = v + 0.25 * EPS11 * abs(A["Avv"][J, I, k, 13])
    got, md, nw = _check(P, A)
    assert nw == 0 and got["Avv"][J, I, k, m] == got["Avv"][J, I + 1, k, 26 - m] == 0.5 * (A["Avv"][J, I, k, m] + v)
    # ... and with the earlier row's diagonal tiny instead, the earlier visit warns once
    A = {n: np.array(S[n], copy=True) for n in BLOCKS}
    A["Avv"][J, I, k, 13] *= 1.0e-9
    A["Avv"][J, I, k, m] = v + 0.25 * EPS11 * abs(A["Avv"][J, I + 1, k, 13])
    got, md, nw = _check(P, A)
    assert nw == 1 and got["Avv"][J, I, k, m] == got["Avv"][J, I + 1, k, 26 - m] == 0.5 * (A["Avv"][J, I, k, m] + v)
    # (4) Avu's own diagonal pair (0,0,0) against Auv's at the same row: checked from both loops
    A = {n: np.array(S[n], copy=True) for n in BLOCKS}
    A["Avu"][J, I, k, 13] += 1.0  # far above tolerance: two warnings (Auv loop, then Avu loop)
    got, md, nw = _check(P, A)
    assert nw == 2 and md == abs(A["Avu"][J, I, k, 13] - A["Auv"][J, I, k, 13])


@pytest.mark.parametrize("case", ["interior", "boundary-periodic", "boundary-outflow"])
def test_symmetry_3d_matches_pairwise_form(case):
    """Random perturbations, small and large, on assembled blocks: the in-place loop and the
    pairwise form agree bit for bit (blocks, maxdiff, warning count).  The boundary cases
    carry halo copies whose partners are not transposes, so they also warn by the thousand."""
    if case == "interior":
        P = problems.slab_3d(seed=42, symmetrize=False)
    else:
        P = problems.slab_3d(seed=43, boundary_ice=True, bc=case.split("-")[1], symmetrize=False)
    rng = np.random.default_rng(7)
    A = _blocks(P)
    for n in BLOCKS:
        sel = rng.random(A[n].shape) < 0.03
        scale = np.where(rng.random(A[n].shape) < 0.5, 1e-14, 1e-9)
        A[n] = np.where(sel, A[n] * (1.0 + scale * rng.standard_normal(A[n].shape)), A[n])
    got, md, nw = _check(P, A)
    want, wmd, wnw = pairwise_3d(P, A)
    assert md == wmd and nw == wnw and nw > 0
    for n in BLOCKS:
        np.testing.assert_array_equal(got[n], want[n])
    assert sum(int(np.count_nonzero(got[n] != A[n])) for n in BLOCKS) > 0


def test_symmetry_2d_reports_only():
    """The 2D check compares the same pairs (jA, iA outer) and changes nothing: maxdiff and the
    warning count follow directly from the blocks, each differing visit counted once."""
    P = problems.slab_2d(seed=44, boundary_ice=True)
    rng = np.random.default_rng(8)
    A = {n: np.array(getattr(P, n), copy=True) for n in BLOCKS}  # (9, NY, NX)
    for n in BLOCKS:
        sel = rng.random(A[n].shape) < 0.05
        A[n] = np.where(sel, A[n] * (1.0 + 1e-12 * rng.standard_normal(A[n].shape)), A[n])
    got, md, nw = _check(P, A)
    assert all(np.array_equal(got[n], A[n]) for n in BLOCKS)
    NY, NX = P.bu.shape
    wmd, wnw = 0.0, 0
    for j, i in _owned_rows(P):
        du, dv = A["Auu"][4, j, i], A["Avv"][4, j, i]
        for jA in (-1, 0, 1):
            for iA in (-1, 0, 1):
                if not (0 <= i + iA < NX and 0 <= j + jA < NY):
                    continue
                m = (iA + 1) + 3 * (jA + 1)
                for n1, n2, dg in (("Auu", "Auu", du), ("Auv", "Avu", du), ("Avv", "Avv", dv), ("Avu", "Auv", dv)):
                    x, y = A[n1][m, j, i], A[n2][8 - m, j + jA, i + iA]
                    if x != y:
                        wmd = max(wmd, abs(y - x))
                        wnw += not (abs(y - x) < EPS11 * abs(dg))
    assert md == wmd and nw == wnw and nw > 0 and md > 0.0


def test_symmetry_check_skips_inactive_rows():
    """Rows of inactive vertices are not visited: a coefficient of an inactive row whose
    partner row is inactive too is left as it is, however asymmetric."""
    P = problems.slab_3d(seed=45, symmetrize=False)
    S = _symmetrized(P)
    act = P.active_vertex != 0
    j, i, iA, jA = next((j, i, iA, jA) for j, i in zip(*np.nonzero(~act))
                        for jA in (-1, 0, 1) for iA in (-1, 0, 1)
                        if (iA, jA) != (0, 0) and 0 < j < act.shape[0] - 1 and 0 < i < act.shape[1] - 1 and
                        not act[j + jA, i + iA])
    m = (iA + 1) + 3 * (jA + 1) + 9
    A = {n: np.array(S[n], copy=True) for n in BLOCKS}
    A["Auu"][j, i, 1, m] = 12345.0
    got, md, nw = _check(P, A)
    assert md == 0.0 and nw == 0 and got["Auu"][j, i, 1, m] == 12345.0


@pytest.mark.parametrize("which", ["dome", "member", "slab-periodic", "slab-outflow", "slab-noslip"])
def test_package_symmetrization_matches_reference_check(which):
    """The synthetic 3D systems end with the reference's pre-solve symmetry check
    (cism_b200.assembly.symmetrize_3d, glissade_velo_higher_solve :2923-2931): the vectorized
    pair averaging gives the oracle's in-place loop result bit for bit, and a second check
    changes nothing."""
    from cism_b200 import assembly as asm
    if which == "dome":
        make = lambda sym: asm.dome(symmetrize=sym)  # noqa: E731
    elif which == "member":
        make = lambda sym: asm.batch_member(30, 5, nz=7, symmetrize=sym)  # noqa: E731
    elif which == "slab-noslip":
        make = lambda sym: problems.slab_3d(seed=5, sliding=False, symmetrize=sym)  # noqa: E731
    else:
        bc = which.split("-")[1]
        make = lambda sym: problems.slab_3d(seed=4, bc=bc, boundary_ice=True, symmetrize=sym)  # noqa: E731
    P, Q = make(True), make(False)
    ou, ouv, ovu, ov, md, nw = oracle.check_symmetry(Q)
    np.testing.assert_array_equal(P.Auu, ou)
    np.testing.assert_array_equal(P.Auv, ouv)
    np.testing.assert_array_equal(P.Avu, ovu)
    np.testing.assert_array_equal(P.Avv, ov)
    ru, ruv, rvu, rv, md2, nw2 = oracle.check_symmetry(P)
    for a, b in zip((ru, ruv, rvu, rv), (P.Auu, P.Auv, P.Avu, P.Avv)):
        np.testing.assert_array_equal(a, b)
    # an assembly with an ice-free outer ring leaves nothing above the tolerance; the slabs with
    # ice on the boundary take their halo rows from the halo update (periodic copies of the far
    # side, outflow zeros), which the element sums of the owned rows do not match
    if not which.startswith("slab-") or which == "slab-noslip":
        assert nw == 0 and nw2 == 0 and md2 == 0.0
