"""Generate tests/golden/dense_kat.npz: dense-LU solutions of small assembled systems.

The reference ships no golden vectors for its PCG; these fixtures pin the oracle
and the GPU library against an independent dense direct solve (numpy LAPACK),
computed on the owned, active nodes of small first-Picard systems from
cism_b200.assembly.  Run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests import problems  # noqa: E402
from tests.test_oracle_kat import _owned_active_dense  # noqa: E402


def main():
    # the 3D slab without the pre-solve symmetry averaging: on its symmetrized form the
    # Chronopoulos-Gear test solve stagnates at a relative residual of 8e-10, short of the
    # 1e-10 these fixtures are checked at
    out = {}
    for name, P in (("slab3d", problems.slab_3d(seed=21, nz=4, symmetrize=False)), ("slab2d", problems.slab_2d(seed=22))):
        idx, A, b = _owned_active_dense(P)
        xs = np.linalg.solve(A, b)
        n = len(idx)
        xu, xv = np.zeros_like(P.bu), np.zeros_like(P.bv)
        for key, r in idx.items():
            xu[key[:P.bu.ndim]] = xs[r]
            xv[key[:P.bv.ndim]] = xs[n + r]
        cond = np.linalg.cond(A)
        out[f"{name}_bu"] = P.bu
        out[f"{name}_xu"] = xu
        out[f"{name}_xv"] = xv
        out[f"{name}_cond"] = cond
        # a converged PCG (err < 1e-10) is within ~cond * 1e-10 of the exact solution
        out[f"{name}_bound"] = max(1e-12, 10.0 * cond * 1e-10)
        print(name, "unknowns", 2 * n, "cond %.3e" % cond)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "dense_kat.npz"), **out)


if __name__ == "__main__":
    main()
