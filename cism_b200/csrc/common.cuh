// common.cuh -- shared device definitions of the structured PCG library.
//
// Device data layout (HBM):
//   columns q = i + NX*j (0-based vertex indices, NX = nx-1, NY = ny-1), NQ = NX*NY;
//   vectors are level-major planes: v[k*NQ + q]  (2D solves: nz = 1);
//   FP64 matrix blocks are coefficient planes: A[((blk*NC + c)*nz + k)*NQ + q],
//   blk in {uu, uv, vu, vv}, c the canonical stencil offset
//   c = (iA+1) + 3(jA+1) + 9(kA+1)  (NC = 27 in 3D; NC = 9 and kA = 0 in 2D),
//   which is the order the reference's matvec loops run (kA, jA, iA).
// One thread owns one column and walks its levels; a CTA of 256 threads owns 256
// consecutive columns.  All loads of matrix planes and vector planes are coalesced.
//
// Every global sum uses one fixed reduction tree, independent of launch shape and
// of other work on the device: per column a double-double sum over k = 1..nz,
// a shuffle-down warp tree, a block tree over the 8 warp sums, chunk partials in
// HBM, and a fixed final tree by the last CTA to finish.  Results are therefore
// bit-reproducible run to run and identical whether a solve runs alone or next to
// others.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cismgpu {

constexpr int kBlock = 256;  // threads per CTA == columns per reduction chunk

struct Geom {
    int NX, NY, nz;
    long long NQ;          // NX*NY
    int ilo, ihi, jlo, jhi;  // owned vertex bounds, 0-based inclusive
    int periodic, outflow, no_ice;
};

__host__ __device__ inline bool owned(const Geom &g, int i, int j) {
    return i >= g.ilo && i <= g.ihi && j >= g.jlo && j <= g.jhi;
}

// ---------------------------------------------------------------------------
// double-double (operation order mirrored by the CPU oracle's restatement)
// ---------------------------------------------------------------------------
struct DD { double hi, lo; };

__device__ __forceinline__ DD dd_add_d(DD a, double x) {
    double s = __dadd_rn(a.hi, x);
    double bb = __dsub_rn(s, a.hi);
    double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(x, bb));
    e = __dadd_rn(e, a.lo);
    double hi = __dadd_rn(s, e);
    double lo = __dsub_rn(e, __dsub_rn(hi, s));
    return DD{hi, lo};
}

__device__ __forceinline__ DD dd_add(DD a, DD b) {
    double s = __dadd_rn(a.hi, b.hi);
    double bb = __dsub_rn(s, a.hi);
    double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b.hi, bb));
    e = __dadd_rn(e, __dadd_rn(a.lo, b.lo));
    double hi = __dadd_rn(s, e);
    double lo = __dsub_rn(e, __dsub_rn(hi, s));
    return DD{hi, lo};
}

__device__ __forceinline__ DD dd_shfl_down(DD v, int off) {
    DD r;
    r.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
    r.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
    return r;
}

// Block tree over 256 threads; result valid in thread 0.  'sm' holds 8 DD.
__device__ __forceinline__ DD block_tree(DD v, DD *sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        DD o = dd_shfl_down(v, off);
        if (lane + off < 32) v = dd_add(v, o);
    }
    __syncthreads();  // protect 'sm' reuse across consecutive calls
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        DD w = (lane < 8) ? sm[lane] : DD{0.0, 0.0};
#pragma unroll
        for (int off = 4; off >= 1; off >>= 1) {
            DD o = dd_shfl_down(w, off);
            if (lane + off < 32) w = dd_add(w, o);
        }
        v = w;
    }
    return v;
}

// ---------------------------------------------------------------------------
// Per-solve scalar state, resident in HBM for the whole solve
// ---------------------------------------------------------------------------
struct SolveState {
    double eta0, eta1, eta2, alpha, beta;     // standard PCG
    double rho_old, sigma, rho, delta;        // Chronopoulos-Gear PCG
    double L2_rhs, err;                       // convergence test
    double tol;
    int done;                                 // 1 once converged or failed: later kernels return at once
    int status;                               // CISMGPU_* status
    int niters;
    int checks;                               // number of residual checks done
    unsigned int ticket[4];                   // last-CTA tickets, one per concurrent reduction slot
    unsigned long long maxbits;               // residual velocity: bits of the largest difference so far
    unsigned long long count;                 // residual velocity (mean): nonzero speeds counted
};

enum Epi {
    EPI_NONE = 0,
    EPI_L2RHS,        // L2_rhs = sqrt(S0)
    EPI_STD_ETA1,     // eta1 = S0; NaN -> fail; beta = eta1/eta0
    EPI_STD_ETA2,     // eta0 = eta1; eta2 = S0; alpha = eta1/eta2; NaN -> fail
    EPI_CHECK,        // err = sqrt(S0)/L2_rhs; err < tol -> done, niters = iter
    EPI_CG_RHO0,      // rho_old = S0
    EPI_CG_FIRST,     // sigma = S0; alpha = rho_old/sigma; NaN -> fail
    EPI_CG_ITER,      // rho = S0; delta = S1; beta, sigma, alpha, rho_old; NaN -> fail
    EPI_RESID_VEC,    // err = sqrt(S0) = |Ax - b|; L2_rhs = sqrt(S1) = |b| (owned active)
    EPI_SUM,          // rho = S0
};

}  // namespace cismgpu
