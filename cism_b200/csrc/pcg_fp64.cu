// pcg_fp64.cu -- plain FP64 structured PCG on B200 (sm_100a), reference-faithful.
//
// Each kernel restates one or more consecutive whole-array statements of
// libglissade/glissade_velo_higher_pcg.F90 with the same floating-point operation
// order (the library is compiled with --fmad=false, so a*b+c is never contracted),
// and global sums go through the fixed double-double tree of common.cuh.  The
// kernels never read the CPU; scalars (alpha, beta, ...) live in SolveState in HBM
// and are produced by the last CTA of the reducing kernel.
#include "common.cuh"
#include "../../include/cismgpu.h"

namespace cismgpu {

// ---------------------------------------------------------------------------
// reduction: per-CTA dd partials -> last CTA finishes with the fixed tree and
// runs the scalar epilogue
// ---------------------------------------------------------------------------
struct RedCtx {
    DD *partials;        // [gridDim.x][2]
    SolveState *st;
    int epi;
    int iter;
};

__device__ void epilogue(SolveState *st, int epi, int iter, double S0, double S1) {
    switch (epi) {
    case EPI_L2RHS:
        st->L2_rhs = sqrt(S0);
        break;
    case EPI_STD_ETA1: {  // :1325-1337
        st->eta1 = S0;
        if (S0 != S0) { st->status = CISMGPU_EBREAKDOWN_ETA1; st->done = 1; st->niters = iter; break; }
        st->beta = st->eta1 / st->eta0;
        break;
    }
    case EPI_STD_ETA2: {  // :1371-1394
        st->eta0 = st->eta1;
        st->eta2 = S0;
        st->alpha = st->eta1 / st->eta2;
        if (st->alpha != st->alpha) { st->status = CISMGPU_EBREAKDOWN_ALPHA; st->done = 1; st->niters = iter; }
        break;
    }
    case EPI_CHECK: {     // :1466-1513, :3516-3563
        st->err = sqrt(S0) / st->L2_rhs;
        st->checks += 1;
        if (st->err < st->tol) { st->niters = iter; st->done = 1; }
        break;
    }
    case EPI_CG_RHO0:     // (r,z) of the first pass, kept until (d,q) is known (:3215, :3258)
        st->rho_old = S0;
        break;
    case EPI_CG_FIRST: {  // :3258-3266
        st->sigma = S0;
        st->alpha = st->rho_old / st->sigma;
        if (st->alpha != st->alpha) { st->status = CISMGPU_EBREAKDOWN_ALPHA; st->done = 1; st->niters = iter; }
        break;
    }
    case EPI_CG_ITER: {   // :3426-3437
        st->rho = S0;
        st->delta = S1;
        st->beta = st->rho / st->rho_old;
        st->sigma = st->delta - st->beta * st->rho / st->alpha;
        st->alpha = st->rho / st->sigma;
        st->rho_old = st->rho;
        if (st->alpha != st->alpha) { st->status = CISMGPU_EBREAKDOWN_ALPHA; st->done = 1; st->niters = iter; }
        break;
    }
    case EPI_RESID_VEC:   // glissade_velo_higher.F90:9858-9859, :9883-9884
        st->err = sqrt(S0);
        st->L2_rhs = sqrt(S1);
        break;
    case EPI_SUM:
        st->rho = S0;
        break;
    default:
        break;
    }
}

// Called by all threads of every CTA with the thread's column partials.
template <int NF>
__device__ void reduce_and_finish(const RedCtx &rc, DD v0, DD v1) {
    __shared__ DD sm[8];
    __shared__ bool last;
    DD b0 = block_tree(v0, sm);
    DD b1 = DD{0.0, 0.0};
    if (NF > 1) b1 = block_tree(v1, sm);
    if (threadIdx.x == 0) {
        rc.partials[2 * blockIdx.x + 0] = b0;
        rc.partials[2 * blockIdx.x + 1] = b1;
        __threadfence();
        unsigned int t = atomicAdd(&rc.st->ticket[0], 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    DD a0{0.0, 0.0}, a1{0.0, 0.0};
    for (unsigned int c = threadIdx.x; c < gridDim.x; c += kBlock) {
        DD p0, p1;
        p0.hi = __ldcg(&rc.partials[2 * c].hi);
        p0.lo = __ldcg(&rc.partials[2 * c].lo);
        a0 = dd_add(a0, p0);
        if (NF > 1) {
            p1.hi = __ldcg(&rc.partials[2 * c + 1].hi);
            p1.lo = __ldcg(&rc.partials[2 * c + 1].lo);
            a1 = dd_add(a1, p1);
        }
    }
    DD r0 = block_tree(a0, sm);
    DD r1 = DD{0.0, 0.0};
    if (NF > 1) r1 = block_tree(a1, sm);
    if (threadIdx.x == 0) {
        rc.st->ticket[0] = 0u;
        epilogue(rc.st, rc.epi, rc.iter, r0.hi + r0.lo, r1.hi + r1.lo);
    }
}

// Block tree over the first 256 threads of a block of any size (the other threads pass
// through the barriers); result in thread 0.  Same order as block_tree.
__device__ __forceinline__ DD block_tree_first(DD v, DD *sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < kBlock / 32) {
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            DD o = dd_shfl_down(v, off);
            if (lane + off < 32) v = dd_add(v, o);
        }
    }
    __syncthreads();  // protect 'sm' reuse across consecutive calls
    if (warp < kBlock / 32 && lane == 0) sm[warp] = v;
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

// reduce_and_finish for blocks of kBlock * L threads whose first kBlock threads hold the
// values (the column sums); identical order and result to reduce_and_finish.
template <int NF>
__device__ void reduce_and_finish_first(const RedCtx &rc, DD v0, DD v1) {
    __shared__ DD sm[8];
    __shared__ bool last;
    DD b0 = block_tree_first(v0, sm);
    DD b1 = DD{0.0, 0.0};
    if (NF > 1) b1 = block_tree_first(v1, sm);
    if (threadIdx.x == 0) {
        rc.partials[2 * blockIdx.x + 0] = b0;
        rc.partials[2 * blockIdx.x + 1] = b1;
        __threadfence();
        unsigned int t = atomicAdd(&rc.st->ticket[0], 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    DD a0{0.0, 0.0}, a1{0.0, 0.0};
    if (threadIdx.x < kBlock)
        for (unsigned int c = threadIdx.x; c < gridDim.x; c += kBlock) {
            DD p0, p1;
            p0.hi = __ldcg(&rc.partials[2 * c].hi);
            p0.lo = __ldcg(&rc.partials[2 * c].lo);
            a0 = dd_add(a0, p0);
            if (NF > 1) {
                p1.hi = __ldcg(&rc.partials[2 * c + 1].hi);
                p1.lo = __ldcg(&rc.partials[2 * c + 1].lo);
                a1 = dd_add(a1, p1);
            }
        }
    DD r0 = block_tree_first(a0, sm);
    DD r1 = DD{0.0, 0.0};
    if (NF > 1) r1 = block_tree_first(a1, sm);
    if (threadIdx.x == 0) {
        rc.st->ticket[0] = 0u;
        epilogue(rc.st, rc.epi, rc.iter, r0.hi + r0.lo, r1.hi + r1.lo);
    }
}

__device__ __forceinline__ void col_of(const Geom &g, long long q, int &i, int &j) {
    j = (int)(q / g.NX);
    i = (int)(q - (long long)j * g.NX);
}

// ---------------------------------------------------------------------------
// structured matvec row (matvec_multiply_structured_3d :5612-5650, _2d :5739-5771)
// ---------------------------------------------------------------------------
template <int NC>
__device__ __forceinline__ void mv_row(const Geom &g, const double *__restrict__ A, const double *__restrict__ xu,
                                       const double *__restrict__ xv, int i, int j, long long q, int k,
                                       double &yu, double &yv) {
    const long long plane = (long long)g.nz * g.NQ;
    const double *Auu = A, *Auv = A + NC * plane, *Avu = A + 2 * NC * plane, *Avv = A + 3 * NC * plane;
    double su = 0.0, sv = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
        if (k + kA >= 0 && k + kA < g.nz && i + iA >= 0 && i + iA < g.NX && j + jA >= 0 && j + jA < g.NY) {
            const long long a = (long long)c * plane + (long long)k * g.NQ + q;
            const long long n = (long long)(k + kA) * g.NQ + q + iA + (long long)jA * g.NX;
            const double x1 = xu[n], x2 = xv[n];
            su = __dadd_rn(__dadd_rn(su, __dmul_rn(Auu[a], x1)), __dmul_rn(Auv[a], x2));
            sv = __dadd_rn(__dadd_rn(sv, __dmul_rn(Avu[a], x1)), __dmul_rn(Avv[a], x2));
        }
    }
    yu = su;
    yv = sv;
}

enum MvMode { MV_PLAIN = 0, MV_RESID, MV_DQ, MV_CG_AZ };

constexpr int kDotChunk = 8;  // levels whose loads a column's dot terms issue together

// The dot terms of column q (modes with dot products), added over k in level order: a chunk's
// loads together, then its terms in order.  Loads through L2 (__ldcg): the other levels' y and
// r were written by other CTAs of the same launch.
template <int MODE>
__device__ __forceinline__ void col_dots(const Geom &g, long long q, const double *__restrict__ xu,
                                         const double *__restrict__ xv, const double *__restrict__ yu,
                                         const double *__restrict__ yv, const double *__restrict__ ru,
                                         const double *__restrict__ rv, DD &s0, DD &s1) {
    for (int k0 = 0; k0 < g.nz; k0 += kDotChunk) {
        double t0[kDotChunk], t1[kDotChunk];
#pragma unroll
        for (int u = 0; u < kDotChunk; ++u) {
            t0[u] = t1[u] = 0.0;
            if (k0 + u >= g.nz) continue;
            const long long e = (long long)(k0 + u) * g.NQ + q;
            if (MODE == MV_RESID) {
                const double r1 = __ldcg(ru + e), r2 = __ldcg(rv + e);
                t0[u] = __dadd_rn(__dmul_rn(r1, r1), __dmul_rn(r2, r2));
            } else if (MODE == MV_DQ) {
                t0[u] = __dadd_rn(__dmul_rn(__ldcg(xu + e), __ldcg(yu + e)), __dmul_rn(__ldcg(xv + e), __ldcg(yv + e)));
            } else if (MODE == MV_CG_AZ) {
                const double z1 = __ldcg(xu + e), z2 = __ldcg(xv + e);
                t0[u] = __dadd_rn(__dmul_rn(__ldcg(ru + e), z1), __dmul_rn(__ldcg(rv + e), z2));
                t1[u] = __dadd_rn(__dmul_rn(__ldcg(yu + e), z1), __dmul_rn(__ldcg(yv + e), z2));
            }
        }
#pragma unroll
        for (int u = 0; u < kDotChunk; ++u)
            if (k0 + u < g.nz) {
                s0 = dd_add_d(s0, t0[u]);
                if (MODE == MV_CG_AZ) s1 = dd_add_d(s1, t1[u]);
            }
    }
}

// y = A x over owned active columns, 0 elsewhere; optional fused statements:
//   MV_RESID : r = b - y (whole array); S0 = (r,r)             [:1454-1466, :3504-3516]
//   MV_DQ    : S0 = (x,y) with x = d, y = q                    [:1376-1381, :3241-3248]
//   MV_CG_AZ : S0 = (r,z), S1 = (y,z) with x = z, y = Az       [:3401-3413]
// k_mv_nodes: one thread per node (column q, level k = blockIdx.y), y = A x with the
// reference's statements (mv_row), and for MV_RESID also r = b - y: every (column, level) is
// independent, so a launch has nz * NQ/256 CTAs and enough loads in flight to stream the 108
// coefficient planes.  Dot products in 3D: the last level block of each column block to
// finish has one thread per column add its terms over k in level order (col_dots), then the
// block tree of the 256 columns and the last-CTA tree: the order the reduction has always
// had.  In 2D a column has one level, so every block adds its terms and reduces.
template <int NC, int MODE>
__global__ void __launch_bounds__(kBlock, 4) k_mv_nodes(Geom g, const double *__restrict__ A,
                                                     const int32_t *__restrict__ act,
                                                     const double *__restrict__ xu, const double *__restrict__ xv,
                                                     double *__restrict__ yu, double *__restrict__ yv,
                                                     const double *__restrict__ bu, const double *__restrict__ bv,
                                                     double *__restrict__ ru, double *__restrict__ rv, RedCtx rc) {
    // 2D (one level per column): the column's dot terms and the reduction in this kernel
    constexpr bool FUSED = (NC == 9) && (MODE == MV_RESID || MODE == MV_DQ || MODE == MV_CG_AZ);
    if (rc.st && rc.st->done) return;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    const int k = blockIdx.y;
    DD s0{0.0, 0.0}, s1{0.0, 0.0};
    if (q < g.NQ) {
        int i, j;
        col_of(g, q, i, j);
        const bool own = owned(g, i, j);
        const bool on = own && act[q] != 0;
        const long long e = (long long)k * g.NQ + q;
        double a = 0.0, b = 0.0;
        if (on) mv_row<NC>(g, A, xu, xv, i, j, q, k, a, b);
        yu[e] = a;
        yv[e] = b;
        double r1 = 0.0, r2 = 0.0;
        if (MODE == MV_RESID) {
            r1 = __dsub_rn(bu[e], a);
            r2 = __dsub_rn(bv[e], b);
            ru[e] = r1;
            rv[e] = r2;
        }
        if (FUSED && own) {
            if (MODE == MV_RESID) {
                s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(r1, r1), __dmul_rn(r2, r2)));
            } else if (MODE == MV_DQ) {
                s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(xu[e], a), __dmul_rn(xv[e], b)));
            } else if (MODE == MV_CG_AZ) {
                const double z1 = xu[e], z2 = xv[e];
                s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(ru[e], z1), __dmul_rn(rv[e], z2)));
                s1 = dd_add_d(s1, __dadd_rn(__dmul_rn(a, z1), __dmul_rn(b, z2)));
            }
        }
    }
    if (FUSED) {
        if (MODE == MV_CG_AZ) reduce_and_finish_first<2>(rc, s0, s1);
        else reduce_and_finish_first<1>(rc, s0, s1);
    }
    if (NC == 27 && MODE != MV_PLAIN) {
        // the last of the gridDim.y level blocks of column block blockIdx.x to finish adds the
        // dot terms of its 256 columns over all levels, then the block tree and the last-CTA
        // tree: the same order as a separate dot pass, without its launch and with the sums of
        // the early column blocks overlapping the rest of the matvec.  The per-column-block
        // counters sit after the partials and return to zero here.
        __shared__ bool lastk;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned *cnt = reinterpret_cast<unsigned *>(rc.partials + 2 * gridDim.x) + blockIdx.x;
            __threadfence();  // this block's y and r before its count
            const unsigned t = atomicAdd(cnt, 1u);
            lastk = t == gridDim.y - 1;
            if (lastk) *cnt = 0u;
        }
        __syncthreads();
        if (!lastk) return;
        __threadfence();
        DD d0{0.0, 0.0}, d1{0.0, 0.0};
        if (q < g.NQ) {
            int i, j;
            col_of(g, q, i, j);
            if (owned(g, i, j)) col_dots<MODE>(g, q, xu, xv, yu, yv, ru, rv, d0, d1);
        }
        if (MODE == MV_CG_AZ) reduce_and_finish_first<2>(rc, d0, d1);
        else reduce_and_finish_first<1>(rc, d0, d1);
    }
}

// y = A x (+ the statement MODE fuses with it, see MvMode) on stream s.
template <int NC, int MODE>
inline void launch_mv(cudaStream_t s, const Geom &g, const double *A, const int32_t *act, const double *xu,
                      const double *xv, double *yu, double *yv, const double *bu, const double *bv, double *ru,
                      double *rv, const RedCtx &rc) {
    const dim3 grid((unsigned)((g.NQ + kBlock - 1) / kBlock), (unsigned)g.nz);
    k_mv_nodes<NC, MODE><<<grid, kBlock, 0, s>>>(g, A, act, xu, xv, yu, yv, bu, bv, ru, rv, rc);
}

// ---------------------------------------------------------------------------
// preconditioner apply over the whole array (halo included)
// ---------------------------------------------------------------------------
// tridiag_solver (:5870-5922) on one column of the SIA matrix (easy_sia_solver :5777-5866).
// M(-1), M(0), M(+1) are the A planes of offsets (0,0,-1), (0,0,0), (0,0,+1).
constexpr int kMaxNz = 64;

__device__ void sia_column(const Geom &g, const double *__restrict__ Mlo, const double *__restrict__ Mdi,
                           const double *__restrict__ Mup, const double *__restrict__ r, double *__restrict__ z,
                           long long q) {
    const int nz = g.nz;
    const long long NQ = g.NQ;
    double gam[kMaxNz];
    double sol[kMaxNz];
    // top layer: sbdiag = 0, diag = M(0), spdiag = M(+1); bottom layer: spdiag = 0
    double beta = Mdi[q];
    sol[0] = r[q] / beta;
    for (int k = 1; k < nz; ++k) {
        const double sp_prev = Mup[(long long)(k - 1) * NQ + q];  // spdiag(k-1), k-1 <= nz-1
        const double sb = Mlo[(long long)k * NQ + q];
        const double dg = Mdi[(long long)k * NQ + q];
        gam[k] = sp_prev / beta;
        beta = __dsub_rn(dg, __dmul_rn(sb, gam[k]));
        sol[k] = __dsub_rn(r[(long long)k * NQ + q], __dmul_rn(sb, sol[k - 1])) / beta;
    }
    for (int k = nz - 2; k >= 0; --k) sol[k] = __dsub_rn(sol[k], __dmul_rn(gam[k + 1], sol[k + 1]));
    for (int k = 0; k < nz; ++k) z[(long long)k * NQ + q] = sol[k];
}

enum PreMode { PRE_ONLY = 0, PRE_STD, PRE_CG_FIRST };

// z = PC(r) over the whole array, then optionally:
//   PRE_STD      : S0 = (r,z)                      [:1320-1326]
//   PRE_CG_FIRST : S0 = (r,z) kept for the first-pass epilogue; d = z   [:3215-3223]
// kind: 0 none (z = r), 1 diag, 2 sia (3D only), 3/4 tridiagonal: in 2D z was written by
// k_tri_lines and the halo update, in 3D the SIA columns plus the summed line solution zs
// ([2][NQ], u then v) on every level; anything else: z unchanged.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_precond(Geom g, int kind, const double *__restrict__ A,
                                                    int NC, const int32_t *__restrict__ act,
                                                    const double *__restrict__ ru, const double *__restrict__ rv,
                                                    double *__restrict__ zu, double *__restrict__ zv,
                                                    double *__restrict__ du, double *__restrict__ dv,
                                                    RedCtx rc, const double *__restrict__ zs = nullptr) {
    if (rc.st->done) return;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    DD s0{0.0, 0.0};
    if (q < g.NQ) {
        int i, j;
        col_of(g, q, i, j);
        const long long plane = (long long)g.nz * g.NQ;
        const int cdiag = (NC == 27) ? 13 : 4;
        const double *Auu = A, *Avv = A + 3LL * NC * plane;
        if (kind == CISMGPU_PRECOND_NONE) {
            for (int k = 0; k < g.nz; ++k) {
                const long long e = (long long)k * g.NQ + q;
                zu[e] = ru[e];
                zv[e] = rv[e];
            }
        } else if (kind == CISMGPU_PRECOND_DIAG) {  // :1238-1253 (3D), :467-480 (2D)
            for (int k = 0; k < g.nz; ++k) {
                const long long e = (long long)k * g.NQ + q;
                const double a = Auu[(long long)cdiag * plane + e], b = Avv[(long long)cdiag * plane + e];
                zu[e] = (a != 0.0) ? ru[e] / a : 0.0;
                zv[e] = (b != 0.0) ? rv[e] / b : 0.0;
            }
        } else if (kind == CISMGPU_PRECOND_SIA && NC == 27) {  // :1255-1263
            if (act[q] != 0) {
                sia_column(g, Auu + 4 * plane, Auu + 13 * plane, Auu + 22 * plane, ru, zu, q);
                sia_column(g, Avv + 4 * plane, Avv + 13 * plane, Avv + 22 * plane, rv, zv, q);
            }
        } else if ((kind == CISMGPU_PRECOND_TRIDIAG_LOCAL || kind == CISMGPU_PRECOND_TRIDIAG_GLOBAL) && NC == 27) {
            // tridiag_solver_{local,global}_3d :4617-4655 / :4876-4911: SIA columns, then + zs
            if (act[q] != 0) {
                sia_column(g, Auu + 4 * plane, Auu + 13 * plane, Auu + 22 * plane, ru, zu, q);
                sia_column(g, Avv + 4 * plane, Avv + 13 * plane, Avv + 22 * plane, rv, zv, q);
            }
            const double su = zs[q], sv = zs[g.NQ + q];
            for (int k = 0; k < g.nz; ++k) {
                const long long e = (long long)k * g.NQ + q;
                zu[e] = __dadd_rn(zu[e], su);
                zv[e] = __dadd_rn(zv[e], sv);
            }
        }
        if (MODE == PRE_STD || MODE == PRE_CG_FIRST) {
            const bool own = owned(g, i, j);
            for (int k = 0; k < g.nz; ++k) {
                const long long e = (long long)k * g.NQ + q;
                const double z1 = zu[e], z2 = zv[e];
                if (own) s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(ru[e], z1), __dmul_rn(rv[e], z2)));
                if (MODE == PRE_CG_FIRST) { du[e] = z1; dv[e] = z2; }
            }
        }
    }
    if (MODE == PRE_STD || MODE == PRE_CG_FIRST) reduce_and_finish<1>(rc, s0, s0);
}

// ---------------------------------------------------------------------------
// nonlinear-iteration diagnostics (glissade_velo_higher.F90)
// ---------------------------------------------------------------------------
// compute_residual_vector_{2d,3d} (:9502-9689 / :9693-9894), after y = A u (k_mv MV_PLAIN,
// the same statements and order): resid = y - b on owned active vertices, 0 elsewhere;
// S0 = sum of resid_u^2 + resid_v^2, S1 = sum of bu^2 + bv^2 over owned active vertices (the
// global sums' fixed tree).
__global__ void __launch_bounds__(kBlock) k_resid_vec(Geom g, const int32_t *__restrict__ act,
                                                      const double *__restrict__ yu, const double *__restrict__ yv,
                                                      const double *__restrict__ bu, const double *__restrict__ bv,
                                                      double *__restrict__ ru, double *__restrict__ rv, RedCtx rc) {
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    DD s0{0.0, 0.0}, s1{0.0, 0.0};
    if (q < g.NQ) {
        int i, j;
        col_of(g, q, i, j);
        const bool on = owned(g, i, j) && act[q] != 0;
        for (int k = 0; k < g.nz; ++k) {
            const long long e = (long long)k * g.NQ + q;
            if (on) {
                const double r1 = __dsub_rn(yu[e], bu[e]), r2 = __dsub_rn(yv[e], bv[e]);
                ru[e] = r1;
                rv[e] = r2;
                s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(r1, r1), __dmul_rn(r2, r2)));
                s1 = dd_add_d(s1, __dadd_rn(__dmul_rn(bu[e], bu[e]), __dmul_rn(bv[e], bv[e])));
            } else {
                ru[e] = 0.0;
                rv[e] = 0.0;
            }
        }
    }
    reduce_and_finish<2>(rc, s0, s1);
}

// compute_residual_velocity_{2d,3d} (:10188-10310 / :10314-10446) over owned vertices and
// levels k < kmax: speed = sqrt(u**2 + v**2); where speed /= 0, d = abs((oldspeed-speed)/speed).
// Max modes: the largest d, as atomicMax on the bits of a non-negative double (a NaN d never
// wins, as "d > resid_velo" is false for it; the state's maxbits starts at +0).  Mean mode: the
// count and the sum of d (the global sums' fixed tree; EPI_SUM).
__global__ void __launch_bounds__(kBlock) k_resid_velo(Geom g, int kmax, int mean, const double *__restrict__ u,
                                                       const double *__restrict__ v, const double *__restrict__ us,
                                                       const double *__restrict__ vs, RedCtx rc) {
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    DD s0{0.0, 0.0};
    unsigned long long cnt = 0;
    if (q < g.NQ) {
        int i, j;
        col_of(g, q, i, j);
        if (owned(g, i, j))
            for (int k = 0; k < kmax; ++k) {
                const long long e = (long long)k * g.NQ + q;
                const double speed = __dsqrt_rn(__dadd_rn(__dmul_rn(u[e], u[e]), __dmul_rn(v[e], v[e])));
                if (speed != 0.0) {
                    const double old = __dsqrt_rn(__dadd_rn(__dmul_rn(us[e], us[e]), __dmul_rn(vs[e], vs[e])));
                    const double d = fabs(__ddiv_rn(__dsub_rn(old, speed), speed));
                    if (mean) {
                        ++cnt;
                        s0 = dd_add_d(s0, d);
                    } else if (d > 0.0) {
                        atomicMax(&rc.st->maxbits, (unsigned long long)__double_as_longlong(d));
                    }
                }
            }
    }
    if (mean) {
        if (cnt) atomicAdd(&rc.st->count, cnt);
        reduce_and_finish<1>(rc, s0, s0);
    }
}

// ---------------------------------------------------------------------------
// check_symmetry_assembled_matrix_{3d,2d} (glissade_velo_higher.F90:10854-11117 and
// :10648-10850) pair by pair
// ---------------------------------------------------------------------------
// The reference visits every owned active row R and compares each coefficient of offset d
// with its transpose partner at row R+d, offset -d: Auu with Auu, Auv with Avu (Auu's
// diagonal in the tolerance), then Avv with Avv, Avu with Auv (Avv's diagonal).  A visit
// whose values differ raises maxdiff to |val2 - val1| and, when that is below
// eps11 * |diag of the visited row|, the 3D check averages the pair in place; otherwise it
// warns.  Every coefficient has exactly one partner, so the in-place loop is a function of
// each pair alone: a pair is seen from R (if R is owned and active) and from R+d (likewise),
// it is averaged when either visit's test passes on the original values, the earlier visit
// warns when its test fails, and the later one when its own fails and the earlier one did not
// average.  "Earlier" is the reference's loop order: rows j, i, k, then the Auu/Auv loop
// before the Avv/Avu loop.  One thread owns each pair (the Auv member of an Auv-Avu pair; of
// an Auu or Avv pair the member with the smaller offset index c < 26 - c), reads both values
// and writes both, and only the owners write; the diagonals that the tolerance reads are
// their own partners and are never written, so no thread reads what another writes.
constexpr double kEps11 = 1.0e-11;  // eps11, libglimmer/glimmer_paramets.F90:77

// Element offsets of coefficient c (canonical offset index (iA+1) + 3(jA+1) + 9(kA+1)) at
// level k of column q: the canonical planes (map = identity) or the caller's Fortran blocks,
// (27, nz, NX, NY) in 3D (raw3) or (NX, NY, 9) in 2D, through the caller's indxA map.
struct SymIdx {
    int32_t map[27];
    long long n;  // nz * NQ
    long long NQ;
    int nz;
    int raw3;
    __device__ __forceinline__ long long at(int c, int k, long long q) const {
        const long long m = map[c] - 1;
        return raw3 ? m + 27LL * (k + (long long)nz * q) : m * n + (long long)k * NQ + q;
    }
};

// blockIdx.y: 0 Auu-Auu pairs, 1 Auv-Avu pairs, 2 Avv-Avv pairs; x: coefficient c, level k,
// column q of the pair's first member.  out[0]: maxdiff as the bits of a non-negative double
// (a NaN difference never wins: "abs(val2 - val1) > maxdiff" is false for it), out[1]: warnings.
template <int NC, bool FIX>
__global__ void __launch_bounds__(kBlock) k_sym_check(Geom g, SymIdx L, const int32_t *__restrict__ act,
                                                      double *Auu, double *Auv, double *Avu, double *Avv,
                                                      unsigned long long *out) {
    const long long n = (long long)g.nz * g.NQ;
    const long long t = (long long)blockIdx.x * kBlock + threadIdx.x;
    const int kind = blockIdx.y;
    unsigned long long dbits = 0ull, nw = 0ull;
    if (t < NC * n) {
        const int c = (int)(t / n);
        const long long r = t - (long long)c * n;
        const int k = (int)(r / g.NQ);
        const long long q = r - (long long)k * g.NQ;
        int i, j;
        col_of(g, q, i, j);
        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
        const int cc = NC - 1 - c, cd = NC / 2;
        const int kp = k + kA, ip = i + iA, jp = j + jA;
        // a partner outside the arrays (owned rows at the array edge) is not compared
        const bool inside = kp >= 0 && kp < g.nz && ip >= 0 && ip < g.NX && jp >= 0 && jp < g.NY;
        if (inside && (kind == 1 || c <= cc)) {
            const long long qp = (long long)jp * g.NX + ip;
            const bool self = kind != 1 && c == cc;  // a diagonal is its own partner
            const bool visA = owned(g, i, j) && act[q] != 0;
            const bool visB = !self && owned(g, ip, jp) && act[qp] != 0;
            double *X = kind == 0 ? Auu : (kind == 1 ? Auv : Avv);
            double *Y = kind == 0 ? Auu : (kind == 1 ? Avu : Avv);
            const long long ea = L.at(c, k, q), eb = L.at(cc, kp, qp);
            const double x = (visA || visB) ? X[ea] : 0.0, y = (visA || visB) ? Y[eb] : 0.0;
            if (y != x) {  // val2 /= val1, true for a NaN
                const double d = fabs(__dsub_rn(y, x));
                if (d > 0.0) dbits = (unsigned long long)__double_as_longlong(d);
                // visit A from R: Auu's diagonal for the Auu and Auv checks, Avv's for Avv;
                // visit B from R+d: Auu's for Auu, Avv's for the Avv and Avu checks
                const double *DA = kind == 2 ? Avv : Auu, *DB = kind == 0 ? Auu : Avv;
                const bool passA = visA && d < __dmul_rn(kEps11, fabs(DA[L.at(cd, k, q)]));
                const bool passB = visB && d < __dmul_rn(kEps11, fabs(DB[L.at(cd, kp, qp)]));
                if (FIX) {
                    const long long rowA = k + (long long)g.nz * q, rowB = kp + (long long)g.nz * qp;
                    const bool aFirst = rowA <= rowB;  // equal rows: the Auv check (A) precedes Avu's (B)
                    const bool v1 = aFirst ? visA : visB, p1 = aFirst ? passA : passB;
                    const bool v2 = aFirst ? visB : visA, p2 = aFirst ? passB : passA;
                    nw = (unsigned long long)(v1 && !p1) + (unsigned long long)(v2 && !p2 && !p1);
                    if (passA || passB) {
                        const double avg = __dmul_rn(0.5, __dadd_rn(x, y));
                        X[ea] = avg;
                        Y[eb] = avg;
                    }
                } else {
                    nw = (unsigned long long)(visA && !passA) + (unsigned long long)(visB && !passB);
                }
            }
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        dbits = max(dbits, __shfl_down_sync(0xffffffffu, dbits, off));
        nw += __shfl_down_sync(0xffffffffu, nw, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (dbits) atomicMax(&out[0], dbits);
        if (nw) atomicAdd(&out[1], nw);
    }
}

// ---------------------------------------------------------------------------
// tridiagonal line preconditioners (precond 3 local, 4 global) on one task
// ---------------------------------------------------------------------------
// On one task the global form's solution is its particular solution (tasks_rc = 1,
// tridiag_solver_global_2d :5495-5497), which is the local form's arithmetic on the owned
// block; the forms differ in the global setup's extra zero-pivot check (:4472-4488), in
// 3D inactive columns (local zeroes all nine summed couplings, :3823-3833; global only sets
// the centre, :4025-4032) and in the local back substitution continuing below the owned
// range (:4999-5001, gamma = omega = 0 there).  Lines: u along rows j (i varies), v along
// columns i (j varies), one thread per line.  Work planes of NQ doubles:
enum TriPlane {
    TU_SUB = 0, TU_DG, TU_SP, TU_ADR, TU_OM, TU_DEN,  // u lines: sub, diag, super, 1/diag, omega, 1/denom
    TV_SUB, TV_DG, TV_SP, TV_ADR, TV_OM, TV_DEN,      // v lines
    TRS_U, TRS_V,                                     // 3D: vertical sums of r
    TZS_U, TZS_V,                                     // 3D: line solution of the summed problem
    NTRI
};

// Coefficient planes of the line systems: [u/v][sub, diag, super] -> the device planes of the
// caller's raw indices m (2D: plane c[..][0]) or m, m+9, m+18 (3D vertical sums), with m the
// raw index (1..9) indxA_2d gives the coupling.
struct TriMap {
    int c[2][3][3];
    int m[2][3];
};

// setup_preconditioner_tridiag_{local,global}_{2d,3d}: the line coefficients, zero-diagonal
// fix (:4306-4313) and 1/diag (:4347), omega = 1/denom = 0 until k_tri_factor.  3D: sums
// over levels of the three vertical offsets, ((s + A(m)) + A(m+9)) + A(m+18) (:3813-3819).
template <int NC>
__global__ void k_tri_coef(Geom g, const double *__restrict__ A, const int32_t *__restrict__ act, TriMap tm,
                           int global, double *__restrict__ T) {
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= g.NQ) return;
    const long long plane = (long long)g.nz * g.NQ;
    for (int comp = 0; comp < 2; ++comp) {
        const double *B = A + (comp ? 3LL : 0LL) * NC * plane;  // Auu or Avv
        double v[3];
        for (int e = 0; e < 3; ++e) {
            if (NC == 9) {
                v[e] = B[(long long)tm.c[comp][e][0] * g.NQ + q];
            } else {
                double sum = 0.0;
                for (int k = 0; k < g.nz; ++k) {
                    const long long o = (long long)k * g.NQ + q;
                    sum = __dadd_rn(__dadd_rn(__dadd_rn(sum, B[tm.c[comp][e][0] * plane + o]),
                                              B[tm.c[comp][e][1] * plane + o]),
                                    B[tm.c[comp][e][2] * plane + o]);
                }
                if (act[q] == 0) {
                    if (tm.m[comp][e] == 5) sum = 1.0;
                    else if (!global) sum = 0.0;
                }
                v[e] = sum;
            }
        }
        if (NC == 27 && global) {
            // the global form's staggered halo update of the nine summed planes (:4055-4058): its
            // outflow / no_ice zeroing, which with no_ice reaches the last owned row and column
            // (its periodic copies reach only halo positions, which no owned line reads)
            const int i = (int)(q % g.NX), j = (int)(q / g.NX);
            bool zero = false;
            if (g.outflow) zero = (i == 0 || i == g.NX - 1 || j == 0 || j == g.NY - 1);
            else if (g.no_ice) zero = (i <= 1 || i >= g.NX - 2 || j <= 1 || j >= g.NY - 2);
            if (zero) v[0] = v[1] = v[2] = 0.0;
        }
        if (v[1] == 0.0) { v[1] = 1.0; v[0] = 0.0; v[2] = 0.0; }
        double *P = T + (comp ? TV_SUB : TU_SUB) * g.NQ;
        P[0 * g.NQ + q] = v[0];
        P[1 * g.NQ + q] = v[1];
        P[2 * g.NQ + q] = v[2];
        P[3 * g.NQ + q] = __ddiv_rn(1.0, v[1]);
        P[4 * g.NQ + q] = 0.0;
        P[5 * g.NQ + q] = 0.0;
    }
}

__device__ __forceinline__ void tri_line(const Geom &g, int t, bool &along_i, int &l, int &s0, int &s1) {
    const int nu = g.jhi - g.jlo + 1;
    along_i = t < nu;
    l = along_i ? g.jlo + t : g.ilo + (t - nu);
    s0 = along_i ? g.ilo : g.jlo;
    s1 = along_i ? g.ihi : g.jhi;
}
__device__ __forceinline__ long long tri_at(const Geom &g, bool along_i, int l, int s) {
    return along_i ? (long long)l * g.NX + s : (long long)s * g.NX + l;
}
__host__ __device__ inline int tri_lines(const Geom &g) { return (g.jhi - g.jlo + 1) + (g.ihi - g.ilo + 1); }

// Forward elimination per owned line (:4324-4342 / :4361-4379; global :4441-4452), and for the
// global form the reverse recurrence it checks for zero pivots (:4464-4488).  A zero pivot
// is GM_FATAL in the reference: the solve ends with CISMGPU_EDIVZERO before it starts.
__global__ void k_tri_factor(Geom g, int global, double *__restrict__ T, SolveState *st) {
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= tri_lines(g)) return;
    bool along_i;
    int l, s0, s1;
    tri_line(g, t, along_i, l, s0, s1);
    double *P = T + (along_i ? TU_SUB : TV_SUB) * g.NQ;
    const double *sub = P, *dg = P + g.NQ, *sp = P + 2 * g.NQ;
    double *om = P + 4 * g.NQ, *den = P + 5 * g.NQ;
    long long e = tri_at(g, along_i, l, s0);
    double omp = __ddiv_rn(sp[e], dg[e]);
    om[e] = omp;
    for (int s = s0 + 1; s <= s1; ++s) {
        e = tri_at(g, along_i, l, s);
        const double d = __dsub_rn(dg[e], __dmul_rn(sub[e], omp));
        if (d == 0.0) {
            st->status = CISMGPU_EDIVZERO;
            st->done = 1;
            return;
        }
        const double dn = __ddiv_rn(1.0, d);
        den[e] = dn;
        omp = __dmul_rn(sp[e], dn);
        om[e] = omp;
    }
    if (global) {
        e = tri_at(g, along_i, l, s1);
        double o = __ddiv_rn(sub[e], dg[e]);
        for (int s = s1 - 1; s >= s0; --s) {
            e = tri_at(g, along_i, l, s);
            const double d = __dsub_rn(dg[e], __dmul_rn(sp[e], o));
            if (d == 0.0) {
                st->status = CISMGPU_EDIVZERO;
                st->done = 1;
                return;
            }
            o = __ddiv_rn(sub[e], d);
        }
    }
}

// sum(ru(:,i,j)) over levels, in level order (tridiag_solver_local_3d :4585-4590)
__global__ void k_tri_vsum(Geom g, const double *__restrict__ ru, const double *__restrict__ rv,
                           double *__restrict__ T, const SolveState *st) {
    if (st->done) return;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= g.NQ) return;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < g.nz; ++k) {
        a = __dadd_rn(a, ru[(long long)k * g.NQ + q]);
        b = __dadd_rn(b, rv[(long long)k * g.NQ + q]);
    }
    T[TRS_U * g.NQ + q] = a;
    T[TRS_V * g.NQ + q] = b;
}

// Line solves of tridiag_solver_local_2d (:4985-5013 u, :5041-5069 v) from planes bu, bv into
// xu, xv, which hold zeros on entry: gamma forward (stored in x), then back substitution.  A
// line is a chain of dependent operations, so the loads of kTriBatch positions are issued before
// the chain runs through them (one memory round trip per batch instead of per position); the
// operations and their order are the reference's.
constexpr int kTriBatch = 8;
__global__ void k_tri_lines(Geom g, int global, const double *__restrict__ bu, const double *__restrict__ bv,
                            double *__restrict__ xu, double *__restrict__ xv, const double *__restrict__ T,
                            const SolveState *st) {
    if (st->done) return;
    const int t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= tri_lines(g)) return;
    bool along_i;
    int l, s0, s1;
    tri_line(g, t, along_i, l, s0, s1);
    const double *P = T + (along_i ? TU_SUB : TV_SUB) * g.NQ;
    const double *sub = P, *adr = P + 3 * g.NQ, *om = P + 4 * g.NQ, *den = P + 5 * g.NQ;
    const double *b = along_i ? bu : bv;
    double *x = along_i ? xu : xv;
    long long e = tri_at(g, along_i, l, s0);
    double gp = __dmul_rn(b[e], adr[e]);
    x[e] = gp;
    for (int s = s0 + 1; s <= s1; s += kTriBatch) {
        double vb[kTriBatch], vs[kTriBatch], vd[kTriBatch];
#pragma unroll
        for (int u = 0; u < kTriBatch; ++u) {
            vb[u] = vs[u] = vd[u] = 0.0;
            if (s + u <= s1) {
                const long long f = tri_at(g, along_i, l, s + u);
                vb[u] = b[f];
                vs[u] = sub[f];
                vd[u] = den[f];
            }
        }
#pragma unroll
        for (int u = 0; u < kTriBatch; ++u)
            if (s + u <= s1) {
                gp = __dmul_rn(__dsub_rn(vb[u], __dmul_rn(vs[u], gp)), vd[u]);
                x[tri_at(g, along_i, l, s + u)] = gp;
            }
    }
    double xn = gp;
    for (int s = s1 - 1; s >= s0; s -= kTriBatch) {
        double vx[kTriBatch], vo[kTriBatch];
#pragma unroll
        for (int u = 0; u < kTriBatch; ++u) {
            vx[u] = vo[u] = 0.0;
            if (s - u >= s0) {
                const long long f = tri_at(g, along_i, l, s - u);
                vx[u] = x[f];  // this thread's forward value
                vo[u] = om[f];
            }
        }
#pragma unroll
        for (int u = 0; u < kTriBatch; ++u)
            if (s - u >= s0) {
                xn = __dsub_rn(vx[u], __dmul_rn(vo[u], xn));
                x[tri_at(g, along_i, l, s - u)] = xn;
            }
    }
    if (!global)
        for (int s = s0 - 1; s >= 0; s -= kTriBatch) {
            double vo[kTriBatch];
#pragma unroll
            for (int u = 0; u < kTriBatch; ++u) vo[u] = (s - u >= 0) ? om[tri_at(g, along_i, l, s - u)] : 0.0;
#pragma unroll
            for (int u = 0; u < kTriBatch; ++u)
                if (s - u >= 0) {
                    xn = __dsub_rn(0.0, __dmul_rn(vo[u], xn));
                    x[tri_at(g, along_i, l, s - u)] = xn;
                }
        }
}

// ---------------------------------------------------------------------------
// whole-array vector statements
// ---------------------------------------------------------------------------
enum VecOp {
    OP_STD_INIT = 0,  // r = b - z; d = 0; z = 0; S0 = (b,b)           [:1190-1216]
    OP_STD_D,         // d = z + beta*d                                  [:1340-1341]
    OP_XR,            // x = x + alpha*d; r = r - alpha*q                [:1399-1403, :3272-3276]
    OP_CG_INIT,       // r = b - z                                       [:3115-3116]
    OP_CG_UPD,        // d = z + beta*d; q = Az + beta*q; x += alpha*d; r -= alpha*q  [:3444-3459]
    OP_DOT_BB,        // S0 = (b,b)                                      [:3067-3074]
};

struct VecArgs {
    const double *bu, *bv;
    double *xu, *xv, *ru, *rv, *du, *dv, *qu, *qv, *zu, *zv;
    const double *Azu, *Azv;
};

template <int OP>
__global__ void __launch_bounds__(kBlock) k_vec(Geom g, VecArgs v, RedCtx rc) {
    if (rc.st->done) return;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    DD s0{0.0, 0.0};
    const double alpha = rc.st->alpha, beta = rc.st->beta;
    if (q < g.NQ) {
        int i, j;
        col_of(g, q, i, j);
        const bool own = owned(g, i, j);
        for (int k = 0; k < g.nz; ++k) {
            const long long e = (long long)k * g.NQ + q;
            if (OP == OP_STD_INIT) {
                v.ru[e] = __dsub_rn(v.bu[e], v.zu[e]);
                v.rv[e] = __dsub_rn(v.bv[e], v.zv[e]);
                v.du[e] = 0.0; v.dv[e] = 0.0;
                v.zu[e] = 0.0; v.zv[e] = 0.0;
                if (own) s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(v.bu[e], v.bu[e]), __dmul_rn(v.bv[e], v.bv[e])));
            } else if (OP == OP_DOT_BB) {
                if (own) s0 = dd_add_d(s0, __dadd_rn(__dmul_rn(v.bu[e], v.bu[e]), __dmul_rn(v.bv[e], v.bv[e])));
            } else if (OP == OP_STD_D) {
                v.du[e] = __dadd_rn(v.zu[e], __dmul_rn(beta, v.du[e]));
                v.dv[e] = __dadd_rn(v.zv[e], __dmul_rn(beta, v.dv[e]));
            } else if (OP == OP_XR) {
                v.xu[e] = __dadd_rn(v.xu[e], __dmul_rn(alpha, v.du[e]));
                v.xv[e] = __dadd_rn(v.xv[e], __dmul_rn(alpha, v.dv[e]));
                v.ru[e] = __dsub_rn(v.ru[e], __dmul_rn(alpha, v.qu[e]));
                v.rv[e] = __dsub_rn(v.rv[e], __dmul_rn(alpha, v.qv[e]));
            } else if (OP == OP_CG_INIT) {
                v.ru[e] = __dsub_rn(v.bu[e], v.zu[e]);
                v.rv[e] = __dsub_rn(v.bv[e], v.zv[e]);
            } else if (OP == OP_CG_UPD) {
                const double d1 = __dadd_rn(v.zu[e], __dmul_rn(beta, v.du[e]));
                const double d2 = __dadd_rn(v.zv[e], __dmul_rn(beta, v.dv[e]));
                const double q1 = __dadd_rn(v.Azu[e], __dmul_rn(beta, v.qu[e]));
                const double q2 = __dadd_rn(v.Azv[e], __dmul_rn(beta, v.qv[e]));
                v.du[e] = d1; v.dv[e] = d2;
                v.qu[e] = q1; v.qv[e] = q2;
                v.xu[e] = __dadd_rn(v.xu[e], __dmul_rn(alpha, d1));
                v.xv[e] = __dadd_rn(v.xv[e], __dmul_rn(alpha, d2));
                v.ru[e] = __dsub_rn(v.ru[e], __dmul_rn(alpha, q1));
                v.rv[e] = __dsub_rn(v.rv[e], __dmul_rn(alpha, q2));
            }
        }
    }
    if (OP == OP_STD_INIT || OP == OP_DOT_BB) reduce_and_finish<1>(rc, s0, s0);
}

// ---------------------------------------------------------------------------
// staggered halo on one rank (parallel_mpi.F90:10772-10936)
// ---------------------------------------------------------------------------
// Threads enumerate the ring columns: rows j in {0,1,NY-2,NY-1} (all i), then
// columns i in {0,1,NX-2,NX-1} for 2 <= j <= NY-3.  A periodic halo position
// (i in {0,1,NX-1} or j in {0,1,NY-1}) takes the value at (pi(i), pj(j)) with
// pi(0)=NX-3, pi(1)=NX-2, pi(NX-1)=2 (identity otherwise): the composite of the
// east-west exchange on owned rows followed by the north-south exchange on all
// columns.  Sources are never halo positions, so one pass is race free.  Outflow
// then zeroes i,j in {0, N-1}; no_ice zeroes i,j in {0,1,N-2,N-1}.  Levels k run over
// blockIdx.y, blockIdx.y + gridDim.y, ... (many planes, such as the 27 nz coefficient planes of
// a block, take a grid with several rows of blocks).
__device__ __forceinline__ int pmap(int i, int N) {
    if (i == 0) return N - 3;
    if (i == 1) return N - 2;
    if (i == N - 1) return 2;
    return i;
}

__global__ void __launch_bounds__(kBlock) k_halo(Geom g, double *__restrict__ au, double *__restrict__ av,
                                                 const SolveState *st) {
    if (st && st->done) return;
    const int NX = g.NX, NY = g.NY;
    const long long nring = 4LL * NX + 4LL * (NY - 4);
    const long long t = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (t >= nring) return;
    int i, j;
    if (t < 4LL * NX) {
        const int r = (int)(t / NX);
        i = (int)(t - (long long)r * NX);
        j = (r < 2) ? r : NY - 4 + r;  // 0,1,NY-2,NY-1
    } else {
        const long long u = t - 4LL * NX;
        const int r = (int)(u / (NY - 4));
        j = 2 + (int)(u - (long long)r * (NY - 4));
        i = (r < 2) ? r : NX - 4 + r;
    }
    bool zero = false;
    if (g.outflow) zero = (i == 0 || i == NX - 1 || j == 0 || j == NY - 1);
    else if (g.no_ice) zero = (i <= 1 || i >= NX - 2 || j <= 1 || j >= NY - 2);
    const long long q = (long long)j * NX + i;
    if (zero) {
        for (int k = blockIdx.y; k < g.nz; k += gridDim.y) {
            au[(long long)k * g.NQ + q] = 0.0;
            av[(long long)k * g.NQ + q] = 0.0;
        }
        return;
    }
    if (g.periodic) {
        const bool halo = (i <= 1 || i == NX - 1 || j <= 1 || j == NY - 1);
        if (!halo) return;
        const long long s = (long long)pmap(j, NY) * NX + pmap(i, NX);
        for (int k = blockIdx.y; k < g.nz; k += gridDim.y) {
            au[(long long)k * g.NQ + q] = au[(long long)k * g.NQ + s];
            av[(long long)k * g.NQ + q] = av[(long long)k * g.NQ + s];
        }
    }
}

// ---------------------------------------------------------------------------
// owned-vertex global sum of arr1 + arr2 (parallel_global_sum_stagger on one rank)
// ---------------------------------------------------------------------------
// FORTRAN_LAYOUT: element (k, q) at k + nz*q (the caller's arrays); otherwise k*NQ + q.
// Same tree as every solver reduction: column dd sums over k, block tree per chunk of
// 256 columns, chunk partials, fixed final tree by the last CTA (which also resets the
// ticket for the next use).
template <bool FORTRAN_LAYOUT>
__global__ void __launch_bounds__(kBlock) k_gsum(Geom g, const double *__restrict__ a1, const double *__restrict__ a2,
                                                 DD *partials, unsigned int *ticket, double *out) {
    __shared__ DD sm[8];
    __shared__ bool last;
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    DD acc{0.0, 0.0};
    if (q < g.NQ) {
        int i, j;
        j = (int)(q / g.NX);
        i = (int)(q - (long long)j * g.NX);
        if (owned(g, i, j))
            for (int k = 0; k < g.nz; ++k) {
                const long long e = FORTRAN_LAYOUT ? (long long)k + (long long)g.nz * q : (long long)k * g.NQ + q;
                acc = dd_add_d(acc, __dadd_rn(a1[e], a2[e]));
            }
    }
    DD b = block_tree(acc, sm);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = b;
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    DD a{0.0, 0.0};
    for (unsigned int c = threadIdx.x; c < gridDim.x; c += kBlock) {
        DD p;
        p.hi = __ldcg(&partials[c].hi);
        p.lo = __ldcg(&partials[c].lo);
        a = dd_add(a, p);
    }
    DD r = block_tree(a, sm);
    if (threadIdx.x == 0) {
        *ticket = 0u;
        *out = r.hi + r.lo;
    }
}

// ---------------------------------------------------------------------------
// layout conversion between the caller's Fortran arrays and device planes
// ---------------------------------------------------------------------------
// 3D block A(27,nz,NX,NY) raw -> planes [c][k][q]; canonical c reads m = indxA(c)
__global__ void k_perm_block3(Geom g, const double *__restrict__ raw, double *__restrict__ dst,
                              const int32_t *__restrict__ map27) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // Fortran order k + nz*q
    const long long n = (long long)g.nz * g.NQ;
    if (node >= n) return;
    const long long q = node / g.nz;
    const int k = (int)(node - q * g.nz);
    const double *src = raw + 27LL * node;
    for (int c = 0; c < 27; ++c) dst[(long long)c * n + (long long)k * g.NQ + q] = src[map27[c] - 1];
}

// 2D block A(NX,NY,9) raw (already planes) -> canonical planes
__global__ void k_perm_block2(Geom g, const double *__restrict__ raw, double *__restrict__ dst,
                              const int32_t *__restrict__ map9) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NQ) return;
    for (int c = 0; c < 9; ++c) dst[(long long)c * g.NQ + q] = raw[(long long)(map9[c] - 1) * g.NQ + q];
}

// vector (nz,NX,NY) Fortran <-> level-major planes
__global__ void k_vec_in(Geom g, const double *__restrict__ raw, double *__restrict__ dst) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)g.nz * g.NQ;
    if (node >= n) return;
    const long long q = node / g.nz;
    const int k = (int)(node - q * g.nz);
    dst[(long long)k * g.NQ + q] = raw[node];
}

__global__ void k_vec_out(Geom g, const double *__restrict__ src, double *__restrict__ raw) {
    const long long node = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)g.nz * g.NQ;
    if (node >= n) return;
    const long long q = node / g.nz;
    const int k = (int)(node - q * g.nz);
    raw[node] = src[(long long)k * g.NQ + q];
}

// Reproducible-sum solves (parallel%reprosum): the two product fields work2u = au*bu and
// work2v = av*bv of one parallel_global_sum_stagger call, written in the caller's layout
// (node k + nz*q) that the reproducible sum reads.  An owned node whose au*bu + av*bv is not
// finite is recorded in *flag (1 NaN, 2 +Inf, 4 -Inf) and its products are written as zero,
// so the integer expansion only ever sees finite summands; the host then returns the IEEE
// sum of the non-finite values instead.
__global__ void __launch_bounds__(kBlock) k_repro_products(Geom g, const double *__restrict__ au,
                                                           const double *__restrict__ bu,
                                                           const double *__restrict__ av,
                                                           const double *__restrict__ bv, double *__restrict__ o1,
                                                           double *__restrict__ o2, int *flag) {
    const long long q = (long long)blockIdx.x * kBlock + threadIdx.x;
    if (q >= g.NQ) return;
    int i, j;
    col_of(g, q, i, j);
    const bool own = owned(g, i, j);
    int f = 0;
    for (int k = 0; k < g.nz; ++k) {
        const long long e = (long long)k * g.NQ + q;
        double p1 = __dmul_rn(au[e], bu[e]);
        double p2 = __dmul_rn(av[e], bv[e]);
        if (own) {
            const double v = __dadd_rn(p1, p2);
            if (v != v) f |= 1;
            else if (v == __longlong_as_double(0x7ff0000000000000LL)) f |= 2;
            else if (v == __longlong_as_double(0xfff0000000000000LL)) f |= 4;
            if (!(v - v == 0.0)) { p1 = 0.0; p2 = 0.0; }
        }
        o1[(long long)k + (long long)g.nz * q] = p1;
        o2[(long long)k + (long long)g.nz * q] = p2;
    }
    if (f) atomicOr(flag, f);
}

// The scalar epilogue of a sum computed on the host side of the stream (the reproducible sum).
__global__ void k_epilogue_value(SolveState *st, int epi, int iter, double S0, double S1) {
    if (st->done) return;
    epilogue(st, epi, iter, S0, S1);
}

// ---------------------------------------------------------------------------
// Global sums in the reference's own order (parallel_global_sum_stagger without reprosum,
// parallel_mpi.F90:6770 (3D), :6637 (2D), nflds forms :7042 (3D), :6904 (2D)):
//   local_sum = local_sum + arr1(k,i,j) + arr2(k,i,j)
// over owned vertices, j outer, then i, then k, every addition rounded in turn, and the
// work arrays products rounded first (worku = ru*zu, ...).  A chain of dependent additions
// has no parallelism, so one thread adds while the other warps of the CTA stage the next
// chunk of summands in shared memory (two buffers).  With two fields (Chronopoulos-Gear's
// nflds = 2 calls) the two chains are independent and run interleaved in the same thread.
// ---------------------------------------------------------------------------
constexpr int kSeqChunk = 512;  // summands per term per chunk

struct SeqArgs {
    const double *a[2][2];  // field f: u term a[f][0], v term a[f][1]
    const double *b[2][2];  // and their second factors (null: the term is a itself)
};

// FLAYOUT: element (k, q) at k + nz*q (the caller's arrays); otherwise planes k*NQ + q.
// epi2 != EPI_NONE: the two sums finish two epilogues, epi with S0 then epi2 with S1 (the
// first pass of Chronopoulos-Gear); otherwise one epilogue epi(S0, S1).  out (optional)
// receives S0.  One CTA of kBlock threads.
template <int NF, bool FLAYOUT>
__global__ void __launch_bounds__(kBlock) k_seq_sum(Geom g, SeqArgs s, SolveState *st, int epi, int epi2, int iter,
                                                    double *out) {
    __shared__ double sm[2][NF][2][kSeqChunk];
    if (st && st->done) return;
    const long long W = (long long)(g.ihi - g.ilo + 1) * g.nz;  // summands of one owned row j
    const long long n = (long long)(g.jhi - g.jlo + 1) * W;
    const long long nchunk = (n + kSeqChunk - 1) / kSeqChunk;
    // stage chunk c into buffer buf with threads [t0, kBlock)
    auto stage = [&](long long c, int buf, int t0) {
        for (int t = threadIdx.x - t0; t < kSeqChunk; t += kBlock - t0) {
            const long long e = c * kSeqChunk + t;
            if (e >= n) break;
            const long long r = e / W, rem = e - r * W;
            const int i = g.ilo + (int)(rem / g.nz), k = (int)(rem % g.nz), j = g.jlo + (int)r;
            const long long q = (long long)j * g.NX + i;
            const long long x = FLAYOUT ? (long long)k + (long long)g.nz * q : (long long)k * g.NQ + q;
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    sm[buf][f][h][t] = s.b[f][h] ? __dmul_rn(s.a[f][h][x], s.b[f][h][x]) : s.a[f][h][x];
        }
    };
    double s0 = 0.0, s1 = 0.0;
    if (nchunk > 0) stage(0, 0, 0);
    __syncthreads();
    for (long long c = 0; c < nchunk; ++c) {
        const int buf = (int)(c & 1);
        if (threadIdx.x >= 32) {
            if (c + 1 < nchunk) stage(c + 1, buf ^ 1, 32);
        } else if (threadIdx.x == 0) {
            const int cnt = (int)min((long long)kSeqChunk, n - c * kSeqChunk);
            const double *u0 = sm[buf][0][0], *v0 = sm[buf][0][1];
            const double *u1 = sm[buf][NF - 1][0], *v1 = sm[buf][NF - 1][1];
#pragma unroll 8
            for (int t = 0; t < cnt; ++t) {
                s0 = __dadd_rn(__dadd_rn(s0, u0[t]), v0[t]);
                if (NF > 1) s1 = __dadd_rn(__dadd_rn(s1, u1[t]), v1[t]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (out) *out = s0;
        if (st) {
            if (epi2 != EPI_NONE) {
                epilogue(st, epi, iter, s0, 0.0);
                if (!st->done) epilogue(st, epi2, iter, s1, 0.0);
            } else {
                epilogue(st, epi, iter, s0, s1);
            }
        }
    }
}

__global__ void k_init_state(SolveState *st, double tol, int maxiters) {
    st->eta0 = 1.0; st->eta1 = 0.0; st->eta2 = 0.0; st->alpha = 0.0; st->beta = 0.0;
    st->rho_old = 0.0; st->sigma = 0.0; st->rho = 0.0; st->delta = 0.0;
    st->L2_rhs = 0.0;
    st->err = __longlong_as_double(0x7ff8000000000000LL);  // NaN until the first check
    st->tol = tol;
    st->done = 0; st->status = 0; st->niters = maxiters; st->checks = 0;
    for (int t = 0; t < 4; ++t) st->ticket[t] = 0u;
}

}  // namespace cismgpu
