// pcg_mixed.cu -- mixed-precision, batched, persistent Chronopoulos-Gear PCG on B200.
//
// Algorithm (per solve): the Chronopoulos-Gear recurrences of
// pcg_solver_chrongear_* (glissade_velo_higher_pcg.F90:3296-3581) with the
// matrix, z, d, q, Az and the recursive residual r stored and multiplied in FP32,
// the solution x accumulated in FP64, every dot product accumulated in FP64
// double-double, and the reference's periodic residual replacement
// (:3482-3579) done in FP64: at every check iteration r = b - A x is computed
// with the FP64 matrix, the FP64 norm gives err, and the FP32 recurrences
// continue from the true residual (a "reliable update": the Krylov directions
// are kept, so the iteration count stays close to FP64 CG while the bulk of the
// traffic moves half the bytes).
//
// Execution: one cooperative persistent kernel runs any number of independent
// solves (a batch, or the slots of the serving loop).  The owned vertices of each
// solve are cut into tiles of TX x TY columns; a CTA processes tiles round robin.
// Per step a tile computes, for its columns and a one-column halo ring, the
// pointwise update of iteration i and the preconditioner of iteration i+1 (the
// halo values are recomputed from the previous step's vectors, which is why r, q
// and Az are double buffered), then the FP32 stencil product of iteration i+1 and
// the tile's partial dot products.  The last CTA to finish a solve's tiles in a
// step reduces that solve's partials with a fixed tree and advances the solve's
// state machine, so every solve needs exactly one grid barrier per iteration and
// its results do not depend on which CTA ran which tile or on what else is in the
// batch.  Grid barriers spin with a clock64 limit and report CISMGPU_ETIMEOUT.
#pragma once

#include "common.cuh"

namespace cismgpu {

constexpr int kTX = 32, kTY = 8;                 // tile of columns (one thread per column)
constexpr int kSlots = (kTX + 2) * (kTY + 2);    // tile + one-column halo ring
constexpr int kMixedMaxNz = 32;                  // shared-memory bound of the mixed kernel (levels)

enum MStep { MS_INIT = 0, MS_A, MS_MERGED, MS_B, MS_CHECK, MS_DONE };

// device-visible description of one solve
struct MDesc {
    Geom g;
    int NC;          // 27 (3D) or 9 (2D)
    int precond;     // 0 none, 1 diag, 2 sia
    int tiles_x, tiles_y, ntiles;
    const float *A32;    // [4][NC][nz][NQ]
    const double *A64;   // [4][NC][nz][NQ]
    const float *pre;    // diag: [2][nz][NQ] inverse diagonal; sia: [2][3][nz][NQ] (1/beta, sb, gamma)
    const int32_t *act;  // [NQ]
    const double *b;     // [2][nz][NQ]
    double *x;           // [2][nz][NQ]
    float *r[2], *q[2], *Az[2];  // [2][nz][NQ] each (u, v planes)
    float *z, *d;                // [2][nz][NQ]
    DD *partials;        // [ntiles][3]
};

struct MState {
    double alpha, beta, rho_old, sigma, L2_rhs, err, tol;
    double rr_inner;     // (r,r) of the recursive FP32 residual, for diagnostics
    int step, iter, par;
    int maxiters, ncheck;
    int done, status, niters;
    int checks, fp32_matvecs, fp64_matvecs;
    unsigned ticket;
};

struct MTile { int solve, tile; };

struct GridBar {
    unsigned count;
    unsigned gen;
    int abort;          // set on a barrier timeout; every CTA leaves at its next wait
    int n_active;       // solves not yet done
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool zero_pos(const Geom &g, int i, int j) {
    if (g.outflow) return i == 0 || i == g.NX - 1 || j == 0 || j == g.NY - 1;
    if (g.no_ice) return i <= 1 || i >= g.NX - 2 || j <= 1 || j >= g.NY - 2;
    return false;
}

// Map a vertex position to the owned position whose value it holds after the
// staggered halo update; returns -1 for positions that hold zero or lie outside
// the array.
__device__ __forceinline__ long long src_col(const Geom &g, int i, int j) {
    if (i < 0 || i >= g.NX || j < 0 || j >= g.NY) return -1;
    if (zero_pos(g, i, j)) return -1;
    if (g.periodic) {
        const bool halo = (i <= 1 || i == g.NX - 1 || j <= 1 || j == g.NY - 1);
        if (halo) {
            i = pmap(i, g.NX);
            j = pmap(j, g.NY);
        }
    }
    if (!owned(g, i, j)) return -1;
    return (long long)j * g.NX + i;
}

// The FP32 unknowns: owned, active, and not forced to zero by the boundary condition.
__device__ __forceinline__ bool live_col(const MDesc &D, int i, int j, long long q) {
    return owned(D.g, i, j) && D.act[q] != 0 && !zero_pos(D.g, i, j);
}

__device__ bool grid_barrier(GridBar *bar, unsigned nblocks) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned *vgen = &bar->gen;
        volatile int *vabort = &bar->abort;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar->count, 1u);
        if (arrived == nblocks - 1) {
            bar->count = 0u;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*vgen == gen) {
                if (*vabort) { ok = 0; break; }
                if (clock64() - t0 > (1LL << 32)) {  // ~2 s at 2 GHz: give up, report
                    atomicExch(&bar->abort, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__device__ __forceinline__ bool is_check_it(int iter, int ncheck) { return (iter % ncheck == 0) || iter == 5; }

// ---------------------------------------------------------------------------
// per-solve state machine, run by the last CTA of a step (thread 0)
// ---------------------------------------------------------------------------
__device__ void advance_state(MState &S, const MDesc &D, double S0, double S1, double S2) {
    switch (S.step) {
    case MS_INIT:  // S0 = (b,b), S1 = (r,r) of r = b - A x0
        S.L2_rhs = sqrt(S0);
        S.err = sqrt(S1) / S.L2_rhs;
        S.fp64_matvecs += 1;
        S.iter = 1;
        if (S.maxiters < 1) {
            S.niters = 0;
            S.done = 1;
            S.step = MS_DONE;
        } else {
            S.step = MS_A;
        }
        break;
    case MS_A:       // S0 = (r,z), S1 = (Az,z) of iteration iter
    case MS_MERGED: {
        if (S.step == MS_MERGED) {  // the merged step finished iteration iter's update: advance
            S.par ^= 1;
            S.iter += 1;
        }
        S.fp32_matvecs += 1;
        const bool first = (S.iter == 1);
        const double rho = S0, delta = S1;
        S.rr_inner = S2;
        S.beta = first ? 0.0 : rho / S.rho_old;
        S.sigma = first ? delta : delta - S.beta * rho / S.alpha;
        S.alpha = rho / S.sigma;
        S.rho_old = rho;
        if (S.alpha != S.alpha) {
            S.status = CISMGPU_EBREAKDOWN_ALPHA;
            S.done = 1;
            S.niters = S.iter;
            S.step = MS_DONE;
            break;
        }
        // iteration iter's update comes next: alone if a check or the last iteration follows
        S.step = (is_check_it(S.iter, S.ncheck) || S.iter >= S.maxiters) ? MS_B : MS_MERGED;
        break;
    }
    case MS_B:
        S.par ^= 1;
        if (is_check_it(S.iter, S.ncheck)) {
            S.step = MS_CHECK;
        } else {  // last iteration without a check
            S.niters = S.maxiters;
            S.done = 1;
            S.step = MS_DONE;
        }
        break;
    case MS_CHECK:  // S0 = (r,r) of the FP64 true residual
        S.checks += 1;
        S.fp64_matvecs += 1;
        S.err = sqrt(S0) / S.L2_rhs;
        if (S.err < S.tol) {
            S.niters = S.iter;
            S.done = 1;
            S.step = MS_DONE;
        } else if (S.iter >= S.maxiters) {
            S.niters = S.maxiters;
            S.done = 1;
            S.step = MS_DONE;
        } else {
            S.iter += 1;
            S.step = MS_A;
        }
        break;
    default:
        break;
    }
}

// ---------------------------------------------------------------------------
// tile work
// ---------------------------------------------------------------------------
template <int NZM>
struct MShared {
    float z[2][NZM][kSlots];       // preconditioned residual on tile + halo
    float rt[2][NZM][kTX * kTY];   // new residual on the tile columns
    DD red[8];
    bool last;
};

// Loads of data that other CTAs wrote earlier in the same launch go through L2
// (ld.global.cg): L1 is not coherent across SMs.
__device__ __forceinline__ float ldf(const float *p) { return __ldcg(p); }
__device__ __forceinline__ double ldd(const double *p) { return __ldcg(p); }

__device__ __forceinline__ MState load_state(const MState *p) {
    MState s;
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(p);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s);
#pragma unroll
    for (int w = 0; w < (int)(sizeof(MState) / 8); ++w) dst[w] = __ldcg(src + w);
    return s;
}

// z = M^-1 r on one column, in place in smem (s = slot), FP32.
template <int NZM>
__device__ __forceinline__ void precond_col(const MDesc &D, float (*zc)[NZM][kSlots], int s, long long q) {
    const int nz = D.g.nz;
    const long long plane = (long long)nz * D.g.NQ;
    for (int c = 0; c < 2; ++c) {
        float (*z)[kSlots] = zc[c];
        if (D.precond == 1) {
            const float *inv = D.pre + c * plane;
            for (int k = 0; k < nz; ++k) z[k][s] = z[k][s] * inv[(long long)k * D.g.NQ + q];
        } else if (D.precond == 2) {
            const float *ib = D.pre + (c * 3 + 0) * plane, *sb = D.pre + (c * 3 + 1) * plane,
                        *gm = D.pre + (c * 3 + 2) * plane;
            // forward: y_1 = r_1/beta_1; y_k = (r_k - sb_k y_{k-1})/beta_k ; back: z_k = y_k - gamma_{k+1} z_{k+1}
            float prev = z[0][s] * ib[q];
            z[0][s] = prev;
            for (int k = 1; k < nz; ++k) {
                const long long e = (long long)k * D.g.NQ + q;
                prev = (z[k][s] - sb[e] * prev) * ib[e];
                z[k][s] = prev;
            }
            for (int k = nz - 2; k >= 0; --k)
                z[k][s] = z[k][s] - gm[(long long)(k + 1) * D.g.NQ + q] * z[k + 1][s];
        }
        // precond 0: z = r
    }
}

// One tile of one solve for the solve's current step.  Returns the three partials.
template <int NC, int NZM>
__device__ void tile_step(const MDesc &D, const MState &S, int tile, MShared<NZM> &sh, DD &p0, DD &p1, DD &p2) {
    const Geom &g = D.g;
    const int nz = g.nz;
    const long long NQ = g.NQ;
    const long long plane = (long long)nz * NQ;
    const int tx = tile % D.tiles_x, ty = tile / D.tiles_x;
    const int i0 = g.ilo + tx * kTX, j0 = g.jlo + ty * kTY;
    const int t = threadIdx.x;
    const int step = S.step;
    const int par = S.par;
    p0 = p1 = p2 = DD{0.0, 0.0};

    if (step == MS_INIT || step == MS_CHECK) {
        // r = b - A64 x (FP64, x read through the halo map); r32 = r on live columns
        const int ti = t % kTX, tj = t / kTX;
        const int i = i0 + ti, j = j0 + tj;
        if (i <= g.ihi && j <= g.jhi) {
            const long long q = (long long)j * g.NX + i;
            const bool on = D.act[q] != 0;
            const bool live = live_col(D, i, j, q);
            const double *Auu = D.A64, *Auv = D.A64 + NC * plane, *Avu = D.A64 + 2 * NC * plane,
                         *Avv = D.A64 + 3 * NC * plane;
            const double *xu = D.x, *xv = D.x + plane;
            for (int k = 0; k < nz; ++k) {
                const long long e = (long long)k * NQ + q;
                double yu = 0.0, yv = 0.0;
                if (on) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
                        if (k + kA < 0 || k + kA >= nz) continue;
                        const long long sc = src_col(g, i + iA, j + jA);
                        if (sc < 0) continue;
                        const long long n = (long long)(k + kA) * NQ + sc;
                        const long long a = (long long)c * plane + e;
                        const double x1 = ldd(xu + n), x2 = ldd(xv + n);
                        yu = fma(Auu[a], x1, yu);
                        yu = fma(Auv[a], x2, yu);
                        yv = fma(Avu[a], x1, yv);
                        yv = fma(Avv[a], x2, yv);
                    }
                }
                const double ru = D.b[e] - yu, rv = D.b[plane + e] - yv;
                p1 = dd_add_d(p1, ru * ru + rv * rv);
                if (step == MS_INIT) p0 = dd_add_d(p0, D.b[e] * D.b[e] + D.b[plane + e] * D.b[plane + e]);
                else p0 = p1;
                D.r[par][e] = live ? (float)ru : 0.0f;
                D.r[par][plane + e] = live ? (float)rv : 0.0f;
            }
        }
        if (step == MS_CHECK) { p0 = p1; p1 = DD{0.0, 0.0}; }
        return;
    }

    const float alpha = (float)S.alpha, beta = (float)S.beta;
    const bool do_b = (step == MS_MERGED || step == MS_B);
    const bool do_a = (step == MS_MERGED || step == MS_A);
    const int rin = par, rout = do_b ? (par ^ 1) : par;  // buffers holding r_i / r_{i+1}

    // ---- pass 1: update (B) on the tile, new residual and z on tile + halo ----
    for (int s = t; s < kSlots; s += blockDim.x) {
        const int li = s % (kTX + 2), lj = s / (kTX + 2);
        const int i = i0 - 1 + li, j = j0 - 1 + lj;
        const bool interior = li >= 1 && li <= kTX && lj >= 1 && lj <= kTY;
        long long m = src_col(g, i, j);
        const bool mine = interior && m >= 0 && owned(g, i, j) && m == (long long)j * g.NX + i;
        bool live = false;
        if (m >= 0) {
            const int mi = (int)(m % g.NX), mj = (int)(m / g.NX);
            live = live_col(D, mi, mj, m);
        }
        if (!live) {
            for (int k = 0; k < nz; ++k) { sh.z[0][k][s] = 0.0f; sh.z[1][k][s] = 0.0f; }
            if (mine && do_b) {  // keep dead columns at zero
                for (int k = 0; k < nz; ++k)
                    for (int c = 0; c < 2; ++c) {
                        const long long e = c * plane + (long long)k * NQ + m;
                        D.q[rout][e] = 0.0f;
                        D.r[rout][e] = 0.0f;
                    }
            }
            if (interior && do_a) {
                const int it = (li - 1) + kTX * (lj - 1);
                for (int k = 0; k < nz; ++k) { sh.rt[0][k][it] = 0.0f; sh.rt[1][k][it] = 0.0f; }
            }
            continue;
        }
        for (int c = 0; c < 2; ++c) {
            for (int k = 0; k < nz; ++k) {
                const long long e = c * plane + (long long)k * NQ + m;
                float rn;
                if (do_b) {
                    const float qn = fmaf(beta, ldf(D.q[rin] + e), ldf(D.Az[rin] + e));  // q_i = Az_i + beta q_{i-1}
                    rn = fmaf(-alpha, qn, ldf(D.r[rin] + e));                          // r_{i+1} = r_i - alpha q_i
                    if (mine) {
                        const float dn = fmaf(beta, D.d[e], D.z[e]);           // d_i = z_i + beta d_{i-1}
                        D.d[e] = dn;
                        D.q[rout][e] = qn;
                        D.r[rout][e] = rn;
                        D.x[e] = fma(S.alpha, (double)dn, D.x[e]);            // x += alpha d_i (FP64)
                    }
                } else {
                    rn = ldf(D.r[rin] + e);
                }
                sh.z[c][k][s] = rn;
                if (interior && do_a) sh.rt[c][k][(li - 1) + kTX * (lj - 1)] = rn;
            }
        }
        if (do_a) precond_col<NZM>(D, sh.z, s, m);
    }
    if (!do_a) return;
    __syncthreads();

    // ---- pass 2: Az = A z on the tile columns, partial dots ----
    {
        const int ti = t % kTX, tj = t / kTX;
        const int i = i0 + ti, j = j0 + tj;
        const int s = (ti + 1) + (kTX + 2) * (tj + 1);
        const int it = ti + kTX * tj;
        if (t < kTX * kTY && i <= g.ihi && j <= g.jhi) {
            const long long q = (long long)j * g.NX + i;
            const bool live = live_col(D, i, j, q);
            const float *Auu = D.A32, *Auv = D.A32 + NC * plane, *Avu = D.A32 + 2 * NC * plane,
                        *Avv = D.A32 + 3 * NC * plane;
            float *Azu = D.Az[rout], *Azv = D.Az[rout] + plane;
            for (int k = 0; k < nz; ++k) {
                const long long e = (long long)k * NQ + q;
                float yu = 0.0f, yv = 0.0f;
                if (live) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
                        const int kk = k + kA;
                        if (kk < 0 || kk >= nz) continue;
                        const int sn = s + iA + (kTX + 2) * jA;
                        const float zu = sh.z[0][kk][sn], zv = sh.z[1][kk][sn];
                        const long long a = (long long)c * plane + e;
                        yu = fmaf(Auu[a], zu, yu);
                        yu = fmaf(Auv[a], zv, yu);
                        yv = fmaf(Avu[a], zu, yv);
                        yv = fmaf(Avv[a], zv, yv);
                    }
                }
                Azu[e] = yu;
                Azv[e] = yv;
                const double zu = sh.z[0][k][s], zv = sh.z[1][k][s];
                D.z[e] = (float)zu;
                D.z[plane + e] = (float)zv;
                const double ru = sh.rt[0][k][it], rv = sh.rt[1][k][it];
                p0 = dd_add_d(p0, ru * zu + rv * zv);
                p1 = dd_add_d(p1, (double)yu * zu + (double)yv * zv);
                p2 = dd_add_d(p2, ru * ru + rv * rv);
            }
        }
    }
}

template <int NC, int NZM>
__global__ void __launch_bounds__(kBlock) k_mixed(const MDesc *__restrict__ descs, MState *states,
                                                  const MTile *__restrict__ tiles, int ntiles, GridBar *bar,
                                                  int max_steps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MShared<NZM> &sh = *reinterpret_cast<MShared<NZM> *>(smem_raw);
    for (int step = 0; step < max_steps; ++step) {
        if (((volatile GridBar *)bar)->n_active <= 0) break;
        for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
            const MTile T = tiles[w];
            const MDesc &D = descs[T.solve];
            MState *Sp = &states[T.solve];
            const MState S = load_state(Sp);
            if (S.done || S.step == MS_DONE) continue;
            DD p0, p1, p2;
            tile_step<NC, NZM>(D, S, T.tile, sh, p0, p1, p2);
            DD b0 = block_tree(p0, sh.red);
            DD b1 = block_tree(p1, sh.red);
            DD b2 = block_tree(p2, sh.red);
            if (threadIdx.x == 0) {
                D.partials[3 * T.tile + 0] = b0;
                D.partials[3 * T.tile + 1] = b1;
                D.partials[3 * T.tile + 2] = b2;
                __threadfence();
                const unsigned tk = atomicAdd(&Sp->ticket, 1u);
                sh.last = (tk == (unsigned)D.ntiles - 1);
            }
            __syncthreads();
            if (sh.last) {
                __threadfence();
                DD a0{0.0, 0.0}, a1{0.0, 0.0}, a2{0.0, 0.0};
                for (int c = threadIdx.x; c < D.ntiles; c += kBlock) {
                    DD v0, v1, v2;
                    v0.hi = __ldcg(&D.partials[3 * c].hi); v0.lo = __ldcg(&D.partials[3 * c].lo);
                    v1.hi = __ldcg(&D.partials[3 * c + 1].hi); v1.lo = __ldcg(&D.partials[3 * c + 1].lo);
                    v2.hi = __ldcg(&D.partials[3 * c + 2].hi); v2.lo = __ldcg(&D.partials[3 * c + 2].lo);
                    a0 = dd_add(a0, v0);
                    a1 = dd_add(a1, v1);
                    a2 = dd_add(a2, v2);
                }
                DD r0 = block_tree(a0, sh.red);
                DD r1 = block_tree(a1, sh.red);
                DD r2 = block_tree(a2, sh.red);
                if (threadIdx.x == 0) {
                    MState NS = load_state(Sp);
                    NS.ticket = 0u;
                    advance_state(NS, D, r0.hi + r0.lo, r1.hi + r1.lo, r2.hi + r2.lo);
                    *Sp = NS;
                    if (NS.done) atomicSub(&bar->n_active, 1);
                    __threadfence();
                }
            }
            __syncthreads();
        }
        if (!grid_barrier(bar, gridDim.x)) return;
    }
}

// ---------------------------------------------------------------------------
// setup kernels: FP32 matrix copy and FP32 preconditioner factors
// ---------------------------------------------------------------------------
__global__ void k_to_f32(const double *__restrict__ src, float *__restrict__ dst, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        dst[e] = (float)src[e];
}

// diag: inverse of the diagonal coefficient (0 where the diagonal is 0), per component
// sia : Thomas factors of the column tridiagonal (0,0,-1)/(0,0,0)/(0,0,+1) couplings
template <int NC>
__global__ void k_mixed_precond_setup(Geom g, int precond, const double *__restrict__ A64, float *__restrict__ pre) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NQ) return;
    const long long plane = (long long)g.nz * g.NQ;
    const int cd = (NC == 27) ? 13 : 4;
    for (int c = 0; c < 2; ++c) {
        const double *Ab = A64 + (c == 0 ? 0 : 3) * NC * plane;  // Auu or Avv
        if (precond == 1) {
            for (int k = 0; k < g.nz; ++k) {
                const long long e = (long long)k * g.NQ + q;
                const double a = Ab[(long long)cd * plane + e];
                pre[c * plane + e] = (a != 0.0) ? (float)(1.0 / a) : 0.0f;
            }
        } else if (precond == 2 && NC == 27) {
            float *ib = pre + (c * 3 + 0) * plane, *sb = pre + (c * 3 + 1) * plane, *gm = pre + (c * 3 + 2) * plane;
            double beta = Ab[13 * plane + q];
            ib[q] = (float)(1.0 / beta);
            sb[q] = 0.0f;
            gm[q] = 0.0f;
            for (int k = 1; k < g.nz; ++k) {
                const long long e = (long long)k * g.NQ + q;
                const double sp_prev = Ab[22 * plane + (long long)(k - 1) * g.NQ + q];
                const double s = Ab[4 * plane + e];
                const double gam = sp_prev / beta;
                beta = Ab[13 * plane + e] - s * gam;
                ib[e] = (float)(1.0 / beta);
                sb[e] = (float)s;
                gm[e] = (float)gam;
            }
        }
    }
}

// Device buffers of the mixed solver for one system (owned by the host Solver).
struct MixedBufs {
    bool valid = false;
    int precond = -1;
    float *A32 = nullptr, *pre = nullptr, *vec = nullptr;
    DD *partials = nullptr;
    MState *state = nullptr;
    MDesc *desc = nullptr;
    MTile *tiles = nullptr;
    GridBar *bar = nullptr;
    size_t nbytes = 0;
    int ntiles = 0;
    void release() {
        for (void *p : {(void *)A32, (void *)pre, (void *)vec, (void *)partials, (void *)state, (void *)desc,
                        (void *)tiles, (void *)bar})
            if (p) cudaFree(p);
        A32 = pre = vec = nullptr;
        partials = nullptr;
        state = nullptr;
        desc = nullptr;
        tiles = nullptr;
        bar = nullptr;
        nbytes = 0;
        valid = false;
        precond = -1;
    }
    size_t bytes() const { return nbytes; }
};

}  // namespace cismgpu
