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
    DD *partials;        // [ntiles][2 step parities][3]
    const int *maps;     // [ntiles][(TX+2)*(TY+2)] slot maps (k_slot_maps)
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
// Tile shapes: one CTA of 256 threads per tile.  2D: 64 x 16 columns (4 per thread);
// 3D: 32 x 8 columns with nz levels each.
template <int NC> struct TileShape;
template <> struct TileShape<9> { static constexpr int TX = 64, TY = 16; };
template <> struct TileShape<27> { static constexpr int TX = 32, TY = 8; };

constexpr int kMaxCtaSolves = 32;  // distinct solves whose tiles one CTA may hold in a launch

template <int NC, int NZM>
struct MShared {
    static constexpr int TX = TileShape<NC>::TX, TY = TileShape<NC>::TY;
    static constexpr int NS = (TX + 2) * (TY + 2), NT = TX * TY;
    static constexpr int KP = (NC == 27) ? NZM + 2 : 1;  // z levels with a zero row above and below
    float z[2][KP][NS];        // preconditioned residual on tile + halo
    float rt[2][NZM][NT];      // new residual on the tile columns
    int map[NS];               // slot map of the current tile (k_slot_maps)
    MDesc D;                   // descriptor of the current tile's solve
    MState st[kMaxCtaSolves];  // this CTA's copy of the state of every solve it holds
    int sid[kMaxCtaSolves];    // solve index of each cached state
    int owner[kMaxCtaSolves];  // 1 if this CTA holds tile 0 of the solve (reports it)
    int nsolve;
    int cur;                   // cache slot described by D
    DD red[8][3];
};

// Loads of data that other CTAs wrote earlier in the same launch go through L2
// (ld.global.cg): L1 is not coherent across SMs.
__device__ __forceinline__ float ldf(const float *p) { return __ldcg(p); }
__device__ __forceinline__ double ldd(const double *p) { return __ldcg(p); }

// Block tree over 256 threads for three dd fields at once; result in thread 0.
__device__ __forceinline__ void block_tree3(DD &a, DD &b, DD &c, DD (*sm)[3]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        DD oa = dd_shfl_down(a, off), ob = dd_shfl_down(b, off), oc = dd_shfl_down(c, off);
        if (lane + off < 32) { a = dd_add(a, oa); b = dd_add(b, ob); c = dd_add(c, oc); }
    }
    __syncthreads();
    if (lane == 0) { sm[warp][0] = a; sm[warp][1] = b; sm[warp][2] = c; }
    __syncthreads();
    if (warp == 0) {
        const DD z0{0.0, 0.0};
        a = lane < 8 ? sm[lane][0] : z0;
        b = lane < 8 ? sm[lane][1] : z0;
        c = lane < 8 ? sm[lane][2] : z0;
#pragma unroll
        for (int off = 4; off >= 1; off >>= 1) {
            DD oa = dd_shfl_down(a, off), ob = dd_shfl_down(b, off), oc = dd_shfl_down(c, off);
            if (lane + off < 32) { a = dd_add(a, oa); b = dd_add(b, ob); c = dd_add(c, oc); }
        }
    }
}

// Slot map entry: (halo source column + 1) << 2 | live | mine << 1.  Source -1 means the
// slot holds zero (zero boundary condition or outside the array).
__device__ __forceinline__ int map_src(int v) { return (v >> 2) - 1; }
__device__ __forceinline__ bool map_live(int v) { return (v & 1) != 0; }
__device__ __forceinline__ bool map_mine(int v) { return (v & 2) != 0; }

template <int TX, int TY>
__global__ void k_slot_maps(MDesc D, int *maps) {
    constexpr int NS = (TX + 2) * (TY + 2);
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)D.ntiles * NS) return;
    const int tile = (int)(id / NS), sl = (int)(id % NS);
    const Geom &g = D.g;
    const int tx = tile % D.tiles_x, ty = tile / D.tiles_x;
    const int i0 = g.ilo + tx * TX, j0 = g.jlo + ty * TY;
    const int li = sl % (TX + 2), lj = sl / (TX + 2);
    const int i = i0 - 1 + li, j = j0 - 1 + lj;
    const long long m = src_col(g, i, j);
    int v = (int)(m + 1) << 2;
    if (m >= 0) {
        const int mi = (int)(m % g.NX), mj = (int)(m / g.NX);
        const bool live = live_col(D, mi, mj, m);
        const bool interior = li >= 1 && li <= TX && lj >= 1 && lj <= TY;
        if (live) v |= 1;
        if (live && interior && m == (long long)j * g.NX + i) v |= 2;
    }
    maps[id] = v;
}

// z = M^-1 r on one column of the SIA tridiagonal, in place in smem (slot s), FP32.
// The column's factors are loaded in one batch first: a load inside the recurrence
// would cost one memory round trip per level.
template <int KP, int NS, int NZM>
__device__ __forceinline__ void sia_col(const MDesc &D, float (*zc)[KP][NS], int s, long long q) {
    const int nz = D.g.nz;
    const long long NQ = D.g.NQ;
    const long long plane = (long long)nz * NQ;
    for (int c = 0; c < 2; ++c) {
        float (*z)[NS] = zc[c] + 1;  // level k is row k+1 (rows 0 and nz+1 are zero padding)
        const float *ib = D.pre + (c * 3 + 0) * plane, *sb = D.pre + (c * 3 + 1) * plane,
                    *gm = D.pre + (c * 3 + 2) * plane;
        float fib[NZM], fsb[NZM], fgm[NZM];
#pragma unroll
        for (int k = 0; k < NZM; ++k) {
            const bool in = k < nz;
            fib[k] = in ? __ldg(ib + (long long)k * NQ + q) : 0.0f;
            fsb[k] = in ? __ldg(sb + (long long)k * NQ + q) : 0.0f;
            fgm[k] = in ? __ldg(gm + (long long)k * NQ + q) : 0.0f;
        }
        // forward: y_1 = r_1/beta_1; y_k = (r_k - sb_k y_{k-1})/beta_k; back: z_k = y_k - gamma_{k+1} z_{k+1}
        float prev = z[0][s] * fib[0];
        z[0][s] = prev;
#pragma unroll
        for (int k = 1; k < NZM; ++k) {
            if (k < nz) {
                prev = (z[k][s] - fsb[k] * prev) * fib[k];
                z[k][s] = prev;
            }
        }
        float next = z[nz - 1][s];
#pragma unroll
        for (int k = NZM - 2; k >= 0; --k) {
            if (k < nz - 1) {
                next = z[k][s] - fgm[k + 1] * next;
                z[k][s] = next;
            }
        }
    }
}

// One tile of one solve for the solve's current step; writes the tile's partials.
template <int NC, int NZM>
__device__ void tile_step(const MState &S, int tile, int pbuf, MShared<NC, NZM> &sh) {
    using SH = MShared<NC, NZM>;
    constexpr int TX = SH::TX, TY = SH::TY, NS = SH::NS, NT = SH::NT, KP = SH::KP;
    constexpr int OFF = (NC == 27) ? 1 : 0;  // z row of level 0
    const MDesc &D = sh.D;
    const Geom &g = D.g;
    const int nz = (NC == 27) ? g.nz : 1;
    const long long NQ = g.NQ;
    const long long plane = (long long)nz * NQ;
    const int tx = tile % D.tiles_x, ty = tile / D.tiles_x;
    const int i0 = g.ilo + tx * TX, j0 = g.jlo + ty * TY;
    const int t = threadIdx.x;
    const int step = S.step;
    const int par = S.par;
    DD p0{0.0, 0.0}, p1{0.0, 0.0}, p2{0.0, 0.0};

    const int *tmap = D.maps + (long long)tile * NS;
    for (int sl = t; sl < NS; sl += kBlock) sh.map[sl] = tmap[sl];
    __syncthreads();

    if (step == MS_INIT || step == MS_CHECK) {
        // r = b - A64 x (FP64, x read through the halo map); r32 = r on live columns
        const double *Auu = D.A64, *Auv = D.A64 + NC * plane, *Avu = D.A64 + 2 * NC * plane,
                     *Avv = D.A64 + 3 * NC * plane;
        const double *xu = D.x, *xv = D.x + plane;
        for (int it = t; it < NT; it += kBlock) {
            const int ti = it % TX, tj = it / TX;
            const int i = i0 + ti, j = j0 + tj;
            if (i > g.ihi || j > g.jhi) continue;
            const long long q = (long long)j * g.NX + i;
            const int s = (ti + 1) + (TX + 2) * (tj + 1);
            const bool on = D.act[q] != 0;
            const bool live = map_live(sh.map[s]);
            int nb[9];
#pragma unroll
            for (int h = 0; h < 9; ++h) nb[h] = map_src(sh.map[s + (h % 3 - 1) + (TX + 2) * (h / 3 - 1)]);
            for (int k = 0; k < nz; ++k) {
                const long long e = (long long)k * NQ + q;
                double yu = 0.0, yv = 0.0;
                if (on) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const int kA = (NC == 27) ? c / 9 - 1 : 0;
                        const int sc = nb[c % 9];
                        if (k + kA < 0 || k + kA >= nz || sc < 0) continue;
                        const long long n = (long long)(k + kA) * NQ + sc;
                        const long long a = (long long)c * plane + e;
                        const double x1 = ldd(xu + n), x2 = ldd(xv + n);
                        yu = fma(Auu[a], x1, yu);
                        yu = fma(Auv[a], x2, yu);
                        yv = fma(Avu[a], x1, yv);
                        yv = fma(Avv[a], x2, yv);
                    }
                }
                const double bu = D.b[e], bv = D.b[plane + e];
                const double ru = bu - yu, rv = bv - yv;
                p1 = dd_add_d(p1, ru * ru + rv * rv);
                if (step == MS_INIT) p0 = dd_add_d(p0, bu * bu + bv * bv);
                D.r[par][e] = live ? (float)ru : 0.0f;
                D.r[par][plane + e] = live ? (float)rv : 0.0f;
            }
        }
        if (step == MS_CHECK) { p0 = p1; p1 = DD{0.0, 0.0}; }
    } else {
        const float alpha = (float)S.alpha, beta = (float)S.beta;
        const double alpha64 = S.alpha;
        const bool do_b = (step == MS_MERGED || step == MS_B);
        const bool do_a = (step == MS_MERGED || step == MS_A);
        const int rin = par, rout = do_b ? (par ^ 1) : par;  // buffers holding r_i / r_{i+1}

        // ---- pass 1: update (B) on the tile, new residual (and diag z) on tile + halo ----
        constexpr int P1 = (2 * NS + kBlock - 1) / kBlock;  // items per thread and level
        for (int k = 0; k < nz; ++k) {
#pragma unroll
            for (int r = 0; r < P1; ++r) {
                const int it = t + r * kBlock;
                if (it >= 2 * NS) break;
                const int c = it / NS, sl = it - c * NS;
                const int v = sh.map[sl];
                const int m = map_live(v) ? map_src(v) : -1;
                float rn = 0.0f;
                if (m >= 0) {
                    const long long e = c * plane + (long long)k * NQ + m;
                    if (do_b) {
                        const float qo = ldf(D.q[rin] + e), az = ldf(D.Az[rin] + e), ro = ldf(D.r[rin] + e);
                        const float qn = fmaf(beta, qo, az);  // q_i = Az_i + beta q_{i-1}
                        rn = fmaf(-alpha, qn, ro);             // r_{i+1} = r_i - alpha q_i
                        if (map_mine(v)) {
                            const float dn = fmaf(beta, D.d[e], D.z[e]);  // d_i = z_i + beta d_{i-1}
                            D.d[e] = dn;
                            D.q[rout][e] = qn;
                            D.r[rout][e] = rn;
                            D.x[e] = fma(alpha64, (double)dn, D.x[e]);  // x += alpha d_i (FP64)
                        }
                    } else {
                        rn = ldf(D.r[rin] + e);
                    }
                }
                if (do_a) {
                    const int li = sl % (TX + 2), lj = sl / (TX + 2);
                    if (li >= 1 && li <= TX && lj >= 1 && lj <= TY) sh.rt[c][k][(li - 1) + TX * (lj - 1)] = rn;
                    float zv = rn;
                    if (D.precond == 1 && m >= 0) zv = rn * D.pre[c * plane + (long long)k * NQ + m];
                    sh.z[c][k + OFF][sl] = zv;
                }
            }
        }
        if (do_a) {
            if (NC == 27) {  // zero padding rows (levels -1 and nz)
                for (int it = t; it < 2 * NS; it += kBlock) {
                    const int c = it / NS, sl = it - c * NS;
                    sh.z[c][0][sl] = 0.0f;
                    sh.z[c][nz + 1][sl] = 0.0f;
                }
            }
            __syncthreads();
            if (NC == 27 && D.precond == 2) {  // column tridiagonal solves on tile + halo
                for (int sl = t; sl < NS; sl += kBlock) {
                    const int v = sh.map[sl];
                    if (map_live(v)) sia_col<KP, NS, NZM>(D, sh.z, sl, map_src(v));
                }
                __syncthreads();
            }

            // ---- pass 2: Az = A z on the tile columns, z to HBM, partial dots ----
            // Couplings that leave the grid are zero in the FP32 copy and the padded z rows
            // and out-of-grid halo slots are zero, so every column sums all NC terms.
            const float *Auu = D.A32, *Auv = D.A32 + NC * plane, *Avu = D.A32 + 2 * NC * plane,
                        *Avv = D.A32 + 3 * NC * plane;
            float *Azu = D.Az[rout], *Azv = D.Az[rout] + plane;
#pragma unroll
            for (int r = 0; r < NT / kBlock; ++r) {
                const int it = t + r * kBlock;
                const int ti = it % TX, tj = it / TX;
                const int i = i0 + ti, j = j0 + tj;
                if (i > g.ihi || j > g.jhi) continue;
                const int s = (ti + 1) + (TX + 2) * (tj + 1);
                const long long q = (long long)j * g.NX + i;
                const bool live = map_live(sh.map[s]);
                for (int k = 0; k < nz; ++k) {
                    const long long e = (long long)k * NQ + q;
                    float yu = 0.0f, yv = 0.0f;
                    if (live) {
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
                            const int sn = s + iA + (TX + 2) * jA;
                            const float zu = sh.z[0][k + OFF + kA][sn], zv = sh.z[1][k + OFF + kA][sn];
                            const long long a = (long long)c * plane + e;
                            yu = fmaf(__ldg(Auu + a), zu, yu);
                            yu = fmaf(__ldg(Auv + a), zv, yu);
                            yv = fmaf(__ldg(Avu + a), zu, yv);
                            yv = fmaf(__ldg(Avv + a), zv, yv);
                        }
                    }
                    Azu[e] = yu;
                    Azv[e] = yv;
                    const float zu = sh.z[0][k + OFF][s], zv = sh.z[1][k + OFF][s];
                    D.z[e] = zu;
                    D.z[plane + e] = zv;
                    const double ru = sh.rt[0][k][it], rv = sh.rt[1][k][it];
                    p0 = dd_add_d(p0, ru * (double)zu + rv * (double)zv);
                    p1 = dd_add_d(p1, (double)yu * zu + (double)yv * zv);
                    p2 = dd_add_d(p2, ru * ru + rv * rv);
                }
            }
        }
    }
    block_tree3(p0, p1, p2, sh.red);
    if (t == 0) {
        DD *pp = D.partials + ((long long)tile * 2 + pbuf) * 3;
        pp[0] = p0;
        pp[1] = p1;
        pp[2] = p2;
    }
    __syncthreads();
}

// Reduce the partials (buffer pbuf) of every running solve this CTA holds and advance
// its cached state.  Every CTA holding a solve does this with the same inputs and the
// same fixed tree, so all copies of a solve's state stay bit-identical.  The CTA holding
// tile 0 publishes a finished solve and decrements n_active before its next barrier.
template <int NC, int NZM>
__device__ void reduce_cached(MShared<NC, NZM> &sh, const MDesc *__restrict__ descs, int pbuf, MState *gstates,
                              GridBar *bar) {
    for (int cs = 0; cs < sh.nsolve; ++cs) {
        if (sh.st[cs].done) continue;
        const MDesc &D = descs[sh.sid[cs]];
        const int ntl = D.ntiles;
        const DD *P = D.partials;
        DD a0{0.0, 0.0}, a1{0.0, 0.0}, a2{0.0, 0.0};
        for (int c = threadIdx.x; c < ntl; c += kBlock) {
            const DD *pp = P + ((long long)c * 2 + pbuf) * 3;
            DD v0, v1, v2;
            v0.hi = __ldcg(&pp[0].hi); v0.lo = __ldcg(&pp[0].lo);
            v1.hi = __ldcg(&pp[1].hi); v1.lo = __ldcg(&pp[1].lo);
            v2.hi = __ldcg(&pp[2].hi); v2.lo = __ldcg(&pp[2].lo);
            a0 = dd_add(a0, v0);
            a1 = dd_add(a1, v1);
            a2 = dd_add(a2, v2);
        }
        block_tree3(a0, a1, a2, sh.red);
        if (threadIdx.x == 0) {
            MState &S = sh.st[cs];
            advance_state(S, D, a0.hi + a0.lo, a1.hi + a1.lo, a2.hi + a2.lo);
            if (S.done && sh.owner[cs]) {
                gstates[sh.sid[cs]] = S;
                __threadfence();
                atomicSub(&bar->n_active, 1);
            }
        }
        __syncthreads();
    }
}

template <int NC, int NZM>
__global__ void __launch_bounds__(kBlock, 2) k_mixed(const MDesc *__restrict__ descs, MState *states,
                                                     const MTile *__restrict__ tiles, int ntiles, GridBar *bar,
                                                     int max_steps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MShared<NC, NZM> &sh = *reinterpret_cast<MShared<NC, NZM> *>(smem_raw);
    // cache the states of the solves this CTA holds (round robin over the tile list)
    if (threadIdx.x == 0) {
        int n = 0;
        for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
            const MTile T = tiles[w];
            int u = 0;
            while (u < n && sh.sid[u] != T.solve) ++u;
            if (u == n && n < kMaxCtaSolves) {
                sh.sid[n] = T.solve;
                sh.owner[n] = 0;
                const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&states[T.solve]);
                unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sh.st[n]);
                for (int w8 = 0; w8 < (int)(sizeof(MState) / 8); ++w8) dst[w8] = __ldcg(src + w8);
                ++n;
            }
            if (u < n && T.tile == 0) sh.owner[u] = 1;
        }
        sh.nsolve = n;
        sh.cur = -1;
    }
    __syncthreads();
    bool finished = false;
    int step = 0;
    for (; step < max_steps; ++step) {
        const int pbuf = step & 1;
        if (step > 0) reduce_cached<NC, NZM>(sh, descs, pbuf ^ 1, states, bar);  // previous step's sums
        for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
            const MTile T = tiles[w];
            int cs = 0;
            while (cs < sh.nsolve && sh.sid[cs] != T.solve) ++cs;
            if (cs >= sh.nsolve || sh.st[cs].done) continue;
            if (sh.cur != cs) {
                __syncthreads();
                if (threadIdx.x == 0) {
                    sh.D = descs[T.solve];
                    sh.cur = cs;
                }
                __syncthreads();
            }
            tile_step<NC, NZM>(sh.st[cs], T.tile, pbuf, sh);
        }
        if (!grid_barrier(bar, gridDim.x)) return;
        if (((volatile GridBar *)bar)->n_active <= 0) {
            finished = true;
            break;
        }
    }
    // out of steps: fold in the last step's sums so that the next launch resumes exactly
    if (!finished && step > 0) reduce_cached<NC, NZM>(sh, descs, (step - 1) & 1, states, bar);
    if (threadIdx.x == 0)
        for (int cs = 0; cs < sh.nsolve; ++cs)
            if (sh.owner[cs]) states[sh.sid[cs]] = sh.st[cs];
}

// ---------------------------------------------------------------------------
// setup kernels: FP32 matrix copy and FP32 preconditioner factors
// ---------------------------------------------------------------------------
// FP32 copy of the coefficient planes; couplings whose neighbour lies outside the
// array (which the reference skips) are stored as zero so the FP32 stencil loop needs
// no bounds tests.
template <int NC>
__global__ void k_to_f32(Geom g, const double *__restrict__ src, float *__restrict__ dst) {
    const long long plane = (long long)g.nz * g.NQ;
    const long long n = 4LL * NC * plane;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)((e / plane) % NC);
        const long long r = e % plane;
        const int k = (int)(r / g.NQ);
        const long long q = r % g.NQ;
        const int i = (int)(q % g.NX), j = (int)(q / g.NX);
        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
        const bool in = i + iA >= 0 && i + iA < g.NX && j + jA >= 0 && j + jA < g.NY && k + kA >= 0 && k + kA < g.nz;
        dst[e] = in ? (float)src[e] : 0.0f;
    }
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
    bool stale = false;        // the FP64 matrix changed since the FP32 copy was made
    long long shape_nvec = 0;
    int shape_nc = 0;
    int precond = -1;
    float *A32 = nullptr, *pre = nullptr, *vec = nullptr;
    int *maps = nullptr;
    DD *partials = nullptr;
    MState *state = nullptr;
    MDesc *desc = nullptr;
    MTile *tiles = nullptr;
    GridBar *bar = nullptr;
    size_t nbytes = 0;
    int ntiles = 0;
    void release() {
        for (void *p : {(void *)A32, (void *)pre, (void *)vec, (void *)partials, (void *)state, (void *)desc,
                        (void *)tiles, (void *)bar, (void *)maps})
            if (p) cudaFree(p);
        A32 = pre = vec = nullptr;
        maps = nullptr;
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
