// pcg_mixed.cu -- mixed-precision, batched, persistent Chronopoulos-Gear PCG on B200.
//
// Algorithm (per solve): the Chronopoulos-Gear recurrences of
// pcg_solver_chrongear_* (glissade_velo_higher_pcg.F90:3296-3581) with the
// matrix, z, d, q, Az and the recursive residual r stored and multiplied in FP32,
// the solution x accumulated in FP64, every dot product accumulated in FP64
// (within and across tiles, in one fixed order), and the reference's periodic residual replacement
// (:3482-3579) done in FP64: at every check iteration r = b - A x is computed
// with the FP64 matrix, the FP64 norm gives err, and the FP32 recurrences
// continue from the true residual (a "reliable update": the Krylov directions
// are kept, so the iteration count stays close to FP64 CG while the bulk of the
// traffic moves half the bytes).
//
// Execution: one cooperative persistent kernel runs any number of independent
// solves (a batch, or the slots of the serving loop).  The owned vertices of each
// solve are cut into tiles of kTX x TY columns (TY fixed per solve); a CTA
// processes tiles round robin.  Per step a tile computes, for its columns and a
// one-column halo ring, the pointwise update of iteration i and the
// preconditioner of iteration i+1 (the halo values are recomputed from the
// previous step's vectors, which is why r, q and Az are double buffered), then the
// FP32 stencil product of iteration i+1 and the tile's partial dot products, and
// publishes them in a record stamped with the solve's step number.  There is no
// grid barrier: before its next step every CTA holding a tile of a solve waits
// for all of that solve's records of the step, and sums them in one fixed order,
// so all CTAs advance identical copies of the solve's scalars, a solve never waits
// for another solve, and its results do not depend on which CTA ran which tile or
// on what else is in the launch.  Every wait is bounded (clock64) and reports
// CISMGPU_ETIMEOUT.
#pragma once

#include "common.cuh"

namespace cismgpu {

constexpr int kMixedMaxNz = 32;                  // shared-memory bound of the mixed kernel (levels)

// Step kinds.  A check iteration ends with one MS_BC step (update and FP64 residual
// replacement together); the owners' in-place d and x writes of that update are deferred
// to the next step (MS_A_UPD, or MS_FIN when the solve stops there), so that no tile reads
// a neighbour's half-updated d or x while it recomputes the halo of x.
// The tridiagonal line preconditioners (precond 3, 4) need the whole domain's residual before any
// line is solved, so an iteration takes three steps: MS_UPD (the update alone, the tile's line
// right-hand sides), MS_LINES (the line solves) and MS_A / MS_A_UPD (the preconditioner, which reads
// the line solution, then the stencil product and the dots).
enum MStep { MS_INIT = 0, MS_A, MS_MERGED, MS_B, MS_CHECK_UNUSED, MS_DONE, MS_BC, MS_A_UPD, MS_FIN, MS_UPD, MS_LINES };

// A tile's partial sums of one step (two sums).  Every 64-bit word carries the step number
// (tag) in its high half and one 32-bit half of a sum in its low half (w[2i] low, w[2i+1]
// high half of sum i), so a reader that finds the tag in all four words has the step's values, with
// relaxed loads and no fence.  The words are stored after a release fence, so an acquire
// load of a word also orders the tile's vector stores of the step before the reader's
// later loads (the halo).  Each tile writes kRecCopies copies ([copy][tile][parity]); a CTA
// reads copy blockIdx % kRecCopies, so the all-to-all reads of a step spread over more L2
// lines.
struct __align__(64) TileRec {
    unsigned long long w[4];
    unsigned long long pad[4];
};
constexpr int kRecCopies = 4;
constexpr size_t kStreamBytes = 32u << 20;  // FP32 matrix size above which L2 cannot keep a solve's matrix
constexpr int kNbrMax = 8;     // tiles whose columns one tile's halo reads (else: fence)
constexpr int kNbrStride = kNbrMax + 1;  // [count or -1, tiles...] per tile

// The scalars a solve's leader broadcasts after summing a step's records (dynamic launches):
// word = tag << 32 | done << 9 | par << 8 | step, written last.  Replicated kBcastCopies
// times, one 256-byte line each, so that polls spread over several L2 slices.
struct __align__(256) Bcast {
    unsigned long long word;
    double alpha, beta;
    double pad[29];
};
constexpr int kBcastCopies = 8;

// device-visible description of one solve
struct MDesc {
    Geom g;
    int NC;          // 27 (3D) or 9 (2D)
    int precond;     // 0 none, 1 diag, 2 sia
    int TY;          // tile height of this solve
    int tiles_x, tiles_y, ntiles;
    const float4 *A32;   // [NC][nz][NQ] of (uu, uv, vu, vv): one 16-byte load per coupling
    const double *A64;   // [4][NC][nz][NQ]
    const double2 *A64i; // [NC][nz][NQ][2] of {uu, uv}, {vu, vv} for streamed matrices (else null): the FP64
                         // residual's two 16-byte loads per coupling
    const float *pre;    // diag: [2][nz][NQ] inverse diagonal; sia: [2][3][nz][NQ] (1/beta, sb, gamma)
    const int32_t *act;  // [NQ]
    const double *b;     // [2][nz][NQ]
    double *x;           // [2][nz][NQ]
    float *r[2], *q[2], *Az[2];  // [2][nz][NQ] each (u, v planes)
    float *z, *d;                // [2][nz][NQ]
    TileRec *recs;       // [kRecCopies][ntiles][2 step parities]
    Bcast *bc;           // [2 step parities][kBcastCopies] (dynamic launches)
    int *dflag;          // set once the solve is done (dynamic launches)
    const int *maps;     // [ntiles][(kTX+2)*(TY+2)] slot maps (k_slot_maps)
    const int *nbrs;     // [ntiles][kNbrStride] tiles owning the tile's live halo columns (k_tile_nbrs)
    int stream;          // matrix loads evict-first (the FP32 matrix exceeds kStreamBytes)
    int sym;             // 3D, exactly symmetric: A32 and A64i hold the symmetric half (k_to_half)
    // precond 3, 4: FP32 line factors [u, v][sub, 1/diag, omega, 1/denom][NQ], the lines' right-hand
    // sides rs and solution zs [u, v][NQ]; u planes transposed (column i, row j at i*NY + j) so that
    // the u lines, one per owned row, load and store coalesced
    const float *tri;
    float *rs, *zs;
};

struct MState {
    double alpha, beta, rho_old, sigma, L2_rhs, err, tol;
    int step, iter, par;
    int maxiters, ncheck;
    int done, status, niters;
    int checks, fp32_matvecs, fp64_matvecs;
    unsigned tick;       // steps completed (the tag of the last records summed)
    int tri;             // precond 3, 4: iterations take the MS_UPD, MS_LINES steps
    int after;           // the step that follows MS_LINES
};

struct MTile { int solve, tile; };

struct MCtl {
    int abort;                 // set on a wait timeout; every CTA leaves at its next wait
    int active;                // dynamic launches: solves not yet done
    unsigned long long next;   // dynamic launches: work counter (step * ntiles + tile list position)
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

__device__ __forceinline__ bool is_check_it(int iter, int ncheck) { return (iter % ncheck == 0) || iter == 5; }

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned *p, unsigned v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Bulk copies global -> shared memory (the copy engine, no registers in flight) completing on
// an mbarrier in the CTA's shared memory.  Addresses 16-byte aligned, sizes multiples of 16.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *m, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *m, unsigned bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(m)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *m, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_u32(m)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// The four words of a record, as two 16-byte relaxed loads (each 64-bit element is a
// single-copy-atomic access).
__device__ __forceinline__ void ld_rec(const TileRec *rp, unsigned long long (&w)[4]) {
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w[0]), "=l"(w[1]) : "l"(rp->w) : "memory");
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w[2]), "=l"(w[3]) : "l"(rp->w + 2) : "memory");
}
__device__ __forceinline__ int ld_acquire_i(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr long long kWaitCycles = 1LL << 31;  // ~1 s at 2 GHz: a wait longer than this is a failure
// The wait bound every spin-wait below uses (kWaitCycles unless a test shortened it), and a
// test hook: with c_withhold_tag != 0, tile 0 of every solve does not publish its record of
// that step, so the waits for it run out (a flag nothing sets) and the launch ends with
// CISMGPU_ETIMEOUT.  Both are set by cismgpu_test_set_device_waits; 0 restores the defaults.
__constant__ long long c_wait_cycles = kWaitCycles;
__constant__ unsigned c_withhold_tag = 0u;

// ---------------------------------------------------------------------------
// per-solve state machine, run by thread 0 of every CTA holding the solve
// ---------------------------------------------------------------------------
__device__ void advance_state(MState &S, double S0, double S1) {
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
            S.step = S.tri ? MS_LINES : MS_A;
            S.after = MS_A;
        }
        break;
    case MS_A:       // S0 = (r,z), S1 = (Az,z) of iteration iter
    case MS_A_UPD:
    case MS_MERGED: {
        if (S.step == MS_MERGED) {  // the merged step finished iteration iter's update: advance
            S.par ^= 1;
            S.iter += 1;
        }
        S.fp32_matvecs += 1;
        const bool first = (S.iter == 1);
        const double rho = S0, delta = S1;
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
        // iteration iter's update comes next: with the FP64 check at check iterations, alone
        // at the last iteration, merged with the next iteration's first half otherwise
        S.step = is_check_it(S.iter, S.ncheck) ? MS_BC
                 : (S.iter >= S.maxiters ? MS_B : (S.tri ? MS_UPD : MS_MERGED));
        break;
    }
    case MS_UPD:  // line preconditioners: iteration iter's update, then the lines of iter + 1
        S.par ^= 1;
        S.iter += 1;
        S.step = MS_LINES;
        S.after = MS_A;
        break;
    case MS_LINES:
        S.step = S.after;
        break;
    case MS_B:  // last iteration without a check
        S.par ^= 1;
        S.niters = S.maxiters;
        S.done = 1;
        S.step = MS_DONE;
        break;
    case MS_BC:  // S0 = (r,r) of the FP64 true residual after iteration iter's update
        S.par ^= 1;
        S.checks += 1;
        S.fp64_matvecs += 1;
        S.err = sqrt(S0) / S.L2_rhs;
        if (S.err < S.tol) {
            S.niters = S.iter;
            S.step = MS_FIN;
        } else if (S.iter >= S.maxiters) {
            S.niters = S.maxiters;
            S.step = MS_FIN;
        } else {
            S.iter += 1;
            S.step = S.tri ? MS_LINES : MS_A_UPD;
            S.after = MS_A_UPD;
        }
        break;
    case MS_FIN:  // the deferred x and d writes are done
        S.done = 1;
        S.step = MS_DONE;
        break;
    default:
        break;
    }
}

// ---------------------------------------------------------------------------
// tile work
// ---------------------------------------------------------------------------
// Tiles are kTX columns wide (one warp per tile row: coalesced 128-byte FP32 rows) and
// TY rows high; TY is chosen per solve by the host (mixed_solve_ty).
constexpr int kTX = 32;
constexpr int kMaxCtaSolves = 64;  // distinct solves whose tiles one CTA may hold in a launch
constexpr int kMaxTY = 64;
constexpr int kMaxAcq = 32;        // neighbour tiles a CTA acquires per step (4 tiles x 8)
constexpr int kTilesCached = 16;   // tile list entries a CTA keeps in shared memory
constexpr int kCh2 = 4;            // stencil items per load batch
constexpr int kChR = 4;            // FP64 residual items per load batch

struct MHead {
    MDesc D;                   // descriptor of the current tile's solve
    MState st[kMaxCtaSolves];  // this CTA's copy of the state of every solve it holds
    int sid[kMaxCtaSolves];    // solve index of each cached state
    int owner[kMaxCtaSolves];  // 1 if this CTA holds tile 0 of the solve (reports it)
    int nsolve;
    int cur;                   // cache slot described by D
    double red[8][2];
    double rsum[8][2];
    unsigned long long mbar;   // resident launches: completion of the matrix's bulk copies
    int nacq;                  // >= 0: the CTA reads the halo of acq[0..nacq) only; -1: fence
    int acq[kMaxAcq];
    int ntl;                   // static launches: tile list entries of this CTA
    MTile tl[kTilesCached];    // the first kTilesCached of them
};

// Dynamic shared memory: head | map[NS] | z[2][KP][NS] | rt[2][NZM][NT]
//                        | (resident launches) A[4][NC][NZM*NT] FP32 matrix of the CTA's tile
// sized for the launch's largest tile height.
template <int NC, int NZM>
struct MLayout {
    static constexpr int KP = (NC == 27) ? NZM + 2 : 1;  // z levels with a zero row above and below
    int NS, NT;
    bool resA;
    __host__ __device__ MLayout(int TY, bool resident) : NS((kTX + 2) * (TY + 2)), NT(kTX * TY), resA(resident) {}
    __host__ __device__ size_t off_map() const { return (sizeof(MHead) + 15) / 16 * 16; }
    __host__ __device__ size_t off_z() const { return (off_map() + 4 * (size_t)NS + 15) / 16 * 16; }
    __host__ __device__ size_t off_rt() const { return off_z() + 4 * (size_t)2 * KP * NS; }
    __host__ __device__ size_t off_A() const { return (off_rt() + 4 * (size_t)2 * NZM * NT + 15) / 16 * 16; }
    // 3D FP64 check steps (up to 16 levels): x (updated by the step's d) of the tile and its halo
    // ring, all levels with a zero row above and below, [2][KP][NS] doubles over the z and rt regions
    __host__ __device__ size_t off_x64() const { return off_z(); }
    __host__ __device__ size_t bytes() const {
        size_t b = off_A() + (resA ? 4 * (size_t)4 * NC * NZM * NT : 0);
        if (NC == 27 && NZM <= 16) {  // (32 levels keep the per-coupling residual_pass: the tile
                                      // would halve their occupancy)
            const size_t bx = off_x64() + 8 * (size_t)2 * KP * NS;
            if (bx > b) b = bx;
        }
        return b;
    }
};

// Matrix loads (read-only for the launch) carry an L2 policy: evict-first for a solve whose
// matrix streams through L2 every step (larger than L2 can keep), so that it does not push
// out the vectors the next pass reads; evict-normal for one L2 can keep between steps.
__device__ __forceinline__ unsigned long long l2_matrix_policy(bool stream) {
    unsigned long long pol;
    if (stream) asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    else asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float4 ld_stream(const float4 *p, unsigned long long pol) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_stream(const double *p, unsigned long long pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ld_stream(const double2 *p, unsigned long long pol) {
    double2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
        : "=d"(v.x), "=d"(v.y)
        : "l"(p), "l"(pol));
    return v;
}

// Loads of the symmetric half copy: every stored coupling is read twice in a step, by its
// node and by its transpose partner's node, close together in time.
__device__ __forceinline__ float4 ld_half(const float4 *p, unsigned long long pol) { return ld_stream(p, pol); }
__device__ __forceinline__ double2 ld_half(const double2 *p, unsigned long long pol) { return ld_stream(p, pol); }

// Loads of data that other CTAs wrote earlier in the same launch go through L2
// (ld.global.cg): L1 is not coherent across SMs.
__device__ __forceinline__ float ldf(const float *p) { return __ldcg(p); }
__device__ __forceinline__ double ldd(const double *p) { return __ldcg(p); }

// Sum of two doubles over the 256 threads in a fixed order (warp shuffle tree, then the
// 8 warp sums in order); result in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b, double (*sm)[2]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    __syncthreads();
    if (lane == 0) { sm[warp][0] = a; sm[warp][1] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = sm[0][0]; b = sm[0][1];
#pragma unroll
        for (int w = 1; w < kBlock / 32; ++w) { a += sm[w][0]; b += sm[w][1]; }
    }
}

// Slot map entry: (halo source column + 1) << 2 | live | mine << 1.  Source -1 means the
// slot holds zero (zero boundary condition or outside the array).
__device__ __forceinline__ int map_src(int v) { return (v >> 2) - 1; }
__device__ __forceinline__ bool map_live(int v) { return (v & 1) != 0; }
__device__ __forceinline__ bool map_mine(int v) { return (v & 2) != 0; }

__global__ void k_slot_maps(MDesc D, int *maps) {
    const int TY = D.TY;
    const int NS = (kTX + 2) * (TY + 2);
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)D.ntiles * NS) return;
    const int tile = (int)(id / NS), sl = (int)(id % NS);
    const Geom &g = D.g;
    const int tx = tile % D.tiles_x, ty = tile / D.tiles_x;
    const int i0 = g.ilo + tx * kTX, j0 = g.jlo + ty * TY;
    const int li = sl % (kTX + 2), lj = sl / (kTX + 2);
    const int i = i0 - 1 + li, j = j0 - 1 + lj;
    const long long m = src_col(g, i, j);
    int v = (int)(m + 1) << 2;
    if (m >= 0) {
        const int mi = (int)(m % g.NX), mj = (int)(m / g.NX);
        const bool live = live_col(D, mi, mj, m);
        const bool interior = li >= 1 && li <= kTX && lj >= 1 && lj <= TY;
        if (live) v |= 1;
        if (live && interior && m == (long long)j * g.NX + i) v |= 2;
    }
    maps[id] = v;
}

// For each tile, the other tiles owning a live column its halo slots read ([count, tiles]),
// or count -1 if there are more than kNbrMax (the readers then fence instead).
__global__ void k_tile_nbrs(MDesc D, const int *maps, int *nbrs) {
    const int tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= D.ntiles) return;
    const Geom &g = D.g;
    const int NS = (kTX + 2) * (D.TY + 2);
    int list[kNbrMax];
    int n = 0;
    bool over = false;
    for (int sl = 0; sl < NS && !over; ++sl) {
        const int v = maps[(size_t)tile * NS + sl];
        if (!map_live(v)) continue;
        const int m = map_src(v);
        const int mi = m % g.NX, mj = m / g.NX;
        const int ot = ((mj - g.jlo) / D.TY) * D.tiles_x + (mi - g.ilo) / kTX;
        if (ot == tile) continue;
        bool seen = false;
        for (int k = 0; k < n; ++k) seen |= (list[k] == ot);
        if (seen) continue;
        if (n == kNbrMax) over = true;
        else list[n++] = ot;
    }
    int *out = nbrs + (size_t)tile * kNbrStride;
    out[0] = over ? -1 : n;
    for (int k = 0; k < n; ++k) out[1 + k] = list[k];
}

// z = M^-1 r on one column of the SIA tridiagonal, in place in smem (zc = z[c][0][0],
// row stride NS; level k at row k+1), FP32.  The column's factors are loaded in one
// batch first: a load inside the recurrence would cost a memory round trip per level.
template <int NZM>
__device__ __forceinline__ void sia_col(const MDesc &D, float *zc, int NS, int s, int q, int c0, int c1) {
    const int nz = D.g.nz;
    const int NQ = (int)D.g.NQ;
    const int plane = nz * NQ;
    constexpr int KP = NZM + 2;
    for (int c = c0; c <= c1; ++c) {
        float *z = zc + c * KP * NS + NS + s;  // z[k * NS] is level k
        const float *ib = D.pre + (c * 3 + 0) * plane, *sb = D.pre + (c * 3 + 1) * plane,
                    *gm = D.pre + (c * 3 + 2) * plane;
        float fib[NZM], fsb[NZM], fgm[NZM];
#pragma unroll
        for (int k = 0; k < NZM; ++k) {
            const bool in = k < nz;
            fib[k] = in ? __ldg(ib + k * NQ + q) : 0.0f;
            fsb[k] = in ? __ldg(sb + k * NQ + q) : 0.0f;
            fgm[k] = in ? __ldg(gm + k * NQ + q) : 0.0f;
        }
        // forward: y_1 = r_1/beta_1; y_k = (r_k - sb_k y_{k-1})/beta_k; back: z_k = y_k - gamma_{k+1} z_{k+1}
        if (NZM <= 16) {
            // the column in registers: its shared-memory loads issue together, and the recurrences
            // wait on arithmetic alone (the same operations in the same order as below)
            float zz[NZM];
#pragma unroll
            for (int k = 0; k < NZM; ++k) zz[k] = (k < nz) ? z[k * NS] : 0.0f;
            float prev = zz[0] * fib[0];
            zz[0] = prev;
#pragma unroll
            for (int k = 1; k < NZM; ++k)
                if (k < nz) {
                    prev = (zz[k] - fsb[k] * prev) * fib[k];
                    zz[k] = prev;
                }
            float next = prev;
#pragma unroll
            for (int k = NZM - 2; k >= 0; --k)
                if (k < nz - 1) {
                    next = zz[k] - fgm[k + 1] * next;
                    zz[k] = next;
                }
#pragma unroll
            for (int k = 0; k < NZM; ++k)
                if (k < nz) z[k * NS] = zz[k];
        } else {
            float prev = z[0] * fib[0];
            z[0] = prev;
#pragma unroll
            for (int k = 1; k < NZM; ++k)
                if (k < nz) {
                    prev = (z[k * NS] - fsb[k] * prev) * fib[k];
                    z[k * NS] = prev;
                }
            float next = prev;
#pragma unroll
            for (int k = NZM - 2; k >= 0; --k)
                if (k < nz - 1) {
                    next = z[k * NS] - fgm[k + 1] * next;
                    z[k * NS] = next;
                }
        }
    }
}

// FP64 r = b - A64 x on the tile (x read through the halo map); r32 = r on live columns,
// into buffer rpar.  With sdn (the MS_BC step) the x of every tile and halo slot is first
// advanced by this iteration's update, x + alpha64 * dn with dn = sdn[c][k][slot] -- the same
// FP64 fma its owner applies later, so the residual sees exactly the updated x.
// Partials: p0 = (b,b), p1 = (r,r).  Loads of kChR items are issued before any store.
// IL: read the interleaved FP64 copy (solves whose matrix streams through L2; a matrix L2
// keeps between checks reads faster from the four planes).  HALF (3D, D.sym): the interleaved
// copy holds the symmetric half only; a lower coupling is read from its transpose partner.
// The coefficients are the same numbers in either layout, so the result is too.
template <int NC, bool IL, bool HALF = false>
__device__ __forceinline__ void residual_pass(const MDesc &D, const int *smap, int TY, int i0, int j0, int rpar,
                                              const float *sdn, double alpha64, double &p0, double &p1) {
    const Geom &g = D.g;
    const int nz = (NC == 27) ? g.nz : 1;
    const int NQ = (int)g.NQ;
    const int plane = nz * NQ;
    const int NT = kTX * TY;
    const double2 *__restrict__ A2 = D.A64i;
    const double *__restrict__ Auu = D.A64;
    const double *__restrict__ Auv = D.A64 + (size_t)NC * plane;
    const double *__restrict__ Avu = D.A64 + (size_t)2 * NC * plane;
    const double *__restrict__ Avv = D.A64 + (size_t)3 * NC * plane;
    const double *__restrict__ xu = D.x;
    const double *__restrict__ xv = D.x + plane;
    float *__restrict__ ru32 = D.r[rpar];
    float *__restrict__ rv32 = D.r[rpar] + plane;
    const int NS = (kTX + 2) * (TY + 2);
    const int nitems = NT * nz;
    const unsigned long long pol = l2_matrix_policy(D.stream != 0);
#pragma unroll 1
    for (int base = threadIdx.x; base < nitems; base += kChR * kBlock) {
        double yu[kChR], yv[kChR], bu[kChR], bv[kChR];
        int ee[kChR];
        bool ok[kChR], lv[kChR];
#pragma unroll
        for (int u = 0; u < kChR; ++u) {
            const int it = base + u * kBlock;
            yu[u] = 0.0; yv[u] = 0.0; bu[u] = 0.0; bv[u] = 0.0;
            ee[u] = 0; ok[u] = false; lv[u] = false;
            if (it < nitems) {
                const int col = it % NT, k = it / NT;
                const int ti = col % kTX, tj = col / kTX;
                const int i = i0 + ti, j = j0 + tj;
                if (i <= g.ihi && j <= g.jhi) {
                    const int q = j * g.NX + i;
                    const int s = (ti + 1) + (kTX + 2) * (tj + 1);
                    const int e = k * NQ + q;
                    ok[u] = true;
                    ee[u] = e;
                    lv[u] = map_live(smap[s]);
                    bu[u] = D.b[e];
                    bv[u] = D.b[plane + e];
                    if (D.act[q] != 0) {
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
                            const int sn = s + iA + (kTX + 2) * jA;
                            const int sc = map_src(smap[sn]);
                            if (k + kA < 0 || k + kA >= nz || sc < 0) continue;
                            const int n = (k + kA) * NQ + sc;
                            const size_t a = (size_t)c * plane + e;
                            // x is not written during this step (owner writes are deferred) and the step
                            // starts after the acquire of the tiles' records and a barrier: plain
                            // loads, so the neighbour reuse of x hits in L1
                            double x1 = xu[n], x2 = xv[n];
                            if (sdn) {
                                x1 = fma(alpha64, (double)sdn[(k + kA) * NS + sn], x1);
                                x2 = fma(alpha64, (double)sdn[(nz + k + kA) * NS + sn], x2);
                            }
                            if (HALF) {
                                double2 au, av;
                                if (c >= 13) {
                                    const size_t h = (size_t)(c - 13) * plane + e;
                                    au = ld_half(A2 + 2 * h, pol);
                                    av = ld_half(A2 + 2 * h + 1, pol);
                                } else {  // partner n = (k+kA, i+iA, j+jA), coupling 26 - c, blocks swapped
                                    const size_t h = (size_t)(13 - c) * plane + (size_t)(k + kA) * NQ +
                                                     (size_t)((j + jA) * g.NX + (i + iA));
                                    const double2 pu = ld_half(A2 + 2 * h, pol), pv = ld_half(A2 + 2 * h + 1, pol);
                                    au = make_double2(pu.x, pv.x);  // uu, uv(R) = vu(n)
                                    av = make_double2(pu.y, pv.y);  // vu(R) = uv(n), vv
                                }
                                yu[u] = fma(au.x, x1, yu[u]);
                                yu[u] = fma(au.y, x2, yu[u]);
                                yv[u] = fma(av.x, x1, yv[u]);
                                yv[u] = fma(av.y, x2, yv[u]);
                            } else if (IL) {
                                const double2 au = ld_stream(A2 + 2 * a, pol), av = ld_stream(A2 + 2 * a + 1, pol);
                                yu[u] = fma(au.x, x1, yu[u]);
                                yu[u] = fma(au.y, x2, yu[u]);
                                yv[u] = fma(av.x, x1, yv[u]);
                                yv[u] = fma(av.y, x2, yv[u]);
                            } else {
                                yu[u] = fma(ld_stream(Auu + a, pol), x1, yu[u]);
                                yu[u] = fma(ld_stream(Auv + a, pol), x2, yu[u]);
                                yv[u] = fma(ld_stream(Avu + a, pol), x1, yv[u]);
                                yv[u] = fma(ld_stream(Avv + a, pol), x2, yv[u]);
                            }
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kChR; ++u) {
            if (!ok[u]) continue;
            const double ru = bu[u] - yu[u], rv = bv[u] - yv[u];
            p1 += ru * ru + rv * rv;
            p0 += bu[u] * bu[u] + bv[u] * bv[u];
            ru32[ee[u]] = lv[u] ? (float)ru : 0.0f;
            rv32[ee[u]] = lv[u] ? (float)rv : 0.0f;
        }
    }
}

// FP64 r = b - A64 x on a 3D tile with x read from the shared-memory tile sx ([2][KP][NS]
// doubles: level k at row k+1, rows 0 and nz+1 and slots that hold zero are zero), the matrix
// from the interleaved copy (HALF: its symmetric half, a lower coupling read from its transpose
// partner).  Every node takes all 27 couplings with no bounds tests: a coupling that leaves the
// array meets a zero x (and in the full copy a zero coefficient), which adds nothing.  The
// multiply-adds run in the reference's coupling order, as residual_pass.  Partials: p0 = (b,b),
// p1 = (r,r); r32 = r on live columns, into buffer rpar.
template <int NZM, bool HALF>
__device__ __forceinline__ void residual_tile(const MDesc &D, const int *smap, int TY, int i0, int j0, int rpar,
                                              const double *sx, double &p0, double &p1) {
    constexpr int KP = NZM + 2;
    const Geom &g = D.g;
    const int nz = g.nz;
    const int NQ = (int)g.NQ;
    const int plane = nz * NQ;
    const int NT = kTX * TY;
    const int NS = (kTX + 2) * (TY + 2);
    const double2 *__restrict__ A2 = D.A64i;
    float *__restrict__ ru32 = D.r[rpar];
    float *__restrict__ rv32 = D.r[rpar] + plane;
    const double *sxu = sx, *sxv = sx + KP * NS;
    const int nitems = NT * nz;
    const unsigned long long pol = l2_matrix_policy(D.stream != 0);
#pragma unroll 1
    for (int base = threadIdx.x; base < nitems; base += kChR * kBlock) {
        double yu[kChR], yv[kChR], bu[kChR], bv[kChR];
        int ee[kChR];
        bool ok[kChR], lv[kChR];
#pragma unroll
        for (int u = 0; u < kChR; ++u) {
            const int it = base + u * kBlock;
            yu[u] = 0.0; yv[u] = 0.0; bu[u] = 0.0; bv[u] = 0.0;
            ee[u] = 0; ok[u] = false; lv[u] = false;
            if (it < nitems) {
                const int col = it % NT, k = it / NT;
                const int ti = col % kTX, tj = col / kTX;
                const int i = i0 + ti, j = j0 + tj;
                if (i <= g.ihi && j <= g.jhi) {
                    const int q = j * g.NX + i;
                    const int s = (ti + 1) + (kTX + 2) * (tj + 1);
                    const int e = k * NQ + q;
                    ok[u] = true;
                    ee[u] = e;
                    lv[u] = map_live(smap[s]);
                    bu[u] = D.b[e];
                    bv[u] = D.b[plane + e];
                    if (D.act[q] != 0) {
#pragma unroll
                        for (int c = 0; c < 27; ++c) {
                            const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = c / 9 - 1;
                            const int zi = (k + 1 + kA) * NS + s + iA + (kTX + 2) * jA;
                            const double x1 = sxu[zi], x2 = sxv[zi];
                            double2 au, av;
                            if (!HALF) {
                                const size_t h = (size_t)c * plane + e;
                                au = ld_stream(A2 + 2 * h, pol);
                                av = ld_stream(A2 + 2 * h + 1, pol);
                            } else if (c >= 13) {
                                const size_t h = (size_t)(c - 13) * plane + e;
                                au = ld_half(A2 + 2 * h, pol);
                                av = ld_half(A2 + 2 * h + 1, pol);
                            } else {  // partner n = (k+kA, i+iA, j+jA), coupling 26 - c, blocks swapped
                                const int kk = k + kA < 0 ? 0 : k + kA;  // level -1: its x row is zero
                                const size_t h = (size_t)(13 - c) * plane + (size_t)kk * NQ +
                                                 (size_t)((j + jA) * g.NX + (i + iA));
                                const double2 pu = ld_half(A2 + 2 * h, pol), pv = ld_half(A2 + 2 * h + 1, pol);
                                au = make_double2(pu.x, pv.x);
                                av = make_double2(pu.y, pv.y);
                            }
                            yu[u] = fma(au.x, x1, yu[u]);
                            yu[u] = fma(au.y, x2, yu[u]);
                            yv[u] = fma(av.x, x1, yv[u]);
                            yv[u] = fma(av.y, x2, yv[u]);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kChR; ++u) {
            if (!ok[u]) continue;
            const double ru = bu[u] - yu[u], rv = bv[u] - yv[u];
            p1 += ru * ru + rv * rv;
            p0 += bu[u] * bu[u] + bv[u] * bv[u];
            ru32[ee[u]] = lv[u] ? (float)ru : 0.0f;
            rv32[ee[u]] = lv[u] ? (float)rv : 0.0f;
        }
    }
}

// x of a 3D tile and its halo ring into the shared-memory tile sx ([2][KP][NS] doubles, level k
// at row k+1, zero rows 0 and nz+1, zero in slots that hold zero); with upd, advanced by this
// step's d: x + alpha64 * dn, dn = z + beta d (the owner applies the same FP64 fma later, so the
// residual sees exactly the updated x), and q = Az + beta q written for the owned columns.
template <int NZM>
__device__ __forceinline__ void fill_x_tile(const MDesc &D, const int *smap, int TY, int par, bool upd, float beta,
                                            double alpha64, double *sx) {
    constexpr int KP = NZM + 2;
    const Geom &g = D.g;
    const int nz = g.nz;
    const int NQ = (int)g.NQ;
    const int plane = nz * NQ;
    const int NS = (kTX + 2) * (TY + 2);
    const float *__restrict__ q_in = D.q[par];
    const float *__restrict__ az_in = D.Az[par];
    float *__restrict__ q_out = D.q[par ^ 1];
    for (int it = threadIdx.x; it < 2 * NS; it += kBlock) {  // zero rows above and below
        const int c = it >= NS ? 1 : 0, sl = it - c * NS;
        sx[(c * KP + 0) * NS + sl] = 0.0;
        sx[(c * KP + nz + 1) * NS + sl] = 0.0;
    }
    const int n1 = 2 * NS * nz;
#pragma unroll 1
    for (int base = threadIdx.x; base < n1; base += 4 * kBlock) {
        float zo[4], dol[4], qo[4], az[4];
        double xo[4];
        int ee[4], vv[4], ix[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int it = base + u * kBlock;
            ix[u] = -1;
            vv[u] = 0;
            ee[u] = 0;
            zo[u] = dol[u] = qo[u] = az[u] = 0.0f;
            xo[u] = 0.0;
            if (it < n1) {
                const int k = it / (2 * NS), rem = it - k * 2 * NS;
                const int c = rem >= NS ? 1 : 0, sl = rem - c * NS;
                ix[u] = (c * KP + k + 1) * NS + sl;
                const int v = smap[sl];
                vv[u] = v;
                if (map_live(v)) {
                    const int e = c * plane + k * NQ + map_src(v);
                    ee[u] = e;
                    xo[u] = ldd(D.x + e);
                    if (upd) {
                        zo[u] = ldf(D.z + e);
                        dol[u] = ldf(D.d + e);
                        if (map_mine(v)) {
                            qo[u] = ldf(q_in + e);
                            az[u] = ldf(az_in + e);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (ix[u] < 0) continue;
            const bool live = map_live(vv[u]);
            double xn = 0.0;
            if (live) {
                xn = xo[u];
                if (upd) {
                    xn = fma(alpha64, (double)fmaf(beta, dol[u], zo[u]), xn);  // x + alpha (z_i + beta d_{i-1})
                    if (map_mine(vv[u])) q_out[ee[u]] = fmaf(beta, qo[u], az[u]);  // q_i = Az_i + beta q_{i-1}
                }
            }
            sx[ix[u]] = xn;
        }
    }
}

// Line preconditioners (precond 3, 4): the right-hand sides of the line solves for the tile's
// owned columns, from the residual rb this step wrote -- per column and component the sum over
// levels in level order (3D, as tridiag_solver_local_3d sums r, glissade_velo_higher_pcg.F90:
// 4585-4590), r itself in 2D -- with the u component transposed.  rb is read back through L2 after
// a barrier (this CTA's threads wrote it).
template <int NC, int NZM>
__device__ __forceinline__ void tri_rhs(const MDesc &D, int TY, int i0, int j0, const float *rb) {
    const Geom &g = D.g;
    const int nz = (NC == 27) ? g.nz : 1;
    const int NQ = (int)g.NQ, plane = nz * NQ, NT = kTX * TY;
    for (int it = threadIdx.x; it < 2 * NT; it += kBlock) {
        const int c = it / NT, col = it - c * NT;
        const int i = i0 + col % kTX, j = j0 + col / kTX;
        if (i > g.ihi || j > g.jhi) continue;
        const int q = j * g.NX + i;
        const float *r = rb + c * plane + q;
        float v[NZM];
#pragma unroll
        for (int k = 0; k < NZM; ++k) v[k] = (k < nz) ? ldf(r + k * NQ) : 0.0f;
        float sum = v[0];
#pragma unroll
        for (int k = 1; k < NZM; ++k)
            if (k < nz) sum += v[k];
        D.rs[c * NQ + (c == 0 ? i * g.NY + j : q)] = sum;
    }
}

// The line solves of one step (tridiag_solver_local_2d, :4985-5013 along rows for u, :5041-5069
// along columns for v), in FP32 with the factors of the FP64 setup: forward elimination
// gamma_s = (b_s - sub_s gamma_{s-1}) / denom_s (gamma_s0 = b_s0 / diag_s0), then back
// substitution z_s = gamma_s - omega_s z_{s+1} over the owned range.  One thread per line: u lines
// over the owned rows, then v lines over the owned columns, spread over the solve's tiles (tile t
// takes lines t*256 + thread, then + ntiles*256).  Both kinds index their planes s*stride + line
// (u planes transposed), so a warp's 32 consecutive lines load and store 128 contiguous bytes per
// position.  Loads of kLineBatch positions are issued before the recurrence runs through them.
// Not inlined: its batch registers would otherwise raise the register pressure of every step
// kind (spills in the 2D kernels' hot passes).
constexpr int kLineBatch = 16;
__device__ __noinline__ void lines_step(const MDesc &D, int tile) {
    const Geom &g = D.g;
    const int NQ = (int)g.NQ;
    const int nu = g.jhi - g.jlo + 1, nv = g.ihi - g.ilo + 1;
    for (int L = tile * kBlock + (int)threadIdx.x; L < nu + nv; L += D.ntiles * kBlock) {
        const bool uline = L < nu;
        const int l = uline ? g.jlo + L : g.ilo + (L - nu);
        const int stride = uline ? g.NY : g.NX;
        const int s0 = uline ? g.ilo : g.jlo, s1 = uline ? g.ihi : g.jhi;
        const float *__restrict__ F = D.tri + (uline ? 0 : 4) * (size_t)NQ;
        const float *__restrict__ sub = F, *__restrict__ adr = F + NQ, *__restrict__ om = F + 2 * NQ,
                                  *__restrict__ den = F + 3 * NQ;
        const float *b = D.rs + (uline ? 0 : NQ);
        float *x = D.zs + (uline ? 0 : NQ);
        float gp = ldf(b + s0 * stride + l) * __ldg(adr + s0 * stride + l);
        x[s0 * stride + l] = gp;
#pragma unroll 1
        for (int s = s0 + 1; s <= s1; s += kLineBatch) {
            float vb[kLineBatch], vs[kLineBatch], vd[kLineBatch];
#pragma unroll
            for (int u = 0; u < kLineBatch; ++u) {
                vb[u] = vs[u] = vd[u] = 0.0f;
                if (s + u <= s1) {
                    const int e = (s + u) * stride + l;
                    vb[u] = ldf(b + e);
                    vs[u] = __ldg(sub + e);
                    vd[u] = __ldg(den + e);
                }
            }
#pragma unroll
            for (int u = 0; u < kLineBatch; ++u)
                if (s + u <= s1) {
                    gp = fmaf(-vs[u], gp, vb[u]) * vd[u];
                    x[(s + u) * stride + l] = gp;
                }
        }
        float xn = gp;
#pragma unroll 1
        for (int s = s1 - 1; s >= s0; s -= kLineBatch) {
            float vg[kLineBatch], vo[kLineBatch];
#pragma unroll
            for (int u = 0; u < kLineBatch; ++u) {
                vg[u] = vo[u] = 0.0f;
                if (s - u >= s0) {
                    const int e = (s - u) * stride + l;
                    vg[u] = ldf(x + e);  // this thread's own forward store
                    vo[u] = __ldg(om + e);
                }
            }
#pragma unroll
            for (int u = 0; u < kLineBatch; ++u)
                if (s - u >= s0) {
                    xn = fmaf(-vo[u], xn, vg[u]);
                    x[(s - u) * stride + l] = xn;
                }
        }
    }
}

// One tile of one solve for the solve's current step; publishes the tile's record.
template <int NC, int NZM>
__device__ void tile_step(const MState &S, int tile, bool resident, int TYmax, MHead &hd, unsigned char *smem) {
    using LY = MLayout<NC, NZM>;
    constexpr int KP = LY::KP;
    constexpr int OFF = (NC == 27) ? 1 : 0;  // z row of level 0
    const LY ly(TYmax, resident);
    const MDesc &D = hd.D;
    const int TY = D.TY;
    const int NS = (kTX + 2) * (TY + 2), NT = kTX * TY;
    int *smap = reinterpret_cast<int *>(smem + ly.off_map());
    float *sz = reinterpret_cast<float *>(smem + ly.off_z());   // [2][KP][NS]
    float *srt = reinterpret_cast<float *>(smem + ly.off_rt()); // [2][NZM][NT]
    const Geom &g = D.g;
    const int nz = (NC == 27) ? g.nz : 1;
    const int NQ = (int)g.NQ;
    const int plane = nz * NQ;
    const int tx = tile % D.tiles_x, ty = tile / D.tiles_x;
    const int i0 = g.ilo + tx * kTX, j0 = g.jlo + ty * TY;
    const int t = threadIdx.x;
    const int step = S.step;
    const int par = S.par;
    const bool tri = D.precond >= 3;  // the line preconditioners
    double p0 = 0.0, p1 = 0.0;

    if (!resident) {  // resident launches keep their single tile's map for the whole launch
        const int *tmap = D.maps + (size_t)tile * NS;
        for (int sl = t; sl < NS; sl += kBlock) smap[sl] = tmap[sl];
        __syncthreads();
    }

    if (NC == 27 && NZM <= 16 && D.A64i && (step == MS_INIT || step == MS_BC)) {
        // 3D: x of the tile and halo (updated by this step's d in MS_BC) into shared memory, then
        // the FP64 residual with branch-free couplings
        double *sx = reinterpret_cast<double *>(smem + ly.off_x64());
        const bool upd = step == MS_BC;
        fill_x_tile<NZM>(D, smap, TY, par, upd, upd ? (float)S.beta : 0.0f, upd ? S.alpha : 0.0, sx);
        __syncthreads();
        if (D.sym) residual_tile<NZM, true>(D, smap, TY, i0, j0, upd ? par ^ 1 : par, sx, p0, p1);
        else residual_tile<NZM, false>(D, smap, TY, i0, j0, upd ? par ^ 1 : par, sx, p0, p1);
        if (upd) {
            p0 = p1;
            p1 = 0.0;
        }
        if (tri) {
            __syncthreads();
            tri_rhs<NC, NZM>(D, TY, i0, j0, D.r[upd ? par ^ 1 : par]);
        }
    } else if (step == MS_LINES) {
        lines_step(D, tile);
    } else if (step == MS_INIT) {
        if (NC == 27 && D.sym) residual_pass<NC, true, true>(D, smap, TY, i0, j0, par, nullptr, 0.0, p0, p1);
        else if (D.A64i) residual_pass<NC, true>(D, smap, TY, i0, j0, par, nullptr, 0.0, p0, p1);
        else residual_pass<NC, false>(D, smap, TY, i0, j0, par, nullptr, 0.0, p0, p1);
        if (tri) {
            __syncthreads();
            tri_rhs<NC, NZM>(D, TY, i0, j0, D.r[par]);
        }
    } else if (step == MS_BC) {
        // update of iteration iter fused with the FP64 check: dn = z + beta d on tile and halo
        // slots (into shared memory, over the z rows), q for the owned columns; the owners'
        // d and x writes wait for the next step
        const float beta = (float)S.beta;
        float *sdn = sz;  // [2][nz][NS]
        const float *__restrict__ q_in = D.q[par];
        const float *__restrict__ az_in = D.Az[par];
        float *__restrict__ q_out = D.q[par ^ 1];
        const int n1 = 2 * NS * nz;
#pragma unroll 1
        for (int base = t; base < n1; base += 4 * kBlock) {
            float zo[4], dol[4], qo[4], az[4];
            int ee[4], vv[4], ix[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int it = base + u * kBlock;
                ix[u] = -1;
                vv[u] = 0;
                ee[u] = 0;
                zo[u] = dol[u] = qo[u] = az[u] = 0.0f;
                if (it < n1) {
                    const int k = it / (2 * NS), rem = it - k * 2 * NS;
                    const int c = rem >= NS ? 1 : 0, sl = rem - c * NS;
                    ix[u] = (c * nz + k) * NS + sl;
                    const int v = smap[sl];
                    vv[u] = v;
                    if (map_live(v)) {
                        const int e = c * plane + k * NQ + map_src(v);
                        ee[u] = e;
                        zo[u] = ldf(D.z + e);
                        dol[u] = ldf(D.d + e);
                        if (map_mine(v)) {
                            qo[u] = ldf(q_in + e);
                            az[u] = ldf(az_in + e);
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (ix[u] < 0) continue;
                const bool live = map_live(vv[u]);
                sdn[ix[u]] = live ? fmaf(beta, dol[u], zo[u]) : 0.0f;  // d_i = z_i + beta d_{i-1}
                if (live && map_mine(vv[u])) q_out[ee[u]] = fmaf(beta, qo[u], az[u]);  // q_i = Az_i + beta q_{i-1}
            }
        }
        __syncthreads();
        if (NC == 27 && D.sym) residual_pass<NC, true, true>(D, smap, TY, i0, j0, par ^ 1, sdn, S.alpha, p0, p1);
        else if (D.A64i) residual_pass<NC, true>(D, smap, TY, i0, j0, par ^ 1, sdn, S.alpha, p0, p1);
        else residual_pass<NC, false>(D, smap, TY, i0, j0, par ^ 1, sdn, S.alpha, p0, p1);
        p0 = p1;
        p1 = 0.0;
        if (tri) {
            __syncthreads();
            tri_rhs<NC, NZM>(D, TY, i0, j0, D.r[par ^ 1]);
        }
    } else if (step == MS_FIN) {
        // the deferred owner writes of the last (checked) update
        const float beta = (float)S.beta;
        const double alpha64 = S.alpha;
        const int nitems = 2 * NT * nz;
        for (int it = t; it < nitems; it += kBlock) {
            const int c = it / (NT * nz), r2 = it - c * NT * nz;
            const int k = r2 / NT, col = r2 - k * NT;
            const int s = (col % kTX + 1) + (kTX + 2) * (col / kTX + 1);
            const int v = smap[s];
            if (!map_mine(v)) continue;
            const int e = c * plane + k * NQ + map_src(v);
            const float dn = fmaf(beta, ldf(D.d + e), ldf(D.z + e));
            D.d[e] = dn;
            D.x[e] = fma(alpha64, (double)dn, ldd(D.x + e));
        }
    } else {
        const float alpha = (float)S.alpha, beta = (float)S.beta;
        const double alpha64 = S.alpha;
        const bool do_b = (step == MS_MERGED || step == MS_B || step == MS_UPD);
        const bool do_a = (step == MS_MERGED || step == MS_A || step == MS_A_UPD);
        const bool upd = (step == MS_A_UPD);  // apply the owners' deferred d and x writes
        const int rin = par, rout = do_b ? (par ^ 1) : par;  // buffers holding r_i / r_{i+1}
        const float *__restrict__ q_in = D.q[rin];
        const float *__restrict__ az_in = D.Az[rin];
        const float *__restrict__ r_in = D.r[rin];
        float *__restrict__ q_out = D.q[rout];
        float *__restrict__ r_out = D.r[rout];
        float *__restrict__ dvec = D.d;
        const float *__restrict__ zvec = D.z;
        double *__restrict__ xvec = D.x;
        const float *__restrict__ dinv = D.pre;
        const bool diag = D.precond == 1;

        // ---- pass 1: update (B) on the tile, new residual (and diag z) on tile + halo ----
        // items (k, c, slot) in the order k, c, slot; kCh1 items' loads are issued together
        constexpr int kCh1 = 6;  // items per load batch (register budget)
        const int per_k = 2 * NS;
        const int n1 = per_k * nz;
#pragma unroll 1
        for (int base = t; base < n1; base += kCh1 * kBlock) {
            float qo[kCh1], az[kCh1], ro[kCh1], dold[kCh1], zold[kCh1], pr[kCh1];
            double xold[kCh1];
            int ee[kCh1], vv[kCh1], ss[kCh1], sr[kCh1];
            int k = base / per_k;
            int rem = base - k * per_k;
#pragma unroll
            for (int u = 0; u < kCh1; ++u) {
                if (u > 0) {
                    rem += kBlock;
                    while (rem >= per_k) { rem -= per_k; ++k; }
                }
                ss[u] = -1;
                sr[u] = -1;
                vv[u] = 0;
                ee[u] = 0;
                qo[u] = az[u] = ro[u] = dold[u] = zold[u] = 0.0f;
                pr[u] = 1.0f;
                xold[u] = 0.0;
                if (k < nz) {
                    const int c = rem >= NS ? 1 : 0, sl = rem - c * NS;
                    ss[u] = (c * KP + k + OFF) * NS + sl;  // the item's z slot in smem
                    const int li = sl % (kTX + 2), lj = sl / (kTX + 2);
                    if (li >= 1 && li <= kTX && lj >= 1 && lj <= TY)  // tile column: keep r for the dots
                        sr[u] = (c * NZM + k) * NT + (li - 1) + kTX * (lj - 1);
                    const int v = smap[sl];
                    vv[u] = v;
                    // an update alone (MS_B, MS_UPD) writes only the tile's own columns
                    const int m = (map_live(v) && (do_a || map_mine(v))) ? map_src(v) : -1;
                    if (m >= 0) {
                        const int e = c * plane + k * NQ + m;
                        ee[u] = e;
                        if (do_b) {
                            qo[u] = ldf(q_in + e);
                            az[u] = ldf(az_in + e);
                            ro[u] = ldf(r_in + e);
                            if (map_mine(v)) {
                                dold[u] = ldf(dvec + e);
                                zold[u] = ldf(zvec + e);
                                xold[u] = ldd(xvec + e);
                            }
                        } else {
                            ro[u] = ldf(r_in + e);
                            if (upd && map_mine(v)) {
                                dold[u] = ldf(dvec + e);
                                zold[u] = ldf(zvec + e);
                                xold[u] = ldd(xvec + e);
                            }
                        }
                        if (do_a && diag) pr[u] = __ldg(dinv + e);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kCh1; ++u) {
                if (ss[u] < 0) continue;
                const int v = vv[u];
                const bool live = map_live(v);
                float rn = 0.0f;
                if (live) {
                    const int e = ee[u];
                    if (do_b) {
                        const float qn = fmaf(beta, qo[u], az[u]);  // q_i = Az_i + beta q_{i-1}
                        rn = fmaf(-alpha, qn, ro[u]);              // r_{i+1} = r_i - alpha q_i
                        if (map_mine(v)) {
                            const float dn = fmaf(beta, dold[u], zold[u]);  // d_i = z_i + beta d_{i-1}
                            dvec[e] = dn;
                            q_out[e] = qn;
                            r_out[e] = rn;
                            xvec[e] = fma(alpha64, (double)dn, xold[u]);  // x += alpha d_i (FP64)
                        }
                    } else {
                        rn = ro[u];
                        if (upd && map_mine(v)) {  // the previous (checked) update's owner writes
                            const float dn = fmaf(beta, dold[u], zold[u]);
                            dvec[e] = dn;
                            xvec[e] = fma(alpha64, (double)dn, xold[u]);
                        }
                    }
                }
                if (do_a) {
                    if (sr[u] >= 0) srt[sr[u]] = rn;
                    sz[ss[u]] = (diag && live) ? rn * pr[u] : rn;
                }
            }
        }
        if (tri && !do_a) {  // MS_UPD: the right-hand sides of the next lines
            __syncthreads();
            tri_rhs<NC, NZM>(D, TY, i0, j0, r_out);
        }
        if (do_a) {
            if (NC == 27) {  // zero padding rows (levels -1 and nz)
                for (int it = t; it < 2 * NS; it += kBlock) {
                    const int c = it >= NS ? 1 : 0, sl = it - c * NS;
                    sz[(c * KP + 0) * NS + sl] = 0.0f;
                    sz[(c * KP + nz + 1) * NS + sl] = 0.0f;
                }
            }
            __syncthreads();
            if (NC == 27 && (D.precond == 2 || tri)) {  // column tridiagonal solves on tile + halo
                // one (column, component) per thread while they fit the block: the two
                // components' recurrences then run side by side instead of one after the other
                const bool split = 2 * NS <= kBlock;
                const int nit = split ? 2 * NS : NS;
                for (int it = t; it < nit; it += kBlock) {
                    const int c = split ? it / NS : 0, sl = split ? it - c * NS : it;
                    const int v = smap[sl];
                    if (map_live(v)) sia_col<NZM>(D, sz, NS, sl, map_src(v), c, split ? c : 1);
                }
                __syncthreads();
            }
            if (tri) {  // + the line solution of the column (3D: on every level), or z = it (2D)
                for (int it = t; it < 2 * NS; it += kBlock) {
                    const int c = it >= NS ? 1 : 0, sl = it - c * NS;
                    const int v = smap[sl];
                    if (!map_live(v)) continue;
                    const int m = map_src(v);
                    const float zl = (c == 0) ? ldf(D.zs + (m % g.NX) * g.NY + m / g.NX) : ldf(D.zs + NQ + m);
                    if (NC == 27) {
                        for (int k = 0; k < nz; ++k) sz[(c * KP + k + OFF) * NS + sl] += zl;
                    } else {
                        sz[(c * KP + OFF) * NS + sl] = zl;
                    }
                }
                __syncthreads();
            }

            // ---- pass 2: Az = A z on (column, level) items, z to HBM, partial dots ----
            // Couplings that leave the grid are zero in the FP32 copy and the padded z rows
            // and out-of-grid halo slots are zero, so every node sums all NC terms.
            const float4 *__restrict__ A4 = D.A32;
            const float4 *sA = reinterpret_cast<const float4 *>(smem + ly.off_A());  // [NC][nz*NT]
            const int NN = nz * NT;
            float *__restrict__ Azu = D.Az[rout];
            float *__restrict__ Azv = D.Az[rout] + plane;
            float *__restrict__ zu_out = D.z;
            float *__restrict__ zv_out = D.z + plane;
            const float *szu = sz, *szv = sz + KP * NS;
            const unsigned long long pol = l2_matrix_policy(D.stream != 0);
#pragma unroll 1
            for (int base = t; base < NN; base += kCh2 * kBlock) {
                float yu[kCh2], yv[kCh2], zu[kCh2], zv[kCh2];
                int ee[kCh2], cc[kCh2];
                bool ok[kCh2];
#pragma unroll
                for (int u = 0; u < kCh2; ++u) {
                    const int it = base + u * kBlock;
                    yu[u] = yv[u] = zu[u] = zv[u] = 0.0f;
                    ok[u] = false;
                    ee[u] = 0;
                    cc[u] = 0;
                    if (it < NN) {
                        const int col = it % NT, k = it / NT;
                        const int ti = col % kTX, tj = col / kTX;
                        const int i = i0 + ti, j = j0 + tj;
                        if (i <= g.ihi && j <= g.jhi) {
                            const int s = (ti + 1) + (kTX + 2) * (tj + 1);
                            const int e = k * NQ + j * g.NX + i;
                            ok[u] = true;
                            ee[u] = e;
                            cc[u] = k * NT + col;
                            zu[u] = szu[(k + OFF) * NS + s];
                            zv[u] = szv[(k + OFF) * NS + s];
                            if (map_live(smap[s])) {
                                if (NC == 27 && D.sym) {
                                    // symmetric half: the diagonal and upper couplings from this node,
                                    // a lower coupling c from its transpose partner (node n = this
                                    // node + offset(c), coupling 26 - c, uv and vu swapped); at level
                                    // 0 a kA = -1 partner row is clamped to level 0, its z row being
                                    // the zero padding
#pragma unroll
                                    for (int c = 0; c < NC; ++c) {
                                        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = c / 9 - 1;
                                        const int zi = (k + OFF + kA) * NS + s + iA + (kTX + 2) * jA;
                                        const float z1 = szu[zi], z2 = szv[zi];
                                        float4 a;
                                        if (c >= 13) {
                                            a = ld_half(A4 + (size_t)(c - 13) * plane + e, pol);
                                        } else {
                                            const int kk = k + kA < 0 ? 0 : k + kA;
                                            const float4 pa = ld_half(A4 + (size_t)(13 - c) * plane + kk * NQ +
                                                                            (j + jA) * g.NX + (i + iA), pol);
                                            a = make_float4(pa.x, pa.z, pa.y, pa.w);
                                        }
                                        yu[u] = fmaf(a.x, z1, yu[u]);
                                        yu[u] = fmaf(a.y, z2, yu[u]);
                                        yv[u] = fmaf(a.z, z1, yv[u]);
                                        yv[u] = fmaf(a.w, z2, yv[u]);
                                    }
                                } else if (resident) {
#pragma unroll
                                    for (int c = 0; c < NC; ++c) {
                                        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
                                        const int zi = (k + OFF + kA) * NS + s + iA + (kTX + 2) * jA;
                                        const float z1 = szu[zi], z2 = szv[zi];
                                        const float4 a = sA[c * NN + it];
                                        yu[u] = fmaf(a.x, z1, yu[u]);
                                        yu[u] = fmaf(a.y, z2, yu[u]);
                                        yv[u] = fmaf(a.z, z1, yv[u]);
                                        yv[u] = fmaf(a.w, z2, yv[u]);
                                    }
                                } else {
#pragma unroll
                                    for (int c = 0; c < NC; ++c) {
                                        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
                                        const int zi = (k + OFF + kA) * NS + s + iA + (kTX + 2) * jA;
                                        const float z1 = szu[zi], z2 = szv[zi];
                                        const float4 a = ld_stream(A4 + (size_t)c * plane + e, pol);
                                        yu[u] = fmaf(a.x, z1, yu[u]);
                                        yu[u] = fmaf(a.y, z2, yu[u]);
                                        yv[u] = fmaf(a.z, z1, yv[u]);
                                        yv[u] = fmaf(a.w, z2, yv[u]);
                                    }
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < kCh2; ++u) {
                    if (!ok[u]) continue;
                    const int e = ee[u];
                    Azu[e] = yu[u];
                    Azv[e] = yv[u];
                    zu_out[e] = zu[u];
                    zv_out[e] = zv[u];
                    const double ru = srt[cc[u]], rv = srt[NZM * NT + cc[u]];
                    p0 += ru * (double)zu[u] + rv * (double)zv[u];
                    p1 += (double)yu[u] * zu[u] + (double)yv[u] * zv[u];
                }
            }
        }
    }
    block_sum2(p0, p1, hd.red);
    if (t < 32) {  // warp 0: lane c*4+k stores word k of copy c, after a release fence
        p0 = __shfl_sync(0xffffffffu, p0, 0);
        p1 = __shfl_sync(0xffffffffu, p1, 0);
        if (t < 4 * kRecCopies) {
            const unsigned tag = S.tick + 1u;
            const int c = t / 4, k = t - 4 * (t / 4);
            const double pv = (k < 2) ? p0 : p1;
            const unsigned half = (k & 1) ? (unsigned)__double2hiint(pv) : (unsigned)__double2loint(pv);
            TileRec *rp = D.recs + (size_t)c * 2 * D.ntiles + 2 * (size_t)tile + (tag & 1u);
            fence_acq_rel();  // the tile's vector stores (every thread's, via the barrier above) first
            if (!(tile == 0 && tag == c_withhold_tag))
                st_relaxed64(&rp->w[k], ((unsigned long long)tag << 32) | half);
        }
    }
    __syncthreads();
}

// Waits for the step-`tag` records of the ntl tiles at R (one record pair per tile) and sums
// them in a fixed order: thread t takes tiles t, t + 256, ... in increasing order, then a
// warp shuffle tree and a tree over the 8 warp sums.  Every CTA summing a solve's records
// runs this with the same inputs, so all of them get bit-identical sums (in thread 0).
// Records validate themselves (the tag in every word), so a thread polls its tiles with
// relaxed loads issued together: one memory round trip once they are there.  Ordering for
// the loads that follow: with nacq >= 0, threads 0..nacq-1 each take an acquire load of a
// record of tile acq[t] (the tiles whose columns the CTA's halo reads) alongside; with
// nacq < 0 every thread ends with an acquire fence (a leader whose sums others rely on).
// Returns false if a wait gave up.
constexpr int kRecPerThread = 2;  // tiles a thread polls at once (ntl <= 512 in one round)
__device__ bool sum_records(const TileRec *R, int ntl, unsigned tag, MCtl *ctl, double (*rsum)[2],
                            const int *acq, int nacq, double &s0, double &s1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double a0 = 0.0, a1 = 0.0;
    int bad = 0;
    const int at = (nacq > 0 && (int)threadIdx.x < nacq) ? acq[threadIdx.x] : -1;
    bool acq_need = at >= 0;
    for (int w0 = threadIdx.x; (w0 < ntl || acq_need) && !bad; w0 += kRecPerThread * kBlock) {
        unsigned need = 0;
#pragma unroll
        for (int u = 0; u < kRecPerThread; ++u)
            if (w0 + u * kBlock < ntl) need |= 1u << u;
        double v[kRecPerThread][2];
#pragma unroll
        for (int u = 0; u < kRecPerThread; ++u) v[u][0] = v[u][1] = 0.0;
        const long long t0 = clock64();
        unsigned spins = 0;
        for (;;) {
#pragma unroll
            for (int u = 0; u < kRecPerThread; ++u) {
                if (!((need >> u) & 1u)) continue;
                unsigned long long wd[4];
                ld_rec(R + 2 * (size_t)(w0 + u * kBlock), wd);
                bool ok = true;
#pragma unroll
                for (int k = 0; k < 4; ++k) ok &= (unsigned)(wd[k] >> 32) == tag;
                if (ok) {
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        v[u][k] = __hiloint2double((int)(unsigned)wd[2 * k + 1], (int)(unsigned)wd[2 * k]);
                    need &= ~(1u << u);
                }
            }
            if (acq_need && (unsigned)(ld_acquire64(&R[2 * (size_t)at].w[3]) >> 32) == tag) acq_need = false;
            if (!need && !acq_need) break;
            __nanosleep(spins < 16 ? 20 : 100);
            if ((++spins & 31u) == 0) {
                if (*(volatile int *)&ctl->abort) { bad = 1; break; }
                if (clock64() - t0 > c_wait_cycles) {
                    atomicExch(&ctl->abort, 1);
                    bad = 1;
                    break;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kRecPerThread; ++u)
            if (w0 + u * kBlock < ntl) { a0 += v[u][0]; a1 += v[u][1]; }
    }
    if (nacq < 0) fence_acq_rel();
    if (__syncthreads_or(bad)) return false;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const double o0 = __shfl_down_sync(0xffffffffu, a0, off), o1 = __shfl_down_sync(0xffffffffu, a1, off);
        if (lane + off < 32) { a0 += o0; a1 += o1; }
    }
    if (lane == 0) { rsum[warp][0] = a0; rsum[warp][1] = a1; }
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = kBlock / 32;
        a0 = lane < NW ? rsum[lane][0] : 0.0;
        a1 = lane < NW ? rsum[lane][1] : 0.0;
#pragma unroll
        for (int off = NW / 2; off >= 1; off >>= 1) {
            const double o0 = __shfl_down_sync(0xffffffffu, a0, off), o1 = __shfl_down_sync(0xffffffffu, a1, off);
            if (lane + off < NW) { a0 += o0; a1 += o1; }
        }
    }
    s0 = a0; s1 = a1;
    return true;
}

// Wait for the records of the step just taken by every running solve this CTA holds, sum
// them (sum_records) and advance the solve's cached state.  Every CTA holding a solve does
// this with the same inputs in the same order, so all copies of a solve's state stay
// bit-identical.  The CTA holding tile 0 publishes a finished solve.
// Returns false if a wait gave up (here or in another CTA).
__device__ bool reduce_wait(MHead &hd, const MDesc *__restrict__ descs, MState *gstates, MCtl *ctl) {
    for (int cs = 0; cs < hd.nsolve; ++cs) {
        if (hd.st[cs].done) continue;  // uniform: only thread 0 writes st, before a barrier
        const MDesc &D = descs[hd.sid[cs]];
        const int ntl = D.ntiles;
        const unsigned tag = hd.st[cs].tick + 1u;
        const TileRec *R = D.recs + (size_t)(blockIdx.x % kRecCopies) * 2 * ntl + (tag & 1u);
        double s0, s1;
        if (!sum_records(R, ntl, tag, ctl, hd.rsum, hd.acq, hd.nsolve == 1 ? hd.nacq : -1, s0, s1)) return false;
        if (threadIdx.x == 0) {
            MState &S = hd.st[cs];
            advance_state(S, s0, s1);
            S.tick = tag;
            if (S.done && hd.owner[cs]) {
                gstates[hd.sid[cs]] = S;
                __threadfence();
            }
        }
        __syncthreads();
    }
    return true;
}

// resident != 0: the launch has exactly one tile per CTA; the CTA keeps that tile's slot
// map and (2D) its FP32 matrix coefficients in shared memory for the whole launch.
// A CTA leaves when every solve it holds is done, or after max_steps steps (a serving
// epoch); then it folds in the last step's sums so that the next launch resumes exactly.
template <int NC, int NZM>
__global__ void __launch_bounds__(kBlock, 2) k_mixed(const MDesc *__restrict__ descs, MState *states,
                                                     const MTile *__restrict__ tiles, int ntiles, int TYmax,
                                                     int resident, MCtl *ctl, int max_steps) {
    extern __shared__ __align__(16) unsigned char smem[];
    MHead &hd = *reinterpret_cast<MHead *>(smem);
    const MLayout<NC, NZM> ly(TYmax, resident != 0);
    // cache the states of the solves this CTA holds (round robin over the tile list)
    if (threadIdx.x == 0) {
        int n = 0;
        for (int w = blockIdx.x; w < ntiles; w += gridDim.x) {
            const MTile T = tiles[w];
            if (T.solve < 0) continue;  // padding of a blocked tile order
            int u = 0;
            while (u < n && hd.sid[u] != T.solve) ++u;
            if (u == n && n < kMaxCtaSolves) {
                hd.sid[n] = T.solve;
                hd.owner[n] = 0;
                const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&states[T.solve]);
                unsigned long long *dst = reinterpret_cast<unsigned long long *>(&hd.st[n]);
                for (int w8 = 0; w8 < (int)(sizeof(MState) / 8); ++w8) dst[w8] = __ldcg(src + w8);
                ++n;
            }
            if (u < n && T.tile == 0) hd.owner[u] = 1;
        }
        hd.nsolve = n;
        hd.cur = -1;
        // one solve: acquire only the tiles whose columns this CTA's halo reads (the line
        // preconditioners read every tile's columns: fence)
        int na = (n == 1) ? 0 : -1;
        for (int w = blockIdx.x; w < ntiles && na >= 0; w += gridDim.x) {
            const MTile T = tiles[w];
            if (T.solve < 0) continue;
            const int *nb = descs[T.solve].nbrs + (size_t)T.tile * kNbrStride;
            const int cnt = nb[0];
            if (cnt < 0 || na + cnt > kMaxAcq || descs[T.solve].precond >= 3) { na = -1; break; }
            for (int k = 0; k < cnt; ++k) hd.acq[na++] = nb[1 + k];
        }
        hd.nacq = na;
        int nt = 0;
        for (int w = blockIdx.x; w < ntiles; w += gridDim.x, ++nt)
            if (nt < kTilesCached) hd.tl[nt] = tiles[w];
        hd.ntl = nt;
    }
    __syncthreads();
    if (resident && blockIdx.x < ntiles) {  // the CTA's only tile: slot map and FP32 matrix
        const MTile T = tiles[blockIdx.x];
        const MDesc &D = descs[T.solve];
        const int TY = D.TY;
        const int NS = (kTX + 2) * (TY + 2), NT = kTX * TY;
        int *smap = reinterpret_cast<int *>(smem + ly.off_map());
        const int *tmap = D.maps + (size_t)T.tile * NS;
        for (int sl = threadIdx.x; sl < NS; sl += kBlock) smap[sl] = tmap[sl];
        float4 *sA = reinterpret_cast<float4 *>(smem + ly.off_A());
        const int nz = (NC == 27) ? D.g.nz : 1;
        const int NQ = (int)D.g.NQ;
        const int plane = nz * NQ;
        const int tx = T.tile % D.tiles_x, ty = T.tile / D.tiles_x;
        const int i0 = D.g.ilo + tx * kTX, j0 = D.g.jlo + ty * TY;
        const int NN = nz * NT;
        // sA[c][k][tj][ti] = A32[c][k][j0+tj][i0+ti]: each (c, k, tj) row of the tile inside the
        // grid is one bulk copy of ncol float4 (16-byte aligned at both ends); the columns past
        // ihi and the rows past jhi are zeros stored by the threads (bytes no copy writes)
        const int ncol = min(kTX, D.g.ihi - i0 + 1), nrow = min(TY, D.g.jhi - j0 + 1);
        const int nrows = NC * nz * nrow;
        if (threadIdx.x == 0) {
            mbar_init(&hd.mbar, 1);
            mbar_expect_tx(&hd.mbar, (unsigned)(nrows * ncol * 16));
        }
        __syncthreads();
        for (int r = threadIdx.x; r < nrows; r += kBlock) {
            const int tj = r % nrow, ck = r / nrow, k = ck % nz, c = ck / nz;
            bulk_g2s(sA + (size_t)c * NN + k * NT + tj * kTX, D.A32 + (size_t)c * plane + k * NQ + (j0 + tj) * D.g.NX + i0,
                     (unsigned)(ncol * 16), &hd.mbar);
        }
        for (int w = threadIdx.x; w < NC * NN; w += kBlock) {
            const int col = (w % NN) % NT;
            if (col % kTX >= ncol || col / kTX >= nrow) sA[w] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        long long t0 = clock64();
        bool ok = true;
        while (!mbar_try_wait(&hd.mbar, 0u))
            if (clock64() - t0 > c_wait_cycles) { ok = false; break; }
        if (__syncthreads_or(!ok)) {  // the copies did not land: fail the launch, after one more
            if (threadIdx.x == 0) atomicExch(&ctl->abort, 1);  // bounded wait for them
            t0 = clock64();
            while (!mbar_try_wait(&hd.mbar, 0u) && clock64() - t0 <= c_wait_cycles) {
            }
            return;
        }
    }
    bool finished = false;
    int step = 0;
    for (; step < max_steps; ++step) {
        if (step > 0 && !reduce_wait(hd, descs, states, ctl)) return;  // previous step's sums
        bool running = false;
        for (int cs = 0; cs < hd.nsolve; ++cs) running |= !hd.st[cs].done;
        if (!running) {
            finished = true;
            break;
        }
        for (int u = 0; u < hd.ntl; ++u) {
            const MTile T = (u < kTilesCached) ? hd.tl[u] : tiles[blockIdx.x + (size_t)u * gridDim.x];
            if (T.solve < 0) continue;  // padding of a blocked tile order
            int cs = 0;
            while (cs < hd.nsolve && hd.sid[cs] != T.solve) ++cs;
            if (cs >= hd.nsolve || hd.st[cs].done) continue;
            if (hd.cur != cs) {
                __syncthreads();
                if (threadIdx.x == 0) {
                    hd.D = descs[T.solve];
                    hd.cur = cs;
                }
                __syncthreads();
            }
            tile_step<NC, NZM>(hd.st[cs], T.tile, resident != 0, TYmax, hd, smem);
        }
    }
    // out of steps: fold in the last step's sums so that the next launch resumes exactly
    if (!finished && step > 0 && !reduce_wait(hd, descs, states, ctl)) return;
    if (threadIdx.x == 0)
        for (int cs = 0; cs < hd.nsolve; ++cs)
            if (hd.owner[cs]) states[hd.sid[cs]] = hd.st[cs];
}

// ---------------------------------------------------------------------------
// dynamic launches (batches and the serving loop)
// ---------------------------------------------------------------------------
// Leader duties of one step for every running solve this CTA leads: wait for the records
// of all the solve's tiles, sum them in the same fixed order as reduce_wait (so results are
// bit-identical to the single-solve kernel), advance the state and broadcast the scalars
// the tiles need.  A finished solve is published to gstates, flagged and counted down.
// Returns false if a wait gave up (here or in another CTA).
__device__ bool lead_duties(MHead &hd, const MDesc *__restrict__ descs, MState *const *gstates, MCtl *ctl) {
    for (int cs = 0; cs < hd.nsolve; ++cs) {
        if (hd.st[cs].done) continue;  // uniform: only thread 0 writes st, before a barrier
        const MDesc &D = descs[hd.sid[cs]];
        const int ntl = D.ntiles;
        const unsigned tag = hd.st[cs].tick + 1u;
        const TileRec *R = D.recs + (size_t)(blockIdx.x % kRecCopies) * 2 * ntl + (tag & 1u);
        double s0, s1;
        if (!sum_records(R, ntl, tag, ctl, hd.rsum, nullptr, -1, s0, s1)) return false;
        if (threadIdx.x == 0) {
            MState &S = hd.st[cs];
            advance_state(S, s0, s1);
            S.tick = tag;
            if (S.done) *gstates[hd.sid[cs]] = S;
            Bcast *B = D.bc + (size_t)(tag & 1u) * kBcastCopies;
            for (int k = 0; k < kBcastCopies; ++k) {
                B[k].alpha = S.alpha;
                B[k].beta = S.beta;
            }
            __threadfence();  // the state, the scalars and (cumulatively) the records before the word
            const unsigned long long word = ((unsigned long long)tag << 32) | (unsigned)(S.done << 9) |
                                            (unsigned)(S.par << 8) | (unsigned)S.step;
            for (int k = 0; k < kBcastCopies; ++k) st_relaxed64(&B[k].word, word);
            if (S.done) {
                st_relaxed(reinterpret_cast<unsigned *>(D.dflag), 1u);
                atomicSub(&ctl->active, 1);
            }
        }
        __syncthreads();
    }
    return true;
}

// Dynamic persistent kernel.  Work items are (step, tile list position), handed out in
// order by one atomic counter, so every CTA works on whatever tiles are left: solves that
// converge early free the GPU for the others.  Solve i is led by CTA i * grid / nsolve,
// which sums its records and broadcasts its scalars (lead_duties); a CTA that takes a tile
// of solve X at step s waits for X's broadcast of step s (tag = ltick0[X] + s).  Before a CTA
// works on any item of step s it finishes its leader duties of every earlier step, so the
// waits cannot form a cycle.  The per-tile arithmetic is tile_step, and the sums are taken
// in the same fixed order as the single-solve kernel, so every result is bit-identical to
// solving the system alone with the same tile height.  Stops when all solves are done or
// after max_steps steps (a serving epoch), after folding in the last step's sums.
// MULTI: the launch holds 2D solves and 3D solves of up to NZM levels together (the serving
// loop's mixed epochs); each work item runs the tile code of its solve's class, 3D tiles laid
// out for height TYmax and 2D tiles for TY2max in the same dynamic shared memory.
template <int NC, int NZM, bool MULTI = false>
__global__ void __launch_bounds__(kBlock, 2) k_mixed_dyn(const MDesc *__restrict__ descs, MState *const *states,
                                                         const unsigned *__restrict__ ltick0, int nsolve,
                                                         const MTile *__restrict__ tiles, int ntiles, int TYmax,
                                                         int TY2max, MCtl *ctl, int max_steps) {
    extern __shared__ __align__(16) unsigned char smem[];
    MHead &hd = *reinterpret_cast<MHead *>(smem);
    __shared__ unsigned long long s_item;
    __shared__ int s_flag;
    __shared__ MState s_view;
    if (threadIdx.x == 0) {  // the solves this CTA leads
        int n = 0;
        for (int i = 0; i < nsolve && n < kMaxCtaSolves; ++i) {
            if ((int)((long long)i * gridDim.x / nsolve) != (int)blockIdx.x) continue;
            hd.sid[n] = i;
            hd.owner[n] = 1;
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(states[i]);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&hd.st[n]);
            for (int w8 = 0; w8 < (int)(sizeof(MState) / 8); ++w8) dst[w8] = __ldcg(src + w8);
            // a solve that finished in an earlier launch (the serving loop queues its next epoch
            // before it has read the previous one) is not running: count it out at once
            if (hd.st[n].done) atomicSub(&ctl->active, 1);
            ++n;
        }
        hd.nsolve = n;
        hd.cur = -1;
    }
    __syncthreads();
    int duty_step = 0;  // leader duties of steps < duty_step are done
    bool epoch_end = false;
    for (;;) {
        __syncthreads();  // every thread is done with the previous item's shared values
        if (threadIdx.x == 0) {
            s_flag = (*(volatile int *)&ctl->active <= 0 || *(volatile int *)&ctl->abort) ? 1 : 0;
            if (!s_flag) s_item = atomicAdd(&ctl->next, 1ull);
        }
        __syncthreads();
        if (s_flag) break;  // all solves done (or a wait gave up somewhere)
        const long long step = (long long)(s_item / (unsigned long long)ntiles);
        const int pos = (int)(s_item % (unsigned long long)ntiles);
        if (step >= max_steps) {
            epoch_end = true;
            break;
        }
        while (duty_step < step) {
            if (!lead_duties(hd, descs, states, ctl)) return;
            ++duty_step;
        }
        const MTile T = tiles[pos];
        if (T.solve < 0) continue;
        // the solve's scalars after `step` steps of this launch
        if (threadIdx.x == 0) {
            const MDesc *Dp = descs + T.solve;
            const unsigned tag = ltick0[T.solve] + (unsigned)step;
            const Bcast *B = Dp->bc + (size_t)(tag & 1u) * kBcastCopies + (blockIdx.x % kBcastCopies);
            const int *dflag = Dp->dflag;
            int st = 0;  // 0 ready, 1 solve done, 2 gave up
            unsigned long long word = ld_acquire64(&B->word);
            if ((unsigned)(word >> 32) != tag) {
                const long long t0 = clock64();
                unsigned spins = 0;
                while ((unsigned)((word = ld_acquire64(&B->word)) >> 32) != tag) {
                    if (ld_acquire_i(dflag)) { st = 1; break; }
                    __nanosleep(spins < 16 ? 20 : 100);
                    if ((++spins & 31u) == 0) {
                        if (*(volatile int *)&ctl->abort) { st = 2; break; }
                        if (clock64() - t0 > c_wait_cycles) {
                            atomicExch(&ctl->abort, 1);
                            st = 2;
                            break;
                        }
                    }
                }
            }
            if (st == 0 && ((word >> 9) & 1u)) st = 1;
            if (st == 0) {
                s_view.step = (int)(word & 0xffu);
                s_view.par = (int)((word >> 8) & 1u);
                s_view.alpha = __ldcg(&B->alpha);
                s_view.beta = __ldcg(&B->beta);
                s_view.tick = tag;
                if (hd.cur != T.solve) {
                    hd.D = *Dp;
                    hd.cur = T.solve;
                }
            }
            s_flag = st;
        }
        __syncthreads();
        if (s_flag == 2) return;
        if (s_flag == 1) continue;
        if (MULTI) {
            if (hd.D.NC == 27) tile_step<27, NZM>(s_view, T.tile, false, TYmax, hd, smem);
            else tile_step<9, 1>(s_view, T.tile, false, TY2max, hd, smem);
        } else {
            tile_step<NC, NZM>(s_view, T.tile, false, TYmax, hd, smem);
        }
    }
    if (threadIdx.x == 0) s_flag = *(volatile int *)&ctl->abort;
    __syncthreads();
    if (s_flag) return;
    // a serving epoch ends: fold in the sums of the last steps so the next launch resumes exactly
    if (epoch_end)
        while (duty_step < max_steps) {
            if (!lead_duties(hd, descs, states, ctl)) return;
            ++duty_step;
        }
    if (threadIdx.x == 0)
        for (int cs = 0; cs < hd.nsolve; ++cs) *states[hd.sid[cs]] = hd.st[cs];
}

// ---------------------------------------------------------------------------
// setup kernels: FP32 matrix copy and FP32 preconditioner factors
// ---------------------------------------------------------------------------
// FP32 copy of the coefficient planes; couplings whose neighbour lies outside the
// array (which the reference skips) are stored as zero so the FP32 stencil loop needs
// no bounds tests.
template <int NC>
__global__ void k_to_f32(Geom g, const double *__restrict__ src, float4 *__restrict__ dst,
                         double2 *__restrict__ dst64) {
    const long long plane = (long long)g.nz * g.NQ;
    const long long n = (long long)NC * plane;  // one float4 (uu, uv, vu, vv) per coupling and node
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e / plane);
        const long long r = e % plane;
        const int k = (int)(r / g.NQ);
        const long long q = r % g.NQ;
        const int i = (int)(q % g.NX), j = (int)(q / g.NX);
        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = (NC == 27) ? c / 9 - 1 : 0;
        const bool in = i + iA >= 0 && i + iA < g.NX && j + jA >= 0 && j + jA < g.NY && k + kA >= 0 && k + kA < g.nz;
        const size_t bs = (size_t)NC * plane;  // FP64 planes [4][NC][nz][NQ]
        const double uu = in ? src[e] : 0.0, uv = in ? src[bs + e] : 0.0;
        const double vu = in ? src[2 * bs + e] : 0.0, vv = in ? src[3 * bs + e] : 0.0;
        dst[e] = make_float4((float)uu, (float)uv, (float)vu, (float)vv);
        if (dst64) {
            dst64[2 * e] = make_double2(uu, uv);
            dst64[2 * e + 1] = make_double2(vu, vv);
        }
    }
}

// Exact symmetry of a 3D system, the condition of the symmetric half storage: every lower
// coupling c < 13 of an owned active row R equals its transpose partner bit for bit -- Auu with
// Auu, Auv with Avu, Avu with Auv, Avv with Avv -- at the neighbour node n = R + (iA, jA, kA)
// and the opposite offset 26 - c.  check_symmetry_assembled_matrix_3d, which the reference runs
// before every 3D solve (glissade_velo_higher.F90:2923-2931), averages such pairs to equality.
// A difference, or a partner outside the array, sets *flag.  One thread per column.
__global__ void k_sym_exact3d(Geom g, const int32_t *__restrict__ act, const double *__restrict__ A, int *flag) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NQ) return;
    const int i = (int)(q % g.NX), j = (int)(q / g.NX);
    if (!owned(g, i, j) || act[q] == 0) return;
    const long long plane = (long long)g.nz * g.NQ, bs = 27 * plane;
    int bad = 0;
    for (int k = 0; k < g.nz && !bad; ++k)
        for (int c = 0; c < 13; ++c) {
            const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = c / 9 - 1;
            const int in = i + iA, jn = j + jA, kn = k + kA;
            if (kn < 0) continue;  // a coupling leaving the column: zero in both layouts
            if (in < 0 || in >= g.NX || jn < 0 || jn >= g.NY) { bad = 1; break; }
            const long long e = (long long)c * plane + (long long)k * g.NQ + q;
            const long long f = (long long)(26 - c) * plane + (long long)kn * g.NQ + (long long)jn * g.NX + in;
            if (A[e] != A[f] || A[bs + e] != A[2 * bs + f] || A[2 * bs + e] != A[bs + f] ||
                A[3 * bs + e] != A[3 * bs + f]) {
                bad = 1;
                break;
            }
        }
    if (bad) atomicOr(flag, 1);
}

// The symmetric half copy (3D): the 14 couplings c = 13..26 (the diagonal and the upper
// offsets) of every node, FP32 as float4 (uu, uv, vu, vv) in planes [c - 13][nz][NQ] and FP64
// interleaved as {uu, uv}, {vu, vv}; couplings leaving the array are stored as zero, as in
// k_to_f32.  The kernels read a lower coupling from its transpose partner.
__global__ void k_to_half(Geom g, const double *__restrict__ src, float4 *__restrict__ dst,
                          double2 *__restrict__ dst64) {
    const long long plane = (long long)g.nz * g.NQ;
    const long long n = 14 * plane;
    const size_t bs = (size_t)27 * plane;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int h = (int)(e / plane), c = 13 + h;
        const long long r = e % plane;
        const int k = (int)(r / g.NQ);
        const long long q = r % g.NQ;
        const int i = (int)(q % g.NX), j = (int)(q / g.NX);
        const int iA = c % 3 - 1, jA = (c / 3) % 3 - 1, kA = c / 9 - 1;
        const bool in = i + iA >= 0 && i + iA < g.NX && j + jA >= 0 && j + jA < g.NY && k + kA >= 0 && k + kA < g.nz;
        const size_t f = (size_t)c * plane + r;
        const double uu = in ? src[f] : 0.0, uv = in ? src[bs + f] : 0.0;
        const double vu = in ? src[2 * bs + f] : 0.0, vv = in ? src[3 * bs + f] : 0.0;
        dst[e] = make_float4((float)uu, (float)uv, (float)vu, (float)vv);
        dst64[2 * e] = make_double2(uu, uv);
        dst64[2 * e + 1] = make_double2(vu, vv);
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

// FP32 factors of the line preconditioners (precond 3, 4) from the FP64 setup's planes (k_tri_coef,
// k_tri_factor): [u, v][sub, 1/diag, omega, 1/denom][NQ], the u planes transposed (column i, row j
// at i*NY + j) for the coalesced u lines of lines_step.
__global__ void k_tri_to_f32(Geom g, const double *__restrict__ T, float *__restrict__ out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.NQ) return;
    const long long i = q % g.NX, j = q / g.NX, tq = i * g.NY + j;
    const int f[4] = {TU_SUB, TU_ADR, TU_OM, TU_DEN};
    for (int k = 0; k < 4; ++k) {
        out[k * g.NQ + tq] = (float)T[(long long)f[k] * g.NQ + q];
        out[(4 + k) * g.NQ + q] = (float)T[(long long)(f[k] - TU_SUB + TV_SUB) * g.NQ + q];
    }
}

// Device buffers of the mixed solver for one system (owned by the host Solver).
struct MixedBufs {
    bool valid = false;
    int TY = 0;                // tile height the slot maps were built for
    bool stale = false;        // the FP64 matrix changed since the FP32 copy was made
    long long shape_nvec = 0;
    int shape_nc = 0;
    int precond = -1;
    float4 *A32 = nullptr;
    double2 *A64i = nullptr;   // FP64 matrix interleaved per coupling (k_to_f32), or its symmetric half
    bool sym = false;          // A32 and A64i hold the symmetric half (k_to_half)
    bool il = false;           // A64i holds the full interleaved FP64 copy (streamed, not symmetric)
    int *flag = nullptr;       // device word of the symmetry test
    float *pre = nullptr, *vec = nullptr;
    float *tri = nullptr;      // precond 3, 4: line factors [8][NQ], rs [2][NQ], zs [2][NQ]
    int *maps = nullptr;
    int *nbrs = nullptr;
    TileRec *recs = nullptr;
    Bcast *bc = nullptr;       // [2][kBcastCopies] broadcast lines, then one line holding the done flag
    MState *state = nullptr;
    MDesc *desc = nullptr;
    MTile *tiles = nullptr;
    MCtl *ctl = nullptr;
    size_t nbytes = 0;
    int ntiles = 0;
    int ntiles_cap = 0;
    long long maps_cap = 0;
    void release() {
        for (void *p : {(void *)A32, (void *)A64i, (void *)pre, (void *)vec, (void *)recs, (void *)state, (void *)desc,
                        (void *)tiles, (void *)ctl, (void *)maps, (void *)nbrs, (void *)bc, (void *)flag, (void *)tri})
            if (p) cudaFree(p);
        tri = nullptr;
        A32 = nullptr;
        A64i = nullptr;
        flag = nullptr;
        sym = false;
        il = false;
        pre = vec = nullptr;
        maps = nullptr;
        nbrs = nullptr;
        ntiles = ntiles_cap = 0;
        maps_cap = 0;
        TY = 0;
        recs = nullptr;
        bc = nullptr;
        state = nullptr;
        desc = nullptr;
        tiles = nullptr;
        ctl = nullptr;
        nbytes = 0;
        valid = false;
        precond = -1;
    }
    size_t bytes() const { return nbytes; }
};

}  // namespace cismgpu
