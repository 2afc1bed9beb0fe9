// pcg_oracle.cpp -- CPU restatement of CISM's native structured PCG solve.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the timed
// CPU baseline for the B200 library; nothing in the product links or calls it.
// It may be used only by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline arm.
//
// PARITY STATUS: the reference is Fortran 90 and no Fortran compiler exists in
// this build environment, and the reference ships no golden vectors or
// known-answer tests for this path.  This restatement is therefore *unpinned*
// against reference outputs; it is pinned against mathematical known answers
// (dense solves, dense matvecs, Thomas vs dense) in tests/test_oracle_kat.py, and
// against a second restatement of the four solvers, their preconditioners, halo,
// matvecs, sums and the residual steps, written separately in Python from the
// reference source (tests/test_oracle_restatement.py), which it equals bit for bit.
//
// It restates, loop for loop and in the same floating-point operation order:
//   libglissade/glissade_velo_higher_pcg.F90
//     pcg_solver_standard_2d          :67-823
//     pcg_solver_standard_3d          :827-1537
//     pcg_solver_chrongear_2d         :1541-2628
//     pcg_solver_chrongear_3d         :2632-3594
//     setup_preconditioner_diag_3d    :3598-3643
//     setup_preconditioner_sia_3d     :3647-3733
//     setup_preconditioner_diag_2d    :4199-4243
//     setup_preconditioner_tridiag_local_3d   :3737-3926
//     setup_preconditioner_tridiag_global_3d  :3930-4195
//     setup_preconditioner_tridiag_local_2d   :4247-4392
//     setup_preconditioner_tridiag_global_2d  :4396-4520  (one task per row and column)
//     tridiag_solver_local_3d         :4524-4658
//     tridiag_solver_global_3d        :4662-4913  (one task: the particular solution)
//     tridiag_solver_local_2d         :4917-5100
//     tridiag_solver_global_2d        :5104-5524  (tasks_rc = 1 branch, :5495-5497)
//   libglissade/glissade_velo_higher.F90
//     compute_residual_vector_2d      :9502-9689
//     compute_residual_vector_3d      :9693-9894
//     compute_residual_velocity_2d    :10188-10310
//     compute_residual_velocity_3d    :10314-10446
//     matvec_multiply_structured_3d   :5528-5652
//     matvec_multiply_structured_2d   :5656-5773
//     easy_sia_solver                 :5777-5866
//     tridiag_solver                  :5870-5922
//   libglimmer/parallel_mpi.F90
//     parallel_global_sum_stagger_*   :6537-7063  (one rank: mpi_allreduce is the identity)
//     staggered_parallel_halo_real8_* :10609-11099 (one rank: periodic self-exchange, BC zero fill)
//
// Compile with -O2 -ffp-contract=off (gfortran on x86-64 does not contract a*b+c
// into an FMA; the reference Linux build uses -O2).
//
// Global sums have three modes:
//   ORACLE_SUM_SEQ    : the reference's non-reprosum order: local_sum = local_sum + arr1 + arr2,
//                       j outer, i, k inner over owned vertices (parallel_mpi.F90:6760-6790).
//   ORACLE_SUM_EXACT  : the exact sum of fl(arr1+arr2) over owned vertices, rounded once to
//                       nearest-even: an order-independent reproducible sum in the spirit of
//                       the reprosum branch (parallel_mpi.F90:6702-6758, cism_reprosum_mod.F90).
//   ORACLE_SUM_DDTREE : a restatement of the B200 library's fixed reduction tree (double-double
//                       column chunks of 256, warp and block trees); with it the whole solve is
//                       bit-identical to the GPU, which isolates summation order as the only
//                       source of difference against ORACLE_SUM_SEQ.
//   ORACLE_SUM_REPRO  : a restatement of the reference's reprosum branch as CISM calls it on one
//                       rank and one thread (parallel_reduce_reprosum, parallel_mpi.F90:9618-9725,
//                       cism_reprosum_calc and cism_reprosum_int, libglimmer/cism_reprosum_mod.F90:
//                       237-1057 and 1063-1818): the integer-vector fixed-point sum.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../include/cismgpu.h"

namespace {

enum { ORACLE_SUM_SEQ = 0, ORACLE_SUM_EXACT = 1, ORACLE_SUM_DDTREE = 2, ORACLE_SUM_REPRO = 3 };

// ---------------------------------------------------------------------------
// Exact summation: a Kulisch-style fixed-point accumulator over the whole
// double range, radix 2^32 digits held in int64 limbs (bit 0 = 2^-1074).
// ---------------------------------------------------------------------------
struct ExactAcc {
    static const int NLIMB = 72;  // 72*32 = 2304 bits > 1074 + 1024 + 64 headroom
    int64_t limb[NLIMB];
    ExactAcc() { std::memset(limb, 0, sizeof(limb)); }
    void add(double v) {
        if (v == 0.0) return;
        int e;
        double f = std::frexp(std::fabs(v), &e);  // |v| = f * 2^e, f in [0.5,1)
        // integer mantissa m = f*2^53, |v| = m * 2^(e-53); lsb exponent e-53 >= -1074
        int64_t m = (int64_t)std::ldexp(f, 53);
        int lsb = e - 53;
        if (lsb < -1074) {  // subnormal: shift mantissa so that lsb = -1074 (exact)
            m >>= (-1074 - lsb);
            lsb = -1074;
        }
        int shift = lsb + 1074;
        int li = shift / 32, off = shift % 32;
        unsigned __int128 w = ((unsigned __int128)(uint64_t)m) << off;
        int64_t sgn = v < 0 ? -1 : 1;
        for (int t = 0; t < 3 && li + t < NLIMB; ++t) {
            int64_t digit = (int64_t)(uint64_t)(w & 0xffffffffu);
            limb[li + t] += sgn * digit;
            w >>= 32;
        }
    }
    double result() const {
        // propagate carries into canonical signed digits
        std::vector<int64_t> d(limb, limb + NLIMB);
        for (int t = 0; t < NLIMB - 1; ++t) {
            int64_t c = d[t] >> 32;      // arithmetic shift: floor division
            d[t] -= c * ((int64_t)1 << 32);
            d[t + 1] += c;
        }
        bool neg = d[NLIMB - 1] < 0;
        if (neg) {  // negate the whole number: two's complement over digits
            for (int t = 0; t < NLIMB; ++t) d[t] = -d[t];
            for (int t = 0; t < NLIMB - 1; ++t) {
                int64_t c = d[t] >> 32;
                d[t] -= c * ((int64_t)1 << 32);
                d[t + 1] += c;
            }
        }
        // now all digits in [0, 2^32)
        int top = -1;
        for (int t = NLIMB - 1; t >= 0; --t) if (d[t] != 0) { top = t; break; }
        if (top < 0) return 0.0;
        int hb = 31;
        while (!((d[top] >> hb) & 1)) --hb;
        long P = (long)top * 32 + hb;  // index of the most significant set bit
        auto bit = [&](long idx) -> int {
            if (idx < 0) return 0;
            return (int)((d[idx / 32] >> (idx % 32)) & 1);
        };
        double res;
        if (P < 53) {
            uint64_t M = 0;
            for (long b = P; b >= 0; --b) M = (M << 1) | (uint64_t)bit(b);
            res = std::ldexp((double)M, -1074);
        } else {
            uint64_t M = 0;
            for (long b = P; b > P - 53; --b) M = (M << 1) | (uint64_t)bit(b);
            long low = P - 53;  // bits low..0 are the remainder
            int g = bit(low);
            bool sticky = false;
            for (long b = low - 1; b >= 0; --b)
                if (bit(b)) { sticky = true; break; }
            if (g && (sticky || (M & 1))) M += 1;
            res = std::ldexp((double)M, (int)(P - 52 - 1074));
        }
        return neg ? -res : res;
    }
};

// ---------------------------------------------------------------------------
// Double-double arithmetic, operation order identical to the device code.
// ---------------------------------------------------------------------------
struct DD { double hi, lo; };

inline DD dd_add_d(DD a, double x) {
    double s = a.hi + x;
    double bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (x - bb);
    e = e + a.lo;
    double hi = s + e;
    double lo = e - (hi - s);
    return DD{hi, lo};
}

inline DD dd_add(DD a, DD b) {
    double s = a.hi + b.hi;
    double bb = s - a.hi;
    double e = (a.hi - (s - bb)) + (b.hi - bb);
    e = e + (a.lo + b.lo);
    double hi = s + e;
    double lo = e - (hi - s);
    return DD{hi, lo};
}

// Restatement of the device reduction tree.  'col_sum(q)' must return, for
// column q (0-based, q = (i-1) + NX*(j-1)), the dd accumulation over its levels
// k = 1..nz in order; non-owned columns return {0,0}.
//   chunk = 256 columns; thread t of chunk c handles column c*256+t;
//   warp tree: for off = 16,8,4,2,1: v[l] = v[l] + v[l+off]  (l+off < 32 else own)
//   block tree over the 8 warp sums: for off = 4,2,1 (lanes >= 8 hold 0)
//   final: 256 "threads" accumulate chunk partials c = t, t+256, ... in order,
//          then the same warp and block trees.
template <class F>
double ddtree_reduce(long nq, F col_sum) {
    const int B = 256;
    long nchunk = (nq + B - 1) / B;
    auto block_tree = [](std::vector<DD> &v) -> DD {
        // v has 256 entries
        DD w[8];
        for (int wp = 0; wp < 8; ++wp) {
            DD lane[32];
            for (int l = 0; l < 32; ++l) lane[l] = v[wp * 32 + l];
            for (int off = 16; off >= 1; off >>= 1) {
                DD nxt[32];
                for (int l = 0; l < 32; ++l)
                    nxt[l] = (l + off < 32) ? dd_add(lane[l], lane[l + off]) : lane[l];
                std::memcpy(lane, nxt, sizeof(lane));
            }
            w[wp] = lane[0];
        }
        DD lane[32];
        for (int l = 0; l < 32; ++l) lane[l] = (l < 8) ? w[l] : DD{0.0, 0.0};
        for (int off = 4; off >= 1; off >>= 1) {
            DD nxt[32];
            for (int l = 0; l < 32; ++l)
                nxt[l] = (l + off < 32) ? dd_add(lane[l], lane[l + off]) : lane[l];
            std::memcpy(lane, nxt, sizeof(lane));
        }
        return lane[0];
    };
    std::vector<DD> partial(nchunk);
    std::vector<DD> v(B);
    for (long c = 0; c < nchunk; ++c) {
        for (int t = 0; t < B; ++t) {
            long q = c * B + t;
            v[t] = (q < nq) ? col_sum(q) : DD{0.0, 0.0};
        }
        partial[c] = block_tree(v);
    }
    for (int t = 0; t < B; ++t) {
        DD acc{0.0, 0.0};
        for (long c = t; c < nchunk; c += B) acc = dd_add(acc, partial[c]);
        v[t] = acc;
    }
    DD r = block_tree(v);
    return r.hi + r.lo;
}

// ---------------------------------------------------------------------------
// Grid and index helpers (Fortran column-major, 1-based)
// ---------------------------------------------------------------------------
struct Geom {
    int nz, NX, NY;  // NX = nx-1, NY = ny-1 vertices; nz = 1 for 2D
    long nq() const { return (long)NX * NY; }
    long ntot() const { return (long)nz * NX * NY; }
    // 3D vector element (k,i,j)
    long v3(int k, int i, int j) const { return (k - 1) + (long)nz * ((i - 1) + (long)NX * (j - 1)); }
    // 3D block element (m,k,i,j)
    long a3(int m, int k, int i, int j) const { return (m - 1) + 27L * v3(k, i, j); }
    // 2D vector element (i,j)
    long v2(int i, int j) const { return (i - 1) + (long)NX * (j - 1); }
    // 2D block element (i,j,m)
    long a2(int i, int j, int m) const { return (i - 1) + (long)NX * ((j - 1) + (long)NY * (m - 1)); }
};

struct Ctx {
    Geom g;
    cismgpu_par_t par;
    int summode;
    const int32_t *indx2;  // indxA_2d(-1:1,-1:1): (iA+1) + 3*(jA+1)
    const int32_t *indx3;  // indxA_3d(-1:1,-1:1,-1:1)
    const int32_t *active; // active_vertex(NX,NY)
    int I2(int iA, int jA) const { return indx2[(iA + 1) + 3 * (jA + 1)]; }
    int I3(int iA, int jA, int kA) const { return indx3[(iA + 1) + 3 * (jA + 1) + 9 * (kA + 1)]; }
    bool act(int i, int j) const { return active[(i - 1) + (long)g.NX * (j - 1)] != 0; }
    bool owned_col(long q) const {
        int i = (int)(q % g.NX) + 1, j = (int)(q / g.NX) + 1;
        return i >= par.staggered_ilo && i <= par.staggered_ihi &&
               j >= par.staggered_jlo && j <= par.staggered_jhi;
    }
};

typedef std::vector<double> Vec;

// parallel_global_sum_stagger (3D and 2D; nz = 1 for 2D), one field with arr2.
// Vectors are in Fortran layout (nz, NX, NY), so element (k, q) is at k-1 + nz*q.
// ---------------------------------------------------------------------------
// reprosum (libglimmer/cism_reprosum_mod.F90), one field, one rank, one OpenMP thread, called
// as parallel_reduce_reprosum does (parallel_mpi.F90:9691-9707): no global-max or level hints,
// so cism_reprosum_calc takes its "recompute" path (:442-525): exponent range of the nonzero
// summands, arr_max_shift from the summand count, max_levels from the range, then
// cism_reprosum_int with validate = .false.  Fortran intrinsics on IEEE doubles: exponent(x)
// and fraction(x) are frexp's exponent and mantissa, scale(x,n) = x*2^n, set_exponent(x,e) =
// fraction(x)*2^e; digits(1.0_r8) = 53, digits(1_i8) = 63, MINEXPONENT(1.0_r8) = -1021,
// MAXEXPONENT(1.0_r8) = 1024; int(x,i8) truncates; i8 division truncates toward zero.
// ---------------------------------------------------------------------------
inline int f_exponent(double x) { int e; std::frexp(x, &e); return e; }
inline double f_fraction(double x) { int e; return std::frexp(x, &e); }
inline double f_set_exponent(double x, int e) { return std::ldexp(f_fraction(x), e); }

double reprosum(const std::vector<double> &arr) {
    const int kDigR8 = 53, kDigI8 = 63, kMinExp = -1021, kMaxExp = 1024;
    const long nsummands = (long)arr.size();
    // Non-finite summands: the reference's NaN/Inf handling is commented out
    // (cism_reprosum_mod.F90:58-62) and int(x, i8) of a NaN or an infinity is processor
    // dependent, so its result is undefined there.  The library and this restatement both
    // return the IEEE sum of the non-finite summands (NaN, +Inf or -Inf), which keeps the
    // solvers' NaN breakdown tests meaningful.
    {
        bool nan = false, pinf = false, ninf = false;
        for (double x : arr) {
            if (x != x) nan = true;
            else if (x == HUGE_VAL) pinf = true;
            else if (x == -HUGE_VAL) ninf = true;
        }
        if (nan || (pinf && ninf)) return NAN;
        if (pinf) return HUGE_VAL;
        if (ninf) return -HUGE_VAL;
    }
    // exponent extremes of the nonzero summands (:455-487)
    int lmin = kMaxExp, lmax = kMinExp;
    for (double x : arr)
        if (x != 0.0) {
            const int e = f_exponent(x);
            lmin = std::min(e, lmin);
            lmax = std::max(e, lmax);
        }
    const int gmax = lmax;
    const int gmin = std::min(gmax, lmin);
    long max_nsummands = nsummands / 1 + 1;      // (max_nsummands/omp_nthreads) + 1 (:501)
    max_nsummands = std::max(max_nsummands, 1L); // max(., tasks*omp_nthreads)
    const int shift = kDigI8 - (f_exponent((double)max_nsummands) + 1);
    if (shift < 2) return NAN;                   // mpi_abort in the reference (:505-510)
    const int max_levels = 2 + (kDigR8 + (gmax - gmin)) / shift;
    const int extra_levels = (kDigI8 - 1) / shift;
    const int min_level = -(extra_levels - 1);
    const int64_t R = (int64_t)1 << shift;       // i8_radix**arr_max_shift
    // levels min_level..max_levels
    std::vector<int64_t> lv(max_levels - min_level + 1, 0);
    auto L = [&](int level) -> int64_t & { return lv[level - min_level]; };
    // integer expansion of every summand (:1199-1262)
    for (double x : arr) {
        if (x == 0.0) continue;
        const int e = f_exponent(x);
        const double f = f_fraction(x);
        int ashift = shift - (gmax - e);
        int ilevel;
        if (ashift < 1) {
            ilevel = (1 + (gmax - e)) / shift;
            ashift = ilevel * shift - (gmax - e);
            while (ashift < 1) {
                ashift += shift;
                ilevel += 1;
            }
        } else {
            ilevel = 1;
        }
        if (ilevel <= max_levels) {
            double rem = std::ldexp(f, ashift);
            int64_t v = (int64_t)rem;
            L(ilevel) += v;
            rem = rem - (double)v;
            while (rem != 0.0 && ilevel < max_levels) {
                ilevel += 1;
                rem = std::ldexp(rem, shift);
                v = (int64_t)rem;
                L(ilevel) += v;
                rem = rem - (double)v;
            }
        }
    }
    auto carry = [&]() {  // (:1266-1276, :1361-1371, :1403-1413)
        for (int l = max_levels; l >= min_level + 1; --l)
            if ((L(l) < 0 ? -L(l) : L(l)) >= R) {
                const int64_t ix = L(l) / R;
                L(l - 1) += ix;
                L(l) -= ix * R;
            }
    };
    carry();  // per thread
    carry();  // after the (one-rank) allreduce
    // sign and same-sign digits (:1373-1401)
    int ilevel = min_level;
    while (L(ilevel) == 0 && ilevel < max_levels) ++ilevel;
    const int64_t sgn = (L(ilevel) < 0) ? -1 : 1;
    auto fsign = [](int64_t v) -> int64_t { return v < 0 ? -1 : 1; };
    if (ilevel < max_levels)
        for (int j = ilevel; j <= max_levels - 1; ++j)
            if (fsign(L(j)) != fsign(L(j + 1)) || L(j + 1) == 0) {
                L(j) -= sgn;
                L(j + 1) += sgn * R;
            }
    if (sgn < 0)
        for (int j = ilevel; j <= max_levels; ++j) L(j) = -L(j);
    carry();
    // floating-point pieces of at most 53 digits each (:1415-1487)
    std::vector<double> sv;
    bool first = true;
    int ash = gmax - min_level * shift;
    int digit_count = 0;
    int begin_level = min_level;
    while (begin_level <= max_levels) {
        int trunc_loc = 0, trunc_level = max_levels;
        for (int l = begin_level; l <= max_levels; ++l) {
            int LX;
            if (first) {
                if (digit_count == 0) LX = (L(l) != 0) ? f_exponent((double)L(l)) : 0;
                else LX = shift;
            } else {
                LX = (l == begin_level && digit_count != 0) ? 0 : shift;
            }
            if (digit_count + LX >= kDigR8) {
                trunc_level = l;
                trunc_loc = (digit_count + LX) - kDigR8;
                break;
            }
            digit_count += LX;
        }
        first = false;
        int64_t trunc_rem = 0;
        if (trunc_loc != 0) {
            const int64_t P = (int64_t)1 << trunc_loc;
            int64_t ix = L(trunc_level) / P;
            ix = ix * P;
            trunc_rem = L(trunc_level) - ix;
            L(trunc_level) = ix;
        }
        double piece = 0.0;
        for (int l = begin_level; l <= trunc_level; ++l) {
            if (L(l) != 0) {
                const double X = (double)L(l);
                const int cur = f_exponent(X) + ash;
                if (cur >= kMinExp) piece = piece + f_set_exponent(X, cur);
                else piece = piece + std::ldexp(f_set_exponent(X, cur - kMinExp), kMinExp);
            }
            if (l < trunc_level || trunc_loc == 0) ash -= shift;
        }
        sv.push_back(piece);
        if (trunc_loc == 0) {
            digit_count = 0;
            begin_level = trunc_level + 1;
        } else {
            digit_count = trunc_loc;
            begin_level = trunc_level;
            L(trunc_level) = trunc_rem;
        }
    }
    // smallest to largest, then the sign (:1489-1495)
    double sum = 0.0;
    for (long j = (long)sv.size() - 1; j >= 0; --j) sum = sum + sv[j];
    return (double)sgn * sum;
}

double global_sum(const Ctx &c, const Vec &a1, const Vec &a2) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    if (c.summode == ORACLE_SUM_SEQ) {
        double local_sum = 0.0;
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i)
                for (int k = 1; k <= g.nz; ++k) {
                    long e = g.v3(k, i, j);
                    local_sum = local_sum + a1[e] + a2[e];
                }
        return local_sum;  // parallel_reduce_sum on one rank
    } else if (c.summode == ORACLE_SUM_REPRO) {  // parallel_mpi.F90:6703-6738: arr(count) = arr1 + arr2
        std::vector<double> arr;
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i)
                for (int k = 1; k <= g.nz; ++k) {
                    long e = g.v3(k, i, j);
                    arr.push_back(a1[e] + a2[e]);
                }
        return reprosum(arr);
    } else if (c.summode == ORACLE_SUM_EXACT) {
        ExactAcc acc;
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i)
                for (int k = 1; k <= g.nz; ++k) {
                    long e = g.v3(k, i, j);
                    acc.add(a1[e] + a2[e]);
                }
        return acc.result();
    } else {
        return ddtree_reduce(g.nq(), [&](long q) -> DD {
            if (!c.owned_col(q)) return DD{0.0, 0.0};
            DD acc{0.0, 0.0};
            for (int k = 0; k < g.nz; ++k) {
                long e = k + (long)g.nz * q;
                acc = dd_add_d(acc, a1[e] + a2[e]);
            }
            return acc;
        });
    }
}

// staggered_parallel_halo on one rank (parallel_mpi.F90:10772-10936), nz = 1 for 2D.
void halo(const Ctx &c, Vec &a) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    const int NX = g.NX, NY = g.NY, nz = g.nz;
    const int lh = 2, uh = 1;
    if (p.periodic_bc) {
        // east-west over owned rows j = jlo..jhi; sends are captured before receives land
        std::vector<double> wsend, esend;
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int k = 1; k <= nz; ++k) wsend.push_back(a[g.v3(k, 1 + lh, j)]);
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int ii = NX - uh - lh + 1; ii <= NX - uh; ++ii)
                for (int k = 1; k <= nz; ++k) esend.push_back(a[g.v3(k, ii, j)]);
        size_t n = 0;
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int k = 1; k <= nz; ++k) a[g.v3(k, NX, j)] = wsend[n++];
        n = 0;
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int ii = 1; ii <= lh; ++ii)
                for (int k = 1; k <= nz; ++k) a[g.v3(k, ii, j)] = esend[n++];
        // north-south over the full i range (after the east-west update)
        std::vector<double> ssend, nsend;
        for (int i = 1; i <= NX; ++i)
            for (int k = 1; k <= nz; ++k) ssend.push_back(a[g.v3(k, i, 1 + lh)]);
        for (int jj = NY - uh - lh + 1; jj <= NY - uh; ++jj)
            for (int i = 1; i <= NX; ++i)
                for (int k = 1; k <= nz; ++k) nsend.push_back(a[g.v3(k, i, jj)]);
        n = 0;
        for (int i = 1; i <= NX; ++i)
            for (int k = 1; k <= nz; ++k) a[g.v3(k, i, NY)] = ssend[n++];
        n = 0;
        for (int jj = 1; jj <= lh; ++jj)
            for (int i = 1; i <= NX; ++i)
                for (int k = 1; k <= nz; ++k) a[g.v3(k, i, jj)] = nsend[n++];
    }
    if (p.outflow_bc) {
        for (int j = 1; j <= NY; ++j)
            for (int k = 1; k <= nz; ++k) { a[g.v3(k, 1, j)] = 0.0; a[g.v3(k, NX, j)] = 0.0; }
        for (int i = 1; i <= NX; ++i)
            for (int k = 1; k <= nz; ++k) { a[g.v3(k, i, 1)] = 0.0; a[g.v3(k, i, NY)] = 0.0; }
    } else if (p.no_ice_bc) {
        for (int j = 1; j <= NY; ++j)
            for (int k = 1; k <= nz; ++k) {
                a[g.v3(k, 1, j)] = 0.0; a[g.v3(k, 2, j)] = 0.0;
                a[g.v3(k, NX - 1, j)] = 0.0; a[g.v3(k, NX, j)] = 0.0;
            }
        for (int i = 1; i <= NX; ++i)
            for (int k = 1; k <= nz; ++k) {
                a[g.v3(k, i, 1)] = 0.0; a[g.v3(k, i, 2)] = 0.0;
                a[g.v3(k, i, NY - 1)] = 0.0; a[g.v3(k, i, NY)] = 0.0;
            }
        // corner flags are false on a single rank (parallel_mpi.F90:2619-2622)
    }
}

// matvec_multiply_structured_3d, :5528-5652
void matvec3(const Ctx &c, const double *Auu, const double *Auv, const double *Avu, const double *Avv,
             const Vec &xu, const Vec &xv, Vec &yu, Vec &yv) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    std::fill(yu.begin(), yu.end(), 0.0);
    std::fill(yv.begin(), yv.end(), 0.0);
    for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
        for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i) {
            if (!c.act(i, j)) continue;
            for (int k = 1; k <= g.nz; ++k) {
                long e = g.v3(k, i, j);
                for (int kA = -1; kA <= 1; ++kA)
                    for (int jA = -1; jA <= 1; ++jA)
                        for (int iA = -1; iA <= 1; ++iA) {
                            if ((k + kA >= 1 && k + kA <= g.nz) && (i + iA >= 1 && i + iA <= g.NX) &&
                                (j + jA >= 1 && j + jA <= g.NY)) {
                                int m = c.I3(iA, jA, kA);
                                long a = g.a3(m, k, i, j);
                                long n = g.v3(k + kA, i + iA, j + jA);
                                yu[e] = yu[e] + Auu[a] * xu[n] + Auv[a] * xv[n];
                                yv[e] = yv[e] + Avu[a] * xu[n] + Avv[a] * xv[n];
                            }
                        }
            }
        }
}

// matvec_multiply_structured_2d, :5656-5773 (jA, iA outer; j, i inner)
void matvec2(const Ctx &c, const double *Auu, const double *Auv, const double *Avu, const double *Avv,
             const Vec &xu, const Vec &xv, Vec &yu, Vec &yv) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    std::fill(yu.begin(), yu.end(), 0.0);
    std::fill(yv.begin(), yv.end(), 0.0);
    for (int jA = -1; jA <= 1; ++jA)
        for (int iA = -1; iA <= 1; ++iA) {
            int m = c.I2(iA, jA);
            for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
                for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i) {
                    if (!c.act(i, j)) continue;
                    if ((i + iA >= 1 && i + iA <= g.NX) && (j + jA >= 1 && j + jA <= g.NY)) {
                        long e = g.v2(i, j);
                        long a = g.a2(i, j, m);
                        long n = g.v2(i + iA, j + jA);
                        yu[e] = yu[e] + Auu[a] * xu[n] + Auv[a] * xv[n];
                        yv[e] = yv[e] + Avu[a] * xu[n] + Avv[a] * xv[n];
                    }
                }
        }
}

// tridiag_solver, :5870-5922
void tridiag_solver(int order, const double *sbdiag, const double *diag, const double *spdiag,
                    const double *rhs, double *soln) {
    std::vector<double> gamma(order + 1);
    double beta = diag[0];
    soln[0] = rhs[0] / beta;
    for (int k = 2; k <= order; ++k) {
        gamma[k - 1] = spdiag[k - 2] / beta;
        beta = diag[k - 1] - sbdiag[k - 1] * gamma[k - 1];
        soln[k - 1] = (rhs[k - 1] - sbdiag[k - 1] * soln[k - 2]) / beta;
    }
    for (int k = order - 1; k >= 1; --k) soln[k - 1] = soln[k - 1] - gamma[k] * soln[k];
}

// easy_sia_solver, :5777-5866.  M is (-1:1, nz, NX, NY): element (l,k,i,j) at (l+1) + 3*v3(k,i,j).
void easy_sia_solver(const Ctx &c, const Vec &M, const Vec &b, Vec &x) {
    const Geom &g = c.g;
    const int nz = g.nz;
    std::vector<double> sb(nz), dg(nz), sp(nz), rhs(nz), soln(nz);
    for (int j = 1; j <= g.NY; ++j)
        for (int i = 1; i <= g.NX; ++i) {
            if (!c.act(i, j)) continue;
            for (int k = 1; k <= nz; ++k) { rhs[k - 1] = b[g.v3(k, i, j)]; soln[k - 1] = x[g.v3(k, i, j)]; }
            int k = 1;
            sb[k - 1] = 0.0;
            dg[k - 1] = M[1 + 3 * g.v3(k, i, j)];
            sp[k - 1] = M[2 + 3 * g.v3(k, i, j)];
            for (k = 2; k <= nz - 1; ++k) {
                sb[k - 1] = M[0 + 3 * g.v3(k, i, j)];
                dg[k - 1] = M[1 + 3 * g.v3(k, i, j)];
                sp[k - 1] = M[2 + 3 * g.v3(k, i, j)];
            }
            k = nz;
            sb[k - 1] = M[0 + 3 * g.v3(k, i, j)];
            dg[k - 1] = M[1 + 3 * g.v3(k, i, j)];
            sp[k - 1] = 0.0;
            tridiag_solver(nz, sb.data(), dg.data(), sp.data(), rhs.data(), soln.data());
            for (int kk = 1; kk <= nz; ++kk) x[g.v3(kk, i, j)] = soln[kk - 1];
        }
}

// Tridiagonal line factors on an (NX, NY) plane, index v2(i,j): the u system runs along
// rows (i), the v system along columns (j).  adr = 1/diag after the zero-diagonal fix.
struct TriLines {
    Vec sub, dg, sp, adr, omega, denom;
};

// Preconditioner state for one solve.
struct Precond {
    int kind;      // 0 none, 1 diag, 2 sia, 3/4 tridiag local/global, other: no branch taken
    Vec Adu, Adv;  // diagonal entries (diag)
    Vec Muu, Mvv;  // (-1:1, nz, NX, NY) (sia; also the vertical part of 3D tridiag)
    TriLines tu, tv;
};

// Line factorization over the owned range (setup_preconditioner_tridiag_local_2d
// :4324-4342 / :4361-4379; the global form :4441-4470 computes the same omega and denom on
// the owned block and, with one task, also runs the reverse recurrence only for its
// zero-pivot check :4472-4488).  along_i: lines are rows j, else columns i.
int tri_factor(const Ctx &c, TriLines &t, bool along_i, bool global) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    const int l0 = along_i ? p.staggered_jlo : p.staggered_ilo, l1 = along_i ? p.staggered_jhi : p.staggered_ihi;
    const int s0 = along_i ? p.staggered_ilo : p.staggered_jlo, s1 = along_i ? p.staggered_ihi : p.staggered_jhi;
    auto at = [&](int line, int s) { return along_i ? g.v2(s, line) : g.v2(line, s); };
    for (int l = l0; l <= l1; ++l) {
        t.omega[at(l, s0)] = t.sp[at(l, s0)] / t.dg[at(l, s0)];
        for (int s = s0 + 1; s <= s1; ++s) {
            const long e = at(l, s);
            double den = t.dg[e] - t.sub[e] * t.omega[at(l, s - 1)];
            if (den == 0.0) return CISMGPU_EDIVZERO;
            t.denom[e] = 1.0 / den;
            t.omega[e] = t.sp[e] * t.denom[e];
        }
        if (global) {
            double om = t.sub[at(l, s1)] / t.dg[at(l, s1)];
            for (int s = s1 - 1; s >= s0; --s) {
                const long e = at(l, s);
                double den_uh = t.dg[e] - t.sp[e] * om;
                if (den_uh == 0.0) return CISMGPU_EDIVZERO;
                om = t.sub[e] / den_uh;
            }
        }
    }
    return CISMGPU_OK;
}

// Coefficients of one line system from a 9-entry plane accessor A(i,j,m): sub/diag/super at
// indxA_2d (-1,0),(0,0),(1,0) for u and (0,-1),(0,0),(0,1) for v; zero diagonals become 1
// with zero off-diagonals (:4306-4313, :4349-4356); omega = denom = 0; adr = 1/diag (:4347).
template <class F>
void tri_coefs(const Ctx &c, TriLines &t, bool along_i, F A) {
    const Geom &g = c.g;
    const long n = g.nq();
    t.sub.assign(n, 0.0); t.dg.assign(n, 0.0); t.sp.assign(n, 0.0);
    t.adr.assign(n, 0.0); t.omega.assign(n, 0.0); t.denom.assign(n, 0.0);
    const int ms = along_i ? c.I2(-1, 0) : c.I2(0, -1), md = c.I2(0, 0), mp = along_i ? c.I2(1, 0) : c.I2(0, 1);
    for (int j = 1; j <= g.NY; ++j)
        for (int i = 1; i <= g.NX; ++i) {
            const long e = g.v2(i, j);
            t.sub[e] = A(i, j, ms);
            t.dg[e] = A(i, j, md);
            t.sp[e] = A(i, j, mp);
            if (t.dg[e] == 0.0) { t.dg[e] = 1.0; t.sub[e] = 0.0; t.sp[e] = 0.0; }
        }
    for (long e = 0; e < n; ++e) t.adr[e] = 1.0 / t.dg[e];
}

// tridiag_solver_local_2d :4985-5013 (u) / :5041-5069 (v) on plane b -> x.  The local form
// back-substitutes down to index 1 (halo entries below the owned range: gamma = omega = 0);
// the global form with one task keeps the owned particular solution and zero elsewhere.
void tri_solve(const Ctx &c, const TriLines &t, bool along_i, bool global, const double *b, double *x) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    const int l0 = along_i ? p.staggered_jlo : p.staggered_ilo, l1 = along_i ? p.staggered_jhi : p.staggered_ihi;
    const int s0 = along_i ? p.staggered_ilo : p.staggered_jlo, s1 = along_i ? p.staggered_ihi : p.staggered_jhi;
    auto at = [&](int line, int s) { return along_i ? g.v2(s, line) : g.v2(line, s); };
    for (long e = 0; e < g.nq(); ++e) x[e] = 0.0;
    std::vector<double> gam((along_i ? g.NX : g.NY) + 1, 0.0);
    for (int l = l0; l <= l1; ++l) {
        std::fill(gam.begin(), gam.end(), 0.0);
        gam[s0] = b[at(l, s0)] * t.adr[at(l, s0)];
        for (int s = s0 + 1; s <= s1; ++s) {
            const long e = at(l, s);
            gam[s] = (b[e] - t.sub[e] * gam[s - 1]) * t.denom[e];
        }
        x[at(l, s1)] = gam[s1];
        const int send = global ? s0 : 1;
        for (int s = s1 - 1; s >= send; --s) {
            const long e = at(l, s);
            x[e] = gam[s] - t.omega[e] * x[at(l, s + 1)];
        }
    }
}

int setup_precond(const Ctx &c, bool is3d, int precond, const double *Auu, const double *Avv, Precond &P) {
    const Geom &g = c.g;
    P.kind = precond;
    const bool tri = (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL);
    const bool global = (precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL);
    if (precond == CISMGPU_PRECOND_DIAG) {
        P.Adu.assign(g.ntot(), 0.0);
        P.Adv.assign(g.ntot(), 0.0);
        if (is3d) {  // setup_preconditioner_diag_3d :3639-3641
            int m = c.I3(0, 0, 0);
            for (int j = 1; j <= g.NY; ++j)
                for (int i = 1; i <= g.NX; ++i)
                    for (int k = 1; k <= g.nz; ++k) {
                        P.Adu[g.v3(k, i, j)] = Auu[g.a3(m, k, i, j)];
                        P.Adv[g.v3(k, i, j)] = Avv[g.a3(m, k, i, j)];
                    }
        } else {     // setup_preconditioner_diag_2d :4239-4241
            int m = c.I2(0, 0);
            for (int j = 1; j <= g.NY; ++j)
                for (int i = 1; i <= g.NX; ++i) {
                    P.Adu[g.v2(i, j)] = Auu[g.a2(i, j, m)];
                    P.Adv[g.v2(i, j)] = Avv[g.a2(i, j, m)];
                }
        }
    } else if (tri && !is3d) {  // setup_preconditioner_tridiag_{local,global}_2d
        tri_coefs(c, P.tu, true, [&](int i, int j, int m) { return Auu[g.a2(i, j, m)]; });
        tri_coefs(c, P.tv, false, [&](int i, int j, int m) { return Avv[g.a2(i, j, m)]; });
        int st = tri_factor(c, P.tu, true, global);
        if (st) return st;
        st = tri_factor(c, P.tv, false, global);
        if (st) return st;
    }
    if ((precond == CISMGPU_PRECOND_SIA || tri) && is3d) {  // setup_preconditioner_sia_3d :3686-3727
        P.Muu.assign(3 * g.ntot(), 0.0);
        P.Mvv.assign(3 * g.ntot(), 0.0);
        for (int j = 1; j <= g.NY; ++j)
            for (int i = 1; i <= g.NX; ++i)
                for (int k = 1; k <= g.nz; ++k) {
                    long e = g.v3(k, i, j);
                    int m = c.I3(0, 0, -1);
                    P.Muu[0 + 3 * e] = Auu[g.a3(m, k, i, j)];
                    P.Mvv[0 + 3 * e] = Avv[g.a3(m, k, i, j)];
                    m = c.I3(0, 0, 0);
                    P.Muu[1 + 3 * e] = Auu[g.a3(m, k, i, j)];
                    P.Mvv[1 + 3 * e] = Avv[g.a3(m, k, i, j)];
                    m = c.I3(0, 0, 1);
                    P.Muu[2 + 3 * e] = Auu[g.a3(m, k, i, j)];
                    P.Mvv[2 + 3 * e] = Avv[g.a3(m, k, i, j)];
                }
    }
    if (tri && is3d) {
        // vertical sums of the 9 horizontal couplings over the 3 vertical offsets and all
        // levels, raw m, m+9, m+18 (:3809-3821 / :4011-4023); inactive columns: the local form
        // zeroes the 9 sums and sets m = 5 to 1 (:3823-3833), the global form only sets m = 5
        // to 1 (:4025-4032) and then runs the staggered halo update on each summed plane
        // (:4055-4058), whose no_ice zeroing reaches the last owned row and column
        const long nq = g.nq();
        Vec su(9 * nq), sv(9 * nq);
        for (int j = 1; j <= g.NY; ++j)
            for (int i = 1; i <= g.NX; ++i)
                for (int m = 1; m <= 9; ++m) {
                    double au = 0.0, av = 0.0;
                    for (int k = 1; k <= g.nz; ++k) {
                        au = au + Auu[g.a3(m, k, i, j)] + Auu[g.a3(m + 9, k, i, j)] + Auu[g.a3(m + 18, k, i, j)];
                        av = av + Avv[g.a3(m, k, i, j)] + Avv[g.a3(m + 9, k, i, j)] + Avv[g.a3(m + 18, k, i, j)];
                    }
                    su[(m - 1) * nq + g.v2(i, j)] = au;
                    sv[(m - 1) * nq + g.v2(i, j)] = av;
                }
        for (int j = 1; j <= g.NY; ++j)
            for (int i = 1; i <= g.NX; ++i) {
                if (c.act(i, j)) continue;
                for (int m = 1; m <= 9; ++m)
                    if (!global || m == 5) {
                        su[(m - 1) * nq + g.v2(i, j)] = (m == 5) ? 1.0 : 0.0;
                        sv[(m - 1) * nq + g.v2(i, j)] = (m == 5) ? 1.0 : 0.0;
                    }
            }
        if (global) {
            Ctx c2 = c;
            c2.g.nz = 1;  // (NX, NY) planes
            for (int m = 0; m < 9; ++m) {
                Vec pu(su.begin() + m * nq, su.begin() + (m + 1) * nq);
                Vec pv(sv.begin() + m * nq, sv.begin() + (m + 1) * nq);
                halo(c2, pu);
                halo(c2, pv);
                std::copy(pu.begin(), pu.end(), su.begin() + m * nq);
                std::copy(pv.begin(), pv.end(), sv.begin() + m * nq);
            }
        }
        tri_coefs(c, P.tu, true, [&](int i, int j, int m) { return su[(m - 1) * nq + g.v2(i, j)]; });
        tri_coefs(c, P.tv, false, [&](int i, int j, int m) { return sv[(m - 1) * nq + g.v2(i, j)]; });
        int st = tri_factor(c, P.tu, true, global);
        if (st) return st;
        st = tri_factor(c, P.tv, false, global);
        if (st) return st;
    }
    return CISMGPU_OK;
}

// z = PC(r), applied over the whole array (halo included), :1231-1263 / :460-480.
void apply_precond(const Ctx &c, bool is3d, const Precond &P, const Vec &ru, const Vec &rv, Vec &zu, Vec &zv) {
    const long n = c.g.ntot();
    if (P.kind == CISMGPU_PRECOND_NONE) {
        zu = ru;
        zv = rv;
    } else if (P.kind == CISMGPU_PRECOND_DIAG) {
        for (long e = 0; e < n; ++e) {
            zu[e] = (P.Adu[e] != 0.0) ? ru[e] / P.Adu[e] : 0.0;
            zv[e] = (P.Adv[e] != 0.0) ? rv[e] / P.Adv[e] : 0.0;
        }
    } else if (P.kind == CISMGPU_PRECOND_SIA && is3d) {
        easy_sia_solver(c, P.Muu, ru, zu);
        easy_sia_solver(c, P.Mvv, rv, zv);
    } else if (P.kind == CISMGPU_PRECOND_TRIDIAG_LOCAL || P.kind == CISMGPU_PRECOND_TRIDIAG_GLOBAL) {
        const bool global = (P.kind == CISMGPU_PRECOND_TRIDIAG_GLOBAL);
        const Geom &g = c.g;
        Ctx c2 = c;
        c2.g.nz = 1;  // (NX, NY) planes
        if (!is3d) {  // line solves, then halo(z) (:502-531 / :533-617)
            tri_solve(c2, P.tu, true, global, ru.data(), zu.data());
            tri_solve(c2, P.tv, false, global, rv.data(), zv.data());
            halo(c2, zu);
            halo(c2, zv);
        } else {  // tridiag_solver_{local,global}_3d: vertical sums of r (sum(ru(:,i,j))), line
                  // solves, halo of the summed solution, SIA columns, z += summed solution
            const long nq = g.nq();
            Vec rsu(nq), rsv(nq), zsu(nq), zsv(nq);
            for (int j = 1; j <= g.NY; ++j)
                for (int i = 1; i <= g.NX; ++i) {
                    double a = 0.0, b = 0.0;
                    for (int k = 1; k <= g.nz; ++k) { a = a + ru[g.v3(k, i, j)]; b = b + rv[g.v3(k, i, j)]; }
                    rsu[g.v2(i, j)] = a;
                    rsv[g.v2(i, j)] = b;
                }
            tri_solve(c2, P.tu, true, global, rsu.data(), zsu.data());
            tri_solve(c2, P.tv, false, global, rsv.data(), zsv.data());
            halo(c2, zsu);
            halo(c2, zsv);
            easy_sia_solver(c, P.Muu, ru, zu);
            easy_sia_solver(c, P.Mvv, rv, zv);
            for (int j = 1; j <= g.NY; ++j)
                for (int i = 1; i <= g.NX; ++i)
                    for (int k = 1; k <= g.nz; ++k) {
                        zu[g.v3(k, i, j)] = zu[g.v3(k, i, j)] + zsu[g.v2(i, j)];
                        zv[g.v3(k, i, j)] = zv[g.v3(k, i, j)] + zsv[g.v2(i, j)];
                    }
        }
    }
    // any other value: no branch taken, z keeps its contents (as in the reference)
}

inline void mul(const Vec &a, const Vec &b, Vec &out) {
    for (size_t e = 0; e < a.size(); ++e) out[e] = a[e] * b[e];
}

int check_args(int nx, int ny, int nz, const cismgpu_par_t *par, int precond, int ncheck, int maxiters) {
    (void)precond;  // every value is accepted: 0-4 have branches, others take none
    if (!par || nx < 5 || ny < 5 || nz < 1) return CISMGPU_EINVAL;
    if (ncheck < 1) return CISMGPU_EINVAL;
    if (maxiters < 0) return CISMGPU_EINVAL;
    if (par->tasks_row * par->tasks_col != 1) return CISMGPU_EUNSUPPORTED;
    if (par->staggered_ilo < 1 || par->staggered_ihi > nx - 1 || par->staggered_ilo > par->staggered_ihi ||
        par->staggered_jlo < 1 || par->staggered_jhi > ny - 1 || par->staggered_jlo > par->staggered_jhi)
        return CISMGPU_EINVAL;
    return CISMGPU_OK;
}

// pcg_solver_standard_{2d,3d}: :67-823 and :827-1537
int standard(bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx2,
             const int32_t *indx3, const int32_t *active, const double *Auu, const double *Auv,
             const double *Avu, const double *Avv, const double *bu_, const double *bv_, double *xu_,
             double *xv_, int precond, int ncheck, double tol, int maxiters, double *err, int *niters,
             int summode) {
    int st = check_args(nx, ny, nz, par, precond, ncheck, maxiters);
    if (st) return st;
    Ctx c{Geom{is3d ? nz : 1, nx - 1, ny - 1}, *par, summode, indx2, indx3, active};
    const long n = c.g.ntot();
    Vec bu(bu_, bu_ + n), bv(bv_, bv_ + n), xu(xu_, xu_ + n), xv(xv_, xv_ + n);
    Vec ru(n), rv(n), du(n), dv(n), qu(n), qv(n), zu(n, 0.0), zv(n, 0.0), w0u(n), w0v(n);
    Precond P;
    *err = NAN;  // intent(out) and never set when no check runs; NaN makes that visible
    *niters = maxiters;
    st = setup_precond(c, is3d, precond, Auu, Avv, P);
    if (st) return st;  // GM_FATAL in the reference: x unchanged
    auto matvec = [&](const Vec &a, const Vec &b, Vec &ya, Vec &yb) {
        if (is3d) matvec3(c, Auu, Auv, Avu, Avv, a, b, ya, yb);
        else matvec2(c, Auu, Auv, Avu, Avv, a, b, ya, yb);
    };
    int status = CISMGPU_OK;

    halo(c, xu); halo(c, xv);
    matvec(xu, xv, zu, zv);
    for (long e = 0; e < n; ++e) { ru[e] = bu[e] - zu[e]; rv[e] = bv[e] - zv[e]; }
    *niters = maxiters;
    double eta0 = 1.0, eta1, eta2, alpha, beta;
    std::fill(du.begin(), du.end(), 0.0); std::fill(dv.begin(), dv.end(), 0.0);
    std::fill(zu.begin(), zu.end(), 0.0); std::fill(zv.begin(), zv.end(), 0.0);
    mul(bu, bu, w0u); mul(bv, bv, w0v);
    double L2_rhs = std::sqrt(global_sum(c, w0u, w0v));

    for (int iter = 1; iter <= maxiters; ++iter) {
        apply_precond(c, is3d, P, ru, rv, zu, zv);
        mul(ru, zu, w0u); mul(rv, zv, w0v);
        eta1 = global_sum(c, w0u, w0v);
        if (eta1 != eta1) { status = CISMGPU_EBREAKDOWN_ETA1; *niters = iter; break; }
        beta = eta1 / eta0;
        for (long e = 0; e < n; ++e) { du[e] = zu[e] + beta * du[e]; dv[e] = zv[e] + beta * dv[e]; }
        halo(c, du); halo(c, dv);
        matvec(du, dv, qu, qv);
        eta0 = eta1;
        mul(du, qu, w0u); mul(dv, qv, w0v);
        eta2 = global_sum(c, w0u, w0v);
        alpha = eta1 / eta2;
        if (alpha != alpha) { status = CISMGPU_EBREAKDOWN_ALPHA; *niters = iter; break; }
        for (long e = 0; e < n; ++e) {
            xu[e] = xu[e] + alpha * du[e]; xv[e] = xv[e] + alpha * dv[e];
            ru[e] = ru[e] - alpha * qu[e]; rv[e] = rv[e] - alpha * qv[e];
        }
        if (iter % ncheck == 0 || iter == 5) {
            halo(c, xu); halo(c, xv);
            matvec(xu, xv, zu, zv);
            for (long e = 0; e < n; ++e) { ru[e] = bu[e] - zu[e]; rv[e] = bv[e] - zv[e]; }
            mul(ru, ru, w0u); mul(rv, rv, w0v);
            double L2_resid = std::sqrt(global_sum(c, w0u, w0v));
            *err = L2_resid / L2_rhs;
            if (*err < tol) { *niters = iter; break; }
        }
    }
    std::memcpy(xu_, xu.data(), n * sizeof(double));
    std::memcpy(xv_, xv.data(), n * sizeof(double));
    return status;
}

// pcg_solver_chrongear_{2d,3d}: :1541-2628 and :2632-3594
int chrongear(bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx2,
              const int32_t *indx3, const int32_t *active, const double *Auu, const double *Auv,
              const double *Avu, const double *Avv, const double *bu_, const double *bv_, double *xu_,
              double *xv_, int precond, int ncheck, double tol, int maxiters, double *err, int *niters,
              int summode) {
    int st = check_args(nx, ny, nz, par, precond, ncheck, maxiters);
    if (st) return st;
    Ctx c{Geom{is3d ? nz : 1, nx - 1, ny - 1}, *par, summode, indx2, indx3, active};
    const long n = c.g.ntot();
    Vec bu(bu_, bu_ + n), bv(bv_, bv_ + n), xu(xu_, xu_ + n), xv(xv_, xv_ + n);
    Vec ru(n, 0.0), rv(n, 0.0), du(n, 0.0), dv(n, 0.0), zu(n, 0.0), zv(n, 0.0), qu(n, 0.0), qv(n, 0.0);
    Vec Azu(n, 0.0), Azv(n, 0.0), wu(n, 0.0), wv(n, 0.0), w1u(n), w1v(n), w2u(n), w2v(n);
    Precond P;
    // 2D with a tridiagonal preconditioner: at most 100 iterations (:1704-1732); 3D keeps
    // maxiters (:2896-2909)
    const bool tri = (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL);
    const int maxiters_chrongear = (tri && !is3d) ? 100 : maxiters;
    *err = NAN;
    *niters = maxiters_chrongear;
    st = setup_precond(c, is3d, precond, Auu, Avv, P);
    if (st) return st;  // GM_FATAL in the reference: x unchanged
    auto matvec = [&](const Vec &a, const Vec &b, Vec &ya, Vec &yb) {
        if (is3d) matvec3(c, Auu, Auv, Avu, Avv, a, b, ya, yb);
        else matvec2(c, Auu, Auv, Avu, Avv, a, b, ya, yb);
    };
    int status = CISMGPU_OK;

    mul(bu, bu, wu); mul(bv, bv, wv);
    double bb = global_sum(c, wu, wv);
    double L2_rhs = std::sqrt(bb);

    // first pass
    halo(c, xu); halo(c, xv);
    matvec(xu, xv, zu, zv);
    for (long e = 0; e < n; ++e) { ru[e] = bu[e] - zu[e]; rv[e] = bv[e] - zv[e]; }
    halo(c, ru); halo(c, rv);
    apply_precond(c, is3d, P, ru, rv, zu, zv);
    mul(ru, zu, w1u); mul(rv, zv, w1v);
    du = zu; dv = zv;
    matvec(du, dv, qu, qv);
    mul(du, qu, w2u); mul(dv, qv, w2v);
    double rho_old = global_sum(c, w1u, w1v);
    double sigma = global_sum(c, w2u, w2v);
    halo(c, qu); halo(c, qv);
    double alpha = rho_old / sigma;
    if (alpha != alpha) {
        status = CISMGPU_EBREAKDOWN_ALPHA;
        *niters = 1;
    } else {
        for (long e = 0; e < n; ++e) {
            xu[e] = xu[e] + alpha * du[e]; xv[e] = xv[e] + alpha * dv[e];
            ru[e] = ru[e] - alpha * qu[e]; rv[e] = rv[e] - alpha * qv[e];
        }
        for (int iter = 2; iter <= maxiters_chrongear; ++iter) {
            apply_precond(c, is3d, P, ru, rv, zu, zv);
            matvec(zu, zv, Azu, Azv);
            mul(ru, zu, w1u); mul(rv, zv, w1v);
            mul(Azu, zu, w2u); mul(Azv, zv, w2v);
            double rho = global_sum(c, w1u, w1v);
            double delta = global_sum(c, w2u, w2v);
            halo(c, Azu); halo(c, Azv);
            double beta = rho / rho_old;
            sigma = delta - beta * rho / alpha;
            alpha = rho / sigma;
            rho_old = rho;
            if (alpha != alpha) { status = CISMGPU_EBREAKDOWN_ALPHA; *niters = iter; break; }
            for (long e = 0; e < n; ++e) {
                du[e] = zu[e] + beta * du[e]; dv[e] = zv[e] + beta * dv[e];
                qu[e] = Azu[e] + beta * qu[e]; qv[e] = Azv[e] + beta * qv[e];
                xu[e] = xu[e] + alpha * du[e]; xv[e] = xv[e] + alpha * dv[e];
                ru[e] = ru[e] - alpha * qu[e]; rv[e] = rv[e] - alpha * qv[e];
            }
            if (iter % ncheck == 0 || iter == 5) {
                matvec(xu, xv, zu, zv);
                for (long e = 0; e < n; ++e) { ru[e] = bu[e] - zu[e]; rv[e] = bv[e] - zv[e]; }
                mul(ru, ru, wu); mul(rv, rv, wv);
                double rr = global_sum(c, wu, wv);
                *err = std::sqrt(rr) / L2_rhs;
                if (*err < tol) { *niters = iter; break; }
                halo(c, ru); halo(c, rv);
            }
        }
    }
    std::memcpy(xu_, xu.data(), n * sizeof(double));
    std::memcpy(xv_, xv.data(), n * sizeof(double));
    return status;
}

// compute_residual_vector_{2d,3d}: resid = A u - b on owned active vertices (the matvec
// statements of matvec_multiply_structured_*, which the residual loops repeat), the L2 norm
// of resid and |b| over owned active vertices through the global sum of the given mode.
void resid_vector(const Ctx &c, bool is3d, const double *Auu, const double *Auv, const double *Avu,
                  const double *Avv, const Vec &bu, const Vec &bv, const Vec &u, const Vec &v, Vec &ru, Vec &rv,
                  double *L2, double *L2rel) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    const long n = g.ntot();
    Vec yu(n, 0.0), yv(n, 0.0);
    if (is3d) matvec3(c, Auu, Auv, Avu, Avv, u, v, yu, yv);
    else matvec2(c, Auu, Auv, Avu, Avv, u, v, yu, yv);
    ru.assign(n, 0.0);
    rv.assign(n, 0.0);
    Vec wu(n, 0.0), wv(n, 0.0), bu2(n, 0.0), bv2(n, 0.0);
    for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
        for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i) {
            if (!c.act(i, j)) continue;
            for (int k = 1; k <= g.nz; ++k) {
                const long e = g.v3(k, i, j);
                ru[e] = yu[e] - bu[e];
                rv[e] = yv[e] - bv[e];
                wu[e] = ru[e] * ru[e];
                wv[e] = rv[e] * rv[e];
                bu2[e] = bu[e] * bu[e];
                bv2[e] = bv[e] * bv[e];
            }
        }
    *L2 = std::sqrt(global_sum(c, wu, wv));
    const double L2b = std::sqrt(global_sum(c, bu2, bv2));
    *L2rel = (L2b > 0.0) ? *L2 / L2b : 0.0;
}

// compute_residual_velocity_{2d,3d}: whichresid 1 (max, bed left out in 3D), 2 (mean, bed
// left out in 3D), anything else (max over all levels).  The mean's sum follows the mode:
// SEQ is the reference's j, i, k order; DDTREE and EXACT as the global sums.
double resid_velocity(const Ctx &c, bool is3d, int whichresid, const Vec &u, const Vec &v, const Vec &us,
                      const Vec &vs) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    const bool mean = whichresid == CISMGPU_RESID_MEANU;
    const int kmax = (is3d && (whichresid == CISMGPU_RESID_MAXU_NO_UBAS || mean)) ? g.nz - 1 : g.nz;
    auto diff = [&](long e, double &d) {
        const double speed = std::sqrt(u[e] * u[e] + v[e] * v[e]);
        if (speed == 0.0) return false;
        const double old = std::sqrt(us[e] * us[e] + vs[e] * vs[e]);
        d = std::fabs((old - speed) / speed);
        return true;
    };
    double r = 0.0;
    if (!mean) {
        for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
            for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i)
                for (int k = 1; k <= kmax; ++k) {
                    double d;
                    if (diff(g.v3(k, i, j), d) && d > r) r = d;
                }
        return r;
    }
    long count = 0;
    Vec w(g.ntot(), 0.0), z(g.ntot(), 0.0);
    for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
        for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i)
            for (int k = 1; k <= kmax; ++k) {
                double d;
                if (diff(g.v3(k, i, j), d)) {
                    ++count;
                    r = r + d;
                    w[g.v3(k, i, j)] = d;
                }
            }
    if (c.summode != ORACLE_SUM_SEQ) r = global_sum(c, w, z);  // the other modes' order (d + 0 = d)
    if (count > 0) r = r / (double)count;
    return r;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI of the oracle (same argument lists as include/cismgpu.h plus a sum mode)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// check_symmetry_assembled_matrix_{3d,2d} (glissade_velo_higher.F90:10648-10850 and
// :10854-11117): every owned active row compares each coefficient with its transpose partner
// (Auu with Auu^T, Auv with Avu^T, Avv with Avv^T, Avu with Auv^T).  A visit whose two values
// differ raises maxdiff to |val2 - val1| and either averages the pair, when the difference is
// below eps11 (glimmer_paramets.F90:77, 1e-11) times |diag| of the visited row's block (Auu's
// diagonal for the Auu and Auv checks, Avv's for Avv and Avu), or prints a warning.  The 3D
// check writes the averages in place; the 2D check only reports (its averaging is commented
// out).  nwarn counts the asymmetry warnings.  A partner outside the arrays (an owned row at
// the array edge) is skipped; the reference would read outside its arrays there.
// ---------------------------------------------------------------------------
constexpr double kEps11 = 1.0e-11;

struct SymCheck {
    double maxdiff = 0.0;
    long nwarn = 0;
};

inline void sym_visit(SymCheck &r, double &x1, double &x2, double diag, bool fix) {
    const double val1 = x1, val2 = x2;
    if (val2 != val1) {
        if (std::fabs(val2 - val1) > r.maxdiff) r.maxdiff = std::fabs(val2 - val1);
        if (std::fabs(val2 - val1) < kEps11 * std::fabs(diag)) {
            if (fix) {
                const double avg = 0.5 * (val1 + val2);
                x1 = avg;
                x2 = avg;
            }
        } else {
            ++r.nwarn;
        }
    }
}

// :10854-11117, rows in j, i, k order; per row the Auu/Auv loop, then the Avv/Avu loop, each
// over jA, iA, kA with k+kA inside 1..nz
SymCheck sym_check3(const Ctx &c, double *Auu, double *Auv, double *Avu, double *Avv) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    SymCheck r;
    const int md = c.I3(0, 0, 0);
    for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
        for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i) {
            if (!c.act(i, j)) continue;
            for (int k = 1; k <= g.nz; ++k)
                for (int pass = 0; pass < 2; ++pass) {
                    const double diag = pass == 0 ? Auu[g.a3(md, k, i, j)] : Avv[g.a3(md, k, i, j)];
                    for (int jA = -1; jA <= 1; ++jA)
                        for (int iA = -1; iA <= 1; ++iA)
                            for (int kA = -1; kA <= 1; ++kA) {
                                if (k + kA < 1 || k + kA > g.nz) continue;
                                if (i + iA < 1 || i + iA > g.NX || j + jA < 1 || j + jA > g.NY) continue;
                                const long a = g.a3(c.I3(iA, jA, kA), k, i, j);
                                const long b = g.a3(c.I3(-iA, -jA, -kA), k + kA, i + iA, j + jA);
                                if (pass == 0) {
                                    sym_visit(r, Auu[a], Auu[b], diag, true);
                                    sym_visit(r, Auv[a], Avu[b], diag, true);
                                } else {
                                    sym_visit(r, Avv[a], Avv[b], diag, true);
                                    sym_visit(r, Avu[a], Auv[b], diag, true);
                                }
                            }
                }
        }
    return r;
}

// :10648-10850, jA, iA outer, owned active rows inner; nothing is modified
SymCheck sym_check2(const Ctx &c, const double *Auu, const double *Auv, const double *Avu, const double *Avv) {
    const Geom &g = c.g;
    const cismgpu_par_t &p = c.par;
    SymCheck r;
    const int md = c.I2(0, 0);
    for (int jA = -1; jA <= 1; ++jA)
        for (int iA = -1; iA <= 1; ++iA) {
            const int m = c.I2(iA, jA), mm = c.I2(-iA, -jA);
            for (int j = p.staggered_jlo; j <= p.staggered_jhi; ++j)
                for (int i = p.staggered_ilo; i <= p.staggered_ihi; ++i) {
                    if (!c.act(i, j)) continue;
                    if (i + iA < 1 || i + iA > g.NX || j + jA < 1 || j + jA > g.NY) continue;
                    const long a = g.a2(i, j, m), b = g.a2(i + iA, j + jA, mm);
                    double v1, v2;
                    const double du = Auu[g.a2(i, j, md)], dv = Avv[g.a2(i, j, md)];
                    sym_visit(r, v1 = Auu[a], v2 = Auu[b], du, false);
                    sym_visit(r, v1 = Auv[a], v2 = Avu[b], du, false);
                    sym_visit(r, v1 = Avv[a], v2 = Avv[b], dv, false);
                    sym_visit(r, v1 = Avu[a], v2 = Auv[b], dv, false);
                }
        }
    return r;
}

extern "C" {

int oracle_pcg_standard_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                           const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                           const double *Auv, const double *Avu, const double *Avv, const double *bu,
                           const double *bv, double *xu, double *xv, int precond, int ncheck,
                           double tolerance, int maxiters, double *err, int *niters, int itest, int jtest,
                           int rtest, int summode) {
    (void)itest; (void)jtest; (void)rtest;
    return standard(true, nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                    xu, xv, precond, ncheck, tolerance, maxiters, err, niters, summode);
}

int oracle_pcg_chrongear_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                            const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                            const double *Auv, const double *Avu, const double *Avv, const double *bu,
                            const double *bv, double *xu, double *xv, int precond, int ncheck,
                            double tolerance, int maxiters, double *err, int *niters, int itest, int jtest,
                            int rtest, int summode) {
    (void)itest; (void)jtest; (void)rtest;
    return chrongear(true, nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                     xu, xv, precond, ncheck, tolerance, maxiters, err, niters, summode);
}

int oracle_pcg_standard_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                           const int32_t *active_vertex, const double *Auu, const double *Auv,
                           const double *Avu, const double *Avv, const double *bu, const double *bv,
                           double *xu, double *xv, int precond, int ncheck, double tolerance, int maxiters,
                           double *err, int *niters, int itest, int jtest, int rtest, int summode) {
    (void)itest; (void)jtest; (void)rtest;
    return standard(false, nx, ny, 1, par, indxA_2d, nullptr, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                    xu, xv, precond, ncheck, tolerance, maxiters, err, niters, summode);
}

int oracle_pcg_chrongear_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                            const int32_t *active_vertex, const double *Auu, const double *Auv,
                            const double *Avu, const double *Avv, const double *bu, const double *bv,
                            double *xu, double *xv, int precond, int ncheck, double tolerance, int maxiters,
                            double *err, int *niters, int itest, int jtest, int rtest, int summode) {
    (void)itest; (void)jtest; (void)rtest;
    return chrongear(false, nx, ny, 1, par, indxA_2d, nullptr, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                     xu, xv, precond, ncheck, tolerance, maxiters, err, niters, summode);
}

int oracle_matvec_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_3d,
                     const int32_t *active_vertex, const double *Auu, const double *Auv, const double *Avu,
                     const double *Avv, const double *xu, const double *xv, double *yu, double *yv) {
    Ctx c{Geom{nz, nx - 1, ny - 1}, *par, 0, nullptr, indxA_3d, active_vertex};
    long n = c.g.ntot();
    Vec a(xu, xu + n), b(xv, xv + n), ya(n), yb(n);
    matvec3(c, Auu, Auv, Avu, Avv, a, b, ya, yb);
    std::memcpy(yu, ya.data(), n * sizeof(double));
    std::memcpy(yv, yb.data(), n * sizeof(double));
    return 0;
}

int oracle_matvec_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                     const int32_t *active_vertex, const double *Auu, const double *Auv, const double *Avu,
                     const double *Avv, const double *xu, const double *xv, double *yu, double *yv) {
    Ctx c{Geom{1, nx - 1, ny - 1}, *par, 0, indxA_2d, nullptr, active_vertex};
    long n = c.g.ntot();
    Vec a(xu, xu + n), b(xv, xv + n), ya(n), yb(n);
    matvec2(c, Auu, Auv, Avu, Avv, a, b, ya, yb);
    std::memcpy(yu, ya.data(), n * sizeof(double));
    std::memcpy(yv, yb.data(), n * sizeof(double));
    return 0;
}

// staggered_parallel_halo on a (nz, nx-1, ny-1) array in place (nz = 1 for 2D)
int oracle_halo(int nx, int ny, int nz, const cismgpu_par_t *par, double *a) {
    Ctx c{Geom{nz, nx - 1, ny - 1}, *par, 0, nullptr, nullptr, nullptr};
    long n = c.g.ntot();
    Vec v(a, a + n);
    halo(c, v);
    std::memcpy(a, v.data(), n * sizeof(double));
    return 0;
}

// parallel_global_sum_stagger(arr1, parallel, arr2) in the given mode
double oracle_global_sum(int nx, int ny, int nz, const cismgpu_par_t *par, const double *a1, const double *a2,
                         int summode) {
    Ctx c{Geom{nz, nx - 1, ny - 1}, *par, summode, nullptr, nullptr, nullptr};
    long n = c.g.ntot();
    Vec x(a1, a1 + n), y(a2, a2 + n);
    return global_sum(c, x, y);
}

// easy_sia_solver on a (-1:1, nz, nx-1, ny-1) matrix
int oracle_easy_sia(int nx, int ny, int nz, const int32_t *active_vertex, const double *M, const double *b,
                    double *x) {
    cismgpu_par_t par{};
    Ctx c{Geom{nz, nx - 1, ny - 1}, par, 0, nullptr, nullptr, active_vertex};
    long n = c.g.ntot();
    Vec MM(M, M + 3 * n), bb(b, b + n), xx(x, x + n);
    easy_sia_solver(c, MM, bb, xx);
    std::memcpy(x, xx.data(), n * sizeof(double));
    return 0;
}

// z = PC(r) for one preconditioner (setup + apply), is3d ? (nz,nx-1,ny-1) : (nx-1,ny-1)
// arrays; z holds the previous z on entry (kept where the reference keeps it)
int oracle_precond_apply(int is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                         const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                         const double *Avv, int precond, const double *ru, const double *rv, double *zu,
                         double *zv) {
    Ctx c{Geom{is3d ? nz : 1, nx - 1, ny - 1}, *par, 0, indxA_2d, indxA_3d, active_vertex};
    const long n = c.g.ntot();
    Precond P;
    int st = setup_precond(c, is3d != 0, precond, Auu, Avv, P);
    if (st) return st;
    Vec a(ru, ru + n), b(rv, rv + n), za(zu, zu + n), zb(zv, zv + n);
    apply_precond(c, is3d != 0, P, a, b, za, zb);
    std::memcpy(zu, za.data(), n * sizeof(double));
    std::memcpy(zv, zb.data(), n * sizeof(double));
    return CISMGPU_OK;
}

// compute_residual_vector_{2d,3d} (is3d: (nz,nx-1,ny-1) arrays, indx = indxA_3d; else 2D, indxA_2d)
int oracle_compute_residual_vector(int is3d, int nx, int ny, int nz, const cismgpu_par_t *par,
                                   const int32_t *indx, const int32_t *active_vertex, const double *Auu,
                                   const double *Auv, const double *Avu, const double *Avv, const double *bu,
                                   const double *bv, const double *uvel, const double *vvel, double *resid_u,
                                   double *resid_v, double *L2, double *L2rel, int summode) {
    Ctx c{Geom{is3d ? nz : 1, nx - 1, ny - 1}, *par, summode, is3d ? nullptr : indx, is3d ? indx : nullptr,
          active_vertex};
    const long n = c.g.ntot();
    Vec b1(bu, bu + n), b2(bv, bv + n), x1(uvel, uvel + n), x2(vvel, vvel + n), r1, r2;
    resid_vector(c, is3d != 0, Auu, Auv, Avu, Avv, b1, b2, x1, x2, r1, r2, L2, L2rel);
    std::memcpy(resid_u, r1.data(), n * sizeof(double));
    std::memcpy(resid_v, r2.data(), n * sizeof(double));
    return 0;
}

// compute_residual_velocity_{2d,3d}
double oracle_compute_residual_velocity(int is3d, int whichresid, int nx, int ny, int nz,
                                        const cismgpu_par_t *par, const double *uvel, const double *vvel,
                                        const double *usav, const double *vsav, int summode) {
    Ctx c{Geom{is3d ? nz : 1, nx - 1, ny - 1}, *par, summode, nullptr, nullptr, nullptr};
    const long n = c.g.ntot();
    Vec u(uvel, uvel + n), v(vvel, vvel + n), us(usav, usav + n), vs(vsav, vsav + n);
    return resid_velocity(c, is3d != 0, whichresid, u, v, us, vs);
}

// check_symmetry_assembled_matrix_{3d,2d}: is3d ? (27,nz,nx-1,ny-1) blocks, averaged in
// place, indx = indxA_3d : (nx-1,ny-1,9) blocks, unchanged, indx = indxA_2d.
int oracle_check_symmetry(int is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx,
                          const int32_t *active_vertex, double *Auu, double *Auv, double *Avu, double *Avv,
                          double *maxdiff, long *nwarn) {
    Ctx c{Geom{is3d ? nz : 1, nx - 1, ny - 1}, *par, 0, is3d ? nullptr : indx, is3d ? indx : nullptr,
          active_vertex};
    const SymCheck r = is3d ? sym_check3(c, Auu, Auv, Avu, Avv) : sym_check2(c, Auu, Auv, Avu, Avv);
    *maxdiff = r.maxdiff;
    *nwarn = r.nwarn;
    return 0;
}

// reprosum of n doubles (the reference's reproducible sum, one rank)
double oracle_reprosum(const double *a, long n) { return reprosum(std::vector<double>(a, a + n)); }

// exact correctly-rounded sum of n doubles
double oracle_exact_sum(const double *a, long n) {
    ExactAcc acc;
    for (long e = 0; e < n; ++e) acc.add(a[e]);
    return acc.result();
}

}  // extern "C"
