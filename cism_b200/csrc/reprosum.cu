// reprosum.cu -- the reproducible global sum of parallel_global_sum_stagger's reprosum
// branch (libglimmer/parallel_mpi.F90:6703-6738) on the device.
//
// The reference sums arr1 + arr2 over the owned vertices with cism_reprosum_calc
// (libglimmer/cism_reprosum_mod.F90:237-1057), called by parallel_reduce_reprosum
// (parallel_mpi.F90:9618-9725) without global-max or level hints: its "recompute" path.
// Each nonzero summand is cut into integer digits of arr_max_shift bits aligned to the
// largest exponent ("levels"); the level sums are exact integers, so their value does not
// depend on the order of the summands, and the device adds them with 64-bit atomics in any
// order.  The host then normalizes the carries, fixes the sign and converts the levels back
// to a double through pieces of at most 53 digits added smallest first
// (cism_reprosum_int:1346-1495), which reproduces the reference's result bit for bit: in
// most cases the correctly rounded exact sum, and near a rounding tie the reference's own
// double rounding.
//
// Fortran intrinsics on IEEE doubles: exponent(x) and fraction(x) are frexp's exponent and
// mantissa, scale(x,n) = x*2^n, set_exponent(x,e) = fraction(x)*2^e; digits(1.0_r8) = 53,
// digits(1_i8) = 63, MINEXPONENT(1.0_r8) = -1021, MAXEXPONENT(1.0_r8) = 1024; int(x,i8)
// truncates toward zero, as does 64-bit integer division.

namespace cismgpu {

constexpr int kReproMaxLevels = 72;  // levels min_level..max_levels (<= 58 for any doubles)
constexpr int kDigR8 = 53, kDigI8 = 63, kMinExpR8 = -1021, kMaxExpR8 = 1024;

// Pass 1: exponent extremes of the nonzero summands (cism_reprosum_calc:455-487); ext[0] is
// the maximum (starts at MINEXPONENT), ext[1] the minimum (starts at MAXEXPONENT).  Arrays in
// the caller's layout (nz, NX, NY).
__global__ void __launch_bounds__(kBlock) k_repro_extremes(Geom g, const double *__restrict__ a1,
                                                           const double *__restrict__ a2, int *ext) {
    const long long n = (long long)g.nz * g.NQ;
    int emax = kMinExpR8, emin = kMaxExpR8;
    for (long long node = (long long)blockIdx.x * kBlock + threadIdx.x; node < n;
         node += (long long)gridDim.x * kBlock) {
        const long long q = node / g.nz;
        const int j = (int)(q / g.NX), i = (int)(q - (long long)j * g.NX);
        if (!owned(g, i, j)) continue;
        const double v = __dadd_rn(a1[node], a2[node]);
        if (v != 0.0) {
            int e;
            frexp(v, &e);
            emax = max(emax, e);
            emin = min(emin, e);
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        emax = max(emax, __shfl_down_sync(0xffffffffu, emax, off));
        emin = min(emin, __shfl_down_sync(0xffffffffu, emin, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&ext[0], emax);
        atomicMin(&ext[1], emin);
    }
}

// Before a one-shot reproducible sum of caller arrays: an owned summand arr1 + arr2 that is
// not finite is recorded in *flag (1 NaN, 2 +Inf, 4 -Inf, as k_repro_products) and both of
// its parts are set to zero in the device copies, so the integer expansion only meets finite
// values; the caller then returns the IEEE sum of the non-finite summands instead.
__global__ void __launch_bounds__(kBlock) k_repro_screen(Geom g, double *__restrict__ a1, double *__restrict__ a2,
                                                         int *flag) {
    const long long n = (long long)g.nz * g.NQ;
    int f = 0;
    for (long long node = (long long)blockIdx.x * kBlock + threadIdx.x; node < n;
         node += (long long)gridDim.x * kBlock) {
        const long long q = node / g.nz;
        const int j = (int)(q / g.NX), i = (int)(q - (long long)j * g.NX);
        if (!owned(g, i, j)) continue;
        const double v = __dadd_rn(a1[node], a2[node]);
        if (v - v == 0.0) continue;
        if (v != v) f |= 1;
        else if (v > 0.0) f |= 2;
        else f |= 4;
        a1[node] = 0.0;
        a2[node] = 0.0;
    }
    if (f) atomicOr(flag, f);
}

// Pass 2: the integer expansion of every summand (cism_reprosum_int:1199-1262) into the level
// sums lv[level - min_level], first in shared memory, then in global memory.  Unsigned 64-bit
// atomics add two's-complement values exactly; no level sum leaves the int64 range, since
// arr_max_shift leaves log2(nsummands + 1) bits of headroom.
__global__ void __launch_bounds__(kBlock) k_repro_levels(Geom g, const double *__restrict__ a1,
                                                         const double *__restrict__ a2, int gmax, int shift,
                                                         int max_levels, int min_level,
                                                         unsigned long long *lv) {
    __shared__ unsigned long long slv[kReproMaxLevels];
    const int nl = max_levels - min_level + 1;
    for (int l = threadIdx.x; l < nl; l += kBlock) slv[l] = 0ull;
    __syncthreads();
    const long long n = (long long)g.nz * g.NQ;
    for (long long node = (long long)blockIdx.x * kBlock + threadIdx.x; node < n;
         node += (long long)gridDim.x * kBlock) {
        const long long q = node / g.nz;
        const int j = (int)(q / g.NX), i = (int)(q - (long long)j * g.NX);
        if (!owned(g, i, j)) continue;
        const double v = __dadd_rn(a1[node], a2[node]);
        if (v == 0.0) continue;
        int e;
        const double f = frexp(v, &e);
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
        if (ilevel > max_levels) continue;
        double rem = ldexp(f, ashift);
        long long iv = (long long)rem;
        atomicAdd(&slv[ilevel - min_level], (unsigned long long)iv);
        rem = __dsub_rn(rem, (double)iv);
        while (rem != 0.0 && ilevel < max_levels) {
            ilevel += 1;
            rem = ldexp(rem, shift);
            iv = (long long)rem;
            atomicAdd(&slv[ilevel - min_level], (unsigned long long)iv);
            rem = __dsub_rn(rem, (double)iv);
        }
    }
    __syncthreads();
    for (int l = threadIdx.x; l < nl; l += kBlock)
        if (slv[l] != 0ull) atomicAdd(&lv[l], slv[l]);
}

static inline int f_exponent(double x) {
    int e;
    std::frexp(x, &e);
    return e;
}

// cism_reprosum_int:1346-1495 on the level sums L[level - min_level]: carry normalization,
// sign, same-sign digits, then the double through pieces of at most 53 digits.
static double repro_convert(std::vector<int64_t> &lv, int min_level, int max_levels, int shift, int gmax) {
    const int64_t R = (int64_t)1 << shift;
    auto L = [&](int level) -> int64_t & { return lv[(size_t)(level - min_level)]; };
    auto carry = [&]() {
        for (int l = max_levels; l >= min_level + 1; --l)
            if ((L(l) < 0 ? -L(l) : L(l)) >= R) {
                const int64_t ix = L(l) / R;
                L(l - 1) += ix;
                L(l) -= ix * R;
            }
    };
    carry();  // per thread (:1266-1276)
    carry();  // after the reduction over ranks (:1361-1371)
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
    carry();  // (:1403-1413)
    std::vector<double> pieces;
    bool first = true;
    int ash = gmax - min_level * shift;
    int digit_count = 0, begin_level = min_level;
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
            const int64_t ix = (L(trunc_level) / P) * P;
            trunc_rem = L(trunc_level) - ix;
            L(trunc_level) = ix;
        }
        double piece = 0.0;
        for (int l = begin_level; l <= trunc_level; ++l) {
            if (L(l) != 0) {
                const double X = (double)L(l);
                int ex;
                const double fx = std::frexp(X, &ex);
                const int cur = ex + ash;
                if (cur >= kMinExpR8) piece = piece + std::ldexp(fx, cur);
                else piece = piece + std::ldexp(std::ldexp(fx, cur - kMinExpR8), kMinExpR8);
            }
            if (l < trunc_level || trunc_loc == 0) ash -= shift;
        }
        pieces.push_back(piece);
        if (trunc_loc == 0) {
            digit_count = 0;
            begin_level = trunc_level + 1;
        } else {
            digit_count = trunc_loc;
            begin_level = trunc_level;
            L(trunc_level) = trunc_rem;
        }
    }
    double sum = 0.0;  // smallest to largest (:1489-1492), then the sign
    for (long k = (long)pieces.size() - 1; k >= 0; --k) sum = sum + pieces[(size_t)k];
    return (double)sgn * sum;
}

// The reprosum of arr1 + arr2 (device arrays in the caller's layout) over the owned vertices.
// Two passes over the arrays and two short host synchronizations on the stream.
static int repro_global_sum(cudaStream_t s, const Geom &g, const double *d1, const double *d2, DevBuf &scratch,
                            double *sum) {
    const long long nsummands =
        (long long)(g.ihi - g.ilo + 1) * (long long)(g.jhi - g.jlo + 1) * (long long)g.nz;
    CU(scratch.ensure(64 + kReproMaxLevels * sizeof(unsigned long long)));
    int *ext = scratch.as<int>();
    unsigned long long *lv = reinterpret_cast<unsigned long long *>(scratch.as<char>() + 64);
    const int init[2] = {kMinExpR8, kMaxExpR8};
    CU(cudaMemcpyAsync(ext, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const long long n = (long long)g.nz * g.NQ;
    const unsigned grid = (unsigned)std::min<long long>((n + kBlock - 1) / kBlock, 1184);
    k_repro_extremes<<<grid, kBlock, 0, s>>>(g, d1, d2, ext);
    CU(cudaGetLastError());
    int he[2];
    CU(cudaMemcpyAsync(he, ext, sizeof(he), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    // parameters of the recompute path (cism_reprosum_calc:489-525), one rank, one thread
    const int gmax = he[0], gmin = std::min(he[0], he[1]);
    long long max_nsummands = nsummands + 1;
    if (max_nsummands < 1) max_nsummands = 1;
    const int shift = kDigI8 - (f_exponent((double)max_nsummands) + 1);
    if (shift < 2) return fail(CISMGPU_EUNSUPPORTED, "too many summands for the reproducible sum");
    const int max_levels = 2 + (kDigR8 + (gmax - gmin)) / shift;
    const int extra_levels = (kDigI8 - 1) / shift;
    const int min_level = -(extra_levels - 1);
    const int nl = max_levels - min_level + 1;
    if (nl > kReproMaxLevels) return fail(CISMGPU_EUNSUPPORTED, "reproducible sum: too many levels");
    CU(cudaMemsetAsync(lv, 0, (size_t)nl * sizeof(unsigned long long), s));
    k_repro_levels<<<grid, kBlock, 0, s>>>(g, d1, d2, gmax, shift, max_levels, min_level, lv);
    CU(cudaGetLastError());
    std::vector<int64_t> hl((size_t)nl);
    CU(cudaMemcpyAsync(hl.data(), lv, (size_t)nl * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    *sum = repro_convert(hl, min_level, max_levels, shift, gmax);
    return CISMGPU_OK;
}

}  // namespace cismgpu
