// cismgpu.cu -- host driver and C ABI of the B200 structured PCG library.
//
// One translation unit: the FP64 reference-faithful kernels (pcg_fp64.cu), the
// mixed-precision kernels (pcg_mixed.cu) and the host code.  A Solver owns the
// device copy of one linear system (coefficient planes, level-major vectors) and
// one stream; it enqueues a solver's kernel sequence and polls the device-side
// convergence flag with one check period of look-ahead, so the GPU never idles
// waiting for the host.  The one-shot reference-signature calls reuse one cached
// Solver (the Picard loop calls them repeatedly with the same sizes).
#include <cstdio>
#include <algorithm>
#include <chrono>
#include <cctype>
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <thread>
#include <sys/stat.h>
#include <string>
#include <vector>

#include "pcg_fp64.cu"
#include "pcg_mixed.cu"
#include "assembly.cu"

namespace cismgpu {

static thread_local std::string g_last_error;

// cismgpu_set_mixed_layout(CISMGPU_MIXED_LAYOUT_FULL): the mixed solver keeps every coupling even
// of an exactly symmetric 3D matrix (for layout comparisons); read when a copy is built.
static std::atomic<bool> g_mixed_full_storage{false};

// CISMGPU_TRACE=1: host-side phase timestamps on stderr (diagnostics only).
static bool trace_on() {
    static const bool on = [] {
        const char *e = std::getenv("CISMGPU_TRACE");
        return e && e[0] == '1';
    }();
    return on;
}
static void trace(const char *what) {
    if (!trace_on()) return;
    static auto t0 = std::chrono::steady_clock::now();
    const double us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    std::fprintf(stderr, "[cismgpu %12.1f us] %s\n", us, what);
}

static int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? CISMGPU_ENOMEM : CISMGPU_ECUDA,     \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

#define TRY(expr)                \
    do {                         \
        int rc_ = (expr);        \
        if (rc_) return rc_;     \
    } while (0)

// Host-to-device copies of the caller's arrays.  Pinned host memory is copied directly.  Pageable
// memory (a Fortran or numpy caller's arrays) goes through two pinned staging buffers shared by the
// process: host threads copy one chunk into a buffer while the previous chunk's DMA runs, where the
// driver's own pageable path copies with one thread (about 11 GB/s measured for a 1.2 GB 3D system
// on the B200 hosts).  A copy holds the staging lock until its last chunk is queued; it returns with
// the chunks queued on stream s, the caller's memory already read.
constexpr size_t kStageChunk = 32u << 20;  // bytes per staging buffer
constexpr size_t kStageMin = 4u << 20;     // smaller copies go straight through the driver

struct HostStage {
    std::mutex mu;
    void *buf[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    int dev = -1;
    bool failed = false;
};
static HostStage g_stage;

static void parallel_copy(char *dst, const char *src, size_t n) {
    const unsigned hc = std::thread::hardware_concurrency();
    const int nt = (int)std::max(1u, std::min(8u, hc / 2));
    if (nt == 1 || n < (1u << 20)) {
        std::memcpy(dst, src, n);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (n / nt + 63) / 64 * 64;
    for (int t = 0; t < nt; ++t) {
        const size_t lo = std::min(n, (size_t)t * per), hi = std::min(n, lo + per);
        if (hi > lo) th.emplace_back([=] { std::memcpy(dst + lo, src + lo, hi - lo); });
    }
    for (auto &x : th) x.join();
}

static cudaError_t h2d_copy(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    cudaPointerAttributes pa;
    const bool pinned = cudaPointerGetAttributes(&pa, src) == cudaSuccess &&
                        (pa.type == cudaMemoryTypeHost || pa.type == cudaMemoryTypeManaged);
    (void)cudaGetLastError();
    if (pinned || bytes < kStageMin) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    std::lock_guard<std::mutex> lk(g_stage.mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (g_stage.failed || (g_stage.dev >= 0 && g_stage.dev != dev))  // one device's staging at a time
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    if (!g_stage.buf[0]) {
        for (int k = 0; k < 2; ++k) {
            if (cudaMallocHost(&g_stage.buf[k], kStageChunk) != cudaSuccess ||
                cudaEventCreateWithFlags(&g_stage.done[k], cudaEventDisableTiming) != cudaSuccess) {
                (void)cudaGetLastError();
                g_stage.failed = true;  // no pinned memory: the driver's pageable path
                return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
            }
        }
        g_stage.dev = dev;
    }
    const char *from = static_cast<const char *>(src);
    char *to = static_cast<char *>(dst);
    for (size_t off = 0, n = 0; off < bytes; off += kStageChunk, ++n) {
        const int k = (int)(n & 1);
        const size_t len = std::min(kStageChunk, bytes - off);
        if ((e = cudaEventSynchronize(g_stage.done[k])) != cudaSuccess) return e;  // its last DMA is done
        parallel_copy(static_cast<char *>(g_stage.buf[k]), from + off, len);
        if ((e = cudaMemcpyAsync(to + off, g_stage.buf[k], len, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(g_stage.done[k], s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Vectors of one solve, level-major planes of nz*NQ doubles each.
enum VecId {
    VB_U, VB_V, VX_U, VX_V, VR_U, VR_V, VD_U, VD_V, VQ_U, VQ_V, VZ_U, VZ_V, VAZ_U, VAZ_V, VX0_U, VX0_V, NVEC
};

static int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(CISMGPU_ENODEV, "no CUDA device");
    int dev = 0;
    CU(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return fail(CISMGPU_ENODEV, std::string("not an sm_100 device: ") + prop.name);
    return CISMGPU_OK;
}

static inline unsigned nblocks(long long n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }
// rows of blocks (levels in parallel) for the halo of a matrix's 27 nz coefficient planes
constexpr unsigned kHaloPlaneRows = 64;
static inline bool is_check(int iter, int ncheck) { return (iter % ncheck == 0) || iter == 5; }

struct Ptrs {
    double *bu, *bv, *xu, *xv, *ru, *rv, *du, *dv, *qu, *qv, *zu, *zv, *Azu, *Azv, *x0u, *x0v;
};

// The reference elements of the assembly kernels in constant memory (glissade_velo_higher.F90
// :314-392, :528-570), once per process.
static int asm_ref_ready() {
    static std::once_flag ref_once;
    static cudaError_t ref_status = cudaSuccess;
    std::call_once(ref_once, [] {
        AsmRef r;
        AsmRef2 r2;
        const double rs = 1.0 / std::sqrt(3.0);
        const double xq[8] = {-rs, rs, rs, -rs, -rs, rs, rs, -rs};
        const double yq[8] = {-rs, -rs, rs, rs, -rs, -rs, rs, rs};
        const double zq[8] = {-rs, -rs, -rs, -rs, rs, rs, rs, rs};
        const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
                     sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};  // node corners of the reference cube
        for (int p = 0; p < 8; ++p) {
            r.wqp[p] = 1.0;
            for (int n = 0; n < 8; ++n) {  // d/dxr of (1 +- x)(1 +- y)(1 +- z)/8, as :362-389
                const double fx = sx[n] < 0 ? 1.0 - xq[p] : 1.0 + xq[p];
                const double fy = sy[n] < 0 ? 1.0 - yq[p] : 1.0 + yq[p];
                const double fz = sz[n] < 0 ? 1.0 - zq[p] : 1.0 + zq[p];
                r.dxr[p][n] = sx[n] * fy * fz / 8.0;
                r.dyr[p][n] = sy[n] * fx * fz / 8.0;
                r.dzr[p][n] = sz[n] * fx * fy / 8.0;
                r.phi[p][n] = fx * fy * fz / 8.0;
            }
        }
        for (int p = 0; p < 4; ++p)  // the square: points and nodes are the cube's first four
            for (int n = 0; n < 4; ++n) {
                const double fx = sx[n] < 0 ? 1.0 - xq[p] : 1.0 + xq[p];
                const double fy = sy[n] < 0 ? 1.0 - yq[p] : 1.0 + yq[p];
                r2.phi[p][n] = fx * fy / 4.0;
                r2.dxr[p][n] = sx[n] * fy / 4.0;
                r2.dyr[p][n] = sy[n] * fx / 4.0;
            }
        ref_status = cudaMemcpyToSymbol(c_asm_ref, &r, sizeof(r));
        if (ref_status == cudaSuccess) ref_status = cudaMemcpyToSymbol(c_asm_ref2, &r2, sizeof(r2));
    });
    CU(ref_status);
    return CISMGPU_OK;
}

static int repro_global_sum(cudaStream_t s, const Geom &g, const double *d1, const double *d2, DevBuf &scratch,
                            double *sum);

struct Solver {
    Geom g{};
    bool is3d = false;
    int NC = 27;
    long long nvec = 0;
    long long n_active_owned = 0;  // active owned columns
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DevBuf A, raw, vec, act, partials, state, map;
    DevBuf tri;       // tridiagonal preconditioner planes (TriPlane), on first use
    DevBuf A_sav, x_sav;      // accelerated Picard's saved matrix and velocity (cismgpu_solver_save)
    DevBuf rsum;              // the reproducible sum's exponent extremes and level sums
    DevBuf rprod;             // reproducible-sum solves: the two product fields and the flag
    bool repro = false;       // parallel%reprosum: the FP64 solvers' global sums are reproducible sums
    DevBuf asm_in;            // the stiffness assembly's inputs (geometry, flow factor, velocity, efvs)
    DevBuf asm_k;             // 3D assembly: element matrices of one slab of cell rows
    DevBuf bc_in;             // the boundary terms' inputs (beta, lsrf, masks, velocity)
    DevBuf diva_in;           // the DIVA assembly's inputs and outputs
    DevBuf diva_eq[2];        // DIVA's layer viscosities per Gauss point, previous and new
    int diva_cur = 0;         // which of diva_eq holds the current state
    bool diva_valid = false;  // diva_eq[diva_cur] holds a state for this geometry
    bool have_sav = false;
    bool x_current = false;   // the x planes hold a solution (a solve ran since the last upload)
    int32_t hindx[27] = {};   // host copy of the uploaded indxA map (27 or 9 entries)
    int32_t hindx2[9] = {};   // indxA_2d: the uploaded map in 2D; in 3D the caller's, else standard
    MixedBufs mixed;  // FP32 copies, created on first mixed solve
    int *h_done = nullptr;          // pinned, 2 slots for look-ahead polling
    SolveState *h_state = nullptr;  // pinned
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // profiling of matvec launches
    bool prof = false;
    std::vector<cudaEvent_t> pev;
    int pused = 0;
    double prof_ms = 0.0;
    int prof_n = 0;
    double prof_bytes = 0.0;
    int last_ty = 0;  // tile height of the last mixed solve

    ~Solver() { destroy(); }

    void destroy() {
        A.release(); raw.release(); vec.release(); act.release(); partials.release(); state.release(); map.release();
        tri.release();
        A_sav.release();
        x_sav.release();
        rsum.release();
        asm_in.release();
        asm_k.release();
        bc_in.release();
        diva_in.release();
        diva_eq[0].release();
        diva_eq[1].release();
        diva_valid = false;
        have_sav = false;
        mixed.release();
        if (h_done) cudaFreeHost(h_done);
        if (h_state) cudaFreeHost(h_state);
        h_done = nullptr;
        h_state = nullptr;
        for (auto &e : ev) if (e) cudaEventDestroy(e), e = nullptr;
        for (auto &e : pev) cudaEventDestroy(e);
        pev.clear();
        if (own_stream && stream) cudaStreamDestroy(stream);
        stream = nullptr;
        own_stream = false;
    }

    int init(cudaStream_t s) {
        if (h_done) return CISMGPU_OK;
        TRY(check_device());
        if (s) {
            stream = s;
            own_stream = false;
        } else {
            CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            own_stream = true;
        }
        CU(cudaMallocHost(&h_done, 2 * sizeof(int)));
        CU(cudaMallocHost(&h_state, sizeof(SolveState)));
        CU(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
        return CISMGPU_OK;
    }

    Ptrs ptrs() const {
        double *V = vec.as<double>();
        auto P = [&](int id) { return V + (size_t)id * nvec; };
        return Ptrs{P(VB_U), P(VB_V), P(VX_U), P(VX_V), P(VR_U), P(VR_V), P(VD_U), P(VD_V),
                    P(VQ_U), P(VQ_V), P(VZ_U), P(VZ_V), P(VAZ_U), P(VAZ_V), P(VX0_U), P(VX0_V)};
    }

    VecArgs vargs() const {
        const Ptrs p = ptrs();
        VecArgs v;
        v.bu = p.bu; v.bv = p.bv; v.xu = p.xu; v.xv = p.xv; v.ru = p.ru; v.rv = p.rv;
        v.du = p.du; v.dv = p.dv; v.qu = p.qu; v.qv = p.qv; v.zu = p.zu; v.zv = p.zv;
        v.Azu = p.Azu; v.Azv = p.Azv;
        return v;
    }

    // Geometry of the arrays that follow, and buffers sized for it.
    int set_geom(const Geom &geom, bool three_d) {
        g = geom;
        is3d = three_d;
        NC = is3d ? 27 : 9;
        nvec = (long long)g.nz * g.NQ;
        x_current = false;
        CU(vec.ensure((size_t)NVEC * nvec * sizeof(double)));
        CU(raw.ensure((size_t)nvec * sizeof(double)));
        // the block partials of a reduction, then one counter per column block (the 3D matvec's
        // dot products: k_mv_nodes), zero between launches
        const size_t nbq = nblocks(g.NQ);
        CU(partials.ensure(nbq * 2 * sizeof(DD) + nbq * sizeof(unsigned)));
        CU(cudaMemsetAsync(partials.as<DD>() + 2 * nbq, 0, nbq * sizeof(unsigned), stream));
        CU(state.ensure(sizeof(SolveState)));
        return CISMGPU_OK;
    }

    // One vector from the caller's layout into level-major planes (null: zeros).
    int put_vec(int id, const double *src) {
        double *dst = vec.as<double>() + (size_t)id * nvec;
        cudaStream_t s = stream;
        if (!src) {
            CU(cudaMemsetAsync(dst, 0, nvec * sizeof(double), s));
        } else if (is3d) {
            CU(raw.ensure((size_t)nvec * sizeof(double)));
            CU(h2d_copy(raw.p, src, nvec * sizeof(double), s));
            k_vec_in<<<nblocks(nvec), kBlock, 0, s>>>(g, raw.as<double>(), dst);
            CU(cudaGetLastError());
        } else {
            CU(h2d_copy(dst, src, nvec * sizeof(double), s));
        }
        return CISMGPU_OK;
    }

    // The coefficient blocks (permuted by the uploaded indxA map) and the right-hand side.
    int put_system(const double *const blocks[4], const double *bu, const double *bv) {
        const size_t blk_bytes = (size_t)NC * nvec * sizeof(double);
        CU(A.ensure(4 * blk_bytes));
        CU(raw.ensure(blk_bytes));
        cudaStream_t s = stream;
        mixed.stale = true;  // new matrix: FP32 copy and factors must be rebuilt
        for (int b = 0; b < 4; ++b) {
            CU(h2d_copy(raw.p, blocks[b], blk_bytes, s));
            double *dst = A.as<double>() + (size_t)b * NC * nvec;
            if (is3d)
                k_perm_block3<<<nblocks(nvec), kBlock, 0, s>>>(g, raw.as<double>(), dst, map.as<int32_t>());
            else
                k_perm_block2<<<nblocks(g.NQ), kBlock, 0, s>>>(g, raw.as<double>(), dst, map.as<int32_t>());
            CU(cudaGetLastError());
        }
        TRY(put_vec(VB_U, bu));
        TRY(put_vec(VB_V, bv));
        return CISMGPU_OK;
    }

    // Upload the caller's arrays: coefficient planes, level-major vectors.  x0 may be null.
    int upload(const Geom &geom, bool three_d, const int32_t *indx, const int32_t *active,
               const double *const blocks[4], const double *bu, const double *bv, const double *xu,
               const double *xv) {
        TRY(set_geom(geom, three_d));
        for (int c = 0; c < NC; ++c) hindx[c] = indx[c];
        for (int c = 0; c < 9; ++c) hindx2[c] = is3d ? c + 1 : indx[c];
        n_active_owned = 0;
        for (int j = g.jlo; j <= g.jhi; ++j)
            for (int i = g.ilo; i <= g.ihi; ++i) n_active_owned += active[(long long)j * g.NX + i] != 0;
        CU(act.ensure((size_t)g.NQ * sizeof(int32_t)));
        CU(map.ensure(32 * sizeof(int32_t)));
        cudaStream_t s = stream;
        CU(cudaMemcpyAsync(map.p, indx, NC * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(act.p, active, (size_t)g.NQ * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        TRY(put_system(blocks, bu, bv));
        TRY(put_vec(VX0_U, xu));
        TRY(put_vec(VX0_V, xv));
        return CISMGPU_OK;
    }

    // compute_residual_vector on the device (glissade_velo_higher.F90:9502-9894): resid = A x - b
    // into the r planes for x = planes (xid, xid+1); L2 = |Ax - b| and |b| over owned active
    // vertices.  Leaves the stream synchronized.
    int residual_vector(int xid, double *L2_norm, double *L2_rhs) {
        const Ptrs p = ptrs();
        double *V = vec.as<double>();
        const double *xu = V + (size_t)xid * nvec, *xv = V + (size_t)(xid + 1) * nvec;
        SolveState *st = state.as<SolveState>();
        cudaStream_t s = stream;
        CU(cudaMemsetAsync(st, 0, sizeof(SolveState), s));
        RedCtx rc0{partials.as<DD>(), st, EPI_NONE, 0};
        RedCtx rc1{partials.as<DD>(), st, EPI_RESID_VEC, 0};
        const unsigned nb = nblocks(g.NQ);
        if (is3d)
            launch_mv<27, MV_PLAIN>(s, g, A.as<double>(), act.as<int32_t>(), xu, xv, p.zu, p.zv,
                                                              nullptr, nullptr, nullptr, nullptr, rc0);
        else
            launch_mv<9, MV_PLAIN>(s, g, A.as<double>(), act.as<int32_t>(), xu, xv, p.zu, p.zv,
                                                            nullptr, nullptr, nullptr, nullptr, rc0);
        k_resid_vec<<<nb, kBlock, 0, s>>>(g, act.as<int32_t>(), p.zu, p.zv, p.bu, p.bv, p.ru, p.rv, rc1);
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(h_state, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        *L2_norm = h_state->err;
        *L2_rhs = h_state->L2_rhs;
        return CISMGPU_OK;
    }

    // check_symmetry_assembled_matrix_{3d,2d} (glissade_velo_higher.F90:10648-11117) on four
    // device blocks in layout L: 3D averages the nearly symmetric pairs in place, 2D only
    // reports.  maxdiff: the largest asymmetry seen; nwarn: the reference's asymmetry warnings.
    // Leaves the stream synchronized.
    int sym_check(const SymIdx &L, double *Auu, double *Auv, double *Avu, double *Avv, double *maxdiff,
                  long long *nwarn) {
        CU(rsum.ensure(2 * sizeof(unsigned long long)));
        unsigned long long *out = rsum.as<unsigned long long>();
        cudaStream_t s = stream;
        CU(cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s));
        const long long n = (long long)NC * nvec;
        const dim3 grid((unsigned)((n + kBlock - 1) / kBlock), 3);
        if (is3d)
            k_sym_check<27, true><<<grid, kBlock, 0, s>>>(g, L, act.as<int32_t>(), Auu, Auv, Avu, Avv, out);
        else
            k_sym_check<9, false><<<grid, kBlock, 0, s>>>(g, L, act.as<int32_t>(), Auu, Auv, Avu, Avv, out);
        CU(cudaGetLastError());
        unsigned long long h[2];
        CU(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        double md;
        std::memcpy(&md, &h[0], sizeof(md));
        if (maxdiff) *maxdiff = md;
        if (nwarn) *nwarn = (long long)h[1];
        return CISMGPU_OK;
    }

    // assemble_stiffness_matrix_3d (glissade_velo_higher.F90:5382-5643) or, with three_d false,
    // the SSA branch of assemble_stiffness_matrix_2d (:4961-5378) on the device into four blocks
    // in layout L.  nzl: the number of sigma levels (the layers of flwafact and efvs).  The host
    // arrays are uploaded; u, v null: the velocity planes vel_id, vel_id+1 instead.  efvs (host,
    // may be null) receives the element viscosity.  Leaves the stream synchronized.
    int assemble(bool three_d, int nzl, const SymIdx &L, double *Auu, double *Auv, double *Avu, double *Avv,
                 int nhalo, const double *sigma, const int32_t *active_cell, const double *xv, const double *yv,
                 const double *u, const double *v, int vel_id, const double *usrf, const double *thck,
                 const double *flwafact, int whichapprox, int whichefvs, double efvs_constant,
                 double effstrain_min, double n_glen, double *efvs, const double *dsdx = nullptr,
                 const double *dsdy = nullptr, const double *flwa = nullptr) {
        // 2D with dsdx given: the L1L2 branch (dsdx, dsdy at the vertices, flwa per layer)
        TRY(asm_ref_ready());
        const int nx = g.NX + 1, ny = g.NY + 1;
        const size_t nq = (size_t)g.NQ, ncell = (size_t)nx * ny, nel = (size_t)(nzl - 1) * ncell;
        const size_t nvel = three_d ? (size_t)nzl * nq : nq;
        const bool host_vel = u != nullptr, l1l2 = !three_d && dsdx != nullptr;
        // doubles: sigma, 4 vertex fields, flwafact, efvs, the 2D averaged flow factor, [u, v],
        // [dsdx, dsdy, flwa]; then active_cell and the flag
        const size_t nd = (size_t)nzl + 4 * nq + 2 * nel + ncell + (host_vel ? 2 * nvel : 0) + (l1l2 ? 2 * nq + nel : 0);
        CU(asm_in.ensure(nd * sizeof(double) + ncell * sizeof(int32_t) + 16));
        double *D = asm_in.as<double>();
        double *d_sigma = D, *d_xv = D + nzl, *d_yv = d_xv + nq, *d_usrf = d_yv + nq, *d_thck = d_usrf + nq;
        double *d_ff = d_thck + nq, *d_efvs = d_ff + nel, *d_ff2 = d_efvs + nel, *d_u = d_ff2 + ncell,
               *d_v = d_u + nvel, *d_sx = d_u + (host_vel ? 2 * nvel : 0), *d_sy = d_sx + nq, *d_fl = d_sy + nq;
        int32_t *d_act = reinterpret_cast<int32_t *>(D + nd);
        int *d_sing = reinterpret_cast<int *>(d_act + ncell);
        cudaStream_t s = stream;
        auto up = [&](void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        };
        CU(up(d_sigma, sigma, nzl * sizeof(double)));
        CU(up(d_xv, xv, nq * sizeof(double)));
        CU(up(d_yv, yv, nq * sizeof(double)));
        if (three_d) CU(up(d_usrf, usrf, nq * sizeof(double)));
        CU(up(d_thck, thck, nq * sizeof(double)));
        CU(up(d_ff, flwafact, nel * sizeof(double)));
        CU(up(d_act, active_cell, ncell * sizeof(int32_t)));
        if (host_vel) {
            CU(up(d_u, u, nvel * sizeof(double)));
            CU(up(d_v, v, nvel * sizeof(double)));
        }
        if (l1l2) {
            CU(up(d_sx, dsdx, nq * sizeof(double)));
            CU(up(d_sy, dsdy, nq * sizeof(double)));
            CU(up(d_fl, flwa, nel * sizeof(double)));
        }
        CU(cudaMemsetAsync(d_efvs, 0, nel * sizeof(double), s));
        CU(cudaMemsetAsync(d_sing, 0, sizeof(int), s));
        AsmArgs a;
        a.nx = nx; a.ny = ny; a.nz = nzl; a.nhalo = nhalo;
        a.whichapprox = whichapprox; a.whichefvs = whichefvs;
        a.efvs_constant = efvs_constant; a.effstrain_min = effstrain_min;
        a.p_half = (1.0 - n_glen) / n_glen / 2.0;
        // HO_EFVS_FLOWFACT: velo_scale / len_scale * scyr (glimmer_paramets.F90:97-98), host pow
        a.flowfact_pow = std::pow(500.0 / 31536000.0 / 200.0e3 * 31536000.0, (1.0 - n_glen) / n_glen);
        a.sigma = d_sigma; a.active_cell = d_act; a.xv = d_xv; a.yv = d_yv; a.usrf = d_usrf; a.thck = d_thck;
        const double *V = vec.as<double>();
        a.u = host_vel ? d_u : V + (size_t)vel_id * nvec;
        a.v = host_vel ? d_v : V + (size_t)(vel_id + 1) * nvec;
        a.vel_planes = host_vel ? 0 : 1;
        a.flwafact = d_ff; a.efvs = d_efvs; a.singular = d_sing;
        if (three_d) {
            // element matrices by slabs of cell rows into a scratch L2 can keep, each slab then
            // gathered into the rows of its vertex rows: vertex rows [ja, jb) take the cell rows
            // ja+1 .. jb+1 (1-based), so consecutive slabs share one cell row
            const long long per_row = (long long)nx * (nzl - 1);  // elements per cell row
            const long long row_bytes = per_row * 256 * (long long)sizeof(double);
            int vrows = (int)g.NY;
            if (row_bytes > 0) {
                const long long fit = (long long)(kAsmScratchBytes / (size_t)row_bytes) - 1;
                vrows = (int)std::max<long long>(1, std::min<long long>(fit, (long long)g.NY));
            }
            const long long ks = std::max<long long>(1, per_row * (vrows + 1));
            CU(asm_k.ensure((size_t)ks * 256 * sizeof(double)));
            double *K = asm_k.as<double>();
            for (int ja = 0; ja < (int)g.NY; ja += vrows) {
                const int jb = std::min((int)g.NY, ja + vrows), nrows = jb - ja + 1;
                const long long nel = per_row * nrows;
                if (nel > 0)
                    k_asm_elements3d<<<(unsigned)((nel + kAsmEl - 1) / kAsmEl), kAsmElThreads, 0, s>>>(
                        a, ja + 1, nrows, ja, jb, K, ks);
                const long long nn = (long long)nzl * (jb - ja) * g.NX;
                k_asm_gather3d<<<dim3((unsigned)((nn + kAsmBlock - 1) / kAsmBlock), 4), kAsmBlock, 0, s>>>(
                    a, L, ja, jb, ja + 1, K, ks, Auu, Auv, Avu, Avv);
            }
        } else if (l1l2) {
            L1l2Args l;
            l.dsdx = d_sx; l.dsdy = d_sy; l.flwa = d_fl;
            l.linear = std::fabs(n_glen - 1.0) < 1.0e-10;
            k_assemble2d_l1l2<<<(unsigned)((g.NQ + kAsmBlock - 1) / kAsmBlock), kAsmBlock, 0, s>>>(a, l, L, Auu, Auv,
                                                                                                   Avu, Avv);
        } else {
            k_asm_vertavg<<<(unsigned)((ncell + kBlock - 1) / kBlock), kBlock, 0, s>>>((int)ncell, nzl, d_sigma, d_ff,
                                                                                       d_ff2);
            k_assemble2d<<<(unsigned)((g.NQ + kAsmBlock - 1) / kAsmBlock), kAsmBlock, 0, s>>>(a, d_ff2, L, Auu, Auv,
                                                                                               Avu, Avv);
        }
        CU(cudaGetLastError());
        int sing = 0;
        CU(cudaMemcpyAsync(&sing, d_sing, sizeof(int), cudaMemcpyDeviceToHost, s));
        if (efvs) CU(cudaMemcpyAsync(efvs, d_efvs, nel * sizeof(double), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (sing) return fail(CISMGPU_EINVAL, "Jacobian matrix is singular (an element of zero volume)");
        return CISMGPU_OK;
    }

    // The boundary terms of the 3D system on four blocks in layout L and b in layout Wb
    // (glissade_velo_higher.F90:2848-2891): the local basal term of basal_sliding_bc_3d when
    // beta is given (lsrf with it), then dirichlet_boundary_conditions_3d when the masks are
    // given.  Host arrays in the caller's layout; uvel = vvel = null: the velocity planes
    // vel_id, vel_id+1.  Leaves the stream synchronized.
    int boundary3d(const SymIdx &L, double *Auu, double *Auv, double *Avu, double *Avv, double *bu, double *bv,
                   VecIdx Wb, int nhalo, double dx, double dy, const int32_t *active_vertex, const double *beta,
                   const double *lsrf, const int32_t *umask, const int32_t *vmask, const double *uvel,
                   const double *vvel, int vel_id, int assemble_beta = 1, const int32_t *active_cell = nullptr,
                   const double *xv = nullptr, const double *yv = nullptr) {
        const int nx = g.NX + 1, ny = g.NY + 1, nz = g.nz;
        const size_t nq = (size_t)g.NQ, ncell = (size_t)nx * ny, nn = (size_t)nz * nq;
        const bool host_vel = uvel != nullptr;
        // doubles: beta, lsrf, xVertex, yVertex, [uvel, vvel]; then int32: active_vertex, umask,
        // vmask, active_cell, the singular-Jacobian flag
        const size_t nd = 3 * nq + ncell + (host_vel ? 2 * nn : 0);
        CU(bc_in.ensure(nd * sizeof(double) + (nq + 2 * nn + ncell + 1) * sizeof(int32_t)));
        double *D = bc_in.as<double>();
        double *d_beta = D, *d_lsrf = D + nq, *d_xv = d_lsrf + ncell, *d_yv = d_xv + nq, *d_u = d_yv + nq,
               *d_v = d_u + nn;
        int32_t *d_act = reinterpret_cast<int32_t *>(D + nd), *d_um = d_act + nq, *d_vm = d_um + nn,
                *d_cell = d_vm + nn, *d_sing = d_cell + ncell;
        cudaStream_t s = stream;
        auto up = [&](void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        };
        CU(up(d_act, active_vertex, nq * sizeof(int32_t)));
        CU(cudaMemsetAsync(d_sing, 0, sizeof(int32_t), s));
        if (beta) {
            CU(up(d_beta, beta, nq * sizeof(double)));
            CU(up(d_lsrf, lsrf, ncell * sizeof(double)));
            if (assemble_beta == 1) {
                k_basal_local3d<<<nblocks((long long)nq), kBlock, 0, s>>>(nx, ny, nz, dx, dy, L, d_act, d_beta,
                                                                          d_lsrf, Auu, Avv);
            } else {
                TRY(asm_ref_ready());
                CU(up(d_cell, active_cell, ncell * sizeof(int32_t)));
                CU(up(d_xv, xv, nq * sizeof(double)));
                CU(up(d_yv, yv, nq * sizeof(double)));
                k_basal_standard<true, true><<<nblocks((long long)nq), kBlock, 0, s>>>(
                    nx, ny, nz, nhalo, L, d_cell, d_xv, d_yv, d_beta, d_beta, d_lsrf, Auu, Avv, d_sing);
            }
            CU(cudaGetLastError());
        }
        if (umask) {
            CU(up(d_um, umask, nn * sizeof(int32_t)));
            CU(up(d_vm, vmask, nn * sizeof(int32_t)));
            if (host_vel) {
                CU(up(d_u, uvel, nn * sizeof(double)));
                CU(up(d_v, vvel, nn * sizeof(double)));
            }
            const double *V = vec.as<double>();
            const double *xu = host_vel ? d_u : V + (size_t)vel_id * nvec;
            const double *xv = host_vel ? d_v : V + (size_t)(vel_id + 1) * nvec;
            const VecIdx Wm{g.NQ, nz, 0}, Wx{g.NQ, nz, host_vel ? 0 : 1};
            k_dirichlet3d<<<nblocks((long long)nn), kBlock, 0, s>>>(nx, ny, nz, nhalo, L, Wb, Wm, Wx, d_act, d_um,
                                                                    d_vm, xu, xv, Auu, Auv, Avu, Avv, bu, bv);
            CU(cudaGetLastError());
        }
        int sing = 0;
        CU(cudaMemcpyAsync(&sing, d_sing, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (sing) return fail(CISMGPU_EINVAL, "Jacobian matrix is singular (a basal cell of zero area)");
        return CISMGPU_OK;
    }

    // The boundary terms of the 2D system on four blocks in layout L (NC = 9) and b (NQ):
    // the local basal term of basal_sliding_bc_2d when beta is given, then
    // dirichlet_boundary_conditions_2d when the masks are given (:2590-2651).  Host arrays in
    // the (nx-1, ny-1) layout; uvel = vvel = null: the velocity planes vel_id, vel_id+1.
    // Leaves the stream synchronized.
    int boundary2d(const SymIdx &L, double *Auu, double *Auv, double *Avu, double *Avv, double *bu, double *bv,
                   int nhalo, double dx, double dy, const int32_t *active_vertex, const double *beta,
                   const int32_t *umask, const int32_t *vmask, const double *uvel, const double *vvel, int vel_id,
                   int assemble_beta = 1, const int32_t *active_cell = nullptr, const double *xv = nullptr,
                   const double *yv = nullptr, const double *beta_v = nullptr, const double *lsrf = nullptr) {
        // beta_v given: the DIVA basal term (basal_sliding_bc_2d_diva) with beta for u, beta_v
        // for v and the lower surface lsrf (nx, ny)
        const int nx = g.NX + 1, ny = g.NY + 1;
        const size_t nq = (size_t)g.NQ, ncell = (size_t)nx * ny;
        const bool host_vel = uvel != nullptr, diva = beta_v != nullptr;
        // doubles: beta, xVertex, yVertex, beta_v, lsrf, [uvel, vvel]; then int32: active_vertex,
        // umask, vmask, active_cell, the singular-Jacobian flag
        const size_t nd = 4 * nq + ncell + (host_vel ? 2 * nq : 0);
        CU(bc_in.ensure(nd * sizeof(double) + (3 * nq + ncell + 1) * sizeof(int32_t)));
        double *D = bc_in.as<double>();
        double *d_beta = D, *d_xv = D + nq, *d_yv = d_xv + nq, *d_bv = d_yv + nq, *d_lsrf = d_bv + nq,
               *d_u = d_lsrf + ncell, *d_v = d_u + nq;
        int32_t *d_act = reinterpret_cast<int32_t *>(D + nd), *d_um = d_act + nq, *d_vm = d_um + nq,
                *d_cell = d_vm + nq, *d_sing = d_cell + ncell;
        cudaStream_t s = stream;
        auto up = [&](void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        };
        CU(up(d_act, active_vertex, nq * sizeof(int32_t)));
        CU(cudaMemsetAsync(d_sing, 0, sizeof(int32_t), s));
        if (beta && diva) {
            CU(up(d_beta, beta, nq * sizeof(double)));
            CU(up(d_bv, beta_v, nq * sizeof(double)));
            CU(up(d_lsrf, lsrf, ncell * sizeof(double)));
            if (assemble_beta == 1) {
                k_basal_local_diva<<<nblocks((long long)nq), kBlock, 0, s>>>(nx, ny, dx, dy, L, d_act, d_beta, d_bv,
                                                                             d_lsrf, Auu, Avv);
            } else {
                TRY(asm_ref_ready());
                CU(up(d_cell, active_cell, ncell * sizeof(int32_t)));
                CU(up(d_xv, xv, nq * sizeof(double)));
                CU(up(d_yv, yv, nq * sizeof(double)));
                k_basal_standard<false, true><<<nblocks((long long)nq), kBlock, 0, s>>>(
                    nx, ny, 1, nhalo, L, d_cell, d_xv, d_yv, d_beta, d_bv, d_lsrf, Auu, Avv, d_sing);
            }
            CU(cudaGetLastError());
        } else if (beta) {
            CU(up(d_beta, beta, nq * sizeof(double)));
            if (assemble_beta == 1) {
                k_basal_local2d<<<nblocks((long long)nq), kBlock, 0, s>>>(g.NQ, dx, dy, L, d_act, d_beta, Auu, Avv);
            } else {
                TRY(asm_ref_ready());
                CU(up(d_cell, active_cell, ncell * sizeof(int32_t)));
                CU(up(d_xv, xv, nq * sizeof(double)));
                CU(up(d_yv, yv, nq * sizeof(double)));
                k_basal_standard<false, false><<<nblocks((long long)nq), kBlock, 0, s>>>(
                    nx, ny, 1, nhalo, L, d_cell, d_xv, d_yv, d_beta, d_beta, d_beta, Auu, Avv, d_sing);
            }
            CU(cudaGetLastError());
        }
        if (umask) {
            CU(up(d_um, umask, nq * sizeof(int32_t)));
            CU(up(d_vm, vmask, nq * sizeof(int32_t)));
            if (host_vel) {
                CU(up(d_u, uvel, nq * sizeof(double)));
                CU(up(d_v, vvel, nq * sizeof(double)));
            }
            const double *V = vec.as<double>();
            const double *xu = host_vel ? d_u : V + (size_t)vel_id * nvec;
            const double *xv = host_vel ? d_v : V + (size_t)(vel_id + 1) * nvec;
            k_dirichlet2d<<<nblocks((long long)nq), kBlock, 0, s>>>(nx, ny, nhalo, L, d_act, d_um, d_vm, xu, xv, Auu,
                                                                    Auv, Avu, Avv, bu, bv);
            CU(cudaGetLastError());
        }
        int sing = 0;
        CU(cudaMemcpyAsync(&sing, d_sing, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (sing) return fail(CISMGPU_EINVAL, "Jacobian matrix is singular (a basal cell of zero area)");
        return CISMGPU_OK;
    }

    // assemble_stiffness_matrix_2d with HO_APPROX_DIVA into four blocks in layout L (NC = 9).
    // eq_old / eq_new: device buffers of the layer viscosities per Gauss point
    // (nz-1, 4, nx, ny); eq_new must already hold eq_old's values for the cells the kernel does
    // not visit.  Host inputs in the reference's layouts; u, v null: the velocity planes
    // vel_id, vel_id+1.  efvs, omega_k, omega (host, may be null) receive the outputs; omega_k
    // and omega of cells that are not assembled come back as the caller passed them.
    int assemble_diva(int nzl, const SymIdx &L, double *Auu, double *Auv, double *Avu, double *Avv, int nhalo,
                      const double *sigma, const double *stagsigma, const int32_t *active_cell, const double *xv,
                      const double *yv, const double *u, const double *v, int vel_id, const double *stagthck,
                      const double *thck, const double *btractx, const double *btracty, const double *dsfx,
                      const double *dsfy, const double *flwafact, int whichefvs, double efvs_constant,
                      double effstrain_min, double n_glen, const double *eq_old, double *eq_new, double *efvs,
                      double *omega_k, double *omega) {
        TRY(asm_ref_ready());
        const int nx = g.NX + 1, ny = g.NY + 1;
        const size_t nq = (size_t)g.NQ, ncell = (size_t)nx * ny, nel = (size_t)(nzl - 1) * ncell;
        const bool host_vel = u != nullptr;
        // doubles: sigma, stagsigma, xv, yv, stagthck, bx, by, thck, dsfx, dsfy, flwafact, efvs,
        // omega_k, omega, [u, v]; then int32: active_cell, the flag
        const size_t nd = (size_t)2 * nzl + 5 * nq + 4 * ncell + nel + nel + (size_t)nzl * ncell + ncell +
                          (host_vel ? 2 * nq : 0);
        CU(diva_in.ensure(nd * sizeof(double) + (ncell + 1) * sizeof(int32_t)));
        double *D = diva_in.as<double>();
        double *d_sigma = D, *d_ss = d_sigma + nzl, *d_xv = d_ss + nzl, *d_yv = d_xv + nq, *d_h = d_yv + nq,
               *d_bx = d_h + nq, *d_by = d_bx + nq, *d_thck = d_by + nq, *d_sx = d_thck + ncell, *d_sy = d_sx + ncell,
               *d_ff = d_sy + ncell, *d_efvs = d_ff + nel, *d_ok = d_efvs + nel, *d_om = d_ok + (size_t)nzl * ncell,
               *d_u = d_om + ncell, *d_v = d_u + nq;
        int32_t *d_act = reinterpret_cast<int32_t *>(D + nd), *d_sing = d_act + ncell;
        cudaStream_t s = stream;
        auto up = [&](void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        };
        CU(up(d_sigma, sigma, nzl * sizeof(double)));
        CU(up(d_ss, stagsigma, (nzl - 1) * sizeof(double)));
        CU(up(d_xv, xv, nq * sizeof(double)));
        CU(up(d_yv, yv, nq * sizeof(double)));
        CU(up(d_h, stagthck, nq * sizeof(double)));
        CU(up(d_bx, btractx, nq * sizeof(double)));
        CU(up(d_by, btracty, nq * sizeof(double)));
        CU(up(d_thck, thck, ncell * sizeof(double)));
        CU(up(d_sx, dsfx, ncell * sizeof(double)));
        CU(up(d_sy, dsfy, ncell * sizeof(double)));
        CU(up(d_ff, flwafact, nel * sizeof(double)));
        CU(up(d_act, active_cell, ncell * sizeof(int32_t)));
        if (omega_k) CU(up(d_ok, omega_k, (size_t)nzl * ncell * sizeof(double)));
        else CU(cudaMemsetAsync(d_ok, 0, (size_t)nzl * ncell * sizeof(double), s));
        if (omega) CU(up(d_om, omega, ncell * sizeof(double)));
        else CU(cudaMemsetAsync(d_om, 0, ncell * sizeof(double), s));
        if (host_vel) {
            CU(up(d_u, u, nq * sizeof(double)));
            CU(up(d_v, v, nq * sizeof(double)));
        }
        CU(cudaMemsetAsync(d_efvs, 0, nel * sizeof(double), s));
        CU(cudaMemsetAsync(d_sing, 0, sizeof(int32_t), s));
        const double p_effstr = (1.0 - n_glen) / n_glen;
        AsmArgs a;
        a.nx = nx; a.ny = ny; a.nz = nzl; a.nhalo = nhalo;
        a.whichapprox = 4; a.whichefvs = whichefvs;
        a.efvs_constant = efvs_constant; a.effstrain_min = effstrain_min;
        a.p_half = p_effstr / 2.0;
        a.flowfact_pow = std::pow(500.0 / 31536000.0 / 200.0e3 * 31536000.0, p_effstr);
        a.sigma = d_sigma; a.active_cell = d_act; a.xv = d_xv; a.yv = d_yv; a.usrf = d_h; a.thck = d_h;
        const double *V = vec.as<double>();
        a.u = host_vel ? d_u : V + (size_t)vel_id * nvec;
        a.v = host_vel ? d_v : V + (size_t)(vel_id + 1) * nvec;
        a.vel_planes = 1;
        a.flwafact = d_ff; a.efvs = d_efvs; a.singular = d_sing;
        DivaArgs dv;
        dv.stagsigma = d_ss; dv.thck = d_thck; dv.bx = d_bx; dv.by = d_by; dv.dsfx = d_sx; dv.dsfy = d_sy;
        dv.eq_old = eq_old; dv.eq_new = eq_new; dv.omega_k = d_ok; dv.omega = d_om;
        dv.init_pow = std::pow(effstrain_min, p_effstr);  // host pow, as the reference's
        k_assemble2d_diva<<<(unsigned)((g.NQ + kAsmBlock - 1) / kAsmBlock), kAsmBlock, 0, s>>>(a, dv, L, Auu, Auv,
                                                                                               Avu, Avv);
        CU(cudaGetLastError());
        int sing = 0;
        CU(cudaMemcpyAsync(&sing, d_sing, sizeof(int), cudaMemcpyDeviceToHost, s));
        if (efvs) CU(cudaMemcpyAsync(efvs, d_efvs, nel * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (omega_k) CU(cudaMemcpyAsync(omega_k, d_ok, (size_t)nzl * ncell * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (omega) CU(cudaMemcpyAsync(omega, d_om, ncell * sizeof(double), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (sing) return fail(CISMGPU_EINVAL, "Jacobian matrix is singular (an element of zero volume)");
        return CISMGPU_OK;
    }

    // load_vector_gravity (glissade_velo_higher.F90:4228-4449) added into the device loads lu, lv
    // (layout W).  Host inputs in the reference's layouts.  Leaves the stream synchronized.
    int load_gravity(VecIdx W, double *lu, double *lv, int nhalo, const double *sigma, const double *stagwbndsigma,
                     double dx, double dy, const int32_t *active_cell, const int32_t *active_vertex,
                     const double *xv, const double *yv, const double *stagusrf, const double *stagthck,
                     const double *dsdx, const double *dsdy, int whichassemble_taud) {
        TRY(asm_ref_ready());
        const int nx = g.NX + 1, ny = g.NY + 1, nz = g.nz;
        const size_t nq = (size_t)g.NQ, ncell = (size_t)nx * ny;
        // doubles: sigma, stagwbndsigma, xv, yv, stagusrf, stagthck, dsdx, dsdy; then int32:
        // active_cell, active_vertex, the flag
        const size_t nd = (size_t)2 * nz + 1 + 6 * nq;
        CU(asm_in.ensure(nd * sizeof(double) + (ncell + nq + 1) * sizeof(int32_t)));
        double *D = asm_in.as<double>();
        double *d_sig = D, *d_sw = d_sig + nz, *d_xv = d_sw + nz + 1, *d_yv = d_xv + nq, *d_us = d_yv + nq,
               *d_th = d_us + nq, *d_sx = d_th + nq, *d_sy = d_sx + nq;
        int32_t *d_cell = reinterpret_cast<int32_t *>(D + nd), *d_av = d_cell + ncell, *d_sing = d_av + nq;
        cudaStream_t s = stream;
        auto up = [&](void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        };
        CU(up(d_sw, stagwbndsigma, (nz + 1) * sizeof(double)));
        CU(up(d_th, stagthck, nq * sizeof(double)));
        CU(up(d_sx, dsdx, nq * sizeof(double)));
        CU(up(d_sy, dsdy, nq * sizeof(double)));
        CU(up(d_av, active_vertex, nq * sizeof(int32_t)));
        CU(cudaMemsetAsync(d_sing, 0, sizeof(int32_t), s));
        if (whichassemble_taud == 1) {
            k_load_local<<<nblocks((long long)nz * g.NQ), kBlock, 0, s>>>(nx, ny, nz, dx, dy, W, d_av, d_sw, d_th, d_sx,
                                                                          d_sy, lu, lv);
        } else {
            CU(up(d_sig, sigma, nz * sizeof(double)));
            CU(up(d_xv, xv, nq * sizeof(double)));
            CU(up(d_yv, yv, nq * sizeof(double)));
            CU(up(d_us, stagusrf, nq * sizeof(double)));
            CU(up(d_cell, active_cell, ncell * sizeof(int32_t)));
            AsmArgs a{};
            a.nx = nx; a.ny = ny; a.nz = nz; a.nhalo = nhalo;
            a.sigma = d_sig; a.active_cell = d_cell; a.xv = d_xv; a.yv = d_yv; a.usrf = d_us; a.thck = d_th;
            a.singular = d_sing;
            const long long n = (long long)nz * g.NQ;
            k_load_standard<<<(unsigned)((n + kAsmBlock - 1) / kAsmBlock), kAsmBlock, 0, s>>>(a, W, d_sx, d_sy, lu,
                                                                                              lv);
        }
        CU(cudaGetLastError());
        int sing = 0;
        CU(cudaMemcpyAsync(&sing, d_sing, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (sing) return fail(CISMGPU_EINVAL, "Jacobian matrix is singular (an element of zero volume)");
        return CISMGPU_OK;
    }

    // The symmetry check on the resident canonical planes.
    int check_symmetry(double *maxdiff, long long *nwarn) {
        SymIdx L{};
        for (int c = 0; c < 27; ++c) L.map[c] = c + 1;
        L.n = nvec;
        L.NQ = g.NQ;
        L.nz = g.nz;
        L.raw3 = 0;
        const size_t bs = (size_t)NC * nvec;
        double *A0 = A.as<double>();
        TRY(sym_check(L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, maxdiff, nwarn));
        if (is3d) mixed.stale = true;  // the FP32 copies follow the averaged matrix
        return CISMGPU_OK;
    }

    // compute_residual_velocity on the device (:10188-10446) between the planes of id_new
    // (uvel, vvel) and id_old (usav, vsav).  Leaves the stream synchronized.
    int residual_velocity(int whichresid, int id_new, int id_old, double *resid_velo) {
        double *V = vec.as<double>();
        SolveState *st = state.as<SolveState>();
        cudaStream_t s = stream;
        CU(cudaMemsetAsync(st, 0, sizeof(SolveState), s));
        const int mean = whichresid == CISMGPU_RESID_MEANU;
        // 3D: the bed level is left out for the "no basal" max and the mean (size(uvel,1) - 1)
        const int kmax = (is3d && (whichresid == CISMGPU_RESID_MAXU_NO_UBAS || mean)) ? g.nz - 1 : g.nz;
        RedCtx rc{partials.as<DD>(), st, EPI_SUM, 0};
        k_resid_velo<<<nblocks(g.NQ), kBlock, 0, s>>>(g, kmax, mean, V + (size_t)id_new * nvec,
                                                      V + (size_t)(id_new + 1) * nvec, V + (size_t)id_old * nvec,
                                                      V + (size_t)(id_old + 1) * nvec, rc);
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(h_state, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (mean) {
            *resid_velo = h_state->count > 0 ? h_state->rho / (double)h_state->count : 0.0;
        } else {
            double d;
            std::memcpy(&d, &h_state->maxbits, sizeof(d));
            *resid_velo = d;
        }
        return CISMGPU_OK;
    }

    int download(int id_u, int id_v, double *xu, double *xv) {
        double *V = vec.as<double>();
        double *out[2] = {xu, xv};
        const int id[2] = {id_u, id_v};
        for (int t = 0; t < 2; ++t) {
            if (is3d) {
                CU(raw.ensure((size_t)nvec * sizeof(double)));  // staging for the layout change
                k_vec_out<<<nblocks(nvec), kBlock, 0, stream>>>(g, V + (size_t)id[t] * nvec, raw.as<double>());
                CU(cudaGetLastError());
                CU(cudaMemcpyAsync(out[t], raw.p, nvec * sizeof(double), cudaMemcpyDeviceToHost, stream));
            } else {
                CU(cudaMemcpyAsync(out[t], V + (size_t)id[t] * nvec, nvec * sizeof(double), cudaMemcpyDeviceToHost,
                                   stream));
            }
        }
        CU(cudaStreamSynchronize(stream));
        return CISMGPU_OK;
    }

    // ---- profiling of matvec launches (CUDA events on this stream) ----
    template <class F>
    int timed(F launch) {
        if (prof) {
            if (pused + 2 > (int)pev.size() && pev.size() < 16384) {
                for (int t = 0; t < 256; ++t) {
                    cudaEvent_t e;
                    CU(cudaEventCreate(&e));
                    pev.push_back(e);
                }
            }
            if (pused + 2 <= (int)pev.size()) {
                CU(cudaEventRecord(pev[pused], stream));
                launch();
                CU(cudaEventRecord(pev[pused + 1], stream));
                pused += 2;
                return CISMGPU_OK;
            }
        }
        launch();
        return CISMGPU_OK;
    }

    int collect_profile() {
        if (!prof) return CISMGPU_OK;
        CU(cudaStreamSynchronize(stream));
        for (int t = 0; t + 1 < pused; t += 2) {
            float ms = 0.f;
            CU(cudaEventElapsedTime(&ms, pev[t], pev[t + 1]));
            prof_ms += ms;
            prof_n += 1;
        }
        pused = 0;
        return CISMGPU_OK;
    }

    // ---- convergence polling with one check period of look-ahead ----
    struct Poller {
        Solver &s;
        int pending = -1, slot = 0;
        explicit Poller(Solver &sv) : s(sv) {}
        int after_check() {
            SolveState *st = s.state.as<SolveState>();
            if (cudaMemcpyAsync(&s.h_done[slot], &st->done, sizeof(int), cudaMemcpyDeviceToHost, s.stream) !=
                cudaSuccess)
                return -1;
            if (cudaEventRecord(s.ev[slot], s.stream) != cudaSuccess) return -1;
            int finished = 0;
            if (pending >= 0) {
                if (cudaEventSynchronize(s.ev[pending]) != cudaSuccess) return -1;
                finished = s.h_done[pending];
            }
            pending = slot;
            slot ^= 1;
            return finished;
        }
    };

    int begin_solve() {
        x_current = true;
        const Ptrs p = ptrs();
        CU(cudaMemcpyAsync(p.xu, p.x0u, 2 * nvec * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        return CISMGPU_OK;
    }

    int finish_solve(double *err, int *niters) {
        trace("finish_solve: begin");
        CU(cudaMemcpyAsync(h_state, state.p, sizeof(SolveState), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        trace("finish_solve: synchronized");
        TRY(collect_profile());
        *err = h_state->err;
        *niters = h_state->niters;
        if (h_state->status == CISMGPU_EBREAKDOWN_ETA1)
            return fail(CISMGPU_EBREAKDOWN_ETA1, "PCG solver has failed, eta1 = NaN");
        if (h_state->status == CISMGPU_EBREAKDOWN_ALPHA)
            return fail(CISMGPU_EBREAKDOWN_ALPHA, "PCG solver has failed, alpha = NaN");
        if (h_state->status == CISMGPU_EDIVZERO)
            return fail(CISMGPU_EDIVZERO, "divzero in the tridiagonal preconditioner setup");
        if (h_state->status == CISMGPU_ETIMEOUT)
            return fail(CISMGPU_ETIMEOUT, "a bounded device wait gave up (the solve was abandoned)");
        if (h_state->status != CISMGPU_OK)
            return fail(h_state->status, "solve failed on the device");
        return CISMGPU_OK;
    }

    double mv_bytes(int extra_vec_streams) const {
        // per active owned node: 4 blocks x NC coefficients + vector streams of 2 components
        return (double)n_active_owned * g.nz * (4.0 * NC * 8.0 + 2.0 * 8.0 * (2 + extra_vec_streams));
    }

    // Device planes of the line-system couplings for precond 3/4 (TriMap): the raw index m that
    // indxA_2d gives each coupling, and in 3D the planes holding raw m, m+9, m+18.
    int tri_map(TriMap &tm) const {
        static const int geo[2][3] = {{3, 4, 5}, {1, 4, 7}};  // (-1,0),(0,0),(1,0) / (0,-1),(0,0),(0,1)
        for (int comp = 0; comp < 2; ++comp)
            for (int e = 0; e < 3; ++e) {
                const int m = hindx2[geo[comp][e]];
                if (m < 1 || m > 9) return fail(CISMGPU_EINVAL, "indxA_2d entry outside 1..9");
                tm.m[comp][e] = m;
                for (int t = 0; t < 3; ++t) tm.c[comp][e][t] = 0;
                if (!is3d) {
                    tm.c[comp][e][0] = geo[comp][e];  // the planes were permuted by this same map
                } else {
                    for (int t = 0; t < 3; ++t) {
                        int c = 0;
                        while (c < 27 && hindx[c] != m + 9 * t) ++c;
                        if (c == 27) return fail(CISMGPU_EINVAL, "indxA_3d does not name a coefficient the "
                                                                 "tridiagonal preconditioner sums");
                        tm.c[comp][e][t] = c;
                    }
                }
            }
        return CISMGPU_OK;
    }

    // Setup of precond 3/4 (after k_init_state: a zero pivot ends the solve with EDIVZERO).
    int tri_setup(int precond) {
        CU(tri.ensure((size_t)NTRI * g.NQ * sizeof(double)));
        TriMap tm;
        TRY(tri_map(tm));
        const int global = precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
        if (is3d)
            k_tri_coef<27><<<nblocks(g.NQ), kBlock, 0, stream>>>(g, A.as<double>(), act.as<int32_t>(), tm, global,
                                                                tri.as<double>());
        else
            k_tri_coef<9><<<nblocks(g.NQ), kBlock, 0, stream>>>(g, A.as<double>(), act.as<int32_t>(), tm, global,
                                                               tri.as<double>());
        k_tri_factor<<<(tri_lines(g) + kBlock - 1) / kBlock, kBlock, 0, stream>>>(g, global, tri.as<double>(),
                                                                                  state.as<SolveState>());
        CU(cudaGetLastError());
        return CISMGPU_OK;
    }

    // z = PC(r) (+ the statement MODE fuses): precond 3/4 first run their line solves
    // (3D: of the vertically summed residual) and halo update, then k_precond finishes.
    template <int NCC, int MODE>
    int apply_precond(int precond, const Ptrs &p, RedCtx rc, double *du, double *dv) {
        cudaStream_t s = stream;
        SolveState *st = state.as<SolveState>();
        const double *zs = nullptr;
        if (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL) {
            const int global = precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
            double *T = tri.as<double>();
            const long long NQ = g.NQ;
            const unsigned lb = (tri_lines(g) + kBlock - 1) / kBlock;
            const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
            if (NCC == 27) {
                k_tri_vsum<<<nblocks(NQ), kBlock, 0, s>>>(g, p.ru, p.rv, T, st);
                CU(cudaMemsetAsync(T + TZS_U * NQ, 0, 2 * NQ * sizeof(double), s));
                k_tri_lines<<<lb, kBlock, 0, s>>>(g, global, T + TRS_U * NQ, T + TRS_V * NQ, T + TZS_U * NQ,
                                                  T + TZS_V * NQ, T, st);
                Geom g1 = g;
                g1.nz = 1;
                k_halo<<<hb, kBlock, 0, s>>>(g1, T + TZS_U * NQ, T + TZS_V * NQ, st);
                zs = T + TZS_U * NQ;
            } else {
                CU(cudaMemsetAsync(p.zu, 0, NQ * sizeof(double), s));
                CU(cudaMemsetAsync(p.zv, 0, NQ * sizeof(double), s));
                k_tri_lines<<<lb, kBlock, 0, s>>>(g, global, p.ru, p.rv, p.zu, p.zv, T, st);
                k_halo<<<hb, kBlock, 0, s>>>(g, p.zu, p.zv, st);
            }
        }
        k_precond<MODE><<<nblocks(g.NQ), kBlock, 0, s>>>(g, precond, A.as<double>(), NCC, act.as<int32_t>(), p.ru,
                                                         p.rv, p.zu, p.zv, du, dv, rc, zs);
        CU(cudaGetLastError());
        return CISMGPU_OK;
    }

    // One global sum of a reproducible-sum solve: parallel_global_sum_stagger(au*bu, av*bv)
    // with parallel%reprosum (parallel_mpi.F90:6703-6738), synchronizing the stream.  Non-finite
    // owned summands give the IEEE sum of those summands (NaN, +Inf or -Inf).
    int repro_dot(const double *au, const double *bu, const double *av, const double *bv, double *S) {
        CU(rprod.ensure((size_t)2 * nvec * sizeof(double) + 256));
        double *o1 = rprod.as<double>(), *o2 = o1 + nvec;
        int *dflag = reinterpret_cast<int *>(o2 + nvec);
        CU(cudaMemsetAsync(dflag, 0, sizeof(int), stream));
        k_repro_products<<<nblocks(g.NQ), kBlock, 0, stream>>>(g, au, bu, av, bv, o1, o2, dflag);
        CU(cudaGetLastError());
        int hflag = 0;
        CU(cudaMemcpyAsync(&hflag, dflag, sizeof(int), cudaMemcpyDeviceToHost, stream));
        TRY(repro_global_sum(stream, g, o1, o2, rsum, S));  // synchronizes the stream
        if ((hflag & 1) || (hflag & 6) == 6) *S = std::nan("");
        else if (hflag & 2) *S = HUGE_VAL;
        else if (hflag & 4) *S = -HUGE_VAL;
        return CISMGPU_OK;
    }

    int repro_epilogue(int epi, int iter, double S0, double S1) {
        k_epilogue_value<<<1, 1, 0, stream>>>(state.as<SolveState>(), epi, iter, S0, S1);
        CU(cudaGetLastError());
        return CISMGPU_OK;
    }

    // One global sum in the reference's own order, parallel_global_sum_stagger(au*bu, av*bv)
    // without reprosum (parallel_mpi.F90:6770, :6637), and its scalar epilogue, on the device.
    int seq_dot(const double *au, const double *bu, const double *av, const double *bv, int epi, int iter) {
        SeqArgs a{};
        a.a[0][0] = au; a.b[0][0] = bu;
        a.a[0][1] = av; a.b[0][1] = bv;
        k_seq_sum<1, false><<<1, kBlock, 0, stream>>>(g, a, state.as<SolveState>(), epi, EPI_NONE, iter, nullptr);
        CU(cudaGetLastError());
        return CISMGPU_OK;
    }

    // The two-field form (nflds = 2, parallel_mpi.F90:7042, :6904): field 1 = (a1, b1), field 2
    // = (a2, b2), each summed in the reference's order.  epi2 != EPI_NONE: epilogue epi of S0,
    // then epi2 of S1; otherwise epi(S0, S1).
    int seq_dot2(const double *a1u, const double *b1u, const double *a1v, const double *b1v, const double *a2u,
                 const double *b2u, const double *a2v, const double *b2v, int epi, int epi2, int iter) {
        SeqArgs a{};
        a.a[0][0] = a1u; a.b[0][0] = b1u;
        a.a[0][1] = a1v; a.b[0][1] = b1v;
        a.a[1][0] = a2u; a.b[1][0] = b2u;
        a.a[1][1] = a2v; a.b[1][1] = b2v;
        k_seq_sum<2, false><<<1, kBlock, 0, stream>>>(g, a, state.as<SolveState>(), epi, epi2, iter, nullptr);
        CU(cudaGetLastError());
        return CISMGPU_OK;
    }

    // The state's done flag (synchronizes the stream).
    int read_done(int *done) {
        CU(cudaMemcpyAsync(h_done, &state.as<SolveState>()->done, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        *done = h_done[0];
        return CISMGPU_OK;
    }

    template <int NCC> int run_standard(int precond, int ncheck, double tol, int maxiters);
    template <int NCC> int run_chrongear(int precond, int ncheck, double tol, int maxiters);
    template <int NCC> int run_standard_repro(int precond, int ncheck, double tol, int maxiters);
    template <int NCC> int run_chrongear_repro(int precond, int ncheck, double tol, int maxiters);
    template <int NCC> int run_standard_seq(int precond, int ncheck, double tol, int maxiters);
    template <int NCC> int run_chrongear_seq(int precond, int ncheck, double tol, int maxiters);
    template <int NCC> int run_mixed(int precond, int ncheck, double tol, int maxiters);
};

// pcg_solver_standard_{2d,3d} launch sequence (:1169-1524 / :392-808)
template <int NCC>
int Solver::run_standard(int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = stream;
    SolveState *st = state.as<SolveState>();
    DD *part = partials.as<DD>();
    const Ptrs p = ptrs();
    const VecArgs v = vargs();
    const double *Ad = A.as<double>();
    const int32_t *ac = act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    auto rc = [&](int epi, int iter) { return RedCtx{part, st, epi, iter}; };
    const Geom gg = g;
    prof_bytes = mv_bytes(0);

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    if (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL)
        TRY(tri_setup(precond));  // pcg_precond_init (:1083-1160 / :263-376)
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
    launch_mv<NCC, MV_PLAIN>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr,
                                              nullptr, rc(EPI_NONE, 0));
    k_vec<OP_STD_INIT><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_L2RHS, 0));
    CU(cudaGetLastError());
    Poller poll(*this);
    for (int iter = 1; iter <= maxiters; ++iter) {
        TRY((apply_precond<NCC, PRE_STD>(precond, p, rc(EPI_STD_ETA1, iter), nullptr, nullptr)));
        k_vec<OP_STD_D><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_NONE, iter));
        k_halo<<<hb, kBlock, 0, s>>>(gg, p.du, p.dv, st);
        TRY(timed([&] {
            launch_mv<NCC, MV_DQ>(s, gg, Ad, ac, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr,
                                                   nullptr, rc(EPI_STD_ETA2, iter));
        }));
        k_vec<OP_XR><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_NONE, iter));
        if (is_check(iter, ncheck)) {
            k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
            launch_mv<NCC, MV_RESID>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv,
                                                      rc(EPI_CHECK, iter));
            CU(cudaGetLastError());
            int f = poll.after_check();
            if (f < 0) return fail(CISMGPU_ECUDA, "polling the convergence flag failed");
            if (f) break;
        }
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

// pcg_solver_chrongear_{2d,3d} launch sequence (:3066-3581 / :1913-2613)
template <int NCC>
int Solver::run_chrongear(int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = stream;
    SolveState *st = state.as<SolveState>();
    DD *part = partials.as<DD>();
    const Ptrs p = ptrs();
    const VecArgs v = vargs();
    const double *Ad = A.as<double>();
    const int32_t *ac = act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    auto rc = [&](int epi, int iter) { return RedCtx{part, st, epi, iter}; };
    const Geom gg = g;
    prof_bytes = mv_bytes(1);  // the fused (r,z) dot also reads r
    // 2D with a tridiagonal preconditioner: at most 100 iterations (:1704-1732); 3D keeps maxiters
    const bool tri = precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
    if (tri && NCC == 9) maxiters = 100;

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    if (tri) TRY(tri_setup(precond));  // pcg_precond_init (:2916-3040 / :1747-1880)
    // r = d = z = q = Az = 0 (:3048-3061)
    CU(cudaMemsetAsync(p.ru, 0, (size_t)(VAZ_V - VR_U + 1) * nvec * sizeof(double), s));
    k_vec<OP_DOT_BB><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_L2RHS, 0));
    // first pass (:3085-3290)
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
    launch_mv<NCC, MV_PLAIN>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr,
                                              nullptr, rc(EPI_NONE, 1));
    k_vec<OP_CG_INIT><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_NONE, 1));
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.ru, p.rv, st);
    TRY((apply_precond<NCC, PRE_CG_FIRST>(precond, p, rc(EPI_CG_RHO0, 1), p.du, p.dv)));
    launch_mv<NCC, MV_DQ>(s, gg, Ad, ac, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr, nullptr,
                                           rc(EPI_CG_FIRST, 1));
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.qu, p.qv, st);
    k_vec<OP_XR><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_NONE, 1));
    CU(cudaGetLastError());
    Poller poll(*this);
    for (int iter = 2; iter <= maxiters; ++iter) {
        TRY((apply_precond<NCC, PRE_ONLY>(precond, p, rc(EPI_NONE, iter), nullptr, nullptr)));
        TRY(timed([&] {
            launch_mv<NCC, MV_CG_AZ>(s, gg, Ad, ac, p.zu, p.zv, p.Azu, p.Azv, nullptr, nullptr, p.ru,
                                                      p.rv, rc(EPI_CG_ITER, iter));
        }));
        k_halo<<<hb, kBlock, 0, s>>>(gg, p.Azu, p.Azv, st);
        k_vec<OP_CG_UPD><<<nb, kBlock, 0, s>>>(gg, v, rc(EPI_NONE, iter));
        if (is_check(iter, ncheck)) {
            launch_mv<NCC, MV_RESID>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv,
                                                      rc(EPI_CHECK, iter));
            k_halo<<<hb, kBlock, 0, s>>>(gg, p.ru, p.rv, st);
            CU(cudaGetLastError());
            int f = poll.after_check();
            if (f < 0) return fail(CISMGPU_ECUDA, "polling the convergence flag failed");
            if (f) break;
        }
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

// pcg_solver_standard_{2d,3d} with parallel%reprosum: the launch sequence of run_standard with
// each global sum taken by the reproducible sum (parallel_global_sum_stagger :1216, :1325,
// :1381, :1466 / :441, :631, :687, :754).  The fused kernels run with no epilogue; the sum
// of the same products then feeds the same scalar epilogue, so alpha, beta and err are the
// reference's reprosum values.  The host drives the loop: two short stream synchronizations
// per sum.
template <int NCC>
int Solver::run_standard_repro(int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = stream;
    SolveState *st = state.as<SolveState>();
    DD *part = partials.as<DD>();
    const Ptrs p = ptrs();
    const VecArgs v = vargs();
    const double *Ad = A.as<double>();
    const int32_t *ac = act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    const RedCtx none{part, st, EPI_NONE, 0};
    const Geom gg = g;
    double S0 = 0.0;

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    if (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL)
        TRY(tri_setup(precond));
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
    launch_mv<NCC, MV_PLAIN>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr, nullptr, none);
    k_vec<OP_STD_INIT><<<nb, kBlock, 0, s>>>(gg, v, none);
    CU(cudaGetLastError());
    TRY(repro_dot(p.bu, p.bu, p.bv, p.bv, &S0));
    TRY(repro_epilogue(EPI_L2RHS, 0, S0, 0.0));
    for (int iter = 1; iter <= maxiters; ++iter) {
        TRY((apply_precond<NCC, PRE_STD>(precond, p, none, nullptr, nullptr)));
        TRY(repro_dot(p.ru, p.zu, p.rv, p.zv, &S0));
        TRY(repro_epilogue(EPI_STD_ETA1, iter, S0, 0.0));
        k_vec<OP_STD_D><<<nb, kBlock, 0, s>>>(gg, v, none);
        k_halo<<<hb, kBlock, 0, s>>>(gg, p.du, p.dv, st);
        launch_mv<NCC, MV_DQ>(s, gg, Ad, ac, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr, nullptr, none);
        CU(cudaGetLastError());
        TRY(repro_dot(p.du, p.qu, p.dv, p.qv, &S0));
        TRY(repro_epilogue(EPI_STD_ETA2, iter, S0, 0.0));
        k_vec<OP_XR><<<nb, kBlock, 0, s>>>(gg, v, none);
        int done = 0;
        if (is_check(iter, ncheck)) {
            k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
            launch_mv<NCC, MV_RESID>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv, none);
            CU(cudaGetLastError());
            TRY(repro_dot(p.ru, p.ru, p.rv, p.rv, &S0));
            TRY(repro_epilogue(EPI_CHECK, iter, S0, 0.0));
        }
        TRY(read_done(&done));
        if (done) break;
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

// pcg_solver_chrongear_{2d,3d} with parallel%reprosum: the launch sequence of run_chrongear with
// each global sum taken by the reproducible sum (parallel_global_sum_stagger :1921, :2181
// and :2447 with two fields, :2572 / :3067, :3258, :3426, :3516); the two fields of one call
// are summed independently, as cism_reprosum_calc does per field.
template <int NCC>
int Solver::run_chrongear_repro(int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = stream;
    SolveState *st = state.as<SolveState>();
    DD *part = partials.as<DD>();
    const Ptrs p = ptrs();
    const VecArgs v = vargs();
    const double *Ad = A.as<double>();
    const int32_t *ac = act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    const RedCtx none{part, st, EPI_NONE, 0};
    const Geom gg = g;
    const bool tri = precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
    if (tri && NCC == 9) maxiters = 100;
    double S0 = 0.0, S1 = 0.0;

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    if (tri) TRY(tri_setup(precond));
    CU(cudaMemsetAsync(p.ru, 0, (size_t)(VAZ_V - VR_U + 1) * nvec * sizeof(double), s));
    TRY(repro_dot(p.bu, p.bu, p.bv, p.bv, &S0));
    TRY(repro_epilogue(EPI_L2RHS, 0, S0, 0.0));
    // first pass
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
    launch_mv<NCC, MV_PLAIN>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr, nullptr, none);
    k_vec<OP_CG_INIT><<<nb, kBlock, 0, s>>>(gg, v, none);
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.ru, p.rv, st);
    TRY((apply_precond<NCC, PRE_CG_FIRST>(precond, p, none, p.du, p.dv)));
    launch_mv<NCC, MV_DQ>(s, gg, Ad, ac, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr, nullptr, none);
    CU(cudaGetLastError());
    TRY(repro_dot(p.ru, p.zu, p.rv, p.zv, &S0));
    TRY(repro_dot(p.du, p.qu, p.dv, p.qv, &S1));
    TRY(repro_epilogue(EPI_CG_RHO0, 1, S0, 0.0));
    TRY(repro_epilogue(EPI_CG_FIRST, 1, S1, 0.0));
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.qu, p.qv, st);
    k_vec<OP_XR><<<nb, kBlock, 0, s>>>(gg, v, none);
    CU(cudaGetLastError());
    for (int iter = 2; iter <= maxiters; ++iter) {
        int done = 0;
        TRY(read_done(&done));
        if (done) break;
        TRY((apply_precond<NCC, PRE_ONLY>(precond, p, none, nullptr, nullptr)));
        launch_mv<NCC, MV_CG_AZ>(s, gg, Ad, ac, p.zu, p.zv, p.Azu, p.Azv, nullptr, nullptr, p.ru, p.rv, none);
        CU(cudaGetLastError());
        TRY(repro_dot(p.ru, p.zu, p.rv, p.zv, &S0));
        TRY(repro_dot(p.Azu, p.zu, p.Azv, p.zv, &S1));
        TRY(repro_epilogue(EPI_CG_ITER, iter, S0, S1));
        k_halo<<<hb, kBlock, 0, s>>>(gg, p.Azu, p.Azv, st);
        k_vec<OP_CG_UPD><<<nb, kBlock, 0, s>>>(gg, v, none);
        if (is_check(iter, ncheck)) {
            launch_mv<NCC, MV_RESID>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv, none);
            CU(cudaGetLastError());
            TRY(repro_dot(p.ru, p.ru, p.rv, p.rv, &S0));
            TRY(repro_epilogue(EPI_CHECK, iter, S0, 0.0));
            k_halo<<<hb, kBlock, 0, s>>>(gg, p.ru, p.rv, st);
        }
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

// pcg_solver_standard_{2d,3d} with the reference's own summation order: the launch sequence of
// run_standard, its fused kernels run without their epilogue, and each global sum (:1216,
// :1325, :1381, :1466 / :441, :631, :687, :754) is k_seq_sum over the same products with
// the same scalar epilogue.  Everything stays on the device: the host polls the done flag
// at the checks, with one check period of look-ahead, as in run_standard.
template <int NCC>
int Solver::run_standard_seq(int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = stream;
    SolveState *st = state.as<SolveState>();
    DD *part = partials.as<DD>();
    const Ptrs p = ptrs();
    const VecArgs v = vargs();
    const double *Ad = A.as<double>();
    const int32_t *ac = act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    const RedCtx none{part, st, EPI_NONE, 0};
    const Geom gg = g;
    prof_bytes = mv_bytes(0);

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    if (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL)
        TRY(tri_setup(precond));
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
    launch_mv<NCC, MV_PLAIN>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr, nullptr, none);
    k_vec<OP_STD_INIT><<<nb, kBlock, 0, s>>>(gg, v, none);
    CU(cudaGetLastError());
    TRY(seq_dot(p.bu, p.bu, p.bv, p.bv, EPI_L2RHS, 0));
    Poller poll(*this);
    for (int iter = 1; iter <= maxiters; ++iter) {
        TRY((apply_precond<NCC, PRE_STD>(precond, p, none, nullptr, nullptr)));
        TRY(seq_dot(p.ru, p.zu, p.rv, p.zv, EPI_STD_ETA1, iter));
        k_vec<OP_STD_D><<<nb, kBlock, 0, s>>>(gg, v, none);
        k_halo<<<hb, kBlock, 0, s>>>(gg, p.du, p.dv, st);
        TRY(timed([&] {
            launch_mv<NCC, MV_DQ>(s, gg, Ad, ac, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr, nullptr, none);
        }));
        TRY(seq_dot(p.du, p.qu, p.dv, p.qv, EPI_STD_ETA2, iter));
        k_vec<OP_XR><<<nb, kBlock, 0, s>>>(gg, v, none);
        if (is_check(iter, ncheck)) {
            k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
            launch_mv<NCC, MV_RESID>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv, none);
            TRY(seq_dot(p.ru, p.ru, p.rv, p.rv, EPI_CHECK, iter));
            int f = poll.after_check();
            if (f < 0) return fail(CISMGPU_ECUDA, "polling the convergence flag failed");
            if (f) break;
        }
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

// pcg_solver_chrongear_{2d,3d} with the reference's own summation order: run_chrongear's
// sequence with each sum (:3074, :3248 and :3413 with two fields, :3516 / :1921, :2181,
// :2447, :2551) taken by k_seq_sum; the two-field calls sum both fields in one kernel.
template <int NCC>
int Solver::run_chrongear_seq(int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = stream;
    SolveState *st = state.as<SolveState>();
    DD *part = partials.as<DD>();
    const Ptrs p = ptrs();
    const VecArgs v = vargs();
    const double *Ad = A.as<double>();
    const int32_t *ac = act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    const RedCtx none{part, st, EPI_NONE, 0};
    const Geom gg = g;
    prof_bytes = mv_bytes(1);
    const bool tri = precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
    if (tri && NCC == 9) maxiters = 100;

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    if (tri) TRY(tri_setup(precond));
    CU(cudaMemsetAsync(p.ru, 0, (size_t)(VAZ_V - VR_U + 1) * nvec * sizeof(double), s));
    TRY(seq_dot(p.bu, p.bu, p.bv, p.bv, EPI_L2RHS, 0));
    // first pass
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.xu, p.xv, st);
    launch_mv<NCC, MV_PLAIN>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr, nullptr, none);
    k_vec<OP_CG_INIT><<<nb, kBlock, 0, s>>>(gg, v, none);
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.ru, p.rv, st);
    TRY((apply_precond<NCC, PRE_CG_FIRST>(precond, p, none, p.du, p.dv)));
    launch_mv<NCC, MV_DQ>(s, gg, Ad, ac, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr, nullptr, none);
    TRY(seq_dot2(p.ru, p.zu, p.rv, p.zv, p.du, p.qu, p.dv, p.qv, EPI_CG_RHO0, EPI_CG_FIRST, 1));
    k_halo<<<hb, kBlock, 0, s>>>(gg, p.qu, p.qv, st);
    k_vec<OP_XR><<<nb, kBlock, 0, s>>>(gg, v, none);
    CU(cudaGetLastError());
    Poller poll(*this);
    for (int iter = 2; iter <= maxiters; ++iter) {
        TRY((apply_precond<NCC, PRE_ONLY>(precond, p, none, nullptr, nullptr)));
        TRY(timed([&] {
            launch_mv<NCC, MV_CG_AZ>(s, gg, Ad, ac, p.zu, p.zv, p.Azu, p.Azv, nullptr, nullptr, p.ru, p.rv, none);
        }));
        TRY(seq_dot2(p.ru, p.zu, p.rv, p.zv, p.Azu, p.zu, p.Azv, p.zv, EPI_CG_ITER, EPI_NONE, iter));
        k_halo<<<hb, kBlock, 0, s>>>(gg, p.Azu, p.Azv, st);
        k_vec<OP_CG_UPD><<<nb, kBlock, 0, s>>>(gg, v, none);
        if (is_check(iter, ncheck)) {
            launch_mv<NCC, MV_RESID>(s, gg, Ad, ac, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv, none);
            TRY(seq_dot(p.ru, p.ru, p.rv, p.rv, EPI_CHECK, iter));
            k_halo<<<hb, kBlock, 0, s>>>(gg, p.ru, p.rv, st);
            CU(cudaGetLastError());
            int f = poll.after_check();
            if (f < 0) return fail(CISMGPU_ECUDA, "polling the convergence flag failed");
            if (f) break;
        }
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

// ---------------------------------------------------------------------------
// mixed-precision persistent solver (pcg_mixed.cu): host side
// ---------------------------------------------------------------------------
__global__ void k_mstate_to_solve(const MState *ms, SolveState *st, const MCtl *ctl) {
    st->err = ms->err;
    st->niters = ms->niters;
    st->status = (ctl->abort && !ms->done) ? CISMGPU_ETIMEOUT : ms->status;
    st->checks = ms->checks;
    st->done = 1;
}

// Batched form: member t's result into its handle's SolveState.
__global__ void k_mstates_to_solves(const MState *ms, SolveState *const *dst, int n, const MCtl *ctl) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    SolveState *st = dst[t];
    st->err = ms[t].err;
    st->niters = ms[t].niters;
    st->status = (ctl->abort && !ms[t].done) ? CISMGPU_ETIMEOUT : ms[t].status;
    st->checks = ms[t].checks;
    st->done = 1;
}

static int tiles_for(const Geom &g, int TY) {
    return ((g.ihi - g.ilo + kTX) / kTX) * ((g.jhi - g.jlo + TY) / TY);
}

// Couplings per node the mixed kernels read from HBM: 14 with the symmetric half, else NC.
static int mixed_couplings(const Solver &sv) { return sv.mixed.sym ? 14 : sv.NC; }

static MDesc mixed_desc(const Solver &sv, int precond, int TY) {  // TY: the solve's tile height
    const MixedBufs &m = sv.mixed;
    const long long nvec = sv.nvec;
    const Ptrs p = sv.ptrs();
    MDesc D;
    D.g = sv.g;
    D.NC = sv.NC;
    D.precond = precond;
    D.TY = TY;
    D.tiles_x = (sv.g.ihi - sv.g.ilo + kTX) / kTX;
    D.tiles_y = (sv.g.jhi - sv.g.jlo + TY) / TY;
    D.ntiles = D.tiles_x * D.tiles_y;
    D.A32 = m.A32;
    D.A64 = sv.A.as<double>();
    D.A64i = (m.sym || m.il) ? m.A64i : nullptr;
    D.sym = m.sym ? 1 : 0;
    D.pre = m.pre;
    D.act = sv.act.as<int32_t>();
    D.b = p.bu;
    D.x = p.xu;
    float *V = m.vec;
    const size_t vs = (size_t)2 * nvec;  // one vector = u and v planes
    D.r[0] = V + 0 * vs; D.r[1] = V + 1 * vs;
    D.q[0] = V + 2 * vs; D.q[1] = V + 3 * vs;
    D.Az[0] = V + 4 * vs; D.Az[1] = V + 5 * vs;
    D.z = V + 6 * vs;
    D.d = V + 7 * vs;
    D.recs = m.recs;
    D.bc = m.bc;
    D.dflag = reinterpret_cast<int *>(m.bc + 2 * kBcastCopies);
    D.maps = m.maps;
    D.nbrs = m.nbrs;
    D.stream = (size_t)mixed_couplings(sv) * (size_t)nvec * sizeof(float4) > kStreamBytes ? 1 : 0;
    D.tri = m.tri;
    D.rs = m.tri ? m.tri + 8 * sv.g.NQ : nullptr;
    D.zs = m.tri ? m.tri + 10 * sv.g.NQ : nullptr;
    return D;
}

// Shared memory of the mixed kernel for a tile height (resident: 2D launches with one tile
// per CTA keep the tile's FP32 matrix in shared memory).
static size_t mixed_smem(bool is3d, int nzm, int TY, bool resident = false) {
    if (!is3d) return MLayout<9, 1>(TY, resident).bytes();
    if (nzm == 16) return MLayout<27, 16>(TY, false).bytes();
    return MLayout<27, 32>(TY, false).bytes();
}

static int mixed_nzm(const Geom &g, bool is3d) { return !is3d ? 1 : (g.nz <= 16 ? 16 : 32); }

static const void *mixed_kernel(bool is3d, int nzm) {
    if (!is3d) return (const void *)k_mixed<9, 1>;
    if (nzm == 16) return (const void *)k_mixed<27, 16>;
    return (const void *)k_mixed<27, 32>;
}

// Co-resident CTAs of kernel k with `smem` bytes of dynamic shared memory (0 if it does not fit).
// The kernel's dynamic shared-memory limit is raised once per device to the device's opt-in
// maximum and never lowered: several host threads (the serving loop's admission and epoch threads,
// solves on handles) size and launch the same kernels with different amounts, and a limit set per
// call by one thread could drop below the amount another thread is about to launch with.
static int smem_grid(const void *k, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<int, const void *>> raised;
    int dev = 0, nsm = 0, optin = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    const long long maxdyn = (long long)optin - (long long)fa.sharedSizeBytes;
    if ((long long)smem > maxdyn) return 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        const std::pair<int, const void *> key(dev, k);
        if (std::find(raised.begin(), raised.end(), key) == raised.end()) {
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxdyn) != cudaSuccess)
                return 0;
            raised.push_back(key);
        }
    }
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kBlock, smem) != cudaSuccess) return 0;
    return nsm * occ;
}

// Co-resident CTAs of the mixed kernel at tile height TY (0 if it does not fit).
static int mixed_grid(bool is3d, int nzm, int TY, bool resident = false) {
    return smem_grid(mixed_kernel(is3d, nzm), mixed_smem(is3d, nzm, TY, resident));
}

// Tile autotuner, per solve (a solve's tiling, and so its rounding, never depends on what
// else shares a launch): the smallest tile height whose tiles fit in the co-resident
// CTAs, so that alone every CTA holds one tile per step; 2D first tries the layout that
// keeps the tile's FP32 matrix in shared memory.  If no height fits (very large grids),
// 16 rows (8 for nz > 16), the best load balance measured for streaming-bound solves.
static int mixed_solve_ty(const Geom &g, bool is3d, int nzm) {
    if (!is3d)
        for (int TY = 1; TY <= kMaxTY; ++TY) {
            const int G = mixed_grid(is3d, nzm, TY, true);
            if (G == 0) break;
            if (tiles_for(g, TY) <= G) return TY;
        }
    for (int TY = 1; TY <= kMaxTY; ++TY) {
        const int G = mixed_grid(is3d, nzm, TY);
        if (G == 0) break;
        if (tiles_for(g, TY) <= G) return TY;
    }
    int TY = (nzm == 32) ? 8 : 16;
    while (TY > 1 && mixed_grid(is3d, nzm, TY) == 0) --TY;
    return TY;
}

// Tile height of a solve in batched and served launches (dynamic kernel): the single-solve
// rule's height, but at least `floor` rows, so that a tile carries enough work to hide its
// fixed costs (descriptor, map, broadcast, record).  Depends on the solve (and the floor of
// its dims and nz class) only, so a system gives the same bits alone and in any mix.
// floor: the least height (batch_floor: tuned per dims and nz class, else 4 rows in 3D and 16 in 2D).
static int mixed_batch_ty(const Geom &g, bool is3d, int nzm, int floor) {
    int ty = std::max(mixed_solve_ty(g, is3d, nzm), floor);
    while (ty > 1 && mixed_grid(is3d, nzm, ty) == 0) --ty;
    return ty;
}

// A launch keeps the FP32 matrix in shared memory (2D only) when its tiles fit one per
// co-resident CTA with the shared-memory layout of its tallest tile.
static bool mixed_resident(bool is3d, int nzm, int TYmax, long long ntiles) {
    if (is3d) return false;
    const int G = mixed_grid(is3d, nzm, TYmax, true);
    return G > 0 && ntiles <= G;
}

// Allocate and fill the FP32 copy of the matrix, the preconditioner factors and, for tile
// height TY, the tile slot maps and partial sums.
static int mixed_prepare(Solver &sv, int precond, int TY) {
    if (sv.g.nz > kMixedMaxNz) return fail(CISMGPU_EUNSUPPORTED, "mixed solver supports nz <= 32");
    if (8LL * sv.nvec >= (1LL << 31))  // the kernel indexes vector planes with 32-bit offsets
        return fail(CISMGPU_EUNSUPPORTED, "mixed solver supports nz*(nx-1)*(ny-1) < 2^28");
    if (!(precond == 0 || precond == 1 || (precond == 2 && sv.is3d) || precond == CISMGPU_PRECOND_TRIDIAG_LOCAL ||
          precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL))
        return fail(CISMGPU_EUNSUPPORTED, "mixed solver preconditioners: 0, 1, 2 (3D only), 3 or 4");
    MixedBufs &m = sv.mixed;
    const long long nvec = sv.nvec;
    const int NC = sv.NC;
    const Geom &g = sv.g;
    if (!(m.valid && m.shape_nvec == nvec && m.shape_nc == NC)) {
        m.release();
        size_t bytes = 0;
        auto alloc = [&](void **p, size_t n) -> cudaError_t {
            bytes += n;
            return cudaMalloc(p, n);
        };
        CU(alloc((void **)&m.A32, (size_t)NC * nvec * sizeof(float4)));
        // the interleaved FP64 copy: for a streamed matrix, and in 3D for the symmetric half
        if (NC == 27 || (size_t)NC * (size_t)nvec * sizeof(float4) > kStreamBytes)
            CU(alloc((void **)&m.A64i, (size_t)NC * nvec * 2 * sizeof(double2)));
        CU(alloc((void **)&m.flag, 256));
        CU(alloc((void **)&m.pre, (size_t)6 * nvec * sizeof(float)));
        CU(alloc((void **)&m.vec, (size_t)16 * nvec * sizeof(float)));
        CU(alloc((void **)&m.state, sizeof(MState)));
        CU(alloc((void **)&m.bc, (2 * kBcastCopies + 1) * sizeof(Bcast)));  // + the done-flag line
        CU(alloc((void **)&m.desc, sizeof(MDesc)));
        CU(alloc((void **)&m.ctl, sizeof(MCtl)));
        m.nbytes = bytes;
        m.shape_nvec = nvec;
        m.shape_nc = NC;
        m.valid = true;
        m.stale = true;
        m.TY = 0;
        m.ntiles = 0;
    }
    if (m.stale) {  // new matrix: FP32 copy (couplings leaving the grid set to zero)
        // 3D: an exactly symmetric matrix is stored as its symmetric half (14 of 27 couplings)
        m.sym = false;
        if (NC == 27) {
            CU(cudaMemsetAsync(m.flag, 0, sizeof(int), sv.stream));
            k_sym_exact3d<<<nblocks(g.NQ), kBlock, 0, sv.stream>>>(g, sv.act.as<int32_t>(), sv.A.as<double>(), m.flag);
            CU(cudaGetLastError());
            int hflag = 1;
            CU(cudaMemcpyAsync(&hflag, m.flag, sizeof(int), cudaMemcpyDeviceToHost, sv.stream));
            CU(cudaStreamSynchronize(sv.stream));
            m.sym = hflag == 0 && !g_mixed_full_storage.load();
        }
        // the interleaved FP64 copy: always in 3D (the check steps read it with the x tile in
        // shared memory), in 2D for a streamed matrix
        m.il = !m.sym && m.A64i != nullptr && (NC == 27 || (size_t)NC * (size_t)nvec * sizeof(float4) > kStreamBytes);
        if (m.sym) k_to_half<<<1184, kBlock, 0, sv.stream>>>(g, sv.A.as<double>(), m.A32, m.A64i);
        else if (NC == 27) k_to_f32<27><<<1184, kBlock, 0, sv.stream>>>(g, sv.A.as<double>(), m.A32, m.il ? m.A64i : nullptr);
        else k_to_f32<9><<<1184, kBlock, 0, sv.stream>>>(g, sv.A.as<double>(), m.A32, m.A64i);
        CU(cudaGetLastError());
        m.stale = false;
        m.precond = -1;
        m.TY = 0;  // the active mask may have changed: rebuild the slot maps
    }
    if (m.TY != TY) {
        const int ntiles = tiles_for(g, TY);
        const int NS = (kTX + 2) * (TY + 2);
        if (ntiles > m.ntiles_cap || (long long)ntiles * NS > m.maps_cap) {
            if (m.recs) cudaFree(m.recs);
            if (m.maps) cudaFree(m.maps);
            if (m.nbrs) cudaFree(m.nbrs);
            if (m.tiles) cudaFree(m.tiles);
            m.recs = nullptr;
            m.maps = nullptr;
            m.nbrs = nullptr;
            m.tiles = nullptr;
            CU(cudaMalloc((void **)&m.recs, (size_t)kRecCopies * ntiles * 2 * sizeof(TileRec)));
            CU(cudaMalloc((void **)&m.maps, (size_t)ntiles * NS * sizeof(int)));
            CU(cudaMalloc((void **)&m.nbrs, (size_t)ntiles * kNbrStride * sizeof(int)));
            CU(cudaMalloc((void **)&m.tiles, (size_t)ntiles * sizeof(MTile)));
            m.ntiles_cap = ntiles;
            m.maps_cap = (long long)ntiles * NS;
        }
        m.ntiles = ntiles;
        const MDesc D = mixed_desc(sv, precond, TY);
        k_slot_maps<<<nblocks((long long)ntiles * NS), kBlock, 0, sv.stream>>>(D, m.maps);
        CU(cudaGetLastError());
        k_tile_nbrs<<<nblocks(ntiles), kBlock, 0, sv.stream>>>(D, m.maps, m.nbrs);
        CU(cudaGetLastError());
        std::vector<MTile> tl(ntiles);
        for (int t = 0; t < ntiles; ++t) tl[t] = MTile{0, t};
        CU(cudaMemcpyAsync(m.tiles, tl.data(), ntiles * sizeof(MTile), cudaMemcpyHostToDevice, sv.stream));
        CU(cudaStreamSynchronize(sv.stream));  // tl goes out of scope
        m.TY = TY;
    }
    if (m.precond != precond) {
        const bool tri = precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
        // the 3D line preconditioners start with the SIA column solves (tridiag_solver_local_3d)
        const int kind = tri ? (NC == 27 ? CISMGPU_PRECOND_SIA : CISMGPU_PRECOND_NONE) : precond;
        if (NC == 27)
            k_mixed_precond_setup<27><<<nblocks(g.NQ), kBlock, 0, sv.stream>>>(g, kind, sv.A.as<double>(), m.pre);
        else
            k_mixed_precond_setup<9><<<nblocks(g.NQ), kBlock, 0, sv.stream>>>(g, kind, sv.A.as<double>(), m.pre);
        CU(cudaGetLastError());
        if (tri) {  // the FP64 setup (its zero-pivot check included), then the FP32 factors
            if (!m.tri) {
                CU(cudaMalloc((void **)&m.tri, (size_t)12 * g.NQ * sizeof(float)));
                m.nbytes += (size_t)12 * g.NQ * sizeof(float);
            }
            SolveState *st = sv.state.as<SolveState>();
            k_init_state<<<1, 1, 0, sv.stream>>>(st, 0.0, 0);
            TRY(sv.tri_setup(precond));
            k_tri_to_f32<<<nblocks(g.NQ), kBlock, 0, sv.stream>>>(g, sv.tri.as<double>(), m.tri);
            CU(cudaGetLastError());
            int hst = 0;
            CU(cudaMemcpyAsync(&hst, &st->status, sizeof(int), cudaMemcpyDeviceToHost, sv.stream));
            CU(cudaStreamSynchronize(sv.stream));
            if (hst == CISMGPU_EDIVZERO) {
                m.precond = -1;
                return fail(CISMGPU_EDIVZERO, "tridiagonal preconditioner setup met a zero pivot");
            }
        }
        m.precond = precond;
    }
    return CISMGPU_OK;
}

// precond 3 and 4 take three steps per iteration (MS_UPD, MS_LINES).  The mixed solver runs them to
// the caller's maxiters: the reference's 2D budget of 100 iterations for these preconditioners
// (maxiters_tridiag, glissade_velo_higher_pcg.F90:1703-1732, which the FP64 solvers keep) is a
// heuristic for FP64 iterations, and the FP32 recurrences can need more of them.
static MState mixed_init_state(double tol, int maxiters, int ncheck, int precond = 0) {
    MState S;
    std::memset(&S, 0, sizeof(S));
    const bool tri = precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL;
    S.tri = tri ? 1 : 0;
    S.tol = tol;
    S.maxiters = maxiters;
    S.ncheck = ncheck;
    S.niters = maxiters;
    S.step = MS_INIT;
    S.err = std::nan("");
    return S;
}

// The reference starts with halo(x) (:3094-3097) and, with inactive halo vertices and the
// diagonal or SIA preconditioner, never changes x there again; the mixed kernel writes
// only owned unknowns, so x leaves with the same halo values.
static int mixed_reset(Solver &sv, cudaStream_t s) {
    const Ptrs p = sv.ptrs();
    sv.x_current = true;
    CU(cudaMemcpyAsync(p.xu, p.x0u, 2 * sv.nvec * sizeof(double), cudaMemcpyDeviceToDevice, s));
    k_halo<<<nblocks(4LL * sv.g.NX + 4LL * (sv.g.NY - 4)), kBlock, 0, s>>>(sv.g, p.xu, p.xv, nullptr);
    CU(cudaGetLastError());
    CU(cudaMemsetAsync(sv.mixed.vec, 0, (size_t)16 * sv.nvec * sizeof(float), s));
    CU(cudaMemsetAsync(sv.mixed.recs, 0, (size_t)kRecCopies * sv.mixed.ntiles * 2 * sizeof(TileRec), s));  // tags restart at 1
    CU(cudaMemsetAsync(sv.mixed.bc, 0, (2 * kBcastCopies + 1) * sizeof(Bcast), s));       // broadcast tag 0 = x0 state
    return CISMGPU_OK;
}

// Co-resident grid of a launch (sets the kernel's shared-memory attribute; call outside any
// stream capture).  0 if the kernel does not fit.
static int mixed_launch_grid(bool is3d, int nzm, int TY, bool resident, int ntiles) {
    const int grid = mixed_grid(is3d, nzm, TY, resident);
    if (grid < 1) return 0;
    if (resident && grid < ntiles) return 0;
    return std::min(grid, ntiles);
}

template <int NC, int NZM>
static int mixed_launch(const MDesc *d_descs, MState *d_states, const MTile *d_tiles, int ntiles, int TY,
                        int resident, MCtl *d_ctl, int max_steps, int grid, cudaStream_t s) {
    const size_t smem = MLayout<NC, NZM>(TY, resident != 0).bytes();
    void *args[] = {(void *)&d_descs, (void *)&d_states, (void *)&d_tiles, (void *)&ntiles, (void *)&TY,
                    (void *)&resident, (void *)&d_ctl, (void *)&max_steps};
    CU(cudaLaunchCooperativeKernel((const void *)k_mixed<NC, NZM>, dim3(grid), dim3(kBlock), args, smem, s));
    return CISMGPU_OK;
}

template <int NC, int NZM>
static int mixed_dyn_launch(const MDesc *d_descs, MState *const *d_states, const unsigned *d_tick0, int nsolve,
                            const MTile *d_tiles, int ntiles, int TY, MCtl *d_ctl, int max_steps, int grid,
                            cudaStream_t s) {
    const size_t smem = MLayout<NC, NZM>(TY, false).bytes();
    int TY2 = TY;
    void *args[] = {(void *)&d_descs, (void *)&d_states, (void *)&d_tick0, (void *)&nsolve, (void *)&d_tiles,
                    (void *)&ntiles, (void *)&TY, (void *)&TY2, (void *)&d_ctl, (void *)&max_steps};
    CU(cudaLaunchCooperativeKernel((const void *)k_mixed_dyn<NC, NZM>, dim3(grid), dim3(kBlock), args, smem, s));
    return CISMGPU_OK;
}

// Shared memory of the 2D + 3D (nz <= 16) dynamic kernel: the larger of the two layouts.
static size_t mixed_multi_smem(int TY3, int TY2) {
    return std::max(MLayout<27, 16>(TY3, false).bytes(), MLayout<9, 1>(TY2, false).bytes());
}

// One launch of 2D and 3D (nz <= 16) solves together: 3D tiles of height at most TY3, 2D at most TY2.
static int mixed_multi_launch(const MDesc *d_descs, MState *const *d_states, const unsigned *d_tick0, int nsolve,
                              const MTile *d_tiles, int ntiles, int TY3, int TY2, MCtl *d_ctl, int max_steps,
                              int grid, cudaStream_t s) {
    const size_t smem = mixed_multi_smem(TY3, TY2);
    void *args[] = {(void *)&d_descs, (void *)&d_states, (void *)&d_tick0, (void *)&nsolve, (void *)&d_tiles,
                    (void *)&ntiles, (void *)&TY3, (void *)&TY2, (void *)&d_ctl, (void *)&max_steps};
    CU(cudaLaunchCooperativeKernel((const void *)k_mixed_dyn<27, 16, true>, dim3(grid), dim3(kBlock), args, smem, s));
    return CISMGPU_OK;
}

static const void *mixed_dyn_kernel(bool is3d, int nzm) {
    if (!is3d) return (const void *)k_mixed_dyn<9, 1>;
    if (nzm == 16) return (const void *)k_mixed_dyn<27, 16>;
    return (const void *)k_mixed_dyn<27, 32>;
}

static int mixed_multi_grid(int TY3, int TY2) {
    return smem_grid((const void *)k_mixed_dyn<27, 16, true>, mixed_multi_smem(TY3, TY2));
}

// Co-resident CTAs of the dynamic kernel at tile height TY (0 if it does not fit).
static int mixed_dyn_grid(bool is3d, int nzm, int TY) {
    return smem_grid(mixed_dyn_kernel(is3d, nzm), mixed_smem(is3d, nzm, TY, false));
}

static int mixed_dyn_dispatch(bool is3d, int nzm, const MDesc *d, MState *const *st, const unsigned *tick0, int nsolve,
                              const MTile *t, int nt, int TY, MCtl *ctl, int max_steps, int grid, cudaStream_t s) {
    if (!is3d) return mixed_dyn_launch<9, 1>(d, st, tick0, nsolve, t, nt, TY, ctl, max_steps, grid, s);
    if (nzm == 16) return mixed_dyn_launch<27, 16>(d, st, tick0, nsolve, t, nt, TY, ctl, max_steps, grid, s);
    return mixed_dyn_launch<27, 32>(d, st, tick0, nsolve, t, nt, TY, ctl, max_steps, grid, s);
}

static int mixed_dispatch(bool is3d, int nzm, const MDesc *d, MState *st, const MTile *t, int nt, int TY,
                          bool resident, MCtl *ctl, int max_steps, int grid, cudaStream_t s) {
    const int res = resident ? 1 : 0;
    if (!is3d) return mixed_launch<9, 1>(d, st, t, nt, TY, res, ctl, max_steps, grid, s);
    if (nzm == 16) return mixed_launch<27, 16>(d, st, t, nt, TY, 0, ctl, max_steps, grid, s);
    return mixed_launch<27, 32>(d, st, t, nt, TY, 0, ctl, max_steps, grid, s);
}

static double mixed_iter_bytes(const Solver &sv, int precond) {
    const double pre = precond == 2 ? 24.0 : (precond == 1 ? 8.0 : 0.0);
    return (double)sv.n_active_owned * sv.g.nz * (4.0 * mixed_couplings(sv) * 4.0 + 40.0 + 32.0 + 40.0 + pre);
}

static double mixed_check_bytes(const Solver &sv) {
    // FP64 residual (matrix, x, b, r32) + the fused update (z, d, q, Az loads, q store) + the
    // deferred owner writes of the next step (d, z, x loads, d, x stores)
    return (double)sv.n_active_owned * sv.g.nz * (4.0 * mixed_couplings(sv) * 8.0 + 16.0 + 16.0 + 8.0 + 20.0 + 28.0);
}

// One mixed solve at tile height TY on the solver's stream (enqueued; the result lands in the
// solver's SolveState).  ms: device time of the persistent launch (synchronizes).
static int mixed_run(Solver &sv, int precond, int ncheck, double tol, int maxiters, int TY, float *ms,
                     MState *out = nullptr) {
    const bool is3d = sv.is3d;
    const int nzm = mixed_nzm(sv.g, is3d);
    cudaStream_t stream = sv.stream;
    TRY(mixed_prepare(sv, precond, TY));
    TRY(mixed_reset(sv, stream));
    MixedBufs &m = sv.mixed;
    const bool resident = mixed_resident(is3d, nzm, TY, m.ntiles);
    const MDesc D = mixed_desc(sv, precond, TY);
    const MState S0 = mixed_init_state(tol, maxiters, ncheck, precond);
    CU(cudaMemcpyAsync(m.desc, &D, sizeof(MDesc), cudaMemcpyHostToDevice, stream));
    CU(cudaMemcpyAsync(m.state, &S0, sizeof(MState), cudaMemcpyHostToDevice, stream));
    CU(cudaMemsetAsync(m.ctl, 0, sizeof(MCtl), stream));
    const int max_steps = 4 * maxiters + 16;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
        CU(cudaEventCreate(&e0));
        CU(cudaEventCreate(&e1));
        CU(cudaEventRecord(e0, stream));
    }
    const int grid = mixed_launch_grid(is3d, nzm, TY, resident, m.ntiles);
    if (grid < 1) return fail(CISMGPU_EUNSUPPORTED, "mixed kernel does not fit on an SM at this tile height");
    TRY(mixed_dispatch(is3d, nzm, m.desc, m.state, m.tiles, m.ntiles, TY, resident, m.ctl, max_steps, grid, stream));
    if (ms) CU(cudaEventRecord(e1, stream));
    k_mstate_to_solve<<<1, 1, 0, stream>>>(m.state, sv.state.as<SolveState>(), m.ctl);
    CU(cudaGetLastError());
    if (out) CU(cudaMemcpyAsync(out, m.state, sizeof(MState), cudaMemcpyDeviceToHost, stream));
    if (ms) {
        CU(cudaStreamSynchronize(stream));
        CU(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return CISMGPU_OK;
}

// ---------------------------------------------------------------------------
// Tile-height tuner
// ---------------------------------------------------------------------------
// The mixed kernels cut a solve's owned vertices into 32 x TY tiles.  TY trades the fixed costs
// of a tile (slot map, record, broadcast wait) and the halo ring recomputed around it against
// parallelism (tiles per co-resident CTA) and shared memory per CTA.  The tuner times the
// candidate heights on the system itself the first time it meets a key, and keeps the winner
// for the rest of the process and in a cache file, so that a system's tiling -- and with it the
// order of its sums -- depends on the system alone:
//  * single solves: key (dims, nz, layout, tile columns, height bucket); every height that fits
//    on an SM is timed on a short solve of the actual system (kTuneIters iterations, tol 0),
//    best of two;
//  * batches and serving: key (dims, nz class): the least height of every member's tiles,
//    timed on a launch of kTuneSteps steps of the first batch that meets the key (48 steps
//    picked a floor that was faster early in the solve and slower over all of it).
// The occupancy rule (mixed_solve_ty; batch floors 4 rows in 3D and 16 in 2D) is the default and
// keeps its place unless a candidate is more than 3 % faster.  The serving loop never times (its
// launches share the GPU) and uses the table or the default.  CISMGPU_TILE_TUNING=0 turns timing
// off; the cache file is $CISMGPU_TILE_CACHE, else $HOME/.cache/cismgpu/tiles-<GPU name>.txt.
constexpr int kTuneIters = 12;
constexpr int kTuneSteps = 400;  // batch floors: long enough to see more than the first check

struct TileTuner {
    std::mutex mu;
    bool loaded = false;
    int timing = -1;  // -1 not read yet
    std::string path;
    std::map<std::string, int> table;
    std::vector<std::string> log;  // what was measured in this process, for cismgpu_tile_table

    bool timing_on() {
        if (timing < 0) {
            const char *e = std::getenv("CISMGPU_TILE_TUNING");
            timing = (e && e[0] == '0') ? 0 : 1;
        }
        return timing == 1;
    }
    void load() {  // caller holds mu
        if (loaded) return;
        loaded = true;
        const char *e = std::getenv("CISMGPU_TILE_CACHE");
        if (e && e[0]) {
            path = e;
        } else {
            const char *home = std::getenv("HOME");
            cudaDeviceProp prop;
            int dev = 0;
            std::string name = "gpu";
            if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) name = prop.name;
            for (char &c : name)
                if (!std::isalnum((unsigned char)c)) c = '_';
            if (home && home[0]) path = std::string(home) + "/.cache/cismgpu/tiles-" + name + ".txt";
        }
        if (path.empty()) return;
        std::ifstream f(path);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string key;
            int v = 0;
            if (ss >> key >> v && v > 0 && v <= kMaxTY) table[key] = v;
        }
    }
    int get(const std::string &key) {
        std::lock_guard<std::mutex> lk(mu);
        load();
        auto it = table.find(key);
        return it == table.end() ? 0 : it->second;
    }
    void put(const std::string &key, int v, const std::string &note) {
        std::lock_guard<std::mutex> lk(mu);
        load();
        table[key] = v;
        log.push_back(key + " " + std::to_string(v) + " # " + note);
        if (path.empty()) return;
        for (size_t p = path.find('/', 1); p != std::string::npos; p = path.find('/', p + 1))
            (void)::mkdir(path.substr(0, p).c_str(), 0755);  // the cache directory, best effort
        std::ofstream f(path, std::ios::app);
        if (f) f << key << " " << v << " # " << note << "\n";
    }
};
static TileTuner g_tiles;

static std::string tile_key_single(const Solver &sv, int nzm) {
    const int W = sv.g.ihi - sv.g.ilo + 1, H = sv.g.jhi - sv.g.jlo + 1;
    const int hb = (int)std::lround(4.0 * std::log2((double)std::max(H, 1)));
    std::ostringstream k;
    k << "solve:" << (sv.is3d ? "3d" : "2d") << ":nzm" << nzm << ":nz" << sv.g.nz << ":" << (sv.mixed.sym ? "half" : "full")
      << ":tx" << (W + kTX - 1) / kTX << ":hb" << hb;
    return k.str();
}

static std::string tile_key_batch(bool is3d, int nzm) {
    return std::string("batch:") + (is3d ? "3d" : "2d") + ":nzm" + std::to_string(nzm);
}

// The single-solve tile height of sv (prepared with the default height, so its layout is set).
static int tuned_solve_ty(Solver &sv, int precond, int nzm, int TYdef, int *TY) {
    const std::string key = tile_key_single(sv, nzm);
    int v = g_tiles.get(key);
    if (v > 0 && mixed_grid(sv.is3d, nzm, v, false) > 0) {
        *TY = v;
        return CISMGPU_OK;
    }
    *TY = TYdef;
    if (!g_tiles.timing_on()) return CISMGPU_OK;
    std::vector<int> cand = {TYdef};
    for (int ty : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32})
        if (ty != TYdef && ty <= kMaxTY && mixed_grid(sv.is3d, nzm, ty, false) > 0) cand.push_back(ty);
    float tdef = 0.f, tbest = 0.f;
    int arg = TYdef;
    std::ostringstream note;
    for (int ty : cand) {
        float t = 0.f, u = 0.f;
        TRY(mixed_run(sv, precond, 5, 0.0, kTuneIters, ty, &t));
        TRY(mixed_run(sv, precond, 5, 0.0, kTuneIters, ty, &u));
        t = std::min(t, u);
        note << ty << ":" << t << "ms ";
        if (ty == TYdef) tdef = t;
        if (ty == TYdef || t < tbest) {
            tbest = t;
            arg = ty;
        }
    }
    if (tbest >= 0.97f * tdef) arg = TYdef;  // the default unless a candidate is clearly faster
    g_tiles.put(key, arg, note.str() + "(default " + std::to_string(TYdef) + ")");
    *TY = arg;
    return CISMGPU_OK;
}

static int batch_floor(bool is3d, int nzm) {
    const int v = g_tiles.get(tile_key_batch(is3d, nzm));
    return v > 0 ? v : (is3d ? 4 : 16);
}

template <int NCC>
int Solver::run_mixed(int precond, int ncheck, double tol, int maxiters) {
    trace("run_mixed: begin");
    const int nzm = mixed_nzm(g, is3d);
    const int TYdef = mixed_solve_ty(g, is3d, nzm);
    TRY(mixed_prepare(*this, precond, TYdef));  // the matrix layout, which the key names
    int TY = TYdef;
    TRY(tuned_solve_ty(*this, precond, nzm, TYdef, &TY));
    trace("run_mixed: tile height chosen");
    MState hs;
    float ms = 0.f;
    TRY(mixed_run(*this, precond, ncheck, tol, maxiters, TY, prof ? &ms : nullptr, prof ? &hs : nullptr));
    last_ty = TY;
    if (prof) {
        prof_ms += ms;
        prof_n += 1;
        prof_bytes = hs.fp32_matvecs * mixed_iter_bytes(*this, precond) + hs.fp64_matvecs * mixed_check_bytes(*this);
    }
    return CISMGPU_OK;
}

enum Algo { ALG_STANDARD = CISMGPU_ALG_STANDARD, ALG_CHRONGEAR = CISMGPU_ALG_CHRONGEAR,
            ALG_MIXED = CISMGPU_ALG_MIXED_CHRONGEAR };

// Order of the FP64 solvers' global sums when parallel%reprosum is off (cismgpu_set_sum_order).
static std::atomic<int> g_sum_order{CISMGPU_SUM_TREE};

static int run_algorithm(Solver &sv, int alg, int precond, int ncheck, double tol, int maxiters) {
    const bool seq = !sv.repro && g_sum_order.load() == CISMGPU_SUM_SEQUENTIAL;
    if (seq && alg == ALG_STANDARD)
        return sv.is3d ? sv.run_standard_seq<27>(precond, ncheck, tol, maxiters)
                       : sv.run_standard_seq<9>(precond, ncheck, tol, maxiters);
    if (seq && alg == ALG_CHRONGEAR)
        return sv.is3d ? sv.run_chrongear_seq<27>(precond, ncheck, tol, maxiters)
                       : sv.run_chrongear_seq<9>(precond, ncheck, tol, maxiters);
    if (sv.repro && alg == ALG_STANDARD)
        return sv.is3d ? sv.run_standard_repro<27>(precond, ncheck, tol, maxiters)
                       : sv.run_standard_repro<9>(precond, ncheck, tol, maxiters);
    if (sv.repro && alg == ALG_CHRONGEAR)
        return sv.is3d ? sv.run_chrongear_repro<27>(precond, ncheck, tol, maxiters)
                       : sv.run_chrongear_repro<9>(precond, ncheck, tol, maxiters);
    if (alg == ALG_STANDARD)
        return sv.is3d ? sv.run_standard<27>(precond, ncheck, tol, maxiters)
                       : sv.run_standard<9>(precond, ncheck, tol, maxiters);
    if (alg == ALG_CHRONGEAR)
        return sv.is3d ? sv.run_chrongear<27>(precond, ncheck, tol, maxiters)
                       : sv.run_chrongear<9>(precond, ncheck, tol, maxiters);
    if (alg == ALG_MIXED)
        return sv.is3d ? sv.run_mixed<27>(precond, ncheck, tol, maxiters)
                       : sv.run_mixed<9>(precond, ncheck, tol, maxiters);
    return fail(CISMGPU_EINVAL, "unknown algorithm");
}

// Grid sizes and owned bounds every entry point shares.
static int validate_geom(int nx, int ny, int nz, const cismgpu_par_t *par) {
    if (!par) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6 || nz < 1 || nz > kMaxNz)
        return fail(CISMGPU_EINVAL, "grid too small or nz outside 1..64");
    if (par->tasks_row * par->tasks_col != 1)
        return fail(CISMGPU_EUNSUPPORTED, "the whole domain must be on one GPU (tasks_row*tasks_col == 1)");
    if (par->staggered_ilo < 1 || par->staggered_ihi > nx - 1 || par->staggered_ilo > par->staggered_ihi ||
        par->staggered_jlo < 1 || par->staggered_jhi > ny - 1 || par->staggered_jlo > par->staggered_jhi)
        return fail(CISMGPU_EINVAL, "owned vertex bounds outside the array");
    return CISMGPU_OK;
}

static int validate(int nx, int ny, int nz, const cismgpu_par_t *par, const void *indx, const void *act,
                    const void *A0, const void *A1, const void *A2, const void *A3, const void *bu,
                    const void *bv) {
    if (!par || !indx || !act || !A0 || !A1 || !A2 || !A3 || !bu || !bv)
        return fail(CISMGPU_EINVAL, "null pointer argument");
    return validate_geom(nx, ny, nz, par);
}

static int validate_solve_args(int precond, int ncheck, int maxiters) {
    if (ncheck < 1) return fail(CISMGPU_EINVAL, "linear_solve_ncheck must be >= 1");
    if (maxiters < 0) return fail(CISMGPU_EINVAL, "maxiters must be >= 0");
    (void)precond;  // every value is accepted: 0-4 have branches, others take none (as the reference)
    return CISMGPU_OK;
}

// indxA entries index the caller's coefficient dimension on the device: each must lie in 1..NC.
static int validate_indx(const int32_t *indx, int NC) {
    for (int c = 0; c < NC; ++c)
        if (indx[c] < 1 || indx[c] > NC) return fail(CISMGPU_EINVAL, "indxA entry outside 1..27 / 1..9");
    return CISMGPU_OK;
}

static Geom make_geom(int nx, int ny, int nz, const cismgpu_par_t *par) {
    Geom g;
    g.NX = nx - 1;
    g.NY = ny - 1;
    g.nz = nz;
    g.NQ = (long long)g.NX * g.NY;
    g.ilo = par->staggered_ilo - 1;
    g.ihi = par->staggered_ihi - 1;
    g.jlo = par->staggered_jlo - 1;
    g.jhi = par->staggered_jhi - 1;
    g.periodic = par->periodic_bc != 0;
    g.outflow = par->outflow_bc != 0;
    g.no_ice = par->no_ice_bc != 0;
    return g;
}

static std::mutex g_mu;
static Solver *g_oneshot = nullptr;  // cached Solver of the one-shot calls
static int g_oneshot_alg = -1;       // -1: the reference algorithm each call names

static int oneshot_solve(int alg, bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx2,
                         const int32_t *indx3, const int32_t *act, const double *Auu, const double *Auv,
                         const double *Avu, const double *Avv, const double *bu, const double *bv, double *xu,
                         double *xv, int precond, int ncheck, double tol, int maxiters, double *err, int *niters) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    const int32_t *indx = is3d ? indx3 : indx2;
    if (!xu || !xv || !err || !niters) return fail(CISMGPU_EINVAL, "null pointer argument");
    TRY(validate(nx, ny, is3d ? nz : 1, par, indx, act, Auu, Auv, Avu, Avv, bu, bv));
    TRY(validate_solve_args(precond, ncheck, maxiters));
    TRY(validate_indx(indx, is3d ? 27 : 9));
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    TRY(sv.upload(make_geom(nx, ny, is3d ? nz : 1, par), is3d, indx, act, blocks, bu, bv, xu, xv));
    sv.repro = par->reprosum != 0;
    if (is3d && indx2)
        for (int c = 0; c < 9; ++c) sv.hindx2[c] = indx2[c];
    TRY(sv.begin_solve());
    TRY(run_algorithm(sv, g_oneshot_alg >= 0 ? g_oneshot_alg : alg, precond, ncheck, tol, maxiters));
    int rc = sv.finish_solve(err, niters);
    TRY(sv.download(VX_U, VX_V, xu, xv));
    return rc;
}

static int oneshot_matvec(bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx,
                          const int32_t *act, const double *Auu, const double *Auv, const double *Avu,
                          const double *Avv, const double *xu, const double *xv, double *yu, double *yv) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    TRY(validate(nx, ny, is3d ? nz : 1, par, indx, act, Auu, Auv, Avu, Avv, xu, xv));
    TRY(validate_indx(indx, is3d ? 27 : 9));
    if (!yu || !yv) return fail(CISMGPU_EINVAL, "null output pointer");
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    TRY(sv.upload(make_geom(nx, ny, is3d ? nz : 1, par), is3d, indx, act, blocks, xu, xv, nullptr, nullptr));
    const Ptrs p = sv.ptrs();
    SolveState *st = sv.state.as<SolveState>();
    k_init_state<<<1, 1, 0, sv.stream>>>(st, 0.0, 0);
    RedCtx rc0{sv.partials.as<DD>(), st, EPI_NONE, 0};
    if (is3d)
        launch_mv<27, MV_PLAIN>(sv.stream, sv.g, sv.A.as<double>(), sv.act.as<int32_t>(),
                                                                      p.bu, p.bv, p.xu, p.xv, nullptr, nullptr,
                                                                      nullptr, nullptr, rc0);
    else
        launch_mv<9, MV_PLAIN>(sv.stream, sv.g, sv.A.as<double>(), sv.act.as<int32_t>(),
                                                                     p.bu, p.bv, p.xu, p.xv, nullptr, nullptr,
                                                                     nullptr, nullptr, rc0);
    CU(cudaGetLastError());
    return sv.download(VX_U, VX_V, yu, yv);
}

static int oneshot_resid_vec(bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx,
                             const int32_t *act, const double *Auu, const double *Auv, const double *Avu,
                             const double *Avv, const double *bu, const double *bv, const double *uvel,
                             const double *vvel, double *resid_u, double *resid_v, double *L2_norm,
                             double *L2_norm_relative) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    TRY(validate(nx, ny, is3d ? nz : 1, par, indx, act, Auu, Auv, Avu, Avv, bu, bv));
    TRY(validate_indx(indx, is3d ? 27 : 9));
    if (!uvel || !vvel || !resid_u || !resid_v || !L2_norm) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    TRY(sv.upload(make_geom(nx, ny, is3d ? nz : 1, par), is3d, indx, act, blocks, bu, bv, uvel, vvel));
    double l2 = 0.0, l2b = 0.0;
    TRY(sv.residual_vector(VX0_U, &l2, &l2b));
    TRY(sv.download(VR_U, VR_V, resid_u, resid_v));
    *L2_norm = l2;
    if (L2_norm_relative) *L2_norm_relative = (l2b > 0.0) ? l2 / l2b : 0.0;  // :9886-9890
    return CISMGPU_OK;
}

// check_symmetry_assembled_matrix_{3d,2d} on the caller's blocks: copied to the device in the
// caller's own layout, checked there and, in 3D, copied back with the averages written in.
static int oneshot_symmetry(bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx,
                            const int32_t *act, double *const blocks[4], double *maxdiff, long long *nwarn) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    if (!par || !indx || !act || !blocks[0] || !blocks[1] || !blocks[2] || !blocks[3] || !maxdiff || !nwarn)
        return fail(CISMGPU_EINVAL, "null pointer argument");
    TRY(validate_geom(nx, ny, is3d ? nz : 1, par));
    TRY(validate_indx(indx, is3d ? 27 : 9));
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, is3d ? nz : 1, par), is3d));
    const Geom &g = sv.g;
    cudaStream_t s = sv.stream;
    CU(sv.act.ensure((size_t)g.NQ * sizeof(int32_t)));
    CU(cudaMemcpyAsync(sv.act.p, act, (size_t)g.NQ * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    const size_t bs = (size_t)sv.NC * sv.nvec;
    CU(sv.A.ensure(4 * bs * sizeof(double)));
    sv.mixed.stale = true;  // the matrix buffer holds the caller's layout until the next upload
    double *A0 = sv.A.as<double>();
    for (int b = 0; b < 4; ++b)
        CU(cudaMemcpyAsync(A0 + b * bs, blocks[b], bs * sizeof(double), cudaMemcpyHostToDevice, s));
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c < sv.NC ? indx[c] : 1;
    L.n = sv.nvec;
    L.NQ = g.NQ;
    L.nz = g.nz;
    L.raw3 = is3d ? 1 : 0;
    TRY(sv.sym_check(L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, maxdiff, nwarn));
    if (is3d) {
        for (int b = 0; b < 4; ++b)
            CU(cudaMemcpyAsync(blocks[b], A0 + b * bs, bs * sizeof(double), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
    }
    return CISMGPU_OK;
}

static int validate_assembly(int nx, int ny, int nz, int nhalo, int whichefvs, double n_glen, const void *sigma,
                             const void *act, const void *xv, const void *yv, const void *usrf, const void *thck,
                             const void *ff) {
    if (!sigma || !act || !xv || !yv || !usrf || !thck || !ff) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6 || nz < 2 || nz > kMaxNz) return fail(CISMGPU_EINVAL, "grid too small or nz outside 2..64");
    if (nhalo < 2 || 2 * nhalo >= nx || 2 * nhalo >= ny)
        return fail(CISMGPU_EINVAL, "nhalo must be >= 2 (element vertices inside the arrays) and fit the grid");
    if (whichefvs < 0 || whichefvs > 2) return fail(CISMGPU_EINVAL, "whichefvs outside 0..2");
    if (!(n_glen > 0.0)) return fail(CISMGPU_EINVAL, "n_glen must be positive");
    return CISMGPU_OK;
}

// assemble_stiffness_matrix_3d / _2d (SSA) on the caller's host arrays: inputs uploaded, the
// blocks written on the device in the caller's layout (through its indxA map) and copied back.
static int oneshot_assemble(bool three_d, int nx, int ny, int nz, int nhalo, const double *sigma,
                            const int32_t *active_cell, const double *xv, const double *yv, const double *u,
                            const double *v, const double *usrf, const double *thck, const double *ff,
                            int whichapprox, int whichefvs, double efvs_constant, double effstrain_min,
                            double n_glen, const int32_t *indx, double *efvs, double *const blocks[4],
                            const double *dsdx = nullptr, const double *dsdy = nullptr,
                            const double *flwa = nullptr) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    TRY(validate_assembly(nx, ny, nz, nhalo, whichefvs, n_glen, sigma, active_cell, xv, yv, three_d ? usrf : thck,
                          thck, ff));
    if (!u || !v || !indx || !blocks[0] || !blocks[1] || !blocks[2] || !blocks[3])
        return fail(CISMGPU_EINVAL, "null pointer argument");
    const int NC = three_d ? 27 : 9;
    TRY(validate_indx(indx, NC));
    if (dsdx && (!dsdy || !flwa)) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (dsdx && whichefvs == 2 && std::fabs(n_glen - 1.0) >= 1.0e-10 && std::fabs(n_glen - 3.0) >= 1.0e-10)
        return fail(CISMGPU_EINVAL, "Invalid value of n_glen for L1L2 solver (1 or 3)");
    cismgpu_par_t par{};
    par.staggered_ilo = 1; par.staggered_ihi = nx - 1; par.staggered_jlo = 1; par.staggered_jhi = ny - 1;
    par.tasks_row = par.tasks_col = 1;
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, three_d ? nz : 1, &par), three_d));
    const size_t bs = (size_t)NC * sv.nvec;
    CU(sv.A.ensure(4 * bs * sizeof(double)));
    sv.mixed.stale = true;  // the matrix buffer holds the caller's layout until the next upload
    double *A0 = sv.A.as<double>();
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c < NC ? indx[c] : 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = sv.g.nz;
    L.raw3 = three_d ? 1 : 0;
    TRY(sv.assemble(three_d, nz, L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, nhalo, sigma, active_cell, xv, yv, u, v,
                    0, usrf, thck, ff, whichapprox, whichefvs, efvs_constant, effstrain_min, n_glen, efvs, dsdx, dsdy,
                    flwa));
    for (int k = 0; k < 4; ++k)
        CU(cudaMemcpyAsync(blocks[k], A0 + k * bs, bs * sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
    CU(cudaStreamSynchronize(sv.stream));
    return CISMGPU_OK;
}

static int oneshot_resid_velo(bool is3d, int whichresid, int nx, int ny, int nz, const cismgpu_par_t *par,
                              const double *uvel, const double *vvel, const double *usav, const double *vsav,
                              double *resid_velo) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    if (!uvel || !vvel || !usav || !vsav || !resid_velo) return fail(CISMGPU_EINVAL, "null pointer argument");
    TRY(validate_geom(nx, ny, is3d ? nz : 1, par));
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, is3d ? nz : 1, par), is3d));
    TRY(sv.put_vec(VX_U, uvel));
    TRY(sv.put_vec(VX_V, vvel));
    TRY(sv.put_vec(VX0_U, usav));
    TRY(sv.put_vec(VX0_V, vsav));
    return sv.residual_velocity(whichresid, VX_U, VX0_U, resid_velo);
}

}  // namespace cismgpu
#include "reprosum.cu"
namespace cismgpu {

static int oneshot_global_sum(int nx, int ny, int nz, const cismgpu_par_t *par, const double *a1, const double *a2,
                              double *sum) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    if (!par || !a1 || !a2 || !sum) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6 || nz < 1) return fail(CISMGPU_EINVAL, "grid too small");
    if (par->tasks_row * par->tasks_col != 1)
        return fail(CISMGPU_EUNSUPPORTED, "the whole domain must be on one GPU (tasks_row*tasks_col == 1)");
    if (par->staggered_ilo < 1 || par->staggered_ihi > nx - 1 || par->staggered_ilo > par->staggered_ihi ||
        par->staggered_jlo < 1 || par->staggered_jhi > ny - 1 || par->staggered_jlo > par->staggered_jhi)
        return fail(CISMGPU_EINVAL, "owned vertex bounds outside the array");
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    const Geom g = make_geom(nx, ny, nz, par);
    const long long n = (long long)nz * g.NQ;
    const unsigned nb = nblocks(g.NQ);
    CU(sv.raw.ensure((size_t)2 * n * sizeof(double)));
    CU(sv.partials.ensure((size_t)nb * 2 * sizeof(DD)));
    CU(sv.state.ensure(sizeof(SolveState)));
    double *d1 = sv.raw.as<double>(), *d2 = d1 + n;
    SolveState *st = sv.state.as<SolveState>();
    CU(cudaMemcpyAsync(d1, a1, n * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
    CU(cudaMemcpyAsync(d2, a2, n * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
    if (par->reprosum) {  // parallel_mpi.F90:6703-6738; non-finite summands give their IEEE sum
        CU(cudaMemsetAsync(st, 0, sizeof(SolveState), sv.stream));
        int *dflag = &st->status;
        const unsigned grid = (unsigned)std::min<long long>((n + kBlock - 1) / kBlock, 1184);
        k_repro_screen<<<grid, kBlock, 0, sv.stream>>>(g, d1, d2, dflag);
        CU(cudaGetLastError());
        int hflag = 0;
        CU(cudaMemcpyAsync(&hflag, dflag, sizeof(int), cudaMemcpyDeviceToHost, sv.stream));
        TRY(repro_global_sum(sv.stream, g, d1, d2, sv.rsum, sum));  // synchronizes the stream
        if ((hflag & 1) || (hflag & 6) == 6) *sum = std::nan("");
        else if (hflag & 2) *sum = HUGE_VAL;
        else if (hflag & 4) *sum = -HUGE_VAL;
        return CISMGPU_OK;
    }
    CU(cudaMemsetAsync(st, 0, sizeof(SolveState), sv.stream));
    if (g_sum_order.load() == CISMGPU_SUM_SEQUENTIAL) {  // parallel_mpi.F90:6770, :6637
        SeqArgs sa{};
        sa.a[0][0] = d1;
        sa.a[0][1] = d2;
        k_seq_sum<1, true><<<1, kBlock, 0, sv.stream>>>(g, sa, nullptr, EPI_NONE, EPI_NONE, 0, &st->err);
    } else {
        k_gsum<true><<<nb, kBlock, 0, sv.stream>>>(g, d1, d2, sv.partials.as<DD>(), &st->ticket[0], &st->err);
    }
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(sum, &st->err, sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
    CU(cudaStreamSynchronize(sv.stream));
    return CISMGPU_OK;
}

// A prepared launch of the mixed solver over several handles: one dynamic persistent kernel
// (k_mixed_dyn) over all their tiles.  The device block holds, 256-byte aligned: descriptors,
// running states, initial states, launch-start ticks, the tile list, the SolveState pointers
// of the members and the control word with its initial value; results come back into pinned
// host memory, so the whole sequence can be captured in a CUDA graph.
struct MixedBatch {
    std::vector<Solver *> svs;
    bool is3d = false;
    int nzm = 0, TYmax = 1, grid = 0, ntl = 0, max_steps = 0;
    void *dmem = nullptr;
    MDesc *d_descs = nullptr;
    MState *d_states = nullptr, *d_states0 = nullptr;
    MState **d_sptr = nullptr;   // d_sptr[t] = d_states + t
    unsigned *d_tick0 = nullptr;
    MTile *d_tiles = nullptr;
    SolveState **d_dst = nullptr;
    MCtl *d_ctl = nullptr, *d_ctl0 = nullptr;
    MState *h_states = nullptr;  // pinned
    MCtl *h_ctl = nullptr;       // pinned
    void release() {
        if (dmem) cudaFree(dmem);
        if (h_states) cudaFreeHost(h_states);
        if (h_ctl) cudaFreeHost(h_ctl);
        dmem = nullptr;
        h_states = nullptr;
        h_ctl = nullptr;
    }
    ~MixedBatch() { release(); }
};

// Prepare every member (FP32 matrix, maps, preconditioner; its own batch tile height), plan
// the launch and upload the descriptors, initial states and the tile list.
static int batch_prepare(MixedBatch &B, int precond, int ncheck, double tol, int maxiters, int floor = 0) {
    const int n = (int)B.svs.size();
    Solver &s0 = *B.svs[0];
    B.is3d = s0.is3d;
    B.nzm = mixed_nzm(s0.g, s0.is3d);
    if (floor <= 0) floor = batch_floor(B.is3d, B.nzm);
    std::vector<int> tys(n);
    std::vector<MTile> tl;
    for (int t = 0; t < n; ++t) {
        Solver &sv = *B.svs[t];
        if (sv.is3d != s0.is3d || mixed_nzm(sv.g, sv.is3d) != B.nzm)
            return fail(CISMGPU_EINVAL, "batch members must share dims and the nz class (<=16 or <=32)");
        tys[t] = mixed_batch_ty(sv.g, sv.is3d, B.nzm, floor);
        B.TYmax = std::max(B.TYmax, tys[t]);
        TRY(mixed_prepare(sv, precond, tys[t]));
        for (int k = 0; k < tiles_for(sv.g, tys[t]); ++k) tl.push_back(MTile{t, k});
    }
    for (int t = 0; t < n; ++t) CU(cudaStreamSynchronize(B.svs[t]->stream));
    B.grid = mixed_dyn_grid(B.is3d, B.nzm, B.TYmax);
    if (B.grid < 1) return fail(CISMGPU_EUNSUPPORTED, "mixed kernel does not fit on an SM at this tile height");
    if ((long long)n > (long long)B.grid * kMaxCtaSolves)
        return fail(CISMGPU_EUNSUPPORTED, "too many systems for one launch");
    B.ntl = (int)tl.size();
    B.max_steps = 4 * maxiters + 16;
    std::vector<MDesc> descs(n);
    std::vector<SolveState *> dst(n);
    for (int t = 0; t < n; ++t) {
        descs[t] = mixed_desc(*B.svs[t], precond, tys[t]);
        dst[t] = B.svs[t]->state.as<SolveState>();
    }
    const std::vector<MState> states(n, mixed_init_state(tol, maxiters, ncheck, precond));
    const std::vector<unsigned> tick0(n, 0u);
    MCtl c0;
    std::memset(&c0, 0, sizeof(c0));
    c0.active = n;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o_desc = 0, o_st = al(n * sizeof(MDesc)), o_st0 = o_st + al(n * sizeof(MState)),
                 o_sp = o_st0 + al(n * sizeof(MState)), o_tk = o_sp + al(n * sizeof(MState *)),
                 o_tl = o_tk + al(n * sizeof(unsigned)),
                 o_dst = o_tl + al(tl.size() * sizeof(MTile)), o_ctl = o_dst + al(n * sizeof(SolveState *)),
                 o_ctl0 = o_ctl + al(sizeof(MCtl)), total = o_ctl0 + al(sizeof(MCtl));
    CU(cudaMalloc(&B.dmem, total));
    char *base = static_cast<char *>(B.dmem);
    B.d_descs = reinterpret_cast<MDesc *>(base + o_desc);
    B.d_states = reinterpret_cast<MState *>(base + o_st);
    B.d_states0 = reinterpret_cast<MState *>(base + o_st0);
    B.d_sptr = reinterpret_cast<MState **>(base + o_sp);
    B.d_tick0 = reinterpret_cast<unsigned *>(base + o_tk);
    B.d_tiles = reinterpret_cast<MTile *>(base + o_tl);
    B.d_dst = reinterpret_cast<SolveState **>(base + o_dst);
    B.d_ctl = reinterpret_cast<MCtl *>(base + o_ctl);
    B.d_ctl0 = reinterpret_cast<MCtl *>(base + o_ctl0);
    CU(cudaMallocHost((void **)&B.h_states, n * sizeof(MState)));
    CU(cudaMallocHost((void **)&B.h_ctl, sizeof(MCtl)));
    CU(cudaMemcpy(B.d_descs, descs.data(), n * sizeof(MDesc), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(B.d_states0, states.data(), n * sizeof(MState), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(B.d_tick0, tick0.data(), n * sizeof(unsigned), cudaMemcpyHostToDevice));
    std::vector<MState *> sptr(n);
    for (int t = 0; t < n; ++t) sptr[t] = B.d_states + t;
    CU(cudaMemcpy(B.d_sptr, sptr.data(), n * sizeof(MState *), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(B.d_tiles, tl.data(), tl.size() * sizeof(MTile), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(B.d_dst, dst.data(), n * sizeof(SolveState *), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(B.d_ctl0, &c0, sizeof(MCtl), cudaMemcpyHostToDevice));
    return CISMGPU_OK;
}

// One batched solve on stream s: member resets, initial states and control word, the
// persistent launch, and the results (each handle's SolveState, and pinned host copies).  No
// host synchronization and no allocation, so it can be captured.
static int batch_enqueue(MixedBatch &B, cudaStream_t s) {
    const int n = (int)B.svs.size();
    for (Solver *sv : B.svs) TRY(mixed_reset(*sv, s));
    CU(cudaMemcpyAsync(B.d_states, B.d_states0, n * sizeof(MState), cudaMemcpyDeviceToDevice, s));
    CU(cudaMemcpyAsync(B.d_ctl, B.d_ctl0, sizeof(MCtl), cudaMemcpyDeviceToDevice, s));
    TRY(mixed_dyn_dispatch(B.is3d, B.nzm, B.d_descs, B.d_sptr, B.d_tick0, n, B.d_tiles, B.ntl, B.TYmax, B.d_ctl,
                           B.max_steps, B.grid, s));
    k_mstates_to_solves<<<(n + 127) / 128, 128, 0, s>>>(B.d_states, B.d_dst, n, B.d_ctl);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(B.h_states, B.d_states, n * sizeof(MState), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(B.h_ctl, B.d_ctl, sizeof(MCtl), cudaMemcpyDeviceToHost, s));
    return CISMGPU_OK;
}

// The batch tile floor of the members' dims and nz class, timed on this batch the first time the
// class is met (the tuner above): each candidate floor runs kTuneSteps steps of the whole batch
// (tol 0, so no member stops).  Outside any stream capture.
static int tune_batch_floor(const std::vector<Solver *> &svs, int precond, int ncheck, cudaStream_t s) {
    if (svs.empty()) return CISMGPU_OK;
    const bool is3d = svs[0]->is3d;
    const int nzm = mixed_nzm(svs[0]->g, is3d);
    for (Solver *sv : svs)
        if (sv->is3d != is3d || mixed_nzm(sv->g, sv->is3d) != nzm) return CISMGPU_OK;  // batch_prepare rejects it
    const std::string key = tile_key_batch(is3d, nzm);
    if (g_tiles.get(key) > 0 || !g_tiles.timing_on()) return CISMGPU_OK;
    const int fdef = is3d ? 4 : 16;
    const std::vector<int> cand = is3d ? std::vector<int>{4, 2, 6, 8} : std::vector<int>{16, 8, 32};
    float tdef = 0.f, tbest = 0.f;
    int arg = fdef;
    std::ostringstream note;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    int rc = CISMGPU_OK;
    for (int f : cand) {
        MixedBatch T;
        T.svs = svs;
        rc = batch_prepare(T, precond, ncheck, 0.0, 1 << 24, f);
        if (rc) break;
        T.max_steps = kTuneSteps;
        float t = 1e30f;
        for (int rep = 0; rep < 1 && !rc; ++rep) {
            if (cudaEventRecord(e0, s) != cudaSuccess) rc = fail(CISMGPU_ECUDA, "event record failed");
            if (!rc) rc = batch_enqueue(T, s);
            if (!rc && cudaEventRecord(e1, s) != cudaSuccess) rc = fail(CISMGPU_ECUDA, "event record failed");
            float ms = 0.f;
            if (!rc && (cudaStreamSynchronize(s) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                rc = fail(CISMGPU_ECUDA, "timing a batch tile floor failed");
            t = std::min(t, ms);
        }
        if (rc) break;
        note << f << ":" << t << "ms ";
        if (f == fdef) tdef = t;
        if (f == fdef || t < tbest) {
            tbest = t;
            arg = f;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (tbest >= 0.97f * tdef) arg = fdef;
    g_tiles.put(key, arg, note.str() + "(" + std::to_string(svs.size()) + " systems, " +
                              std::to_string(kTuneSteps) + " steps; default " + std::to_string(fdef) + ")");
    return CISMGPU_OK;
}

// Per-member results of the last completed batch_enqueue (after the stream is synchronized).
static int batch_results(const MixedBatch &B, double *errs, int *niters, int *statuses) {
    int first = CISMGPU_OK;
    for (size_t t = 0; t < B.svs.size(); ++t) {
        const MState &S = B.h_states[t];
        errs[t] = S.err;
        niters[t] = S.niters;
        statuses[t] = (B.h_ctl->abort && !S.done) ? CISMGPU_ETIMEOUT : S.status;
        if (statuses[t] && !first) first = statuses[t];
    }
    if (first) return fail(first, "batch member failed (see statuses)");
    return CISMGPU_OK;
}

}  // namespace cismgpu

// ---------------------------------------------------------------------------
// C ABI (include/cismgpu.h)
// ---------------------------------------------------------------------------
using namespace cismgpu;

struct cismgpu_solver {
    Solver sv;
    std::mutex mu;
    bool in_batch = false;               // a graph batch replays this handle's buffers
    cudaStream_t batch_stream = nullptr; // that batch's stream
};

struct cismgpu_batch {
    cismgpu::MixedBatch b;
    std::vector<cismgpu_solver *> members;  // marked in_batch while the batch exists
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};


extern "C" {

int cismgpu_pcg_standard_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                            const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                            const double *Auv, const double *Avu, const double *Avv, const double *bu,
                            const double *bv, double *xu, double *xv, int precond, int linear_solve_ncheck,
                            double tolerance, int maxiters, double *err, int *niters, int itest, int jtest,
                            int rtest) {
    (void)itest; (void)jtest; (void)rtest;  // debug-print location only (verbose_pcg = .false.)
    return oneshot_solve(ALG_STANDARD, true, nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv,
                         bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_pcg_chrongear_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                             const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                             const double *Auv, const double *Avu, const double *Avv, const double *bu,
                             const double *bv, double *xu, double *xv, int precond, int linear_solve_ncheck,
                             double tolerance, int maxiters, double *err, int *niters, int itest, int jtest,
                             int rtest) {
    (void)itest; (void)jtest; (void)rtest;
    return oneshot_solve(ALG_CHRONGEAR, true, nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu,
                         Avv, bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_pcg_standard_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                            const int32_t *active_vertex, const double *Auu, const double *Auv, const double *Avu,
                            const double *Avv, const double *bu, const double *bv, double *xu, double *xv,
                            int precond, int linear_solve_ncheck, double tolerance, int maxiters, double *err,
                            int *niters, int itest, int jtest, int rtest) {
    (void)itest; (void)jtest; (void)rtest;
    return oneshot_solve(ALG_STANDARD, false, nx, ny, 1, par, indxA_2d, nullptr, active_vertex, Auu, Auv, Avu, Avv,
                         bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_pcg_chrongear_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                             const int32_t *active_vertex, const double *Auu, const double *Auv, const double *Avu,
                             const double *Avv, const double *bu, const double *bv, double *xu, double *xv,
                             int precond, int linear_solve_ncheck, double tolerance, int maxiters, double *err,
                             int *niters, int itest, int jtest, int rtest) {
    (void)itest; (void)jtest; (void)rtest;
    return oneshot_solve(ALG_CHRONGEAR, false, nx, ny, 1, par, indxA_2d, nullptr, active_vertex, Auu, Auv, Avu, Avv,
                         bu, bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_matvec_structured_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_3d,
                                 const int32_t *active_vertex, const double *Auu, const double *Auv,
                                 const double *Avu, const double *Avv, const double *xu, const double *xv,
                                 double *yu, double *yv) {
    return oneshot_matvec(true, nx, ny, nz, par, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, xu, xv, yu, yv);
}

int cismgpu_matvec_structured_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                                 const int32_t *active_vertex, const double *Auu, const double *Auv,
                                 const double *Avu, const double *Avv, const double *xu, const double *xv,
                                 double *yu, double *yv) {
    return oneshot_matvec(false, nx, ny, 1, par, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, xu, xv, yu, yv);
}

int cismgpu_global_sum_stagger(int nx, int ny, int nz, const cismgpu_par_t *par, const double *arr1,
                               const double *arr2, double *sum) {
    return oneshot_global_sum(nx, ny, nz, par, arr1, arr2, sum);
}

int cismgpu_compute_residual_vector_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_3d,
                                       const int32_t *active_vertex, const double *Auu, const double *Auv,
                                       const double *Avu, const double *Avv, const double *bu, const double *bv,
                                       const double *uvel, const double *vvel, double *resid_u, double *resid_v,
                                       double *L2_norm, double *L2_norm_relative) {
    return oneshot_resid_vec(true, nx, ny, nz, par, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu, bv, uvel,
                             vvel, resid_u, resid_v, L2_norm, L2_norm_relative);
}

int cismgpu_compute_residual_vector_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                                       const int32_t *active_vertex, const double *Auu, const double *Auv,
                                       const double *Avu, const double *Avv, const double *bu, const double *bv,
                                       const double *uvel, const double *vvel, double *resid_u, double *resid_v,
                                       double *L2_norm, double *L2_norm_relative) {
    return oneshot_resid_vec(false, nx, ny, 1, par, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, bu, bv, uvel,
                             vvel, resid_u, resid_v, L2_norm, L2_norm_relative);
}

int cismgpu_compute_residual_velocity_3d(int whichresid, int nx, int ny, int nz, const cismgpu_par_t *par,
                                         const double *uvel, const double *vvel, const double *usav,
                                         const double *vsav, double *resid_velo) {
    return oneshot_resid_velo(true, whichresid, nx, ny, nz, par, uvel, vvel, usav, vsav, resid_velo);
}

int cismgpu_compute_residual_velocity_2d(int whichresid, int nx, int ny, const cismgpu_par_t *par,
                                         const double *uvel, const double *vvel, const double *usav,
                                         const double *vsav, double *resid_velo) {
    return oneshot_resid_velo(false, whichresid, nx, ny, 1, par, uvel, vvel, usav, vsav, resid_velo);
}

int cismgpu_check_symmetry_assembled_matrix_3d(int nx, int ny, int nz, const cismgpu_par_t *par,
                                               const int32_t *indxA_3d, const int32_t *active_vertex, double *Auu,
                                               double *Auv, double *Avu, double *Avv, double *maxdiff,
                                               long long *nwarn) {
    double *const blocks[4] = {Auu, Auv, Avu, Avv};
    return oneshot_symmetry(true, nx, ny, nz, par, indxA_3d, active_vertex, blocks, maxdiff, nwarn);
}

int cismgpu_check_symmetry_assembled_matrix_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                                               const int32_t *active_vertex, const double *Auu, const double *Auv,
                                               const double *Avu, const double *Avv, double *maxdiff,
                                               long long *nwarn) {
    // the 2D check writes nothing: the blocks stay const through the shared path
    double *const blocks[4] = {const_cast<double *>(Auu), const_cast<double *>(Auv), const_cast<double *>(Avu),
                               const_cast<double *>(Avv)};
    return oneshot_symmetry(false, nx, ny, 1, par, indxA_2d, active_vertex, blocks, maxdiff, nwarn);
}

int cismgpu_solver_create(cismgpu_solver_t **out, int dims, int nx, int ny, int nz, const cismgpu_par_t *par,
                          const int32_t *indxA, const int32_t *active_vertex, const double *Auu, const double *Auv,
                          const double *Avu, const double *Avv, const double *bu, const double *bv,
                          const double *xu0, const double *xv0, void *cuda_stream) {
    g_last_error.clear();
    if (!out) return fail(CISMGPU_EINVAL, "null handle pointer");
    *out = nullptr;
    if (dims != 2 && dims != 3) return fail(CISMGPU_EINVAL, "dims must be 2 or 3");
    const bool is3d = dims == 3;
    TRY(validate(nx, ny, is3d ? nz : 1, par, indxA, active_vertex, Auu, Auv, Avu, Avv, bu, bv));
    TRY(validate_indx(indxA, is3d ? 27 : 9));
    cismgpu_solver *h = new cismgpu_solver();
    int rc = h->sv.init((cudaStream_t)cuda_stream);
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    if (!rc) rc = h->sv.upload(make_geom(nx, ny, is3d ? nz : 1, par), is3d, indxA, active_vertex, blocks, bu, bv,
                               xu0, xv0);
    if (!rc && cudaStreamSynchronize(h->sv.stream) != cudaSuccess) rc = fail(CISMGPU_ECUDA, "upload failed");
    h->sv.repro = par->reprosum != 0;
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return CISMGPU_OK;
}

int cismgpu_solver_solve(cismgpu_solver_t *h, int algorithm, int precond, int linear_solve_ncheck, double tolerance,
                         int maxiters, double *err, int *niters) {
    g_last_error.clear();
    if (!h || !err || !niters) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    trace("solver_solve: begin");
    TRY(validate_solve_args(precond, linear_solve_ncheck, maxiters));
    Solver &sv = h->sv;
    TRY(sv.begin_solve());
    TRY(run_algorithm(sv, algorithm, precond, linear_solve_ncheck, tolerance, maxiters));
    return sv.finish_solve(err, niters);
}


int cismgpu_solver_solve_batch(cismgpu_solver_t **solvers, int n, int algorithm, int precond, int linear_solve_ncheck,
                               double tolerance, int maxiters, double *errs, int *niters, int *statuses,
                               void *cuda_stream) {
    g_last_error.clear();
    if (!solvers || n < 1 || !errs || !niters || !statuses) return fail(CISMGPU_EINVAL, "null argument");
    TRY(validate_solve_args(precond, linear_solve_ncheck, maxiters));
    if (algorithm != CISMGPU_ALG_MIXED_CHRONGEAR) {  // FP64 reference algorithms: one solve after another
        int first = CISMGPU_OK;
        for (int t = 0; t < n; ++t) {
            statuses[t] = cismgpu_solver_solve(solvers[t], algorithm, precond, linear_solve_ncheck, tolerance,
                                               maxiters, &errs[t], &niters[t]);
            if (statuses[t] && !first) first = statuses[t];
        }
        return first;
    }
    std::vector<std::unique_lock<std::mutex>> locks;
    MixedBatch B;
    for (int t = 0; t < n; ++t) {
        if (!solvers[t]) return fail(CISMGPU_EINVAL, "null handle in batch");
        locks.emplace_back(solvers[t]->mu);
        if (solvers[t]->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch");
        B.svs.push_back(&solvers[t]->sv);
    }
    cudaStream_t s = cuda_stream ? (cudaStream_t)cuda_stream : B.svs[0]->stream;
    TRY(tune_batch_floor(B.svs, precond, linear_solve_ncheck, s));
    TRY(batch_prepare(B, precond, linear_solve_ncheck, tolerance, maxiters));
    TRY(batch_enqueue(B, s));
    CU(cudaStreamSynchronize(s));
    return batch_results(B, errs, niters, statuses);
}

int cismgpu_batch_create(cismgpu_batch_t **out, cismgpu_solver_t **solvers, int n, int precond,
                         int linear_solve_ncheck, double tolerance, int maxiters, void *cuda_stream) {
    g_last_error.clear();
    if (!out || !solvers || n < 1) return fail(CISMGPU_EINVAL, "null argument");
    *out = nullptr;
    TRY(validate_solve_args(precond, linear_solve_ncheck, maxiters));
    for (int t = 0; t < n; ++t) {
        if (!solvers[t]) return fail(CISMGPU_EINVAL, "null handle in batch");
        for (int u = 0; u < t; ++u)
            if (solvers[u] == solvers[t]) return fail(CISMGPU_EINVAL, "handle listed twice in batch");
    }
    cismgpu_batch *h = new cismgpu_batch();
    int rc = CISMGPU_OK;
    {
        std::vector<std::unique_lock<std::mutex>> locks;  // held during preparation only
        for (int t = 0; t < n && !rc; ++t) {
            locks.emplace_back(solvers[t]->mu);
            if (solvers[t]->in_batch) rc = fail(CISMGPU_EINVAL, "handle already belongs to a graph batch");
            h->b.svs.push_back(&solvers[t]->sv);
        }
        if (!rc) rc = tune_batch_floor(h->b.svs, precond, linear_solve_ncheck,
                                       cuda_stream ? (cudaStream_t)cuda_stream : h->b.svs[0]->stream);
        if (!rc) rc = batch_prepare(h->b, precond, linear_solve_ncheck, tolerance, maxiters);
        if (!rc) {
            if (cuda_stream) {
                h->stream = (cudaStream_t)cuda_stream;
            } else if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess) {
                h->own_stream = true;
            } else {
                rc = fail(CISMGPU_ECUDA, "stream creation failed");
            }
        }
        if (!rc) {  // capture one batched solve into a graph
            cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) rc = fail(CISMGPU_ECUDA, std::string("begin capture: ") + cudaGetErrorString(e));
            if (!rc) {
                const int rce = batch_enqueue(h->b, h->stream);
                cudaGraph_t g = nullptr;
                e = cudaStreamEndCapture(h->stream, &g);
                h->graph = g;
                if (rce) rc = rce;
                else if (e != cudaSuccess) rc = fail(CISMGPU_ECUDA, std::string("end capture: ") + cudaGetErrorString(e));
            }
            if (!rc) {
                e = cudaGraphInstantiate(&h->exec, h->graph, 0);
                if (e != cudaSuccess) rc = fail(CISMGPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            }
        }
        if (!rc)
            for (int t = 0; t < n; ++t) {
                solvers[t]->in_batch = true;
                solvers[t]->batch_stream = h->stream;
                h->members.push_back(solvers[t]);
            }
    }
    if (rc) {
        cismgpu_batch_destroy(h);
        return rc;
    }
    *out = h;
    return CISMGPU_OK;
}

int cismgpu_batch_run(cismgpu_batch_t *h) {
    g_last_error.clear();
    if (!h || !h->exec) return fail(CISMGPU_EINVAL, "null batch");
    CU(cudaGraphLaunch(h->exec, h->stream));
    return CISMGPU_OK;
}

int cismgpu_batch_wait(cismgpu_batch_t *h, double *errs, int *niters, int *statuses) {
    g_last_error.clear();
    if (!h || !errs || !niters || !statuses) return fail(CISMGPU_EINVAL, "null argument");
    CU(cudaStreamSynchronize(h->stream));
    return batch_results(h->b, errs, niters, statuses);
}

int cismgpu_batch_destroy(cismgpu_batch_t *h) {
    if (!h) return CISMGPU_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (cismgpu_solver *m : h->members) {
        std::lock_guard<std::mutex> lk(m->mu);
        m->in_batch = false;
        m->batch_stream = nullptr;
    }
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CISMGPU_OK;
}

int cismgpu_solver_get_x(cismgpu_solver_t *h, double *xu, double *xv) {
    g_last_error.clear();
    if (!h || !xu || !xv) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) CU(cudaStreamSynchronize(h->batch_stream));  // the batch may be writing x
    return h->sv.download(VX_U, VX_V, xu, xv);
}

int cismgpu_solver_set_system(cismgpu_solver_t *h, const double *Auu, const double *Auv, const double *Avu,
                              const double *Avv, const double *bu, const double *bv, int x0_from_solution) {
    g_last_error.clear();
    if (!h || !Auu || !Auv || !Avu || !Avv || !bu || !bv) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    if (x0_from_solution && sv.x_current) {
        const Ptrs p = sv.ptrs();
        CU(cudaMemcpyAsync(p.x0u, p.xu, 2 * sv.nvec * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream));
    }
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    TRY(sv.put_system(blocks, bu, bv));
    sv.x_current = false;
    CU(cudaStreamSynchronize(sv.stream));  // the caller's arrays may be reused on return
    return CISMGPU_OK;
}

int cismgpu_solver_residual_vector(cismgpu_solver_t *h, double *resid_u, double *resid_v, double *L2_norm,
                                   double *L2_norm_relative) {
    g_last_error.clear();
    if (!h || !L2_norm || (!resid_u) != (!resid_v)) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    double l2 = 0.0, l2b = 0.0;
    TRY(sv.residual_vector(sv.x_current ? VX_U : VX0_U, &l2, &l2b));
    if (resid_u) TRY(sv.download(VR_U, VR_V, resid_u, resid_v));
    *L2_norm = l2;
    if (L2_norm_relative) *L2_norm_relative = (l2b > 0.0) ? l2 / l2b : 0.0;
    return CISMGPU_OK;
}

int cismgpu_assemble_stiffness_matrix_3d(int nx, int ny, int nz, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel, const double *vvel, const double *stagusrf,
                                         const double *stagthck, const double *flwafact, int whichapprox,
                                         int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                         const int32_t *indxA_3d, double *efvs, double *Auu, double *Auv,
                                         double *Avu, double *Avv) {
    double *const blocks[4] = {Auu, Auv, Avu, Avv};
    return oneshot_assemble(true, nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel, vvel, stagusrf,
                            stagthck, flwafact, whichapprox, whichefvs, efvs_constant, effstrain_min, n_glen, indxA_3d,
                            efvs, blocks);
}

int cismgpu_assemble_stiffness_matrix_2d(int nx, int ny, int nz, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel_2d, const double *vvel_2d, const double *stagthck,
                                         const double *flwafact, int whichefvs, double efvs_constant,
                                         double effstrain_min, double n_glen, const int32_t *indxA_2d, double *efvs,
                                         double *Auu, double *Auv, double *Avu, double *Avv) {
    double *const blocks[4] = {Auu, Auv, Avu, Avv};
    return oneshot_assemble(false, nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel_2d, vvel_2d, nullptr,
                            stagthck, flwafact, 1, whichefvs, efvs_constant, effstrain_min, n_glen, indxA_2d, efvs,
                            blocks);
}

// One-shot boundary terms on the caller's 3D blocks (and b): uploaded in the caller's layout,
// modified on the device, copied back.  which: 0 Dirichlet, 1 local basal term.
static int oneshot_boundary3d(int which, int nx, int ny, int nz, int nhalo, double dx, double dy,
                              const int32_t *active_vertex, const double *beta, const double *lsrf,
                              const int32_t *umask, const int32_t *vmask, const double *uvel, const double *vvel,
                              const int32_t *indx, double *Auu, double *Auv, double *Avu, double *Avv, double *bu,
                              double *bv, int assemble_beta = 1, const int32_t *active_cell = nullptr,
                              const double *xv = nullptr, const double *yv = nullptr) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    if (!active_vertex || !indx || !Auu || !Avv) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (which == 0 && (!umask || !vmask || !uvel || !vvel || !Auv || !Avu || !bu || !bv))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (which == 1 && (!beta || !lsrf)) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (which == 1 && assemble_beta == 0 && (!active_cell || !xv || !yv))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6 || nz < 1 || nz > kMaxNz) return fail(CISMGPU_EINVAL, "grid too small or nz outside 1..64");
    if (nhalo < 1 || 2 * nhalo >= nx || 2 * nhalo >= ny) return fail(CISMGPU_EINVAL, "nhalo outside the grid");
    if (which == 1 && assemble_beta == 0 && nhalo < 2)  // the cells' vertices must lie inside the arrays
        return fail(CISMGPU_EINVAL, "the standard basal form needs nhalo >= 2");
    TRY(validate_indx(indx, 27));
    cismgpu_par_t par{};
    par.staggered_ilo = 1; par.staggered_ihi = nx - 1; par.staggered_jlo = 1; par.staggered_jhi = ny - 1;
    par.tasks_row = par.tasks_col = 1;
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, nz, &par), true));
    const size_t bs = (size_t)27 * sv.nvec;
    CU(sv.A.ensure(4 * bs * sizeof(double)));
    sv.mixed.stale = true;  // the matrix buffer holds the caller's layout until the next upload
    double *A0 = sv.A.as<double>();
    double *blk[4] = {A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs};
    double *host[4] = {Auu, Auv, Avu, Avv};
    cudaStream_t s = sv.stream;
    for (int b = 0; b < 4; ++b)
        if (which == 0 || b == 0 || b == 3)
            CU(cudaMemcpyAsync(blk[b], host[b], bs * sizeof(double), cudaMemcpyHostToDevice, s));
    double *V = sv.vec.as<double>();  // b in the caller's layout, in the right-hand-side planes
    double *dbu = V + (size_t)VB_U * sv.nvec, *dbv = V + (size_t)VB_V * sv.nvec;
    if (which == 0) {
        CU(cudaMemcpyAsync(dbu, bu, sv.nvec * sizeof(double), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(dbv, bv, sv.nvec * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = indx[c];
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = nz;
    L.raw3 = 1;
    const VecIdx Wb{sv.g.NQ, nz, 0};
    TRY(sv.boundary3d(L, blk[0], blk[1], blk[2], blk[3], dbu, dbv, Wb, nhalo, dx, dy, active_vertex,
                      which == 1 ? beta : nullptr, lsrf, which == 0 ? umask : nullptr, vmask, uvel, vvel, 0,
                      assemble_beta, active_cell, xv, yv));
    for (int b = 0; b < 4; ++b)
        if (which == 0 || b == 0 || b == 3)
            CU(cudaMemcpyAsync(host[b], blk[b], bs * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (which == 0) {
        CU(cudaMemcpyAsync(bu, dbu, sv.nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(bv, dbv, sv.nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    return CISMGPU_OK;
}

// One-shot 2D boundary terms on the caller's blocks (nx-1,ny-1,9) and b.  which: 0 Dirichlet,
// 1 local basal term.
static int oneshot_boundary2d(int which, int nx, int ny, int nhalo, double dx, double dy,
                              const int32_t *active_vertex, const double *beta, const int32_t *umask,
                              const int32_t *vmask, const double *uvel, const double *vvel, const int32_t *indx,
                              double *Auu, double *Auv, double *Avu, double *Avv, double *bu, double *bv,
                              int assemble_beta = 1, const int32_t *active_cell = nullptr,
                              const double *xv = nullptr, const double *yv = nullptr, const double *beta_v = nullptr,
                              const double *lsrf = nullptr) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    if (!active_vertex || !indx || !Auu || !Avv) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (which == 0 && (!umask || !vmask || !uvel || !vvel || !Auv || !Avu || !bu || !bv))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (which == 1 && !beta) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (beta_v && !lsrf) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (which == 1 && assemble_beta == 0 && (!active_cell || !xv || !yv))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6) return fail(CISMGPU_EINVAL, "grid too small");
    if (nhalo < 1 || 2 * nhalo >= nx || 2 * nhalo >= ny) return fail(CISMGPU_EINVAL, "nhalo outside the grid");
    if (which == 1 && assemble_beta == 0 && nhalo < 2)  // the cells' vertices must lie inside the arrays
        return fail(CISMGPU_EINVAL, "the standard basal form needs nhalo >= 2");
    TRY(validate_indx(indx, 9));
    cismgpu_par_t par{};
    par.staggered_ilo = 1; par.staggered_ihi = nx - 1; par.staggered_jlo = 1; par.staggered_jhi = ny - 1;
    par.tasks_row = par.tasks_col = 1;
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, 1, &par), false));
    const size_t bs = (size_t)9 * sv.nvec;
    CU(sv.A.ensure(4 * bs * sizeof(double)));
    sv.mixed.stale = true;
    double *A0 = sv.A.as<double>();
    double *blk[4] = {A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs};
    double *host[4] = {Auu, Auv, Avu, Avv};
    cudaStream_t s = sv.stream;
    for (int b = 0; b < 4; ++b)
        if (which == 0 || b == 0 || b == 3)
            CU(cudaMemcpyAsync(blk[b], host[b], bs * sizeof(double), cudaMemcpyHostToDevice, s));
    double *V = sv.vec.as<double>();
    double *dbu = V + (size_t)VB_U * sv.nvec, *dbv = V + (size_t)VB_V * sv.nvec;
    if (which == 0) {
        CU(cudaMemcpyAsync(dbu, bu, sv.nvec * sizeof(double), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(dbv, bv, sv.nvec * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c < 9 ? indx[c] : 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = 1;
    L.raw3 = 0;
    TRY(sv.boundary2d(L, blk[0], blk[1], blk[2], blk[3], dbu, dbv, nhalo, dx, dy, active_vertex,
                      which == 1 ? beta : nullptr, which == 0 ? umask : nullptr, vmask, uvel, vvel, 0,
                      assemble_beta, active_cell, xv, yv, beta_v, lsrf));
    for (int b = 0; b < 4; ++b)
        if (which == 0 || b == 0 || b == 3)
            CU(cudaMemcpyAsync(host[b], blk[b], bs * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (which == 0) {
        CU(cudaMemcpyAsync(bu, dbu, sv.nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(bv, dbv, sv.nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    return CISMGPU_OK;
}

// assemble_stiffness_matrix_2d with HO_APPROX_DIVA on the caller's host arrays; efvs_qp_3d is
// the caller's state, read and updated; omega_k and omega change only in assembled cells.
static int oneshot_assemble_diva(int nx, int ny, int nz, int nhalo, const double *sigma, const double *stagsigma,
                                 const int32_t *active_cell, const double *xv, const double *yv, const double *u,
                                 const double *v, const double *stagthck, const double *thck, const double *bx,
                                 const double *by, const double *dsfx, const double *dsfy, const double *ff,
                                 int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                 const int32_t *indx, double *efvs_qp_3d, double *efvs, double *omega_k, double *omega,
                                 double *const blocks[4]) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    TRY(validate_assembly(nx, ny, nz, nhalo, whichefvs, n_glen, sigma, active_cell, xv, yv, stagthck, stagthck, ff));
    if (!stagsigma || !u || !v || !thck || !bx || !by || !dsfx || !dsfy || !indx || !efvs_qp_3d || !blocks[0] ||
        !blocks[1] || !blocks[2] || !blocks[3])
        return fail(CISMGPU_EINVAL, "null pointer argument");
    TRY(validate_indx(indx, 9));
    cismgpu_par_t par{};
    par.staggered_ilo = 1; par.staggered_ihi = nx - 1; par.staggered_jlo = 1; par.staggered_jhi = ny - 1;
    par.tasks_row = par.tasks_col = 1;
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, 1, &par), false));
    const size_t bs = (size_t)9 * sv.nvec, neq = (size_t)(nz - 1) * 4 * nx * ny;
    CU(sv.A.ensure(4 * bs * sizeof(double)));
    sv.mixed.stale = true;
    CU(sv.diva_eq[0].ensure(neq * sizeof(double)));
    CU(sv.diva_eq[1].ensure(neq * sizeof(double)));
    sv.diva_valid = false;  // the one-shot solver's state buffers hold the caller's state only
    double *eo = sv.diva_eq[0].as<double>(), *en = sv.diva_eq[1].as<double>();
    cudaStream_t s = sv.stream;
    CU(cudaMemcpyAsync(eo, efvs_qp_3d, neq * sizeof(double), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(en, eo, neq * sizeof(double), cudaMemcpyDeviceToDevice, s));
    double *A0 = sv.A.as<double>();
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c < 9 ? indx[c] : 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = 1;
    L.raw3 = 0;
    TRY(sv.assemble_diva(nz, L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, nhalo, sigma, stagsigma, active_cell, xv, yv,
                         u, v, 0, stagthck, thck, bx, by, dsfx, dsfy, ff, whichefvs, efvs_constant, effstrain_min,
                         n_glen, eo, en, efvs, omega_k, omega));
    for (int k = 0; k < 4; ++k)
        CU(cudaMemcpyAsync(blocks[k], A0 + k * bs, bs * sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(efvs_qp_3d, en, neq * sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return CISMGPU_OK;
}

int cismgpu_assemble_stiffness_matrix_2d_l1l2(int nx, int ny, int nz, int nhalo, const double *sigma,
                                              const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                              const double *uvel_2d, const double *vvel_2d, const double *stagthck,
                                              const double *dusrf_dx, const double *dusrf_dy, const double *flwa,
                                              const double *flwafact, int whichefvs, double efvs_constant,
                                              double effstrain_min, double n_glen, const int32_t *indxA_2d,
                                              double *efvs, double *Auu, double *Auv, double *Avu, double *Avv) {
    if (!dusrf_dx) {
        g_last_error.clear();
        return fail(CISMGPU_EINVAL, "null pointer argument");
    }
    double *const blocks[4] = {Auu, Auv, Avu, Avv};
    return oneshot_assemble(false, nx, ny, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel_2d, vvel_2d, nullptr,
                            stagthck, flwafact, 3, whichefvs, efvs_constant, effstrain_min, n_glen, indxA_2d, efvs,
                            blocks, dusrf_dx, dusrf_dy, flwa);
}

int cismgpu_load_vector_gravity(int nx, int ny, int nz, int nhalo, const double *sigma, const double *stagwbndsigma,
                                double dx, double dy, const int32_t *active_cell, const int32_t *active_vertex,
                                const double *xVertex, const double *yVertex, const double *stagusrf,
                                const double *stagthck, const double *dusrf_dx, const double *dusrf_dy,
                                int whichassemble_taud, double *loadu, double *loadv) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    if (!stagwbndsigma || !active_vertex || !stagthck || !dusrf_dx || !dusrf_dy || !loadu || !loadv)
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (whichassemble_taud != 0 && whichassemble_taud != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_taud must be 0 (standard) or 1 (local)");
    if (whichassemble_taud == 0)
        TRY(validate_assembly(nx, ny, nz, nhalo, 2, 3.0, sigma, active_cell, xVertex, yVertex, stagusrf, stagthck,
                              stagthck));
    else if (nx < 6 || ny < 6 || nz < 1 || nz > kMaxNz)
        return fail(CISMGPU_EINVAL, "grid too small or nz outside 1..64");
    cismgpu_par_t par{};
    par.staggered_ilo = 1; par.staggered_ihi = nx - 1; par.staggered_jlo = 1; par.staggered_jhi = ny - 1;
    par.tasks_row = par.tasks_col = 1;
    if (!g_oneshot) g_oneshot = new Solver();
    Solver &sv = *g_oneshot;
    TRY(sv.init(nullptr));
    TRY(sv.set_geom(make_geom(nx, ny, nz, &par), true));
    double *V = sv.vec.as<double>();  // the loads in the caller's layout, in the right-hand-side planes
    double *lu = V + (size_t)VB_U * sv.nvec, *lv = V + (size_t)VB_V * sv.nvec;
    cudaStream_t s = sv.stream;
    CU(cudaMemcpyAsync(lu, loadu, sv.nvec * sizeof(double), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(lv, loadv, sv.nvec * sizeof(double), cudaMemcpyHostToDevice, s));
    TRY(sv.load_gravity(VecIdx{sv.g.NQ, nz, 0}, lu, lv, nhalo, sigma, stagwbndsigma, dx, dy, active_cell,
                        active_vertex, xVertex, yVertex, stagusrf, stagthck, dusrf_dx, dusrf_dy, whichassemble_taud));
    CU(cudaMemcpyAsync(loadu, lu, sv.nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(loadv, lv, sv.nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return CISMGPU_OK;
}

// The handle's assembly: blocks into the resident canonical planes.
static int solver_assemble(cismgpu_solver_t *h, bool three_d, int nzl, int nhalo, const double *sigma,
                           const int32_t *active_cell, const double *xVertex, const double *yVertex,
                           const double *uvel, const double *vvel, const double *stagusrf, const double *stagthck,
                           const double *flwafact, int whichapprox, int whichefvs, double efvs_constant,
                           double effstrain_min, double n_glen, double *efvs) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    if (sv.is3d != three_d) return fail(CISMGPU_EINVAL, "the handle's dimension differs from the assembly's");
    if ((!uvel) != (!vvel)) return fail(CISMGPU_EINVAL, "give both velocity components or neither");
    TRY(validate_assembly(sv.g.NX + 1, sv.g.NY + 1, nzl, nhalo, whichefvs, n_glen, sigma, active_cell, xVertex,
                          yVertex, three_d ? stagusrf : stagthck, stagthck, flwafact));
    if (three_d && nzl != sv.g.nz) return fail(CISMGPU_EINVAL, "nz differs from the handle's");
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c + 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = sv.g.nz;
    L.raw3 = 0;
    const size_t bs = (size_t)sv.NC * sv.nvec;
    double *A0 = sv.A.as<double>();
    sv.mixed.stale = true;  // the FP32 copies follow the new matrix
    return sv.assemble(three_d, nzl, L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, nhalo, sigma, active_cell, xVertex,
                       yVertex, uvel, vvel, sv.x_current ? VX_U : VX0_U, stagusrf, stagthck, flwafact, whichapprox,
                       whichefvs, efvs_constant, effstrain_min, n_glen, efvs);
}

int cismgpu_solver_assemble_stiffness_3d(cismgpu_solver_t *h, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel, const double *vvel, const double *stagusrf,
                                         const double *stagthck, const double *flwafact, int whichapprox,
                                         int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                         double *efvs) {
    const int nz = h ? h->sv.g.nz : 0;
    return solver_assemble(h, true, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel, vvel, stagusrf, stagthck,
                           flwafact, whichapprox, whichefvs, efvs_constant, effstrain_min, n_glen, efvs);
}

int cismgpu_solver_assemble_stiffness_2d(cismgpu_solver_t *h, int nz, int nhalo, const double *sigma,
                                         const int32_t *active_cell, const double *xVertex, const double *yVertex,
                                         const double *uvel_2d, const double *vvel_2d, const double *stagthck,
                                         const double *flwafact, int whichefvs, double efvs_constant,
                                         double effstrain_min, double n_glen, double *efvs) {
    return solver_assemble(h, false, nz, nhalo, sigma, active_cell, xVertex, yVertex, uvel_2d, vvel_2d, nullptr,
                           stagthck, flwafact, 1, whichefvs, efvs_constant, effstrain_min, n_glen, efvs);
}

int cismgpu_dirichlet_boundary_conditions_3d(int nx, int ny, int nz, int nhalo, const int32_t *active_vertex,
                                             const int32_t *umask_dirichlet, const int32_t *vmask_dirichlet,
                                             const double *uvel, const double *vvel, const int32_t *indxA_3d,
                                             double *Auu, double *Auv, double *Avu, double *Avv, double *bu,
                                             double *bv) {
    return oneshot_boundary3d(0, nx, ny, nz, nhalo, 0.0, 0.0, active_vertex, nullptr, nullptr, umask_dirichlet,
                              vmask_dirichlet, uvel, vvel, indxA_3d, Auu, Auv, Avu, Avv, bu, bv);
}

int cismgpu_basal_sliding_bc_3d(int nx, int ny, int nz, int nhalo, double dx, double dy,
                                const int32_t *active_cell, const int32_t *active_vertex, const double *beta,
                                const double *lsrf, const double *xVertex, const double *yVertex,
                                int whichassemble_beta, const int32_t *indxA_3d, double *Auu, double *Avv) {
    g_last_error.clear();
    if (whichassemble_beta != 0 && whichassemble_beta != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_beta must be 0 (standard) or 1 (local)");
    return oneshot_boundary3d(1, nx, ny, nz, nhalo, dx, dy, active_vertex, beta, lsrf, nullptr, nullptr, nullptr,
                              nullptr, indxA_3d, Auu, nullptr, nullptr, Avv, nullptr, nullptr, whichassemble_beta,
                              active_cell, xVertex, yVertex);
}

int cismgpu_solver_assemble_system_3d(cismgpu_solver_t *h, int nhalo, double dx, double dy, const double *sigma,
                                      const int32_t *active_cell, const int32_t *active_vertex,
                                      const double *xVertex, const double *yVertex, const double *stagusrf,
                                      const double *stagthck, const double *flwafact, int whichapprox,
                                      int whichefvs, double efvs_constant, double effstrain_min, double n_glen,
                                      const double *beta, const double *lsrf, int whichassemble_beta,
                                      const double *loadu, const double *loadv, const int32_t *umask_dirichlet,
                                      const int32_t *vmask_dirichlet, double *efvs) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    if (!active_vertex || !loadu || !loadv || (!beta) != (!lsrf) || (!umask_dirichlet) != (!vmask_dirichlet))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (whichassemble_beta != 0 && whichassemble_beta != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_beta must be 0 (standard) or 1 (local)");
    // the stiffness blocks from the handle's current velocity (takes and releases the lock)
    TRY(cismgpu_solver_assemble_stiffness_3d(h, nhalo, sigma, active_cell, xVertex, yVertex, nullptr, nullptr,
                                             stagusrf, stagthck, flwafact, whichapprox, whichefvs, efvs_constant,
                                             effstrain_min, n_glen, efvs));
    std::lock_guard<std::mutex> lk(h->mu);
    Solver &sv = h->sv;
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c + 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = sv.g.nz;
    L.raw3 = 0;
    const size_t bs = (size_t)27 * sv.nvec;
    double *A0 = sv.A.as<double>();
    const Ptrs p = sv.ptrs();
    TRY(sv.put_vec(VB_U, loadu));  // bu = loadu, bv = loadv (:2868-2869)
    TRY(sv.put_vec(VB_V, loadv));
    TRY(sv.boundary3d(L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, p.bu, p.bv, VecIdx{sv.g.NQ, sv.g.nz, 1}, nhalo, dx,
                      dy, active_vertex, beta, lsrf, umask_dirichlet, vmask_dirichlet, nullptr, nullptr,
                      sv.x_current ? VX_U : VX0_U, whichassemble_beta, active_cell, xVertex, yVertex));
    // staggered_parallel_halo of the four blocks (every (m, k) plane) and of b (:2893-2904)
    Geom gA = sv.g;
    gA.nz = 27 * sv.g.nz;
    const unsigned hb = nblocks(4LL * sv.g.NX + 4LL * (sv.g.NY - 4));
    cudaStream_t s = sv.stream;
    k_halo<<<dim3(hb, kHaloPlaneRows), kBlock, 0, s>>>(gA, A0, A0 + bs, nullptr);
    k_halo<<<dim3(hb, kHaloPlaneRows), kBlock, 0, s>>>(gA, A0 + 2 * bs, A0 + 3 * bs, nullptr);
    k_halo<<<hb, kBlock, 0, s>>>(sv.g, p.bu, p.bv, nullptr);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    sv.mixed.stale = true;
    return CISMGPU_OK;
}

int cismgpu_dirichlet_boundary_conditions_2d(int nx, int ny, int nhalo, const int32_t *active_vertex,
                                             const int32_t *umask_dirichlet, const int32_t *vmask_dirichlet,
                                             const double *uvel, const double *vvel, const int32_t *indxA_2d,
                                             double *Auu, double *Auv, double *Avu, double *Avv, double *bu,
                                             double *bv) {
    return oneshot_boundary2d(0, nx, ny, nhalo, 0.0, 0.0, active_vertex, nullptr, umask_dirichlet, vmask_dirichlet,
                              uvel, vvel, indxA_2d, Auu, Auv, Avu, Avv, bu, bv);
}

int cismgpu_basal_sliding_bc_2d(int nx, int ny, int nhalo, double dx, double dy, const int32_t *active_cell,
                                const int32_t *active_vertex, const double *beta, const double *xVertex,
                                const double *yVertex, int whichassemble_beta, const int32_t *indxA_2d, double *Auu,
                                double *Avv) {
    g_last_error.clear();
    if (whichassemble_beta != 0 && whichassemble_beta != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_beta must be 0 (standard) or 1 (local)");
    return oneshot_boundary2d(1, nx, ny, nhalo, dx, dy, active_vertex, beta, nullptr, nullptr, nullptr, nullptr,
                              indxA_2d, Auu, nullptr, nullptr, Avv, nullptr, nullptr, whichassemble_beta, active_cell,
                              xVertex, yVertex);
}

int cismgpu_basal_sliding_bc_2d_diva(int nx, int ny, int nhalo, double dx, double dy, const int32_t *active_cell,
                                     const int32_t *active_vertex, const double *beta_eff_x, const double *beta_eff_y,
                                     const double *lsrf, const double *xVertex, const double *yVertex,
                                     int whichassemble_beta, const int32_t *indxA_2d, double *Auu, double *Avv) {
    g_last_error.clear();
    if (whichassemble_beta != 0 && whichassemble_beta != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_beta must be 0 (standard) or 1 (local)");
    if (!beta_eff_y || !lsrf) return fail(CISMGPU_EINVAL, "null pointer argument");
    return oneshot_boundary2d(1, nx, ny, nhalo, dx, dy, active_vertex, beta_eff_x, nullptr, nullptr, nullptr, nullptr,
                              indxA_2d, Auu, nullptr, nullptr, Avv, nullptr, nullptr, whichassemble_beta, active_cell,
                              xVertex, yVertex, beta_eff_y, lsrf);
}

int cismgpu_solver_assemble_system_2d(cismgpu_solver_t *h, int nz, int nhalo, double dx, double dy,
                                      const double *sigma, const int32_t *active_cell, const int32_t *active_vertex,
                                      const double *xVertex, const double *yVertex, const double *stagthck,
                                      const double *flwafact, int whichefvs, double efvs_constant,
                                      double effstrain_min, double n_glen, const double *beta, int whichassemble_beta,
                                      const double *loadu, const double *loadv, const int32_t *umask_dirichlet,
                                      const int32_t *vmask_dirichlet, double *efvs) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    if (!active_vertex || !loadu || !loadv || (!umask_dirichlet) != (!vmask_dirichlet))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (whichassemble_beta != 0 && whichassemble_beta != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_beta must be 0 (standard) or 1 (local)");
    TRY(cismgpu_solver_assemble_stiffness_2d(h, nz, nhalo, sigma, active_cell, xVertex, yVertex, nullptr, nullptr,
                                             stagthck, flwafact, whichefvs, efvs_constant, effstrain_min, n_glen,
                                             efvs));
    std::lock_guard<std::mutex> lk(h->mu);
    Solver &sv = h->sv;
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c + 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = 1;
    L.raw3 = 0;
    const size_t bs = (size_t)9 * sv.nvec;
    double *A0 = sv.A.as<double>();
    const Ptrs p = sv.ptrs();
    TRY(sv.put_vec(VB_U, loadu));  // bu_2d = loadu_2d, bv_2d = loadv_2d (:2620-2621)
    TRY(sv.put_vec(VB_V, loadv));
    TRY(sv.boundary2d(L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, p.bu, p.bv, nhalo, dx, dy, active_vertex, beta,
                      umask_dirichlet, vmask_dirichlet, nullptr, nullptr, sv.x_current ? VX_U : VX0_U,
                      whichassemble_beta, active_cell, xVertex, yVertex));
    // staggered_parallel_halo of every coefficient plane and of b (:2652-2666)
    Geom gA = sv.g;
    gA.nz = 9;
    const unsigned hb = nblocks(4LL * sv.g.NX + 4LL * (sv.g.NY - 4));
    cudaStream_t s = sv.stream;
    k_halo<<<dim3(hb, kHaloPlaneRows), kBlock, 0, s>>>(gA, A0, A0 + bs, nullptr);
    k_halo<<<dim3(hb, kHaloPlaneRows), kBlock, 0, s>>>(gA, A0 + 2 * bs, A0 + 3 * bs, nullptr);
    k_halo<<<hb, kBlock, 0, s>>>(sv.g, p.bu, p.bv, nullptr);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    sv.mixed.stale = true;
    return CISMGPU_OK;
}

int cismgpu_assemble_stiffness_matrix_2d_diva(int nx, int ny, int nz, int nhalo, const double *sigma,
                                              const double *stagsigma, const int32_t *active_cell,
                                              const double *xVertex, const double *yVertex, const double *uvel_2d,
                                              const double *vvel_2d, const double *stagthck, const double *thck,
                                              const double *btractx, const double *btracty,
                                              const double *diva_slope_factor_x, const double *diva_slope_factor_y,
                                              const double *flwafact, int whichefvs, double efvs_constant,
                                              double effstrain_min, double n_glen, const int32_t *indxA_2d,
                                              double *efvs_qp_3d, double *efvs, double *omega_k, double *omega,
                                              double *Auu, double *Auv, double *Avu, double *Avv) {
    double *const blocks[4] = {Auu, Auv, Avu, Avv};
    return oneshot_assemble_diva(nx, ny, nz, nhalo, sigma, stagsigma, active_cell, xVertex, yVertex, uvel_2d, vvel_2d,
                                 stagthck, thck, btractx, btracty, diva_slope_factor_x, diva_slope_factor_y, flwafact,
                                 whichefvs, efvs_constant, effstrain_min, n_glen, indxA_2d, efvs_qp_3d, efvs, omega_k,
                                 omega, blocks);
}

int cismgpu_solver_assemble_stiffness_2d_diva(cismgpu_solver_t *h, int nz, int nhalo, const double *sigma,
                                              const double *stagsigma, const int32_t *active_cell,
                                              const double *xVertex, const double *yVertex, const double *uvel_2d,
                                              const double *vvel_2d, const double *stagthck, const double *thck,
                                              const double *btractx, const double *btracty,
                                              const double *diva_slope_factor_x, const double *diva_slope_factor_y,
                                              const double *flwafact, int whichefvs, double efvs_constant,
                                              double effstrain_min, double n_glen, const double *efvs_qp_3d_in,
                                              double *efvs, double *omega_k, double *omega) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    if (sv.is3d) return fail(CISMGPU_EINVAL, "the handle holds a 3D system");
    if ((!uvel_2d) != (!vvel_2d)) return fail(CISMGPU_EINVAL, "give both velocity components or neither");
    const int nx = sv.g.NX + 1, ny = sv.g.NY + 1;
    TRY(validate_assembly(nx, ny, nz, nhalo, whichefvs, n_glen, sigma, active_cell, xVertex, yVertex, stagthck,
                          stagthck, flwafact));
    if (!stagsigma || !thck || !btractx || !btracty || !diva_slope_factor_x || !diva_slope_factor_y)
        return fail(CISMGPU_EINVAL, "null pointer argument");
    const size_t neq = (size_t)(nz - 1) * 4 * nx * ny;
    CU(sv.diva_eq[0].ensure(neq * sizeof(double)));
    CU(sv.diva_eq[1].ensure(neq * sizeof(double)));
    cudaStream_t s = sv.stream;
    double *eo = sv.diva_eq[sv.diva_cur].as<double>(), *en = sv.diva_eq[1 - sv.diva_cur].as<double>();
    if (efvs_qp_3d_in) CU(cudaMemcpyAsync(eo, efvs_qp_3d_in, neq * sizeof(double), cudaMemcpyHostToDevice, s));
    else if (!sv.diva_valid) CU(cudaMemsetAsync(eo, 0, neq * sizeof(double), s));  // the reference starts at zero
    CU(cudaMemcpyAsync(en, eo, neq * sizeof(double), cudaMemcpyDeviceToDevice, s));
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c + 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = 1;
    L.raw3 = 0;
    const size_t bs = (size_t)9 * sv.nvec;
    double *A0 = sv.A.as<double>();
    sv.mixed.stale = true;
    TRY(sv.assemble_diva(nz, L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, nhalo, sigma, stagsigma, active_cell, xVertex,
                         yVertex, uvel_2d, vvel_2d, sv.x_current ? VX_U : VX0_U, stagthck, thck, btractx, btracty,
                         diva_slope_factor_x, diva_slope_factor_y, flwafact, whichefvs, efvs_constant, effstrain_min,
                         n_glen, eo, en, efvs, omega_k, omega));
    sv.diva_cur = 1 - sv.diva_cur;
    sv.diva_valid = true;
    return CISMGPU_OK;
}

int cismgpu_solver_assemble_system_2d_diva(
    cismgpu_solver_t *h, int nz, int nhalo, double dx, double dy, const double *sigma, const double *stagsigma,
    const int32_t *active_cell, const int32_t *active_vertex, const double *xVertex, const double *yVertex,
    const double *stagthck, const double *thck, const double *btractx, const double *btracty,
    const double *diva_slope_factor_x, const double *diva_slope_factor_y, const double *flwafact, int whichefvs,
    double efvs_constant, double effstrain_min, double n_glen, const double *beta_eff_x, const double *beta_eff_y,
    const double *lsrf, int whichassemble_beta, const double *loadu, const double *loadv,
    const int32_t *umask_dirichlet, const int32_t *vmask_dirichlet, double *efvs, double *omega_k, double *omega) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    if (!active_vertex || !loadu || !loadv || (!beta_eff_x) != (!beta_eff_y) || (beta_eff_x && !lsrf) ||
        (!umask_dirichlet) != (!vmask_dirichlet))
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (whichassemble_beta != 0 && whichassemble_beta != 1)
        return fail(CISMGPU_EINVAL, "whichassemble_beta must be 0 (standard) or 1 (local)");
    // the DIVA stiffness from the handle's current velocity and its kept layer viscosities
    TRY(cismgpu_solver_assemble_stiffness_2d_diva(h, nz, nhalo, sigma, stagsigma, active_cell, xVertex, yVertex,
                                                  nullptr, nullptr, stagthck, thck, btractx, btracty,
                                                  diva_slope_factor_x, diva_slope_factor_y, flwafact, whichefvs,
                                                  efvs_constant, effstrain_min, n_glen, nullptr, efvs, omega_k, omega));
    std::lock_guard<std::mutex> lk(h->mu);
    Solver &sv = h->sv;
    SymIdx L{};
    for (int c = 0; c < 27; ++c) L.map[c] = c + 1;
    L.n = sv.nvec;
    L.NQ = sv.g.NQ;
    L.nz = 1;
    L.raw3 = 0;
    const size_t bs = (size_t)9 * sv.nvec;
    double *A0 = sv.A.as<double>();
    const Ptrs p = sv.ptrs();
    TRY(sv.put_vec(VB_U, loadu));
    TRY(sv.put_vec(VB_V, loadv));
    // basal_sliding_bc_2d_diva (:2575-2589), b = load, dirichlet_boundary_conditions_2d
    TRY(sv.boundary2d(L, A0, A0 + bs, A0 + 2 * bs, A0 + 3 * bs, p.bu, p.bv, nhalo, dx, dy, active_vertex, beta_eff_x,
                      umask_dirichlet, vmask_dirichlet, nullptr, nullptr, sv.x_current ? VX_U : VX0_U,
                      whichassemble_beta, active_cell, xVertex, yVertex, beta_eff_y, lsrf));
    Geom gA = sv.g;
    gA.nz = 9;
    const unsigned hb = nblocks(4LL * sv.g.NX + 4LL * (sv.g.NY - 4));
    cudaStream_t s = sv.stream;
    k_halo<<<dim3(hb, kHaloPlaneRows), kBlock, 0, s>>>(gA, A0, A0 + bs, nullptr);
    k_halo<<<dim3(hb, kHaloPlaneRows), kBlock, 0, s>>>(gA, A0 + 2 * bs, A0 + 3 * bs, nullptr);
    k_halo<<<hb, kBlock, 0, s>>>(sv.g, p.bu, p.bv, nullptr);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    sv.mixed.stale = true;
    return CISMGPU_OK;
}

int cismgpu_solver_check_symmetry(cismgpu_solver_t *h, double *maxdiff, long long *nwarn) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    return h->sv.check_symmetry(maxdiff, nwarn);
}

int cismgpu_solver_save(cismgpu_solver_t *h) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    const size_t abytes = (size_t)4 * sv.NC * sv.nvec * sizeof(double), xbytes = (size_t)2 * sv.nvec * sizeof(double);
    CU(sv.A_sav.ensure(abytes));
    CU(sv.x_sav.ensure(xbytes));
    const Ptrs p = sv.ptrs();
    CU(cudaMemcpyAsync(sv.A_sav.p, sv.A.p, abytes, cudaMemcpyDeviceToDevice, sv.stream));
    CU(cudaMemcpyAsync(sv.x_sav.p, sv.x_current ? p.xu : p.x0u, xbytes, cudaMemcpyDeviceToDevice, sv.stream));
    CU(cudaStreamSynchronize(sv.stream));
    sv.have_sav = true;
    return CISMGPU_OK;
}

int cismgpu_solver_restore(cismgpu_solver_t *h) {
    g_last_error.clear();
    if (!h) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    if (!sv.have_sav) return fail(CISMGPU_EINVAL, "nothing saved on this handle");
    const size_t abytes = (size_t)4 * sv.NC * sv.nvec * sizeof(double), xbytes = (size_t)2 * sv.nvec * sizeof(double);
    const Ptrs p = sv.ptrs();
    CU(cudaMemcpyAsync(sv.A.p, sv.A_sav.p, abytes, cudaMemcpyDeviceToDevice, sv.stream));
    CU(cudaMemcpyAsync(p.x0u, sv.x_sav.p, xbytes, cudaMemcpyDeviceToDevice, sv.stream));
    CU(cudaStreamSynchronize(sv.stream));
    sv.mixed.stale = true;  // the FP32 copies follow the restored matrix
    sv.x_current = false;   // the current velocity is the saved one, and the next solve starts from it
    return CISMGPU_OK;
}

int cismgpu_solver_residual_velocity(cismgpu_solver_t *h, int whichresid, double *resid_velo) {
    g_last_error.clear();
    if (!h || !resid_velo) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
    Solver &sv = h->sv;
    if (!sv.x_current) return fail(CISMGPU_EINVAL, "no solve since the system was set");
    return sv.residual_velocity(whichresid, VX_U, VX0_U, resid_velo);
}

int cismgpu_solver_profile(cismgpu_solver_t *h, int enable) {
    if (!h) return fail(CISMGPU_EINVAL, "null handle");
    std::lock_guard<std::mutex> lk(h->mu);
    h->sv.prof = enable != 0;
    h->sv.prof_ms = 0.0;
    h->sv.prof_n = 0;
    h->sv.pused = 0;
    return CISMGPU_OK;
}

int cismgpu_solver_profile_read(cismgpu_solver_t *h, double *total_ms, int *launches, double *bytes_per_launch) {
    if (!h || !total_ms || !launches || !bytes_per_launch) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(h->mu);
    *total_ms = h->sv.prof_ms;
    *launches = h->sv.prof_n;
    *bytes_per_launch = h->sv.prof_bytes;
    return CISMGPU_OK;
}

size_t cismgpu_solver_device_bytes(const cismgpu_solver_t *h) {
    if (!h) return 0;
    const Solver &s = h->sv;
    return s.A.n + s.raw.n + s.vec.n + s.act.n + s.partials.n + s.state.n + s.map.n + s.mixed.bytes();
}

int cismgpu_solver_destroy(cismgpu_solver_t *h) {
    if (!h) return CISMGPU_OK;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        if (h->in_batch) return fail(CISMGPU_EINVAL, "handle belongs to a graph batch (destroy the batch first)");
        if (h->sv.stream) cudaStreamSynchronize(h->sv.stream);
    }
    delete h;
    return CISMGPU_OK;
}

int cismgpu_set_oneshot_algorithm(int algorithm) {
    std::lock_guard<std::mutex> lk(g_mu);
    const int prev = g_oneshot_alg;
    g_oneshot_alg = (algorithm >= CISMGPU_ALG_STANDARD && algorithm <= CISMGPU_ALG_MIXED_CHRONGEAR) ? algorithm : -1;
    return prev;
}

int cismgpu_test_set_device_waits(long long wait_cycles, unsigned int withhold_step) {
    g_last_error.clear();
    TRY(check_device());
    const long long w = wait_cycles > 0 ? wait_cycles : kWaitCycles;
    CU(cudaMemcpyToSymbol(c_wait_cycles, &w, sizeof(w)));
    CU(cudaMemcpyToSymbol(c_withhold_tag, &withhold_step, sizeof(withhold_step)));
    return CISMGPU_OK;
}

size_t cismgpu_tile_table(char *buf, size_t len) {
    std::string out;
    {
        std::lock_guard<std::mutex> lk(g_tiles.mu);
        g_tiles.load();
        for (const auto &kv : g_tiles.table) {
            std::string line = kv.first + " " + std::to_string(kv.second);
            for (const std::string &l : g_tiles.log)
                if (l.compare(0, kv.first.size() + 1, kv.first + " ") == 0) line = l;
            out += line + "\n";
        }
    }
    if (buf && len > 0) {
        const size_t n = std::min(len - 1, out.size());
        std::memcpy(buf, out.data(), n);
        buf[n] = '\0';
    }
    return out.size() + 1;
}

int cismgpu_set_mixed_layout(int layout) {
    return g_mixed_full_storage.exchange(layout == CISMGPU_MIXED_LAYOUT_FULL) ? CISMGPU_MIXED_LAYOUT_FULL
                                                                               : CISMGPU_MIXED_LAYOUT_AUTO;
}

int cismgpu_solver_mixed_layout(const cismgpu_solver_t *h, int *symmetric_half) {
    g_last_error.clear();
    if (!h || !symmetric_half) return fail(CISMGPU_EINVAL, "null argument");
    *symmetric_half = (h->sv.mixed.valid && h->sv.mixed.sym) ? 1 : 0;
    return CISMGPU_OK;
}

int cismgpu_set_sum_order(int order) {
    const int v = order == CISMGPU_SUM_SEQUENTIAL ? CISMGPU_SUM_SEQUENTIAL : CISMGPU_SUM_TREE;
    return g_sum_order.exchange(v);
}

const char *cismgpu_last_error(void) { return g_last_error.c_str(); }

const char *cismgpu_version(void) { return "cismgpu 0.2 (sm_100a)"; }

}  // extern "C"

#include "server.cu"
#include "noalloc.cu"
