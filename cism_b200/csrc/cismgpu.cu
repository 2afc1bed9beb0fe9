// cismgpu.cu -- host driver and C ABI of the B200 structured PCG library.
//
// One translation unit: the FP64 reference-faithful kernels (pcg_fp64.cu) plus the
// host code that uploads the caller's Fortran arrays, re-lays them into coefficient
// planes, enqueues the solver's kernel sequence on one stream and polls the
// device-side convergence flag with one check period of look-ahead.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pcg_fp64.cu"

namespace cismgpu {

static thread_local std::string g_last_error;

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

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Vectors of one solve, level-major planes of nz*NQ doubles each.
enum VecId { VB_U, VB_V, VX_U, VX_V, VR_U, VR_V, VD_U, VD_V, VQ_U, VQ_V, VZ_U, VZ_V, VAZ_U, VAZ_V, NVEC };

struct Workspace {
    int device = -1;
    bool ready = false;
    cudaStream_t stream = nullptr;
    DevBuf A, raw, vec, act, partials, state, map;
    int *h_done = nullptr;          // pinned, 2 slots for look-ahead polling
    SolveState *h_state = nullptr;  // pinned
    cudaEvent_t ev[2];
};

static std::mutex g_mu;
static Workspace g_ws;

static int init_device(Workspace &ws) {
    if (ws.ready) return CISMGPU_OK;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(CISMGPU_ENODEV, "no CUDA device");
    int dev = 0;
    CU(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return fail(CISMGPU_ENODEV, std::string("not an sm_100 device: ") + prop.name);
    CU(cudaStreamCreateWithFlags(&ws.stream, cudaStreamNonBlocking));
    CU(cudaMallocHost(&ws.h_done, 2 * sizeof(int)));
    CU(cudaMallocHost(&ws.h_state, sizeof(SolveState)));
    CU(cudaEventCreateWithFlags(&ws.ev[0], cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&ws.ev[1], cudaEventDisableTiming));
    ws.device = dev;
    ws.ready = true;
    return CISMGPU_OK;
}

static int validate(int nx, int ny, int nz, const cismgpu_par_t *par, const void *indx, const void *act,
                    const void *A0, const void *A1, const void *A2, const void *A3, const void *bu,
                    const void *bv, const void *xu, const void *xv, int precond, int ncheck, int maxiters,
                    const void *err, const void *niters) {
    if (!par || !indx || !act || !A0 || !A1 || !A2 || !A3 || !bu || !bv || !xu || !xv || !err || !niters)
        return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6 || nz < 1 || nz > kMaxNz)
        return fail(CISMGPU_EINVAL, "grid too small or nz outside 1..64");
    if (ncheck < 1) return fail(CISMGPU_EINVAL, "linear_solve_ncheck must be >= 1");
    if (maxiters < 0) return fail(CISMGPU_EINVAL, "maxiters must be >= 0");
    if (par->tasks_row * par->tasks_col != 1)
        return fail(CISMGPU_EUNSUPPORTED, "the whole domain must be on one GPU (tasks_row*tasks_col == 1)");
    if (precond == CISMGPU_PRECOND_TRIDIAG_LOCAL || precond == CISMGPU_PRECOND_TRIDIAG_GLOBAL)
        return fail(CISMGPU_EUNSUPPORTED, "tridiagonal preconditioners (3, 4) are not implemented");
    if (par->staggered_ilo < 1 || par->staggered_ihi > nx - 1 || par->staggered_ilo > par->staggered_ihi ||
        par->staggered_jlo < 1 || par->staggered_jhi > ny - 1 || par->staggered_jlo > par->staggered_jhi)
        return fail(CISMGPU_EINVAL, "owned vertex bounds outside the array");
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

static inline unsigned nblocks(long long n, int b = kBlock) { return (unsigned)((n + b - 1) / b); }

// Upload the caller's arrays into the workspace (coefficient planes, level-major vectors).
static int upload(Workspace &ws, const Geom &g, bool is3d, const int32_t *indx, const int32_t *act,
                  const double *const blocks[4], const double *bu, const double *bv, const double *xu,
                  const double *xv) {
    const int NC = is3d ? 27 : 9;
    const long long nvec = (long long)g.nz * g.NQ;
    const size_t blk_bytes = (size_t)NC * nvec * sizeof(double);
    CU(ws.A.ensure(4 * blk_bytes));
    CU(ws.raw.ensure(blk_bytes));
    CU(ws.vec.ensure((size_t)NVEC * nvec * sizeof(double)));
    CU(ws.act.ensure((size_t)g.NQ * sizeof(int32_t)));
    CU(ws.partials.ensure((size_t)nblocks(g.NQ) * 2 * sizeof(DD)));
    CU(ws.state.ensure(sizeof(SolveState)));
    CU(ws.map.ensure(32 * sizeof(int32_t)));
    cudaStream_t s = ws.stream;
    CU(cudaMemcpyAsync(ws.map.p, indx, NC * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(ws.act.p, act, (size_t)g.NQ * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    for (int b = 0; b < 4; ++b) {
        CU(cudaMemcpyAsync(ws.raw.p, blocks[b], blk_bytes, cudaMemcpyHostToDevice, s));
        double *dst = ws.A.as<double>() + (size_t)b * NC * nvec;
        if (is3d)
            k_perm_block3<<<nblocks(nvec), kBlock, 0, s>>>(g, ws.raw.as<double>(), dst, ws.map.as<int32_t>());
        else
            k_perm_block2<<<nblocks(g.NQ), kBlock, 0, s>>>(g, ws.raw.as<double>(), dst, ws.map.as<int32_t>());
        CU(cudaGetLastError());
    }
    double *V = ws.vec.as<double>();
    const double *src[4] = {bu, bv, xu, xv};
    const int dst_id[4] = {VB_U, VB_V, VX_U, VX_V};
    for (int t = 0; t < 4; ++t) {
        double *dst = V + (size_t)dst_id[t] * nvec;
        if (is3d) {
            CU(cudaMemcpyAsync(ws.raw.p, src[t], nvec * sizeof(double), cudaMemcpyHostToDevice, s));
            k_vec_in<<<nblocks(nvec), kBlock, 0, s>>>(g, ws.raw.as<double>(), dst);
            CU(cudaGetLastError());
        } else {
            CU(cudaMemcpyAsync(dst, src[t], nvec * sizeof(double), cudaMemcpyHostToDevice, s));
        }
    }
    return CISMGPU_OK;
}

static int download_x(Workspace &ws, const Geom &g, bool is3d, double *xu, double *xv) {
    const long long nvec = (long long)g.nz * g.NQ;
    double *V = ws.vec.as<double>();
    cudaStream_t s = ws.stream;
    double *out[2] = {xu, xv};
    const int id[2] = {VX_U, VX_V};
    for (int t = 0; t < 2; ++t) {
        if (is3d) {
            k_vec_out<<<nblocks(nvec), kBlock, 0, s>>>(g, V + (size_t)id[t] * nvec, ws.raw.as<double>());
            CU(cudaGetLastError());
            CU(cudaMemcpyAsync(out[t], ws.raw.p, nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
        } else {
            CU(cudaMemcpyAsync(out[t], V + (size_t)id[t] * nvec, nvec * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
    }
    CU(cudaMemcpyAsync(ws.h_state, ws.state.p, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return CISMGPU_OK;
}

// Enqueue-and-poll helper: after the kernels of a check iteration are enqueued,
// copy 'done' to pinned memory; wait for the *previous* check's copy so the GPU
// always has one check period of work queued.
struct Poller {
    Workspace &ws;
    SolveState *st;
    int pending = -1;  // slot index of the outstanding copy, -1 if none
    int slot = 0;
    explicit Poller(Workspace &w, SolveState *s) : ws(w), st(s) {}
    // returns 1 when the solve is finished, 0 to continue, <0 on CUDA error
    int after_check() {
        cudaStream_t s = ws.stream;
        if (cudaMemcpyAsync(&ws.h_done[slot], &st->done, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return -1;
        if (cudaEventRecord(ws.ev[slot], s) != cudaSuccess) return -1;
        int finished = 0;
        if (pending >= 0) {
            if (cudaEventSynchronize(ws.ev[pending]) != cudaSuccess) return -1;
            finished = ws.h_done[pending];
        }
        pending = slot;
        slot ^= 1;
        return finished;
    }
};

static inline bool is_check(int iter, int ncheck) { return (iter % ncheck == 0) || iter == 5; }

struct Ptrs {
    double *bu, *bv, *xu, *xv, *ru, *rv, *du, *dv, *qu, *qv, *zu, *zv, *Azu, *Azv;
};

static Ptrs ptrs(Workspace &ws, const Geom &g) {
    const long long nvec = (long long)g.nz * g.NQ;
    double *V = ws.vec.as<double>();
    auto P = [&](int id) { return V + (size_t)id * nvec; };
    return Ptrs{P(VB_U), P(VB_V), P(VX_U), P(VX_V), P(VR_U), P(VR_V), P(VD_U), P(VD_V),
                P(VQ_U), P(VQ_V), P(VZ_U), P(VZ_V), P(VAZ_U), P(VAZ_V)};
}

static VecArgs vargs(const Ptrs &p) {
    VecArgs v;
    v.bu = p.bu; v.bv = p.bv; v.xu = p.xu; v.xv = p.xv; v.ru = p.ru; v.rv = p.rv;
    v.du = p.du; v.dv = p.dv; v.qu = p.qu; v.qv = p.qv; v.zu = p.zu; v.zv = p.zv;
    v.Azu = p.Azu; v.Azv = p.Azv;
    return v;
}

// pcg_solver_standard_{2d,3d} launch sequence (:1169-1524 / :392-808)
template <int NC>
static int run_standard(Workspace &ws, const Geom &g, int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = ws.stream;
    SolveState *st = ws.state.as<SolveState>();
    DD *part = ws.partials.as<DD>();
    const Ptrs p = ptrs(ws, g);
    const VecArgs v = vargs(p);
    const double *A = ws.A.as<double>();
    const int32_t *act = ws.act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    auto rc = [&](int epi, int iter) { return RedCtx{part, st, epi, iter}; };

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    k_halo<<<hb, kBlock, 0, s>>>(g, p.xu, p.xv, st);
    k_mv<NC, MV_PLAIN><<<nb, kBlock, 0, s>>>(g, A, act, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr,
                                             nullptr, rc(EPI_NONE, 0));
    k_vec<OP_STD_INIT><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_L2RHS, 0));
    CU(cudaGetLastError());
    Poller poll(ws, st);
    for (int iter = 1; iter <= maxiters; ++iter) {
        k_precond<PRE_STD><<<nb, kBlock, 0, s>>>(g, precond, A, NC, act, p.ru, p.rv, p.zu, p.zv, nullptr, nullptr,
                                                 rc(EPI_STD_ETA1, iter));
        k_vec<OP_STD_D><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_NONE, iter));
        k_halo<<<hb, kBlock, 0, s>>>(g, p.du, p.dv, st);
        k_mv<NC, MV_DQ><<<nb, kBlock, 0, s>>>(g, A, act, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr,
                                              nullptr, rc(EPI_STD_ETA2, iter));
        k_vec<OP_XR><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_NONE, iter));
        if (is_check(iter, ncheck)) {
            k_halo<<<hb, kBlock, 0, s>>>(g, p.xu, p.xv, st);
            k_mv<NC, MV_RESID><<<nb, kBlock, 0, s>>>(g, A, act, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv,
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
template <int NC>
static int run_chrongear(Workspace &ws, const Geom &g, int precond, int ncheck, double tol, int maxiters) {
    cudaStream_t s = ws.stream;
    SolveState *st = ws.state.as<SolveState>();
    DD *part = ws.partials.as<DD>();
    const Ptrs p = ptrs(ws, g);
    const VecArgs v = vargs(p);
    const double *A = ws.A.as<double>();
    const int32_t *act = ws.act.as<int32_t>();
    const unsigned nb = nblocks(g.NQ);
    const unsigned hb = nblocks(4LL * g.NX + 4LL * (g.NY - 4));
    auto rc = [&](int epi, int iter) { return RedCtx{part, st, epi, iter}; };
    const long long nvec = (long long)g.nz * g.NQ;

    k_init_state<<<1, 1, 0, s>>>(st, tol, maxiters);
    // r = d = z = q = Az = 0 (:3048-3061)
    CU(cudaMemsetAsync(p.ru, 0, (size_t)(NVEC - VR_U) * nvec * sizeof(double), s));
    k_vec<OP_DOT_BB><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_L2RHS, 0));
    // first pass (:3085-3290)
    k_halo<<<hb, kBlock, 0, s>>>(g, p.xu, p.xv, st);
    k_mv<NC, MV_PLAIN><<<nb, kBlock, 0, s>>>(g, A, act, p.xu, p.xv, p.zu, p.zv, nullptr, nullptr, nullptr,
                                             nullptr, rc(EPI_NONE, 1));
    k_vec<OP_CG_INIT><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_NONE, 1));
    k_halo<<<hb, kBlock, 0, s>>>(g, p.ru, p.rv, st);
    k_precond<PRE_CG_FIRST><<<nb, kBlock, 0, s>>>(g, precond, A, NC, act, p.ru, p.rv, p.zu, p.zv, p.du, p.dv,
                                                  rc(EPI_CG_RHO0, 1));
    k_mv<NC, MV_DQ><<<nb, kBlock, 0, s>>>(g, A, act, p.du, p.dv, p.qu, p.qv, nullptr, nullptr, nullptr, nullptr,
                                          rc(EPI_CG_FIRST, 1));
    k_halo<<<hb, kBlock, 0, s>>>(g, p.qu, p.qv, st);
    k_vec<OP_XR><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_NONE, 1));
    CU(cudaGetLastError());
    Poller poll(ws, st);
    for (int iter = 2; iter <= maxiters; ++iter) {
        k_precond<PRE_ONLY><<<nb, kBlock, 0, s>>>(g, precond, A, NC, act, p.ru, p.rv, p.zu, p.zv, nullptr, nullptr,
                                                  rc(EPI_NONE, iter));
        k_mv<NC, MV_CG_AZ><<<nb, kBlock, 0, s>>>(g, A, act, p.zu, p.zv, p.Azu, p.Azv, nullptr, nullptr, p.ru,
                                                 p.rv, rc(EPI_CG_ITER, iter));
        k_halo<<<hb, kBlock, 0, s>>>(g, p.Azu, p.Azv, st);
        k_vec<OP_CG_UPD><<<nb, kBlock, 0, s>>>(g, v, rc(EPI_NONE, iter));
        if (is_check(iter, ncheck)) {
            k_mv<NC, MV_RESID><<<nb, kBlock, 0, s>>>(g, A, act, p.xu, p.xv, p.zu, p.zv, p.bu, p.bv, p.ru, p.rv,
                                                     rc(EPI_CHECK, iter));
            k_halo<<<hb, kBlock, 0, s>>>(g, p.ru, p.rv, st);
            CU(cudaGetLastError());
            int f = poll.after_check();
            if (f < 0) return fail(CISMGPU_ECUDA, "polling the convergence flag failed");
            if (f) break;
        }
    }
    CU(cudaGetLastError());
    return CISMGPU_OK;
}

enum Algo { ALG_STANDARD, ALG_CHRONGEAR };

static int solve(Algo alg, bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx2,
                 const int32_t *indx3, const int32_t *act, const double *Auu, const double *Auv, const double *Avu,
                 const double *Avv, const double *bu, const double *bv, double *xu, double *xv, int precond,
                 int ncheck, double tol, int maxiters, double *err, int *niters) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    const int32_t *indx = is3d ? indx3 : indx2;
    int rc = validate(nx, ny, is3d ? nz : 1, par, indx, act, Auu, Auv, Avu, Avv, bu, bv, xu, xv, precond, ncheck,
                      maxiters, err, niters);
    if (rc) return rc;
    if ((rc = validate_indx(indx, is3d ? 27 : 9))) return rc;
    Workspace &ws = g_ws;
    if ((rc = init_device(ws))) return rc;
    const Geom g = make_geom(nx, ny, is3d ? nz : 1, par);
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    if ((rc = upload(ws, g, is3d, indx, act, blocks, bu, bv, xu, xv))) return rc;
    if (alg == ALG_STANDARD)
        rc = is3d ? run_standard<27>(ws, g, precond, ncheck, tol, maxiters)
                  : run_standard<9>(ws, g, precond, ncheck, tol, maxiters);
    else
        rc = is3d ? run_chrongear<27>(ws, g, precond, ncheck, tol, maxiters)
                  : run_chrongear<9>(ws, g, precond, ncheck, tol, maxiters);
    if (rc) return rc;
    if ((rc = download_x(ws, g, is3d, xu, xv))) return rc;
    *err = ws.h_state->err;
    *niters = ws.h_state->niters;
    if (ws.h_state->status == CISMGPU_EBREAKDOWN_ETA1)
        return fail(CISMGPU_EBREAKDOWN_ETA1, "PCG solver has failed, eta1 = NaN");
    if (ws.h_state->status == CISMGPU_EBREAKDOWN_ALPHA)
        return fail(CISMGPU_EBREAKDOWN_ALPHA, "PCG solver has failed, alpha = NaN");
    return CISMGPU_OK;
}

static int matvec(bool is3d, int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indx,
                  const int32_t *act, const double *Auu, const double *Auv, const double *Avu, const double *Avv,
                  const double *xu, const double *xv, double *yu, double *yv) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error.clear();
    int dummy_i = 0;
    double dummy_d = 0.0;
    int rc = validate(nx, ny, is3d ? nz : 1, par, indx, act, Auu, Auv, Avu, Avv, xu, xv, xu, xv, 0, 1, 0,
                      &dummy_d, &dummy_i);
    if (rc) return rc;
    if ((rc = validate_indx(indx, is3d ? 27 : 9))) return rc;
    if (!yu || !yv) return fail(CISMGPU_EINVAL, "null output pointer");
    Workspace &ws = g_ws;
    if ((rc = init_device(ws))) return rc;
    const Geom g = make_geom(nx, ny, is3d ? nz : 1, par);
    const double *blocks[4] = {Auu, Auv, Avu, Avv};
    // x is uploaded into the b slots and the product lands in the x slots
    if ((rc = upload(ws, g, is3d, indx, act, blocks, xu, xv, xu, xv))) return rc;
    const Ptrs p = ptrs(ws, g);
    SolveState *st = ws.state.as<SolveState>();
    cudaStream_t s = ws.stream;
    k_init_state<<<1, 1, 0, s>>>(st, 0.0, 0);
    RedCtx rc0{ws.partials.as<DD>(), st, EPI_NONE, 0};
    if (is3d)
        k_mv<27, MV_PLAIN><<<nblocks(g.NQ), kBlock, 0, s>>>(g, ws.A.as<double>(), ws.act.as<int32_t>(), p.bu, p.bv,
                                                           p.xu, p.xv, nullptr, nullptr, nullptr, nullptr, rc0);
    else
        k_mv<9, MV_PLAIN><<<nblocks(g.NQ), kBlock, 0, s>>>(g, ws.A.as<double>(), ws.act.as<int32_t>(), p.bu, p.bv,
                                                          p.xu, p.xv, nullptr, nullptr, nullptr, nullptr, rc0);
    CU(cudaGetLastError());
    return download_x(ws, g, is3d, yu, yv);
}

}  // namespace cismgpu

// ---------------------------------------------------------------------------
// C ABI (include/cismgpu.h)
// ---------------------------------------------------------------------------
using namespace cismgpu;

extern "C" {

int cismgpu_pcg_standard_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                            const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                            const double *Auv, const double *Avu, const double *Avv, const double *bu,
                            const double *bv, double *xu, double *xv, int precond, int linear_solve_ncheck,
                            double tolerance, int maxiters, double *err, int *niters, int itest, int jtest,
                            int rtest) {
    (void)itest; (void)jtest; (void)rtest;  // debug-print location only (verbose_pcg = .false.)
    return solve(ALG_STANDARD, true, nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu,
                 bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_pcg_chrongear_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_2d,
                             const int32_t *indxA_3d, const int32_t *active_vertex, const double *Auu,
                             const double *Auv, const double *Avu, const double *Avv, const double *bu,
                             const double *bv, double *xu, double *xv, int precond, int linear_solve_ncheck,
                             double tolerance, int maxiters, double *err, int *niters, int itest, int jtest,
                             int rtest) {
    (void)itest; (void)jtest; (void)rtest;
    return solve(ALG_CHRONGEAR, true, nx, ny, nz, par, indxA_2d, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, bu,
                 bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_pcg_standard_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                            const int32_t *active_vertex, const double *Auu, const double *Auv, const double *Avu,
                            const double *Avv, const double *bu, const double *bv, double *xu, double *xv,
                            int precond, int linear_solve_ncheck, double tolerance, int maxiters, double *err,
                            int *niters, int itest, int jtest, int rtest) {
    (void)itest; (void)jtest; (void)rtest;
    return solve(ALG_STANDARD, false, nx, ny, 1, par, indxA_2d, nullptr, active_vertex, Auu, Auv, Avu, Avv, bu, bv,
                 xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_pcg_chrongear_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                             const int32_t *active_vertex, const double *Auu, const double *Auv, const double *Avu,
                             const double *Avv, const double *bu, const double *bv, double *xu, double *xv,
                             int precond, int linear_solve_ncheck, double tolerance, int maxiters, double *err,
                             int *niters, int itest, int jtest, int rtest) {
    (void)itest; (void)jtest; (void)rtest;
    return solve(ALG_CHRONGEAR, false, nx, ny, 1, par, indxA_2d, nullptr, active_vertex, Auu, Auv, Avu, Avv, bu,
                 bv, xu, xv, precond, linear_solve_ncheck, tolerance, maxiters, err, niters);
}

int cismgpu_matvec_structured_3d(int nx, int ny, int nz, const cismgpu_par_t *par, const int32_t *indxA_3d,
                                 const int32_t *active_vertex, const double *Auu, const double *Auv,
                                 const double *Avu, const double *Avv, const double *xu, const double *xv,
                                 double *yu, double *yv) {
    return matvec(true, nx, ny, nz, par, indxA_3d, active_vertex, Auu, Auv, Avu, Avv, xu, xv, yu, yv);
}

int cismgpu_matvec_structured_2d(int nx, int ny, const cismgpu_par_t *par, const int32_t *indxA_2d,
                                 const int32_t *active_vertex, const double *Auu, const double *Auv,
                                 const double *Avu, const double *Avv, const double *xu, const double *xv,
                                 double *yu, double *yv) {
    return matvec(false, nx, ny, 1, par, indxA_2d, active_vertex, Auu, Auv, Avu, Avv, xu, xv, yu, yv);
}

const char *cismgpu_last_error(void) { return g_last_error.c_str(); }

const char *cismgpu_version(void) { return "cismgpu 0.1 (sm_100a)"; }

}  // extern "C"
