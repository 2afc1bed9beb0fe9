// server.cu -- continuous-batching serving loop for the mixed-precision solver.
//
// Requests (one linear system each, in the caller's Fortran layout) are queued by
// cismgpu_server_submit and served by one host thread:
//   * admission (its own host thread): in arrival order while the HBM budget allows; an admitted request gets
//     its own device-resident handle (matrix, FP32 copy, preconditioner, Krylov vectors),
//     uploaded on the handle's own stream while the GPU runs the current epoch;
//   * epochs: a large 2D request runs a launch of the single-solve kernel of its own (its FP32
//     matrix resident in shared memory where its tiles fit one per CTA); every other active
//     request of a kernel class (2D and 3D with nz <= 16 together; 3D with 16 < nz <= 32) takes
//     part in one launch of the dynamic persistent kernel
//     (k_mixed_dyn; with 2D and 3D requests both present, its multi-class form, in which
//     every work item runs its own solve's tile code, so 2D and 3D requests share the SMs in
//     the same launch) for up to epoch_steps steps; a request's state (scalars in its MState,
//     vectors in its buffers) stays on the device between epochs, so a request joins and
//     leaves between any two epochs without restarting anyone;
//   * retirement: a finished request's x is copied into the caller's arrays, its handle
//     freed and its bytes returned to the budget.
// Tile heights and the order of every sum depend on the request only, so a result is
// bit-identical whether the request is served alone or in any mix.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace cismgpu {

__global__ void k_gather_states(MState *const *src, MState *dst, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = *src[t];
}

struct SrvReq {
    long long id = 0;
    cismgpu_request_t rq{};
    cismgpu_par_t par{};
    int phase = 0;  // 0 queued, 1 admitted, 2 done
    int status = CISMGPU_OK, niters = 0, checks = 0;
    double err = 0.0;
    double t_submit = 0.0, t_admit = 0.0, t_done = 0.0;  // ms since the server started
    cismgpu_solver *h = nullptr;
    size_t bytes = 0;
    int cls = 0;       // kernel class: 0 2D or 3D nz <= 16, 1 3D 16 < nz <= 32, 2 large 2D on the
                       // single-solve kernel
    MState *h_st = nullptr;  // class 2: pinned copy of the state after each epoch
    MCtl *h_ctl = nullptr;   // class 2: pinned copy of the launch's control word
    int TY = 0;
    unsigned tick = 0; // steps completed, as of the last epoch
};

// Device bytes a request's handle holds at most (the FP64 system, its staging block, the
// FP64 and FP32 vectors, the FP32 matrix, the interleaved FP64 matrix of a 3D or streamed
// solve, the factors, tile maps and records; with the line preconditioners their FP64 setup
// planes and FP32 factors and work planes).
static size_t request_bytes(const cismgpu_request_t &r) {
    const long long NQ = (long long)(r.nx - 1) * (r.ny - 1);
    const long long nvec = NQ * (r.dims == 3 ? r.nz : 1);
    const long long NC = r.dims == 3 ? 27 : 9;
    const bool il = r.dims == 3 || (size_t)(NC * nvec) * 16 > kStreamBytes;
    const long long per = 4 * NC * 8 + NC * 8 + NVEC * 8 + 4 * NC * 4 + (il ? 4 * NC * 8 : 0) + 6 * 4 + 16 * 4;
    const long long lines = r.precond >= 3 ? NQ * (NTRI * 8 + 12 * 4) : 0;
    return (size_t)(nvec * per + NQ * 16 + lines + (8 << 20));
}

static constexpr int kSrvClasses = 2;       // classes served by the dynamic kernel
static constexpr long long kSrvResidentMin = 65536;  // owned vertices from which a 2D request runs on
                                                     // the single-solve kernel

static int request_class(const cismgpu_request_t &r) { return (r.dims == 3 && r.nz > 16) ? 1 : 0; }

}  // namespace cismgpu

struct cismgpu_server {
    size_t budget = 0, used = 0;
    int epoch_steps = 64;
    std::mutex mu;
    std::condition_variable cv;     // work arrived / a request finished
    std::deque<cismgpu::SrvReq *> queued;   // submitted, waiting for admission
    std::vector<cismgpu::SrvReq *> ready;   // admitted and uploaded, joining at the next epoch
    std::vector<cismgpu::SrvReq *> active;  // taking part in epochs
    int uploading = 0;                      // admitted, upload in progress
    std::unordered_map<long long, cismgpu::SrvReq *> reqs;
    long long next_id = 1;
    long long inflight = 0;         // submitted and not yet done
    long long epochs = 0;
    long long launches = 0;         // kernel launches (one per class and epoch)
    long long multi_launches = 0;   // launches that held 2D and 3D requests together
    bool stop = false;
    int device = 0;
    std::thread th;                 // epoch loop
    std::thread up;                 // admissions and uploads
    cudaStream_t es = nullptr;      // epoch stream
    std::chrono::steady_clock::time_point t0;
    double now() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace cismgpu {

// Per-class launch scratch, reused across epochs.
struct SrvLaunch {
    DevBuf blk;                 // descriptors | state pointers | ticks | tiles | ctl | gathered states
    char *h_blk = nullptr;      // pinned staging of the same layout (rewritten only after the epoch)
    size_t h_cap = 0;
    MState *h_states = nullptr; // pinned
    MCtl *h_ctl = nullptr;      // pinned
    int cap = 0;
    std::vector<SrvReq *> members;
    ~SrvLaunch() {
        blk.release();
        if (h_blk) cudaFreeHost(h_blk);
        if (h_states) cudaFreeHost(h_states);
        if (h_ctl) cudaFreeHost(h_ctl);
    }
};

// Create, upload and prepare the handle of an admitted request (on the handle's stream).
static int srv_admit(SrvReq &r) {
    const cismgpu_request_t &q = r.rq;
    cismgpu_solver_t *h = nullptr;
    TRY(cismgpu_solver_create(&h, q.dims, q.nx, q.ny, q.nz, &r.par, q.indxA, q.active_vertex, q.Auu, q.Auv,
                              q.Avu, q.Avv, q.bu, q.bv, q.xu0, q.xv0, nullptr));
    r.h = h;
    Solver &sv = h->sv;
    const int nzm = mixed_nzm(sv.g, sv.is3d);
    r.TY = mixed_batch_ty(sv.g, sv.is3d, nzm, batch_floor(sv.is3d, nzm));
    if (!sv.is3d) {
        // a large 2D system runs its epochs on the single-solve kernel, a launch of its own, with
        // its FP32 matrix resident in shared memory where the tiles fit one per co-resident CTA
        // (2D steps are latency-bound: no leader hop, and no matrix stream where resident)
        const int ty1 = mixed_solve_ty(sv.g, false, 1);
        const long long owned = (long long)(sv.g.ihi - sv.g.ilo + 1) * (sv.g.jhi - sv.g.jlo + 1);
        if (owned >= kSrvResidentMin) {
            r.cls = 2;
            r.TY = ty1;
            CU(cudaMallocHost((void **)&r.h_st, sizeof(MState)));
            CU(cudaMallocHost((void **)&r.h_ctl, sizeof(MCtl)));
        }
    }
    TRY(mixed_prepare(sv, q.precond, r.TY));
    TRY(mixed_reset(sv, sv.stream));
    const MState S0 = mixed_init_state(q.tolerance, q.maxiters, q.linear_solve_ncheck, q.precond);
    CU(cudaMemcpyAsync(sv.mixed.state, &S0, sizeof(MState), cudaMemcpyHostToDevice, sv.stream));
    if (r.cls == 2) {
        const MDesc D = mixed_desc(sv, q.precond, r.TY);
        CU(cudaMemcpyAsync(sv.mixed.desc, &D, sizeof(MDesc), cudaMemcpyHostToDevice, sv.stream));
    }
    CU(cudaStreamSynchronize(sv.stream));
    r.tick = 0;
    return CISMGPU_OK;
}

// One epoch of a class-2 request: the single-solve kernel for up to epoch_steps steps
// (it resumes exactly where the previous epoch stopped), then its state and control word into
// the request's pinned copies (asynchronous on the epoch stream).
static int srv_launch_resident(cismgpu_server *S, SrvReq &r) {
    Solver &sv = r.h->sv;
    MixedBufs &m = sv.mixed;
    cudaStream_t s = S->es;
    const bool res = mixed_resident(false, 1, r.TY, m.ntiles);
    const int grid = mixed_launch_grid(false, 1, r.TY, res, m.ntiles);
    if (grid < 1) return fail(CISMGPU_EUNSUPPORTED, "mixed kernel does not fit on an SM at this tile height");
    CU(cudaMemsetAsync(m.ctl, 0, sizeof(MCtl), s));
    TRY(mixed_dispatch(false, 1, m.desc, m.state, m.tiles, m.ntiles, r.TY, res, m.ctl, S->epoch_steps, grid, s));
    CU(cudaMemcpyAsync(r.h_st, m.state, sizeof(MState), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(r.h_ctl, m.ctl, sizeof(MCtl), cudaMemcpyDeviceToHost, s));
    return CISMGPU_OK;
}

// Launch one epoch of class cls over its active requests (asynchronous on the epoch stream).
// *multi: the launch held 2D and 3D requests together (the multi-class kernel).
static int srv_launch(cismgpu_server *S, SrvLaunch &L, int cls, bool *multi) {
    const int n = (int)L.members.size();
    *multi = false;
    if (n == 0) return CISMGPU_OK;
    int TY2 = 1, TY3 = 1, n3 = 0;
    std::vector<MDesc> descs(n);
    std::vector<MState *> sptr(n);
    std::vector<unsigned> tick(n);
    std::vector<MTile> tl;
    for (int t = 0; t < n; ++t) {
        SrvReq &r = *L.members[t];
        Solver &sv = r.h->sv;
        descs[t] = mixed_desc(sv, r.rq.precond, r.TY);
        sptr[t] = sv.mixed.state;
        tick[t] = r.tick;
        if (sv.is3d) {
            TY3 = std::max(TY3, r.TY);
            ++n3;
        } else {
            TY2 = std::max(TY2, r.TY);
        }
        for (int k = 0; k < descs[t].ntiles; ++k) tl.push_back(MTile{t, k});
    }
    const bool is3d = n3 > 0;
    *multi = n3 > 0 && n3 < n;  // class 0 with both kinds: one multi-class launch
    const int nzm = cls == 1 ? 32 : 16;
    const int TYmax = is3d ? TY3 : TY2;
    const int grid = *multi ? mixed_multi_grid(TY3, TY2) : mixed_dyn_grid(is3d, is3d ? nzm : 1, TYmax);
    if (grid < 1) return fail(CISMGPU_EUNSUPPORTED, "mixed kernel does not fit on an SM at this tile height");
    if ((long long)n > (long long)grid * kMaxCtaSolves) return fail(CISMGPU_EUNSUPPORTED, "too many requests");
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o_d = 0, o_p = al(n * sizeof(MDesc)), o_t = o_p + al(n * sizeof(MState *)),
                 o_l = o_t + al(n * sizeof(unsigned)), o_c = o_l + al(tl.size() * sizeof(MTile)),
                 o_g = o_c + al(sizeof(MCtl)), total = o_g + al(n * sizeof(MState));
    CU(L.blk.ensure(total));
    if (total > L.h_cap) {
        if (L.h_blk) cudaFreeHost(L.h_blk);
        L.h_blk = nullptr;
        L.h_cap = 0;
        CU(cudaMallocHost((void **)&L.h_blk, total));
        L.h_cap = total;
    }
    if (n > L.cap) {
        if (L.h_states) cudaFreeHost(L.h_states);
        L.h_states = nullptr;
        CU(cudaMallocHost((void **)&L.h_states, n * sizeof(MState)));
        L.cap = n;
    }
    if (!L.h_ctl) CU(cudaMallocHost((void **)&L.h_ctl, sizeof(MCtl)));
    char *base = static_cast<char *>(L.blk.p);
    MCtl c0;
    std::memset(&c0, 0, sizeof(c0));
    c0.active = n;
    cudaStream_t s = S->es;
    std::memcpy(L.h_blk + o_d, descs.data(), n * sizeof(MDesc));
    std::memcpy(L.h_blk + o_p, sptr.data(), n * sizeof(MState *));
    std::memcpy(L.h_blk + o_t, tick.data(), n * sizeof(unsigned));
    std::memcpy(L.h_blk + o_l, tl.data(), tl.size() * sizeof(MTile));
    std::memcpy(L.h_blk + o_c, &c0, sizeof(MCtl));
    CU(cudaMemcpyAsync(base, L.h_blk, o_g, cudaMemcpyHostToDevice, s));
    if (*multi)
        TRY(mixed_multi_launch(reinterpret_cast<MDesc *>(base + o_d), reinterpret_cast<MState **>(base + o_p),
                               reinterpret_cast<unsigned *>(base + o_t), n, reinterpret_cast<MTile *>(base + o_l),
                               (int)tl.size(), TY3, TY2, reinterpret_cast<MCtl *>(base + o_c), S->epoch_steps, grid,
                               s));
    else
        TRY(mixed_dyn_dispatch(is3d, is3d ? nzm : 1, reinterpret_cast<MDesc *>(base + o_d),
                               reinterpret_cast<MState **>(base + o_p), reinterpret_cast<unsigned *>(base + o_t), n,
                               reinterpret_cast<MTile *>(base + o_l), (int)tl.size(), TYmax,
                               reinterpret_cast<MCtl *>(base + o_c), S->epoch_steps, grid, s));
    k_gather_states<<<(n + 127) / 128, 128, 0, s>>>(reinterpret_cast<MState **>(base + o_p),
                                                   reinterpret_cast<MState *>(base + o_g), n);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(L.h_states, base + o_g, n * sizeof(MState), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(L.h_ctl, base + o_c, sizeof(MCtl), cudaMemcpyDeviceToHost, s));
    return CISMGPU_OK;
}

// A request's result: x to the caller's arrays, its status and counters; it is done for the
// caller (poll and drain see it) from here on.
static void srv_deliver(cismgpu_server *S, SrvReq &r, int status, double err, int niters, int checks) {
    if (r.h) {
        const int rc = cismgpu_solver_get_x(r.h, r.rq.xu, r.rq.xv);
        if (rc && status == CISMGPU_OK) status = rc;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    r.status = status;
    r.err = err;
    r.niters = niters;
    r.checks = checks;
    r.t_done = S->now();
    r.phase = 2;
    S->inflight -= 1;
    S->cv.notify_all();
}

// The handle of a delivered request freed and its bytes returned to the budget.
static void srv_free(cismgpu_server *S, SrvReq &r) {
    if (r.h) {
        cismgpu_solver_destroy(r.h);
        r.h = nullptr;
    }
    if (r.h_st) cudaFreeHost(r.h_st);
    if (r.h_ctl) cudaFreeHost(r.h_ctl);
    r.h_st = nullptr;
    r.h_ctl = nullptr;
    std::lock_guard<std::mutex> lk(S->mu);
    S->used -= r.bytes;
    r.bytes = 0;
    S->cv.notify_all();
}

// Finish a request: delivered, then freed.
static void srv_retire(cismgpu_server *S, SrvReq &r, int status, double err, int niters, int checks) {
    srv_deliver(S, r, status, err, niters, checks);
    srv_free(S, r);
}

// Admission thread: takes queued requests in arrival order as the HBM budget allows and
// uploads and prepares each on its own stream, so that uploads run while the epoch loop keeps
// the GPU busy.  A request larger than the whole budget fails with CISMGPU_ENOMEM.
static void srv_admit_loop(cismgpu_server *S) {
    cudaSetDevice(S->device);
    for (;;) {
        SrvReq *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv.wait(lk, [&] {
                if (S->queued.empty()) return S->stop;
                const SrvReq *f = S->queued.front();
                return f->bytes > S->budget || S->used + f->bytes <= S->budget;
            });
            if (S->queued.empty()) break;  // stopping, nothing left to admit
            r = S->queued.front();
            S->queued.pop_front();
            if (r->bytes > S->budget) {
                r->bytes = 0;  // never counted against the budget
            } else {
                S->used += r->bytes;
            }
            S->uploading += 1;
        }
        int rc = r->bytes == 0 ? fail(CISMGPU_ENOMEM, "request larger than the HBM budget") : srv_admit(*r);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->uploading -= 1;
            if (!rc) {
                r->t_admit = S->now();
                r->phase = 1;
                S->ready.push_back(r);
            }
            S->cv.notify_all();
        }
        if (rc) srv_retire(S, *r, rc, std::nan(""), 0, 0);
    }
}

// Epoch loop: one epoch per kernel class over the active requests (2D and 3D requests share the
// class-0 launch), then the finished ones are delivered and freed; requests admitted meanwhile
// join at the next epoch.  The host waits for each epoch before it queues the next: a pipelined
// form that queued epoch e before reading e-1 measured slower on the served stream (6.9 against
// 8.3 solves/s), because a 3D result's layout change is a kernel that cannot start beside a
// cooperative launch holding every SM, and freeing a finished request's memory synchronizes the
// device, so the host waited for the queued epoch anyway and every request spent one more epoch
// as a skipped member.
static void srv_loop(cismgpu_server *S) {
    cudaSetDevice(S->device);
    SrvLaunch L[kSrvClasses];
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv.wait(lk, [&] {
                return !S->ready.empty() || !S->active.empty() ||
                       (S->stop && S->queued.empty() && S->uploading == 0);
            });
            if (S->ready.empty() && S->active.empty()) break;  // stopping and nothing left
            S->active.insert(S->active.end(), S->ready.begin(), S->ready.end());
            S->ready.clear();
        }
        for (int c = 0; c < kSrvClasses; ++c) L[c].members.clear();
        std::vector<SrvReq *> resident;
        for (SrvReq *r : S->active) {
            if (r->cls == 2) resident.push_back(r);
            else L[r->cls].members.push_back(r);
        }
        int launched = 0, multi = 0;
        std::vector<SrvReq *> res_run;
        for (SrvReq *r : resident) {
            const int rc = srv_launch_resident(S, *r);
            if (rc) srv_retire(S, *r, rc, std::nan(""), 0, 0);
            else {
                res_run.push_back(r);
                ++launched;
            }
        }
        for (int c = 0; c < kSrvClasses; ++c) {
            if (L[c].members.empty()) continue;
            bool m = false;
            const int rc = srv_launch(S, L[c], c, &m);
            if (rc) {  // the class cannot run: fail its requests
                for (SrvReq *r : L[c].members) srv_retire(S, *r, rc, std::nan(""), 0, 0);
                L[c].members.clear();
            } else {
                ++launched;
                multi += m ? 1 : 0;
            }
        }
        if (launched) {
            cudaStreamSynchronize(S->es);
            std::lock_guard<std::mutex> lk(S->mu);
            ++S->epochs;
            S->launches += launched;
            S->multi_launches += multi;
        }
        std::vector<SrvReq *> still;
        for (SrvReq *r : res_run) {
            const MState &st = *r->h_st;
            if (st.done) srv_retire(S, *r, st.status, st.err, st.niters, st.checks);
            else if (r->h_ctl->abort) srv_retire(S, *r, CISMGPU_ETIMEOUT, st.err, st.niters, st.checks);
            else still.push_back(r);
        }
        for (int c = 0; c < kSrvClasses; ++c) {
            const bool aborted = L[c].h_ctl && !L[c].members.empty() && L[c].h_ctl->abort;
            for (size_t t = 0; t < L[c].members.size(); ++t) {
                SrvReq *r = L[c].members[t];
                const MState &st = L[c].h_states[t];
                r->tick = st.tick;
                if (st.done) srv_retire(S, *r, st.status, st.err, st.niters, st.checks);
                else if (aborted) srv_retire(S, *r, CISMGPU_ETIMEOUT, st.err, st.niters, st.checks);
                else still.push_back(r);
            }
        }
        std::lock_guard<std::mutex> lk(S->mu);
        S->active.swap(still);
    }
}

}  // namespace cismgpu

extern "C" {

int cismgpu_server_create(cismgpu_server_t **out, size_t hbm_budget_bytes, int epoch_steps) {
    using namespace cismgpu;
    g_last_error.clear();
    if (!out) return fail(CISMGPU_EINVAL, "null argument");
    *out = nullptr;
    if (hbm_budget_bytes == 0 || epoch_steps < 1) return fail(CISMGPU_EINVAL, "budget and epoch_steps must be > 0");
    TRY(check_device());
    cismgpu_server *S = new cismgpu_server();
    S->budget = hbm_budget_bytes;
    S->epoch_steps = epoch_steps;
    S->t0 = std::chrono::steady_clock::now();
    cudaGetDevice(&S->device);
    const cudaError_t e = cudaStreamCreateWithFlags(&S->es, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete S;
        return fail(CISMGPU_ECUDA, std::string("server stream creation failed: ") + cudaGetErrorString(e));
    }
    S->th = std::thread(srv_loop, S);
    S->up = std::thread(srv_admit_loop, S);
    *out = S;
    return CISMGPU_OK;
}

int cismgpu_server_submit(cismgpu_server_t *S, const cismgpu_request_t *rq, long long *id) {
    using namespace cismgpu;
    g_last_error.clear();
    if (!S || !rq || !id || !rq->par || !rq->xu || !rq->xv) return fail(CISMGPU_EINVAL, "null argument");
    if (rq->dims != 2 && rq->dims != 3) return fail(CISMGPU_EINVAL, "dims must be 2 or 3");
    TRY(validate_solve_args(rq->precond, rq->linear_solve_ncheck, rq->maxiters));
    if (!(rq->precond >= 0 && rq->precond <= 4 && (rq->precond != 2 || rq->dims == 3)))
        return fail(CISMGPU_EUNSUPPORTED, "mixed solver preconditioners: 0, 1, 2 (3D only), 3 or 4");
    if (rq->dims == 3 && (rq->nz < 1 || rq->nz > kMixedMaxNz)) return fail(CISMGPU_EUNSUPPORTED, "nz must be 1..32");
    SrvReq *r = new SrvReq();
    r->rq = *rq;
    r->par = *rq->par;
    r->rq.par = &r->par;
    if (rq->dims == 2) r->rq.nz = 1;
    r->bytes = request_bytes(r->rq);
    r->cls = request_class(r->rq);
    std::lock_guard<std::mutex> lk(S->mu);
    r->id = S->next_id++;
    r->t_submit = S->now();
    S->reqs[r->id] = r;
    S->queued.push_back(r);
    S->inflight += 1;
    *id = r->id;
    S->cv.notify_all();
    return CISMGPU_OK;
}

int cismgpu_server_poll(cismgpu_server_t *S, long long id, int *done, double *err, int *niters, int *status,
                        double *latency_ms, double *queue_ms) {
    using namespace cismgpu;
    if (!S || !done) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return fail(CISMGPU_EINVAL, "unknown request id");
    const SrvReq &r = *it->second;
    *done = r.phase == 2;
    if (err) *err = r.err;
    if (niters) *niters = r.niters;
    if (status) *status = r.status;
    if (latency_ms) *latency_ms = r.phase == 2 ? r.t_done - r.t_submit : S->now() - r.t_submit;
    if (queue_ms) *queue_ms = r.phase >= 1 ? r.t_admit - r.t_submit : S->now() - r.t_submit;
    return CISMGPU_OK;
}

int cismgpu_server_drain(cismgpu_server_t *S) {
    using namespace cismgpu;
    if (!S) return fail(CISMGPU_EINVAL, "null argument");
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv.wait(lk, [&] { return S->inflight == 0 && S->used == 0; });  // done and their memory released
    return CISMGPU_OK;
}

int cismgpu_server_stats(cismgpu_server_t *S, long long *epochs, size_t *bytes_in_use, int *active, int *queued) {
    using namespace cismgpu;
    if (!S) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    if (epochs) *epochs = S->epochs;
    if (bytes_in_use) *bytes_in_use = S->used;
    if (active) *active = (int)S->active.size();
    if (queued) *queued = (int)S->queued.size();
    return CISMGPU_OK;
}

int cismgpu_server_launch_stats(cismgpu_server_t *S, long long *launches, long long *multi_class_launches) {
    using namespace cismgpu;
    if (!S) return fail(CISMGPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    if (launches) *launches = S->launches;
    if (multi_class_launches) *multi_class_launches = S->multi_launches;
    return CISMGPU_OK;
}

int cismgpu_server_destroy(cismgpu_server_t *S) {
    if (!S) return CISMGPU_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    if (S->up.joinable()) S->up.join();
    if (S->th.joinable()) S->th.join();
    for (auto &kv : S->reqs) {
        if (kv.second->h) cismgpu_solver_destroy(kv.second->h);
        delete kv.second;
    }
    if (S->es) cudaStreamDestroy(S->es);
    delete S;
    return CISMGPU_OK;
}

}  // extern "C"
