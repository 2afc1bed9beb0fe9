// noalloc.cu -- the owned-vertex global sum for callers that cannot allocate
// device memory.
//
// cismgpu_global_sum_stagger copies host arrays into buffers the library
// allocates.  Some callers cannot let a library call cudaMalloc: a host whose
// own allocator owns the whole device (a pool carved out at start-up, as large
// CISM runs on a shared node do), code that must not synchronize the device in
// the middle of a time step (cudaMalloc and cudaFree can), and code that only
// holds device pointers handed to it by another component.  For them this file
// adds one entry point that takes device pointers and a stream and allocates
// nothing: the reduction's scratch (one double-double partial per 256-column
// block and the last-block ticket) lives in a fixed-size array in the module's
// own device memory, g_noalloc_scratch below.
//
// Limits and sharing rules:
//  * at most CISMGPU_NOALLOC_MAX_COLUMNS vertex columns ((nx-1)*(ny-1)); larger
//    grids are rejected with CISMGPU_EINVAL before anything is enqueued;
//  * parallel%reprosum is rejected (CISMGPU_EUNSUPPORTED): the reproducible sum needs
//    host steps between its kernels, which an asynchronous call cannot take; with the
//    sequential sum order (cismgpu_set_sum_order) the sum runs in one CTA and uses no
//    scratch at all;
//  * the three buffers must be readable by the current device (its own memory, managed
//    or mapped pinned memory);
//  * every call on a device shares the one array, so two calls whose kernels
//    overlap on the GPU (different streams, no ordering between them) race and
//    give wrong sums; calls on one stream, or otherwise ordered, are safe;
//  * the ticket must start at zero: each call clears it with cudaMemsetAsync on
//    the caller's stream before its kernel (the partials are written before they
//    are read and need no clearing);
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (this also loads the library's kernels onto that
//    device if nothing else has); make that first call before any stream
//    capture begins.

#define CISMGPU_NOALLOC_BLOCKS (CISMGPU_NOALLOC_MAX_COLUMNS / 256)

namespace cismgpu {

struct NoAllocScratch {
    unsigned int ticket;
    unsigned int pad[63];                   // keeps the partials 256-byte aligned
    DD partials[CISMGPU_NOALLOC_BLOCKS];
};
static_assert(CISMGPU_NOALLOC_MAX_COLUMNS % kBlock == 0, "scratch sized in whole blocks");
static_assert(sizeof(NoAllocScratch) == 256 + CISMGPU_NOALLOC_BLOCKS * sizeof(DD), "scratch layout");

// 256 B + 16 B per block: 256 KiB + 256 B for CISMGPU_NOALLOC_MAX_COLUMNS = 2^22.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

static constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static NoAllocScratch *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set-up on first use).
static int noalloc_scratch(NoAllocScratch **out) {
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(CISMGPU_ENODEV, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        TRY(check_device());
        void *p = nullptr;
        CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        if (!p || (reinterpret_cast<uintptr_t>(p) & 255u))
            return fail(CISMGPU_ECUDA, "scratch symbol address missing or misaligned");
        g_noalloc_ptr[dev] = static_cast<NoAllocScratch *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CISMGPU_OK;
}

// The pointer must be readable by the current device: its own device memory, managed memory
// or mapped pinned memory.  Device memory of another GPU is rejected (the kernel would read
// it over the peer link, or fault where peer access is off).
static int noalloc_check_ptr(const void *p, const char *name) {
    cudaPointerAttributes a;
    CU(cudaPointerGetAttributes(&a, p));
    if (a.type == cudaMemoryTypeUnregistered || (a.type == cudaMemoryTypeHost && !a.devicePointer))
        return fail(CISMGPU_EINVAL, std::string(name) + " is not device-accessible memory");
    if (a.type == cudaMemoryTypeDevice) {
        int dev = 0;
        CU(cudaGetDevice(&dev));
        if (a.device != dev)
            return fail(CISMGPU_EINVAL, std::string(name) + " is memory of another device than the current one");
    }
    return CISMGPU_OK;
}

}  // namespace cismgpu

extern "C" int cismgpu_global_sum_stagger_noalloc(int nx, int ny, int nz, const cismgpu_par_t *par,
                                                  const double *arr1_dev, const double *arr2_dev, double *sum_dev,
                                                  void *cuda_stream) {
    using namespace cismgpu;
    g_last_error.clear();
    if (!par || !arr1_dev || !arr2_dev || !sum_dev) return fail(CISMGPU_EINVAL, "null pointer argument");
    if (nx < 6 || ny < 6 || nz < 1) return fail(CISMGPU_EINVAL, "grid too small");
    if (par->tasks_row * par->tasks_col != 1)
        return fail(CISMGPU_EUNSUPPORTED, "the whole domain must be on one GPU (tasks_row*tasks_col == 1)");
    if (par->reprosum)
        return fail(CISMGPU_EUNSUPPORTED, "parallel%reprosum: the reproducible sum needs host steps; "
                                          "use cismgpu_global_sum_stagger");
    if (par->staggered_ilo < 1 || par->staggered_ihi > nx - 1 || par->staggered_ilo > par->staggered_ihi ||
        par->staggered_jlo < 1 || par->staggered_jhi > ny - 1 || par->staggered_jlo > par->staggered_jhi)
        return fail(CISMGPU_EINVAL, "owned vertex bounds outside the array");
    const long long cols = (long long)(nx - 1) * (long long)(ny - 1);
    if (cols > CISMGPU_NOALLOC_MAX_COLUMNS)
        return fail(CISMGPU_EINVAL, "(nx-1)*(ny-1) = " + std::to_string(cols) +
                                        " exceeds the no-allocation scratch limit of " +
                                        std::to_string(CISMGPU_NOALLOC_MAX_COLUMNS) + " columns");
    TRY(noalloc_check_ptr(arr1_dev, "arr1"));
    TRY(noalloc_check_ptr(arr2_dev, "arr2"));
    TRY(noalloc_check_ptr(sum_dev, "sum"));
    NoAllocScratch *s = nullptr;
    TRY(noalloc_scratch(&s));
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    const Geom g = make_geom(nx, ny, nz, par);
    const unsigned nb = nblocks(g.NQ);
    if (g_sum_order.load() == CISMGPU_SUM_SEQUENTIAL) {  // the reference's order; no scratch
        SeqArgs sa{};
        sa.a[0][0] = arr1_dev;
        sa.a[0][1] = arr2_dev;
        k_seq_sum<1, true><<<1, kBlock, 0, stream>>>(g, sa, nullptr, EPI_NONE, EPI_NONE, 0, sum_dev);
        CU(cudaGetLastError());
        return CISMGPU_OK;
    }
    CU(cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned int), stream));
    k_gsum<true><<<nb, kBlock, 0, stream>>>(g, arr1_dev, arr2_dev, s->partials, &s->ticket, sum_dev);
    CU(cudaGetLastError());
    return CISMGPU_OK;
}
