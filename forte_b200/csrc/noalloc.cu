// fcib_spin2_device_noalloc: <S^2> of a device vector with no allocation of any kind.
//
// For callers that cannot allocate device memory: a host program whose memory pool owns the
// whole GPU (a framework caching allocator, a fixed arena sized at start-up), or a loop that
// must not pay for cudaMalloc/cudaFree, which can synchronise the device and fail when memory
// is fragmented.  fcib_spin2 allocates a copy of the vector and its reduction buffers on
// every call; this entry point takes the vector already on the device and allocates nothing.
//
// The same k_spin2 / k_final_reduce kernels and the same grid as fcib_spin2, but the per-block
// partial sums and the reduced result live in a file-scope device array instead of buffers
// allocated per call.  Host code cannot use that array's name as a device address, so the
// first call on each device, with that device current, takes the address with
// cudaGetSymbolAddress (return code checked) and keeps it together with the unique ID of the
// device's current CUDA context; later calls reuse it while that context is still current.
// A device reset (cudaDeviceReset) or a torn-down and recreated primary context loads the
// module again at a new address: the next call sees a different context ID and looks the
// address up again, so a stale address is never launched on.  Make the first call on a device
// (and the first call after a reset) before any stream capture that might include the entry
// point.
//
// Scratch limits: kNoAllocMaxBlocks partial-sum blocks of kSlots doubles plus one result row,
// (1024 + 1) * 73 * 8 B = 598,600 B per device.  The grid is min(4 * SMs, ceil(ndet / 256)), so a
// launch that would need more than kNoAllocMaxBlocks blocks is rejected with FCIB_ERR_UNSUPPORTED.
// Every partial slot read by k_final_reduce is written by k_spin2 first in the same call, so
// nothing in the scratch has to start at zero.
//
// The scratch is shared by every context on a device: calls that overlap in time (concurrent
// host threads, or work still in flight on another stream) race on it; callers serialise them.
#include <mutex>

#include "fcib_internal.h"

namespace fcib {

constexpr int kNoAllocMaxBlocks = 1024;
constexpr int kNoAllocMaxDevices = 64;
constexpr size_t kNoAllocDoubles = (size_t)(kNoAllocMaxBlocks + 1) * kSlots;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Unique ID of the calling thread's current CUDA context (0 when none), through driver entry
// points fetched once from the runtime, so the library needs no link dependency on libcuda.
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);
static unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        void* f1 = nullptr;
        void* f2 = nullptr;
        FCIB_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1));
        FCIB_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2));
        FCIB_CHECK(q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess && f1 && f2,
                   FCIB_ERR_CUDA, "fcib_spin2_device_noalloc: driver entry points cuCtxGetCurrent/cuCtxGetId missing");
        get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    void* ctx = nullptr;
    FCIB_CHECK(get_current(&ctx) == 0, FCIB_ERR_CUDA, "fcib_spin2_device_noalloc: cuCtxGetCurrent failed");
    if (!ctx) return 0;
    unsigned long long id = 0;
    FCIB_CHECK(get_id(ctx, &id) == 0, FCIB_ERR_CUDA, "fcib_spin2_device_noalloc: cuCtxGetId failed");
    return id;
}

static double* noalloc_scratch(int device) {
    static std::mutex mu;
    static double* addr[kNoAllocMaxDevices] = {};
    static unsigned long long ctx_id[kNoAllocMaxDevices] = {};
    FCIB_CHECK(device >= 0 && device < kNoAllocMaxDevices, FCIB_ERR_UNSUPPORTED,
               "fcib_spin2_device_noalloc: device ordinal above the scratch table size (64)");
    std::lock_guard<std::mutex> lock(mu);
    int cur = -1;
    FCIB_CUDA(cudaGetDevice(&cur));
    FCIB_CHECK(cur == device, FCIB_ERR_STATE, "fcib_spin2_device_noalloc: context device is not current");
    // binds the device's primary context to this thread (CUDA 12: created if needed; the device
    // is already the current one, so nothing else changes) before its ID is read
    FCIB_CUDA(cudaSetDevice(cur));
    const unsigned long long id = current_context_id();
    FCIB_CHECK(id != 0, FCIB_ERR_STATE, "fcib_spin2_device_noalloc: no current CUDA context");
    if (!addr[device] || ctx_id[device] != id) {
        void* p = nullptr;
        FCIB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        addr[device] = static_cast<double*>(p);
        ctx_id[device] = id;
    }
    return addr[device];
}

}  // namespace fcib

extern "C" int fcib_spin2_device_noalloc(fcib_ctx* ctx, const double* d_c, double* s2, void* stream) {
    if (!ctx || !d_c || !s2) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.has_ints && c.has_state && c.tables_ready, FCIB_ERR_STATE,
                   "fcib_spin2_device_noalloc: string tables not built (call fcib_size, fcib_solve or "
                   "fcib_spin2 on this context first)");
        const size_t N = (size_t)c.nvec;
        const int nblk = std::max(1, std::min(4 * c.num_sms, (int)((N + kRedThreads - 1) / kRedThreads)));
        FCIB_CHECK(nblk <= kNoAllocMaxBlocks, FCIB_ERR_UNSUPPORTED,
                   "fcib_spin2_device_noalloc: launch needs more partial-sum blocks than the static "
                   "scratch holds (1024)");
        double* partial = noalloc_scratch(c.device);
        double* out = partial + (size_t)kNoAllocMaxBlocks * kSlots;
        cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
        k_spin2<<<nblk, kRedThreads, 0, st>>>(d_c, c.A.str.p, c.B.str.p, (int)c.nas, (int)c.nbs, c.n, partial,
                                              sym_dev(c), (size_t)c.nvec);
        FCIB_KCHECK();
        k_final_reduce<<<1, 256, 0, st>>>(partial, nblk, out);
        FCIB_KCHECK();
        double s = 0.0;
        FCIB_CUDA(cudaMemcpyAsync(&s, out, sizeof(double), cudaMemcpyDeviceToHost, st));
        FCIB_CUDA(cudaStreamSynchronize(st));
        const double na = c.na, nb = c.nb;
        *s2 = -s + 0.25 * (na - nb) * (na - nb) + 0.5 * (na + nb);
    });
}
