// Inner products without any device allocation.
//
// xamg_dot needs a caller-provided scratch buffer for its per-chunk partial
// sums.  Some callers cannot provide one: code that runs while a host
// framework owns every device allocation (a plug-in handed only its input and
// output buffers), code on a latency-critical path where cudaMalloc's implicit
// device synchronisation is not acceptable, or code that must not allocate
// between the set-up and the end of a run.  xamg_dot_noalloc serves them: it
// computes exactly the same numbers as xamg_dot (same kernels, same reduction
// order, nd = 1..4 pairs), but keeps the partial sums in a fixed array that is
// part of this library's device image.
//
// Limits and sharing rules:
//   * the array holds kScratchDoubles doubles (8 MiB); calls whose partial
//     sums need more (xamg_dot_part_size(n, nd, nv) > kScratchDoubles) are
//     rejected with code 2 before anything runs;
//   * every GPU on which the library is loaded holds these 8 MiB until the
//     process exits;
//   * all calls share the one array: calls that overlap on the GPU (different
//     streams, or different host threads) race on it.  Calls issued to one
//     stream are ordered and safe;
//   * a NULL stream means the library's own stream, as for xamg_dot and every
//     other kernel-level entry point, so NULL calls of both are ordered;
//   * the partial sums are always fully written before they are read, so the
//     array needs no clearing between calls;
//   * the first call in a CUDA context looks up the array's device address
//     (cudaGetSymbolAddress) with that context current and keeps it for that
//     context; make that first call before any stream capture.  A context
//     created after cudaDeviceReset gets its own look-up.
#include <cuda.h>
#include <mutex>
#include <string>
#include "kernels.cuh"

namespace xamg {
void set_last_error(const std::string &msg);
cudaStream_t library_stream();
}

namespace {

constexpr long long kScratchDoubles = 1ll << 20;
__device__ __align__(256) double g_dot_scratch[kScratchDoubles];

// One cached address per CUDA context: the module holding the array is loaded
// once per context, so the address is a property of the context (a device can
// see a new context after cudaDeviceReset, or a driver-API context the caller
// made current).
constexpr int kMaxContexts = 64;
struct Slot {
    CUcontext ctx = nullptr;
    double *ptr = nullptr;
};
Slot g_slots[kMaxContexts];
std::mutex g_setup_mutex;

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

CUcontext current_context(std::string &why) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f) {
            why = "cuCtxGetCurrent is not available";
            return nullptr;
        }
        fn = (CtxGetCurrentFn)f;
    }
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS || !c) {
        why = "no current CUDA context";
        return nullptr;
    }
    return c;
}

// Device address of the scratch array in the current context (set-up once
// per context, with that context current).  Returns nullptr on failure.
double *scratch_for_current_context(std::string &why) {
    CUcontext c = current_context(why);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (c)
        for (Slot &s : g_slots)
            if (s.ctx == c) return s.ptr;
    // first call in this context (or no context bound yet: the look-up binds
    // the runtime's primary context, which is then the one to key on)
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
    if (e != cudaSuccess) {
        why = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (!c) c = current_context(why);
    if (!c) return nullptr;
    for (Slot &s : g_slots)
        if (s.ctx == c) return s.ptr;
    for (Slot &s : g_slots)
        if (!s.ctx) {
            s.ctx = c;
            s.ptr = (double *)p;
            return s.ptr;
        }
    why = "more CUDA contexts than the allocation-free path tracks";
    return nullptr;
}

}  // namespace

extern "C" int xamg_dot_noalloc(int prec, int nv, int64_t n, int nd, const void *const *a,
                                const void *const *b, double *out, void *stream) {
    if ((prec != 0 && prec != 1) || nd < 1 || nd > 4 || n < 0 || !a || !b || !out ||
        !(nv == 1 || nv == 2 || nv == 4 || nv == 8 || nv == 16 || nv == 32)) {
        xamg::set_last_error("xamg_dot_noalloc: bad argument");
        return 2;
    }
    long long need = (long long)xk::dot_part_size(n, nd, nv);
    if (need > kScratchDoubles) {
        xamg::set_last_error("xamg_dot_noalloc: n*nd*nv needs " + std::to_string(need) +
                             " partial sums, more than the fixed " +
                             std::to_string(kScratchDoubles) + " of the allocation-free path");
        return 2;
    }
    std::string why;
    double *part = scratch_for_current_context(why);
    if (!part) {
        xamg::set_last_error("xamg_dot_noalloc: " + why);
        return 3;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : xamg::library_stream();
    xk::dots((xk::Prec)prec, nv, n, nd, a, b, part, out, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        xamg::set_last_error(std::string("xamg_dot_noalloc: ") + cudaGetErrorString(e));
        return 3;
    }
    return 0;
}
