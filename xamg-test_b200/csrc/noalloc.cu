// Inner products without any device allocation.
//
// xamg_dot needs a caller-provided scratch buffer for its per-chunk partial
// sums.  Some callers cannot provide one: code that runs while a host
// framework owns every device allocation (a plug-in handed only its input and
// output buffers), code on a latency-critical path where cudaMalloc's implicit
// device synchronisation is not acceptable, or code that must not allocate
// between the set-up and the end of a run.  xamg_dot_noalloc serves them: it
// computes exactly the same numbers as xamg_dot (same kernels, same reduction
// order), but keeps the partial sums in a fixed array that is part of this
// library's device image.
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
//   * the partial sums are always fully written before they are read, so the
//     array needs no clearing between calls;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
#include <mutex>
#include <string>
#include "kernels.cuh"

namespace xamg {
void set_last_error(const std::string &msg);
}

namespace {

constexpr long long kScratchDoubles = 1ll << 20;
__device__ __align__(256) double g_dot_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// Device address of the scratch array for the current device (set-up once
// per device, with that device current).  Returns nullptr on failure.
double *scratch_for_current_device(std::string &why) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        why = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        why = "device index beyond the supported range";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess) {
            why = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_scratch_ptr[dev] = (double *)p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace

extern "C" int xamg_dot_noalloc(int prec, int nv, int64_t n, int nd, const void *const *a,
                                const void *const *b, double *out, void *stream) {
    if ((prec != 0 && prec != 1) || nd < 1 || nd > 3 || n < 0 || !a || !b || !out ||
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
    double *part = scratch_for_current_device(why);
    if (!part) {
        xamg::set_last_error("xamg_dot_noalloc: " + why);
        return 3;
    }
    xk::dots((xk::Prec)prec, nv, n, nd, a, b, part, out, (cudaStream_t)stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        xamg::set_last_error(std::string("xamg_dot_noalloc: ") + cudaGetErrorString(e));
        return 3;
    }
    return 0;
}
