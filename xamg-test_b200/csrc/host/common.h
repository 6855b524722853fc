// Shared host-side types of the XAMG B200 solve phase.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../kernels.cuh"

namespace xamg {

typedef int64_t i64;
using xk::Prec;

// Error reporting: host code throws xamg::Error; the C ABI catches it, stores
// the message (XAMG_b200_last_error) and returns a non-zero code instead of
// aborting a shared-GPU job.
struct Error : std::runtime_error {
    int code;
    Error(const std::string &m, int c = 1) : std::runtime_error(m), code(c) {}
};

#define XCUDA(call)                                                                               \
    do {                                                                                          \
        cudaError_t _e = (call);                                                                  \
        if (_e != cudaSuccess)                                                                    \
            throw ::xamg::Error(std::string("CUDA: ") + cudaGetErrorString(_e) + " at " +         \
                                    __FILE__ + ":" + std::to_string(__LINE__),                    \
                                3);                                                               \
    } while (0)

#define XCHECK(cond, msg)                                                                         \
    do {                                                                                          \
        if (!(cond)) throw ::xamg::Error(msg, 2);                                                 \
    } while (0)

inline size_t prec_size(Prec p) { return p == Prec::F64 ? 8 : 4; }

// Owning device allocation.
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DBuf() {}
    explicit DBuf(size_t b) { alloc(b); }
    void alloc(size_t b) {
        release();
        if (b) XCUDA(cudaMalloc(&p, b));
        bytes = b;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    ~DBuf() { release(); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    template <class T> T *as() const { return (T *)p; }
};

// Host CSR (setup side, FP64 values, int32 indices).
struct HostCsr {
    i64 n = 0, ncols = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
    i64 nnz() const { return rp.empty() ? 0 : rp[n]; }
};

// Process-wide execution context: one stream per library instance.
struct Context {
    cudaStream_t stream = nullptr;
    int device = 0;
    bool inited = false;
    void init() {
        if (inited) return;
        XCUDA(cudaGetDevice(&device));
        XCUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        inited = true;
    }
};
Context &ctx();

// Optional CUDA-event timing of the hot kernels inside solves (off unless
// enabled through XAMG_b200_kernel_timing).  A record is one launch: its
// kernel class, the rows of its operator, its algorithmic bytes and the
// event pair around it on the launching stream.  The level-ordered
// Gauss-Seidel sweep is recorded by its form: cooperative grid, hybrid blocks
// (one CTA per block) with the x tile in shared memory, with the slot window,
// or gathering x per level, and the same three forms with one warp per block
// (GS covers the other sweep paths).
enum class KClass : int {
    GS = 0, SPMV = 1, GS_GRID = 2, GS_TILE = 3, GS_WINDOW = 4, GS_GATHER = 5,
    GSW_TILE = 6, GSW_WINDOW = 7, GSW_GATHER = 8
};
bool ktime_on();
struct KTimeScope {
    bool on;
    int slot = -1;
    KTimeScope(KClass k, i64 rows, double bytes, cudaStream_t s);
    ~KTimeScope();
    cudaStream_t s;
};

}  // namespace xamg
