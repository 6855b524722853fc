// XAMG solve-phase kernels for sm_100a.  See kernels.cuh for the contract.
//
// Design notes (B200):
//  * All kernels here are HBM-bound; they are written for coalesced 16-byte
//    accesses: a CSR row is served by TPR = NV*sizeof(T)/16 threads, each
//    owning 16 contiguous bytes of the NV-wide x/y rows, so a warp reads whole
//    128-byte lines of x and writes whole lines of y.
//  * Matrix entries are read once per product and are streamed with evict-first
//    loads (__ldcs) so that the x block vector, which is re-read ~nnz/N times
//    through the 126 MB L2, keeps its lines resident.
//  * Row sums keep the stored CSR order (a sequential fma chain per (row,col)),
//    which makes the result independent of the launch shape and bit-identical
//    to the oracle.
#include "kernels.cuh"
#include <cooperative_groups.h>
#include <atomic>
#include <algorithm>
#include <cstdio>

namespace xk {

// ------------------------------------------------------------- vector access
template <class T, int V> struct VT;
template <> struct VT<double, 1> { typedef double type; };
template <> struct VT<double, 2> { typedef double2 type; };
template <> struct VT<float, 1> { typedef float type; };
template <> struct VT<float, 2> { typedef float2 type; };
template <> struct VT<float, 4> { typedef float4 type; };

template <class T, int NV> struct Shape {
    static constexpr int V = (NV * (int)sizeof(T) >= 16) ? 16 / (int)sizeof(T) : NV;
    static constexpr int TPR = NV / V;  // threads per row
};

template <class T, int V>
__device__ __forceinline__ void ld(const T *p, T (&r)[V]) {
    typedef typename VT<T, V>::type W;
    W w = __ldg(reinterpret_cast<const W *>(p));
    memcpy(r, &w, sizeof(W));
}
template <class T, int V>
__device__ __forceinline__ void ld_cg(const T *p, T (&r)[V]) {
    typedef typename VT<T, V>::type W;
    W w = __ldcg(reinterpret_cast<const W *>(p));
    memcpy(r, &w, sizeof(W));
}
template <class T, int V>
__device__ __forceinline__ void st(T *p, const T (&r)[V]) {
    typedef typename VT<T, V>::type W;
    W w;
    memcpy(&w, r, sizeof(W));
    *reinterpret_cast<W *>(p) = w;
}
template <class T, int V>
__device__ __forceinline__ void st_cg(T *p, const T (&r)[V]) {
    typedef typename VT<T, V>::type W;
    W w;
    memcpy(&w, r, sizeof(W));
    __stcg(reinterpret_cast<W *>(p), w);
}

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
template <class T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return dmul(a, b); }
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return fmul(a, b); }
template <class T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn<double>(double a, double b) { return dadd(a, b); }
template <> __device__ __forceinline__ float add_rn<float>(float a, float b) { return fadd(a, b); }

#define NV_DISPATCH(nv, FN)                                                                       \
    switch (nv) {                                                                                  \
    case 1: FN(1); break;                                                                          \
    case 2: FN(2); break;                                                                          \
    case 4: FN(4); break;                                                                          \
    case 8: FN(8); break;                                                                          \
    case 16: FN(16); break;                                                                        \
    case 32: FN(32); break;                                                                        \
    default: fprintf(stderr, "xamg: unsupported nv=%d\n", nv); break;                              \
    }

// ---------------------------------------------------------------- SpMV
// mode 0: y = A x; mode 1: y += A x; mode 2: y = 1*b + (-1)*(A x)
// GB entries of a row are fetched per batch (column indices and values first,
// then all GB x gathers), so a row costs about nnz_row/GB dependent memory
// round trips; the accumulation order is the stored order for every GB.
template <class T, int NV, int MODE, int GB>
__global__ void __launch_bounds__(256) k_spmv(i64 n, const int *__restrict__ rp,
                                              const int *__restrict__ ci,
                                              const T *__restrict__ va, const T *__restrict__ x,
                                              T *__restrict__ y, const T *__restrict__ b) {
    constexpr int V = Shape<T, NV>::V, TPR = Shape<T, NV>::TPR, RPB = 256 / TPR;
    i64 row = (i64)blockIdx.x * RPB + threadIdx.x / TPR;
    int lane = threadIdx.x % TPR;
    if (row >= n) return;
    T acc[V];
    if (MODE == 1) {
        ld<T, V>(y + row * NV + lane * V, acc);
    } else {
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] = T(0);
    }
    const int j0 = __ldg(rp + row), j1 = __ldg(rp + row + 1);
    const T *xb = x + lane * V;
    for (int j = j0; j < j1; j += GB) {
        int c[GB];
        T v[GB];
#pragma unroll
        for (int k = 0; k < GB; ++k) {
            const bool in = j + k < j1;
            c[k] = in ? __ldcs(ci + j + k) : 0;
            v[k] = in ? __ldcs(va + j + k) : T(0);
        }
        T xv[GB][V];
#pragma unroll
        for (int k = 0; k < GB; ++k)
            if (j + k < j1) ld<T, V>(xb + (i64)c[k] * NV, xv[k]);
#pragma unroll
        for (int k = 0; k < GB; ++k)
            if (j + k < j1) {
#pragma unroll
                for (int e = 0; e < V; ++e) acc[e] = fma(v[k], xv[k][e], acc[e]);
            }
    }
    if (MODE == 2) {
        T bb[V];
        ld<T, V>(b + row * NV + lane * V, bb);
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] = add_rn<T>(mul_rn<T>(T(1), bb[e]), mul_rn<T>(T(-1), acc[e]));
    }
    st<T, V>(y + row * NV + lane * V, acc);
}

// Streaming variant: a tile of RPB rows has its CSR entries copied into shared
// memory with coalesced loads (when they fit), then every row is summed from
// shared memory with its x gathers issued GB at a time.  Each CTA walks `tpc`
// consecutive tiles, so the x rows of the stencil neighbourhood stay in L1
// between tiles.  Same per-row summation order as k_spmv.
template <class T, int NV, int MODE>
__global__ void __launch_bounds__(256) k_spmv_stream(i64 n, int tpc, const int *__restrict__ rp,
                                                     const int *__restrict__ ci,
                                                     const T *__restrict__ va,
                                                     const T *__restrict__ x, T *__restrict__ y,
                                                     const T *__restrict__ b) {
    constexpr int V = Shape<T, NV>::V, TPR = Shape<T, NV>::TPR, RPB = 256 / TPR, GB = 8;
    constexpr int EMAX = sizeof(T) == 8 ? 2048 : 3072;
    __shared__ int s_c[EMAX];
    __shared__ T s_v[EMAX];
    const int lane = threadIdx.x % TPR;
    const i64 ntiles = (n + RPB - 1) / RPB;
    for (i64 tile = (i64)blockIdx.x * tpc, te = min(ntiles, tile + tpc); tile < te; ++tile) {
        const i64 r0 = tile * RPB, r1 = min(n, r0 + RPB);
        const int e0 = __ldg(rp + r0), cnt = __ldg(rp + r1) - e0;
        const bool staged = cnt <= EMAX;
        if (staged) {
            for (int q = threadIdx.x; q < cnt; q += 256) {
                s_c[q] = __ldcs(ci + e0 + q);
                s_v[q] = __ldcs(va + e0 + q);
            }
            __syncthreads();
        }
        const i64 row = r0 + threadIdx.x / TPR;
        if (row < r1) {
            T acc[V];
            if (MODE == 1) {
                ld<T, V>(y + row * NV + lane * V, acc);
            } else {
#pragma unroll
                for (int e = 0; e < V; ++e) acc[e] = T(0);
            }
            const int j0 = __ldg(rp + row), j1 = __ldg(rp + row + 1);
            const T *xb = x + lane * V;
            for (int j = j0; j < j1; j += GB) {
                int c[GB];
                T v[GB];
#pragma unroll
                for (int k = 0; k < GB; ++k) {
                    bool ok = j + k < j1;
                    c[k] = ok ? (staged ? s_c[j + k - e0] : __ldcs(ci + j + k)) : 0;
                    v[k] = ok ? (staged ? s_v[j + k - e0] : __ldcs(va + j + k)) : T(0);
                }
                T xv[GB][V];
#pragma unroll
                for (int k = 0; k < GB; ++k)
                    if (j + k < j1) ld<T, V>(xb + (i64)c[k] * NV, xv[k]);
#pragma unroll
                for (int k = 0; k < GB; ++k)
                    if (j + k < j1) {
#pragma unroll
                        for (int e = 0; e < V; ++e) acc[e] = fma(v[k], xv[k][e], acc[e]);
                    }
            }
            if (MODE == 2) {
                T bb[V];
                ld<T, V>(b + row * NV + lane * V, bb);
#pragma unroll
                for (int e = 0; e < V; ++e) acc[e] = add_rn<T>(mul_rn<T>(T(1), bb[e]), mul_rn<T>(T(-1), acc[e]));
            }
            st<T, V>(y + row * NV + lane * V, acc);
        }
        if (staged) __syncthreads();
    }
}

// Row sum over entries [j0, j1) read at cidx/vals[j - off] (shared memory
// when SMEM, global with the streaming hint otherwise).  LOOP 0: the entries
// are fetched GB at a time into register arrays, then the GB gathers, then
// the GB FMAs; LOOP 1: a plain loop over the entries unrolled GB times (the
// compiler hoists the unrolled gathers ahead of the FMA chain).
template <class T, int NV, int V, int GB, int LOOP, bool SMEM>
__device__ __forceinline__ void tile_row_sum(int j0, int j1, int off, const int *cidx,
                                             const T *vals, const T *xb, T (&acc)[V]) {
    if (LOOP == 1 && SMEM) {
        const int *cr = cidx + (j0 - off);
        const T *vr = vals + (j0 - off);
        const int m = j1 - j0;
#pragma unroll GB
        for (int k = 0; k < m; ++k) {
            T xv[V];
            ld<T, V>(xb + (i64)cr[k] * NV, xv);
            const T a = vr[k];
#pragma unroll
            for (int e = 0; e < V; ++e) acc[e] = fma(a, xv[e], acc[e]);
        }
        return;
    }
    constexpr int GBB = LOOP == 1 ? 2 : GB;  // batch of the global-memory fallback
    for (int j = j0; j < j1; j += GBB) {
        int c[GBB];
        T v[GBB];
#pragma unroll
        for (int k = 0; k < GBB; ++k) {
            const bool in = j + k < j1;
            if (SMEM) {
                c[k] = in ? cidx[j + k - off] : 0;
                v[k] = in ? vals[j + k - off] : T(0);
            } else {
                c[k] = in ? __ldcs(cidx + j + k) : 0;
                v[k] = in ? __ldcs(vals + j + k) : T(0);
            }
        }
        T xv[GBB][V];
#pragma unroll
        for (int k = 0; k < GBB; ++k)
            if (j + k < j1) ld<T, V>(xb + (i64)c[k] * NV, xv[k]);
#pragma unroll
        for (int k = 0; k < GBB; ++k)
            if (j + k < j1) {
#pragma unroll
                for (int e = 0; e < V; ++e) acc[e] = fma(v[k], xv[k][e], acc[e]);
            }
    }
}

// Tile-staged variant: the CSR entries of a tile of RPB rows are copied into
// shared memory with coalesced streaming loads, so the per-entry column index
// and value reads of the row sums are shared-memory broadcasts (one wavefront
// serves every row of a warp) and L1 carries only the x gathers.  Tiles with
// more than EMAX entries read their entries from global memory.  Same
// per-row summation order as k_spmv.
template <class T, int NV, int MODE, int GB, int LOOP>
__global__ void __launch_bounds__(256, LOOP == 1 ? 6 : 1) k_spmv_tile(i64 n, const int *__restrict__ rp,
                                                   const int *__restrict__ ci,
                                                   const T *__restrict__ va,
                                                   const T *__restrict__ x, T *__restrict__ y,
                                                   const T *__restrict__ b) {
    constexpr int V = Shape<T, NV>::V, TPR = Shape<T, NV>::TPR, RPB = 256 / TPR;
    constexpr int EMAX = RPB * 32 < 2048 ? RPB * 32 : 2048;
    __shared__ int s_c[EMAX];
    __shared__ T s_v[EMAX];
    const i64 r0 = (i64)blockIdx.x * RPB, r1 = min(n, r0 + RPB);
    const int e0 = __ldg(rp + r0), cnt = __ldg(rp + r1) - e0;
    const bool staged = cnt <= EMAX;
    if (staged)
        for (int q = threadIdx.x; q < cnt; q += 256) {
            s_c[q] = __ldcs(ci + e0 + q);
            s_v[q] = __ldcs(va + e0 + q);
        }
    const i64 row = r0 + threadIdx.x / TPR;
    const int lane = threadIdx.x % TPR;
    const bool live = row < r1;
    int j0 = 0, j1 = 0;
    T acc[V];
#pragma unroll
    for (int e = 0; e < V; ++e) acc[e] = T(0);
    if (live) {
        j0 = __ldg(rp + row);
        j1 = __ldg(rp + row + 1);
        if (MODE == 1) ld<T, V>(y + row * NV + lane * V, acc);
    }
    __syncthreads();
    if (!live) return;
    const T *xb = x + lane * V;
    if (staged) tile_row_sum<T, NV, V, GB, LOOP, true>(j0, j1, e0, s_c, s_v, xb, acc);
    else tile_row_sum<T, NV, V, GB, LOOP, false>(j0, j1, 0, ci, va, xb, acc);
    if (MODE == 2) {
        T bb[V];
        ld<T, V>(b + row * NV + lane * V, bb);
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] = add_rn<T>(mul_rn<T>(T(1), bb[e]), mul_rn<T>(T(-1), acc[e]));
    }
    st<T, V>(y + row * NV + lane * V, acc);
}

// SpMV variant selection: 0, 1, 2 = row kernel with gather batches of 4, 8,
// 16 entries; 3, 4 = tile-staged kernel with batches of 4, 8; 5, 6 = the same
// with a plain row loop unrolled 4, 8 times; 10 + k = streaming kernel
// walking k tiles per CTA; -1 = default (6 when NV*sizeof(T) >= 64 bytes,
// else 0).
static thread_local int g_spmv_variant = -1;
void set_spmv_variant(int v) { g_spmv_variant = v; }
static int g_run_rows = 8;
void set_spmv_run_rows(int r) { g_run_rows = r == 8 ? 8 : 0; }
int get_spmv_run_rows() { return g_run_rows; }

// kernels launched by this library (all launchers count here)
static std::atomic<long long> g_launches{0};
void note_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
int get_spmv_variant() { return g_spmv_variant; }

static int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

template <class T, int NV>
static void spmv_t(i64 n, const int *rp, const int *ci, const T *va, const T *x, T *y, int mode,
                   const T *b, cudaStream_t s, int choice) {
    constexpr int RPB = 256 / Shape<T, NV>::TPR;
    if (n <= 0) return;
    note_launch();
    i64 ntiles = (n + RPB - 1) / RPB;
    // default: the tile-staged kernel when a row spans at least 4 threads (its
    // tile of RPB rows then fits the shared-memory stage), else batches of 4
    const int want = choice >= 0 ? choice : g_spmv_variant;
    int var = (want >= 0 && want != 7) ? want : (Shape<T, NV>::TPR >= 4 ? 6 : 0);
    if (var >= 3 && var <= 6) {
        unsigned g = (unsigned)ntiles;
#define L(GB, LOOP)                                                                                \
    if (mode == 0) k_spmv_tile<T, NV, 0, GB, LOOP><<<g, 256, 0, s>>>(n, rp, ci, va, x, y, b);      \
    else if (mode == 1) k_spmv_tile<T, NV, 1, GB, LOOP><<<g, 256, 0, s>>>(n, rp, ci, va, x, y, b); \
    else k_spmv_tile<T, NV, 2, GB, LOOP><<<g, 256, 0, s>>>(n, rp, ci, va, x, y, b);
        if (var == 3) { L(4, 0) } else if (var == 4) { L(8, 0) } else if (var == 5) { L(4, 1) } else { L(8, 1) }
#undef L
        return;
    }
    if (var < 10) {
        unsigned g = (unsigned)ntiles;
#define L(GB)                                                                                      \
    if (mode == 0) k_spmv<T, NV, 0, GB><<<g, 256, 0, s>>>(n, rp, ci, va, x, y, b);                \
    else if (mode == 1) k_spmv<T, NV, 1, GB><<<g, 256, 0, s>>>(n, rp, ci, va, x, y, b);           \
    else k_spmv<T, NV, 2, GB><<<g, 256, 0, s>>>(n, rp, ci, va, x, y, b);
        if (var == 0) { L(4) } else if (var == 2) { L(16) } else { L(8) }
#undef L
        return;
    }
    int tpc = var - 10 > 0 ? var - 10 : (int)std::max<i64>(1, ntiles / ((i64)sm_count() * 8));
    unsigned g = (unsigned)((ntiles + tpc - 1) / tpc);
    if (mode == 0) k_spmv_stream<T, NV, 0><<<g, 256, 0, s>>>(n, tpc, rp, ci, va, x, y, b);
    else if (mode == 1) k_spmv_stream<T, NV, 1><<<g, 256, 0, s>>>(n, tpc, rp, ci, va, x, y, b);
    else k_spmv_stream<T, NV, 2><<<g, 256, 0, s>>>(n, tpc, rp, ci, va, x, y, b);
}

void spmv(Prec p, int nv, i64 n, const int *rp, const int *ci, const void *val, const void *x,
          void *y, int mode, const void *b, cudaStream_t s, int variant) {
    if (p == Prec::F64) {
#define F(NV) spmv_t<double, NV>(n, rp, ci, (const double *)val, (const double *)x, (double *)y, mode, (const double *)b, s, variant)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) spmv_t<float, NV>(n, rp, ci, (const float *)val, (const float *)x, (float *)y, mode, (const float *)b, s, variant)
        NV_DISPATCH(nv, F)
#undef F
    }
}

// ---------------------------------------------------------------- shifted-row runs
// A chunk is up to R = 8 consecutive rows r0 .. r0+cnt-1 with the same entry
// count m whose column indices are those of row r0 shifted by the row offset,
// ci(r0+q, e) = ci(r0, e) + q (the interior rows of a stencil operator).  The
// first row's column list is cut into segments of at most 3 consecutive
// columns, stored as c0 | len << 30; row q's entry j of a segment has column
// c0 + q + j, so the chunk's rows gather the len + cnt - 1 x rows c0 ..
// c0+len+cnt-2 once, into registers, instead of len * cnt times.  TPR threads
// (NV/TPR elements each) evaluate one chunk.  Chunks are grouped four
// to a tile; tile t stores its segments segment-major, sg[toff[t].y + 4s +
// slot], and its values entry-major, vt[(toff[t].x + 4e + slot) * R + q], so
// the loads of one entry by the chunks of a warp fall in one or two 128-byte
// lines.  A CTA of 128 threads first copies the segments and values of its
// chunks (one contiguous range of each) into shared memory with 16-byte
// cp.async; five CTAs share an SM (96 registers a thread), so one CTA's copy
// overlaps the others' gathers.  Each
// row's FMA chain runs over its entries in CSR order starting from 0 (or y),
// the order of every other SpMV kernel here.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <class T, int R, bool SMEM>
__device__ __forceinline__ void ld_vals(const T *p, T (&a)[R]) {
    constexpr int PER = 16 / (int)sizeof(T), NB = R / PER;
    typedef typename VT<T, PER>::type W;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        W w = SMEM ? reinterpret_cast<const W *>(p)[k] : __ldcs(reinterpret_cast<const W *>(p) + k);
        memcpy(a + k * PER, &w, sizeof(W));
    }
}

constexpr int RUN_ROWS = 8, RUN_SEG = 3;
// chunks per CTA of NT threads and the value slots a CTA can stage (32
// entries per chunk on average)
template <class T, int NV, int NT> struct RunShape {
    static constexpr int TPR = Shape<T, NV>::TPR, CPC = NT / TPR, TPC = CPC / 4, SLOTS = TPC * 128;
    static constexpr int SMEM_BYTES = SLOTS * (4 + RUN_ROWS * (int)sizeof(T));
};

// STX: the x rows of each segment are copied by cp.async into this thread's
// own slice of a two-segment shared-memory buffer (xs, NX pieces of 16 bytes
// per segment and thread, strided by the CTA's thread count), one segment
// ahead of their use, instead of being held in registers: fewer registers a
// thread and two segments of gathers in flight.  Same FMA chains.
template <class T, int NV, int MODE, bool SMEM, bool STX = false, int NT = 128>
__device__ __forceinline__ void run_rows(const int4 cd, int smax, const int *sg, const T *val, const T *xb,
                                         T *__restrict__ y, const T *__restrict__ b, int l, T *xs = nullptr) {
    constexpr int V = Shape<T, NV>::V, R = RUN_ROWS, NX = RUN_SEG + R - 1;
    T acc[R][V];
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) acc[q][v] = T(0);
    if (MODE == 1) {
#pragma unroll
        for (int q = 0; q < R; ++q)
            if (q < cd.y) ld<T, V>(y + ((i64)cd.x + q) * NV + l * V, acc[q]);
    }
    auto seg = [&](int s) { return s < cd.w ? (SMEM ? sg[4 * s] : __ldcs(sg + 4 * s)) : 0; };
    int e = 0;
    int sc = seg(0);
    if constexpr (STX) {
        // xs slice of this thread: piece k of buffer u at xs[((u * NX + k) * NT + tid) * V]
        const int tid = threadIdx.x;
        auto issue = [&](int scv, int u) {
            const int c0 = scv & 0x3fffffff, len = (int)((unsigned)scv >> 30);
            const int nx = len + cd.y - 1;
#pragma unroll
            for (int k = 0; k < NX; ++k)
                if (k < nx && len > 0)
                    cp_async16(xs + ((i64)(u * NX + k) * NT + tid) * V, xb + ((i64)c0 + k) * NV);
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        issue(sc, 0);
        for (int s = 0; s < smax; ++s) {
            const int c0 = sc & 0x3fffffff, len = (int)((unsigned)sc >> 30);
            (void)c0;
            const int scn = seg(s + 1);
            issue(s + 1 < smax ? scn : 0, (s + 1) & 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
            const T *xu = xs + (i64)((s & 1) * NX) * NT * V + (i64)tid * V;
#pragma unroll
            for (int j = 0; j < RUN_SEG; ++j) {
                if (j < len) {
                    T a[R];
                    ld_vals<T, R, SMEM>(val + (i64)4 * (e + j) * R, a);
#pragma unroll
                    for (int q = 0; q < R; ++q) {
                        // a shared-memory read (not the read-only global path)
                        typedef typename VT<T, V>::type W;
                        const W xw = *reinterpret_cast<const W *>(xu + (i64)(q + j) * NT * V);
                        T X[V];
                        memcpy(X, &xw, sizeof(W));
#pragma unroll
                        for (int v = 0; v < V; ++v) acc[q][v] = fma(a[q], X[v], acc[q][v]);
                    }
                }
            }
            e += len;
            sc = scn;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else {
    for (int s = 0; s < smax; ++s) {
        const int c0 = sc & 0x3fffffff, len = (int)((unsigned)sc >> 30);
        const int nx = len + cd.y - 1;
        T X[NX][V];
#pragma unroll
        for (int k = 0; k < NX; ++k)
            if (k < nx) ld<T, V>(xb + ((i64)c0 + k) * NV, X[k]);
        sc = seg(s + 1);
#pragma unroll
        for (int j = 0; j < RUN_SEG; ++j) {
            if (j < len) {
                T a[R];
                ld_vals<T, R, SMEM>(val + (i64)4 * (e + j) * R, a);
#pragma unroll
                for (int q = 0; q < R; ++q)
#pragma unroll
                    for (int v = 0; v < V; ++v) acc[q][v] = fma(a[q], X[q + j][v], acc[q][v]);
            }
        }
        e += len;
    }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
        if (q >= cd.y) break;
        const i64 row = (i64)cd.x + q;
        if (MODE == 2) {
            T bb[V];
            ld<T, V>(b + row * NV + l * V, bb);
#pragma unroll
            for (int v = 0; v < V; ++v)
                acc[q][v] = add_rn<T>(mul_rn<T>(T(1), bb[v]), mul_rn<T>(T(-1), acc[q][v]));
        }
        st<T, V>(y + row * NV + l * V, acc[q]);
    }
}

constexpr int RUN_NT = 128;
// x staging buffer of the STX form: two segments of NX 16-byte pieces a thread
template <int NT> struct RunXs {
    static constexpr int BYTES = 2 * (RUN_SEG + RUN_ROWS - 1) * NT * 16;
};
template <class T, int NV, int MODE, int NT, bool STX = false>
__global__ void __launch_bounds__(NT, STX ? 3 : 5) k_spmv_runs(i64 nchunks, i64 ntiles, const int4 *__restrict__ chunks,
                                                      const longlong2 *__restrict__ toff,
                                                      const int *__restrict__ sg,
                                                      const T *__restrict__ vt,
                                                      const T *__restrict__ x, T *__restrict__ y,
                                                      const T *__restrict__ b) {
    typedef RunShape<T, NV, NT> RS;
    constexpr int V = Shape<T, NV>::V, TPR = RS::TPR, CPC = RS::CPC, TPC = RS::TPC, SLOTS = RS::SLOTS;
    static_assert(TPR >= 4 && (RUN_ROWS * (int)sizeof(T)) % 16 == 0, "run kernel shape");
    extern __shared__ __align__(16) unsigned char run_smem[];
    int *s_sg = reinterpret_cast<int *>(run_smem);
    T *s_vt = reinterpret_cast<T *>(run_smem + SLOTS * 4);
    const i64 t0 = (i64)blockIdx.x * TPC, t1 = min(ntiles, t0 + TPC);
    const longlong2 o0 = __ldg(toff + t0), o1 = __ldg(toff + t1);
    const i64 ne = o1.x - o0.x, nsg = o1.y - o0.y;
    const bool staged = ne <= SLOTS;  // segments never outnumber entries
    if (staged) {
        const int np = (int)(nsg / 4), nvb = (int)(ne * RUN_ROWS * (int)sizeof(T) / 16);
        for (int k = threadIdx.x; k < np; k += NT) cp_async16(s_sg + 4 * k, sg + o0.y + 4 * k);
        const char *gv = reinterpret_cast<const char *>(vt + o0.x * RUN_ROWS);
        for (int k = threadIdx.x; k < nvb; k += NT)
            cp_async16(reinterpret_cast<char *>(s_vt) + 16 * k, gv + 16 * k);
        cp_async_wait_all();
    }
    __syncthreads();
    const i64 gid = (i64)blockIdx.x * CPC + threadIdx.x / TPR;
    const int l = threadIdx.x % TPR;
    const bool live = gid < nchunks;
    const int4 cd = live ? __ldg(chunks + gid) : make_int4(0, 0, 0, 0);  // r0, cnt, m, segments
    const int smax = __reduce_max_sync(0xffffffffu, cd.w);
    const longlong2 ot = live ? __ldg(toff + (gid >> 2)) : o0;
    const int slot = (int)(gid & 3);
    const i64 le = ot.x - o0.x + slot, ls = ot.y - o0.y + slot;  // CTA-local first value / segment slot
    const T *xb = x + l * V;
    T *xs = reinterpret_cast<T *>(run_smem + RunShape<T, NV, NT>::SMEM_BYTES);
    if (staged)
        run_rows<T, NV, MODE, true, STX, NT>(cd, smax, s_sg + ls, s_vt + le * RUN_ROWS, xb, y, b, l, xs);
    else
        run_rows<T, NV, MODE, false, STX, NT>(cd, smax, sg + o0.y + ls, vt + (o0.x + le) * RUN_ROWS, xb, y, b, l,
                                             xs);
}

// kernel form of the run product: 0 = x rows in registers, 1 = x rows staged
// in shared memory one segment ahead (per host thread; same results).  A
// register budget of 6 or 8 CTAs per SM for form 0 spills the gathered rows
// and runs 2-4x slower (measured), so it is not offered.
static thread_local int g_run_form = 0;
void set_spmv_run_form(int f) { g_run_form = f ? 1 : 0; }
int get_spmv_run_form() { return g_run_form; }

bool spmv_runs_supported(Prec p, int nv) {
    return p == Prec::F64 ? (nv == 8 || nv == 16 || nv == 32) : (nv == 16 || nv == 32);
}

template <class T, int NV, int NT, bool STX>
static void spmv_runs_p(i64 nchunks, i64 ntiles, const int4 *chunks, const longlong2 *toff, const int *sg,
                        const T *vt, const T *x, T *y, int mode, const T *b, cudaStream_t s) {
    typedef RunShape<T, NV, NT> RS;
    constexpr int SM = RS::SMEM_BYTES + (STX ? RunXs<NT>::BYTES : 0);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_spmv_runs<T, NV, 0, NT, STX>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
        cudaFuncSetAttribute(k_spmv_runs<T, NV, 1, NT, STX>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
        cudaFuncSetAttribute(k_spmv_runs<T, NV, 2, NT, STX>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
        attr = true;
    }
    unsigned g = (unsigned)((ntiles + RS::TPC - 1) / RS::TPC);
    if (mode == 0)
        k_spmv_runs<T, NV, 0, NT, STX><<<g, NT, SM, s>>>(nchunks, ntiles, chunks, toff, sg, vt, x, y, b);
    else if (mode == 1)
        k_spmv_runs<T, NV, 1, NT, STX><<<g, NT, SM, s>>>(nchunks, ntiles, chunks, toff, sg, vt, x, y, b);
    else
        k_spmv_runs<T, NV, 2, NT, STX><<<g, NT, SM, s>>>(nchunks, ntiles, chunks, toff, sg, vt, x, y, b);
}

template <class T, int NV>
static void spmv_runs_t(i64 nchunks, i64 ntiles, const int4 *chunks, const longlong2 *toff, const int *sg,
                        const T *vt, const T *x, T *y, int mode, const T *b, cudaStream_t s) {
    if constexpr (NV >= 8 && NV * sizeof(T) >= 64) {
        if (nchunks <= 0) return;
        note_launch();
        if (g_run_form) spmv_runs_p<T, NV, RUN_NT, true>(nchunks, ntiles, chunks, toff, sg, vt, x, y, mode, b, s);
        else spmv_runs_p<T, NV, RUN_NT, false>(nchunks, ntiles, chunks, toff, sg, vt, x, y, mode, b, s);
    }
}

void spmv_runs(Prec p, int nv, i64 nchunks, i64 ntiles, const int4 *chunks, const longlong2 *toff, const int *sg,
               const void *vt, const void *x, void *y, int mode, const void *b, cudaStream_t s) {
    if (p == Prec::F64) {
#define F(NV) spmv_runs_t<double, NV>(nchunks, ntiles, chunks, toff, sg, (const double *)vt, (const double *)x, (double *)y, mode, (const double *)b, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) spmv_runs_t<float, NV>(nchunks, ntiles, chunks, toff, sg, (const float *)vt, (const float *)x, (float *)y, mode, (const float *)b, s)
        NV_DISPATCH(nv, F)
#undef F
    }
}

// ---------------------------------------------------------------- Gauss-Seidel
// One Gauss-Seidel row update (csr_gs.inl:77-99): sum = t_i - sum_j a_ij x_j
// in CSR order, x_i += relax*invdiag_i*sum.  The row's column indices and
// values are fetched GB entries at a time and the x gathers of a batch are
// issued together, so a level costs a few memory round trips instead of one
// per entry; the fma chain itself keeps the stored order.  CG selects L2-only
// access to x for sweeps whose rows are shared between CTAs.
template <class T, int NV, bool CG>
__device__ __forceinline__ void gs_row(i64 row, int lane, const int *__restrict__ rp,
                                       const int *__restrict__ ci, const T *__restrict__ va,
                                       const T *__restrict__ invd, const T *__restrict__ t, T *x,
                                       const T *__restrict__ relax, i64 brows) {
    constexpr int V = Shape<T, NV>::V, GB = 8;
    T sum[V], xo[V];
    if (CG) {
        ld_cg<T, V>(t + row * NV + lane * V, sum);
        ld_cg<T, V>(x + row * NV + lane * V, xo);
    } else {
        ld<T, V>(t + row * NV + lane * V, sum);
        typedef typename VT<T, V>::type W;
        W w = *reinterpret_cast<const W *>(x + row * NV + lane * V);
        memcpy(xo, &w, sizeof(W));
    }
    const T di = __ldg(invd + row);
    const int j0 = __ldg(rp + row), j1 = __ldg(rp + row + 1);
    i64 lo = 0, hi = INT64_MAX;
    if (brows > 0) { lo = (row / brows) * brows; hi = lo + brows; }
    for (int j = j0; j < j1; j += GB) {
        int c[GB];
        T v[GB];
#pragma unroll
        for (int k = 0; k < GB; ++k) {
            bool ok = j + k < j1;
            c[k] = ok ? __ldg(ci + j + k) : -1;
            v[k] = ok ? -__ldg(va + j + k) : T(0);
        }
        T xv[GB][V];
#pragma unroll
        for (int k = 0; k < GB; ++k) {
            if (c[k] >= lo && c[k] < hi) {
                if (CG) {
                    ld_cg<T, V>(x + (i64)c[k] * NV + lane * V, xv[k]);
                } else {
                    typedef typename VT<T, V>::type W;
                    W w = *reinterpret_cast<const W *>(x + (i64)c[k] * NV + lane * V);
                    memcpy(xv[k], &w, sizeof(W));
                }
            }
        }
#pragma unroll
        for (int k = 0; k < GB; ++k)
            if (c[k] >= lo && c[k] < hi) {
#pragma unroll
                for (int e = 0; e < V; ++e) sum[e] = fma(v[k], xv[k][e], sum[e]);
            }
    }
#pragma unroll
    for (int e = 0; e < V; ++e) {
        T cf = mul_rn<T>(__ldg(relax + lane * V + e), di);
        xo[e] = fma(cf, sum[e], xo[e]);
    }
    if (CG) {
        st_cg<T, V>(x + row * NV + lane * V, xo);
    } else {
        st<T, V>(x + row * NV + lane * V, xo);
    }
}

// Hybrid Gauss-Seidel, one CTA per block of `brows` rows: the forward then the
// backward sweep of the block run level by level with CTA barriers only (the
// blocks are independent by construction, blas2.h:225-263).  Block b owns the
// level range [blev[b], blev[b+1]) of lptr; level l covers perm[lptr[l]..lptr[l+1]).
template <class T, int NV>
__global__ void __launch_bounds__(256) k_gs_blocks(const int *__restrict__ blevf,
                                                   const int *__restrict__ lptrf,
                                                   const int *__restrict__ permf,
                                                   const int *__restrict__ blevb,
                                                   const int *__restrict__ lptrb,
                                                   const int *__restrict__ permb,
                                                   const int *__restrict__ rp,
                                                   const int *__restrict__ ci,
                                                   const T *__restrict__ va,
                                                   const T *__restrict__ invd,
                                                   const T *__restrict__ t, T *x,
                                                   const T *__restrict__ relax, i64 brows) {
    constexpr int TPR = Shape<T, NV>::TPR;
    const int b = blockIdx.x;
    for (int pass = 0; pass < 2; ++pass) {
        const int *blev = pass ? blevb : blevf;
        const int *lptr = pass ? lptrb : lptrf;
        const int *perm = pass ? permb : permf;
        for (int l = __ldg(blev + b), le = __ldg(blev + b + 1); l < le; ++l) {
            int lo = __ldg(lptr + l), items = (__ldg(lptr + l + 1) - lo) * TPR;
            for (int it = threadIdx.x; it < items; it += 256)
                gs_row<T, NV, false>(__ldg(perm + lo + it / TPR), it % TPR, rp, ci, va, invd, t, x,
                                     relax, brows);
            __syncthreads();
        }
    }
}

void gs_blocks(Prec p, int nv, int nblocks, const int *blevf, const int *lptrf, const int *permf,
               const int *blevb, const int *lptrb, const int *permb, const int *rp, const int *ci,
               const void *val, const void *invd, const void *t, void *x, const void *relax,
               i64 brows, cudaStream_t s) {
    if (nblocks <= 0) return;
    note_launch();
    if (p == Prec::F64) {
#define F(NV) k_gs_blocks<double, NV><<<nblocks, 256, 0, s>>>(blevf, lptrf, permf, blevb, lptrb, permb, rp, ci, (const double *)val, (const double *)invd, (const double *)t, (double *)x, (const double *)relax, brows)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) k_gs_blocks<float, NV><<<nblocks, 256, 0, s>>>(blevf, lptrf, permf, blevb, lptrb, permb, rp, ci, (const float *)val, (const float *)invd, (const float *)t, (float *)x, (const float *)relax, brows)
        NV_DISPATCH(nv, F)
#undef F
    }
}

template <class T, int NV>
__global__ void __launch_bounds__(256) k_gs_level(int cnt, const int *__restrict__ rows,
                                                  const int *__restrict__ rp,
                                                  const int *__restrict__ ci,
                                                  const T *__restrict__ va,
                                                  const T *__restrict__ invd,
                                                  const T *__restrict__ t, T *x,
                                                  const T *__restrict__ relax, i64 brows) {
    constexpr int TPR = Shape<T, NV>::TPR;
    int item = blockIdx.x * 256 + threadIdx.x;
    if (item >= cnt * TPR) return;
    gs_row<T, NV, true>(__ldg(rows + item / TPR), item % TPR, rp, ci, va, invd, t, x, relax, brows);
}

void gs_level(Prec p, int nv, int cnt, const int *rows, const int *rp, const int *ci,
              const void *val, const void *invd, const void *t, void *x, const void *relax,
              i64 brows, cudaStream_t s) {
    if (cnt <= 0) return;
    note_launch();
    if (p == Prec::F64) {
#define F(NV) k_gs_level<double, NV><<<(cnt * Shape<double, NV>::TPR + 255) / 256, 256, 0, s>>>(cnt, rows, rp, ci, (const double *)val, (const double *)invd, (const double *)t, (double *)x, (const double *)relax, brows)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) k_gs_level<float, NV><<<(cnt * Shape<float, NV>::TPR + 255) / 256, 256, 0, s>>>(cnt, rows, rp, ci, (const float *)val, (const float *)invd, (const float *)t, (float *)x, (const float *)relax, brows)
        NV_DISPATCH(nv, F)
#undef F
    }
}

// Grid-wide barrier for cooperative launches.  bar[0] counts arrivals,
// bar[1] is the generation.  Every wait is bounded by a wall-clock limit
// (%globaltimer); on expiry the error flag is raised and the caller leaves.
static constexpr unsigned long long kWaitLimitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool grid_sync(unsigned *bar, int *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        unsigned g = *gen;
        __threadfence();
        unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long t0 = gtime();
            while (*gen == g) {
                if (*(volatile int *)err) break;
                if (gtime() - t0 > kWaitLimitNs) {
                    atomicExch(err, 1);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)err == 0;
}

template <class T, int NV>
__global__ void __launch_bounds__(256) k_gs_sweep(int nlev, const int *__restrict__ lptr,
                                                  const int *__restrict__ perm,
                                                  const int *__restrict__ rp,
                                                  const int *__restrict__ ci,
                                                  const T *__restrict__ va,
                                                  const T *__restrict__ invd,
                                                  const T *__restrict__ t, T *x,
                                                  const T *__restrict__ relax, i64 brows,
                                                  unsigned *bar, int *err) {
    constexpr int TPR = Shape<T, NV>::TPR;
    const int stride = gridDim.x * 256;
    for (int l = 0; l < nlev; ++l) {
        int lo = __ldg(lptr + l), hi = __ldg(lptr + l + 1);
        int items = (hi - lo) * TPR;
        for (int it = blockIdx.x * 256 + threadIdx.x; it < items; it += stride)
            gs_row<T, NV, true>(__ldg(perm + lo + it / TPR), it % TPR, rp, ci, va, invd, t, x, relax, brows);
        if (l + 1 < nlev) {
            __threadfence();
            if (!grid_sync(bar, err)) return;
        }
    }
}

template <class T, int NV>
static cudaError_t gs_sweep_t(int nlev, const int *lptr, const int *perm, const int *rp,
                              const int *ci, const T *va, const T *invd, const T *t, T *x,
                              const T *relax, i64 brows, unsigned *bar, int *err, cudaStream_t s) {
    static int nblk = 0;
    if (nblk == 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gs_sweep<T, NV>, 256, 0);
        if (per < 1) per = 1;
        if (per > 2) per = 2;
        nblk = sms * per;
    }
    void *args[] = {&nlev, &lptr, &perm, &rp, &ci, &va, &invd, &t, &x, &relax, &brows, &bar, &err};
    note_launch();
    return cudaLaunchCooperativeKernel((const void *)k_gs_sweep<T, NV>, dim3(nblk), dim3(256),
                                       args, 0, s);
}

cudaError_t gs_sweep_persistent(Prec p, int nv, int nlev, const int *lptr, const int *perm,
                                const int *rp, const int *ci, const void *val, const void *invd,
                                const void *t, void *x, const void *relax, i64 brows,
                                unsigned *bar, int *err, cudaStream_t s) {
    cudaError_t e = cudaErrorInvalidValue;
    if (p == Prec::F64) {
#define F(NV) e = gs_sweep_t<double, NV>(nlev, lptr, perm, rp, ci, (const double *)val, (const double *)invd, (const double *)t, (double *)x, (const double *)relax, brows, bar, err, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) e = gs_sweep_t<float, NV>(nlev, lptr, perm, rp, ci, (const float *)val, (const float *)invd, (const float *)t, (float *)x, (const float *)relax, brows, bar, err, s)
        NV_DISPATCH(nv, F)
#undef F
    }
    return e;
}

// t = 1*b + (-1)*(off-block part of A x)
template <class T, int NV>
__global__ void __launch_bounds__(256) k_offblock(i64 n, const int *__restrict__ rp,
                                                  const int *__restrict__ ci,
                                                  const T *__restrict__ va,
                                                  const T *__restrict__ b,
                                                  const T *__restrict__ x, T *__restrict__ t,
                                                  i64 brows) {
    constexpr int V = Shape<T, NV>::V, TPR = Shape<T, NV>::TPR, RPB = 256 / TPR;
    i64 row = (i64)blockIdx.x * RPB + threadIdx.x / TPR;
    int lane = threadIdx.x % TPR;
    if (row >= n) return;
    i64 lo = (row / brows) * brows, hi = lo + brows;
    T acc[V];
#pragma unroll
    for (int e = 0; e < V; ++e) acc[e] = T(0);
    const T *xb = x + lane * V;
    for (int j = __ldg(rp + row), j1 = __ldg(rp + row + 1); j < j1; ++j) {
        int c = __ldg(ci + j);
        if (c >= lo && c < hi) continue;
        T v = __ldg(va + j);
        T xv[V];
        ld<T, V>(xb + (i64)c * NV, xv);
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] = fma(v, xv[e], acc[e]);
    }
    T bb[V];
    ld<T, V>(b + row * NV + lane * V, bb);
#pragma unroll
    for (int e = 0; e < V; ++e) acc[e] = add_rn<T>(mul_rn<T>(T(1), bb[e]), mul_rn<T>(T(-1), acc[e]));
    st<T, V>(t + row * NV + lane * V, acc);
}

void offblock_resid(Prec p, int nv, i64 n, const int *rp, const int *ci, const void *val,
                    const void *b, const void *x, void *t, i64 brows, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    if (p == Prec::F64) {
#define F(NV) k_offblock<double, NV><<<(unsigned)((n + 256 / Shape<double, NV>::TPR - 1) / (256 / Shape<double, NV>::TPR)), 256, 0, s>>>(n, rp, ci, (const double *)val, (const double *)b, (const double *)x, (double *)t, brows)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) k_offblock<float, NV><<<(unsigned)((n + 256 / Shape<float, NV>::TPR - 1) / (256 / Shape<float, NV>::TPR)), 256, 0, s>>>(n, rp, ci, (const float *)val, (const float *)b, (const float *)x, (float *)t, brows)
        NV_DISPATCH(nv, F)
#undef F
    }
}

// ---------------------------------------------------------------- Jacobi
template <class T, int NV>
__global__ void __launch_bounds__(256) k_jacobi(i64 n, const int *__restrict__ rp,
                                                const int *__restrict__ ci,
                                                const T *__restrict__ va,
                                                const T *__restrict__ invd,
                                                const T *__restrict__ b,
                                                const T *__restrict__ xi, T *__restrict__ xo,
                                                const T *__restrict__ relax) {
    constexpr int V = Shape<T, NV>::V, TPR = Shape<T, NV>::TPR, RPB = 256 / TPR;
    i64 row = (i64)blockIdx.x * RPB + threadIdx.x / TPR;
    int lane = threadIdx.x % TPR;
    if (row >= n) return;
    T acc[V];
#pragma unroll
    for (int e = 0; e < V; ++e) acc[e] = T(0);
    const T *xb = xi + lane * V;
    for (int j = __ldg(rp + row), j1 = __ldg(rp + row + 1); j < j1; ++j) {
        int c = __ldcs(ci + j);
        T v = __ldcs(va + j);
        T xv[V];
        ld<T, V>(xb + (i64)c * NV, xv);
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] = fma(v, xv[e], acc[e]);
    }
    T bb[V], xx[V];
    ld<T, V>(b + row * NV + lane * V, bb);
    ld<T, V>(xi + row * NV + lane * V, xx);
    T di = __ldg(invd + row);
#pragma unroll
    for (int e = 0; e < V; ++e) {
        T cf = mul_rn<T>(__ldg(relax + lane * V + e), di);
        T d = add_rn<T>(bb[e], -acc[e]);
        xx[e] = fma(cf, d, xx[e]);
    }
    st<T, V>(xo + row * NV + lane * V, xx);
}

void jacobi(Prec p, int nv, i64 n, const int *rp, const int *ci, const void *val,
            const void *invd, const void *b, const void *xi, void *xo, const void *relax,
            cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    if (p == Prec::F64) {
#define F(NV) k_jacobi<double, NV><<<(unsigned)((n + 256 / Shape<double, NV>::TPR - 1) / (256 / Shape<double, NV>::TPR)), 256, 0, s>>>(n, rp, ci, (const double *)val, (const double *)invd, (const double *)b, (const double *)xi, (double *)xo, (const double *)relax)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) k_jacobi<float, NV><<<(unsigned)((n + 256 / Shape<float, NV>::TPR - 1) / (256 / Shape<float, NV>::TPR)), 256, 0, s>>>(n, rp, ci, (const float *)val, (const float *)invd, (const float *)b, (const float *)xi, (float *)xo, (const float *)relax)
        NV_DISPATCH(nv, F)
#undef F
    }
}

// ---------------------------------------------------------------- dense
// thread (i, k): y[i,k] = sum_j AinvT[j*n + i] * b[j*nv + k], j ascending, fma.
// The chain is sequential, but its operands are not: they are loaded DU
// steps at a time, the next DU while the current DU multiply (two register
// sets), so the chain runs at FMA latency instead of one L2 round trip per
// few steps.
template <class T>
__global__ void __launch_bounds__(256) k_dense(int n, int nv, const T *__restrict__ AT,
                                               const T *__restrict__ b, T *__restrict__ y) {
    constexpr int DU = 16;
    i64 idx = (i64)blockIdx.x * 256 + threadIdx.x;
    if (idx >= (i64)n * nv) return;
    int i = (int)(idx % n), k = (int)(idx / n);
    T a0[DU], b0[DU], a1[DU], b1[DU];
    auto load = [&](int j0, T(&a)[DU], T(&bb)[DU]) {
#pragma unroll
        for (int u = 0; u < DU; ++u) {
            const bool in = j0 + u < n;
            a[u] = in ? __ldg(AT + (i64)(j0 + u) * n + i) : T(0);
            bb[u] = in ? __ldg(b + (i64)(j0 + u) * nv + k) : T(0);
        }
    };
    auto chain = [&](int j0, T &s, const T(&a)[DU], const T(&bb)[DU]) {
#pragma unroll
        for (int u = 0; u < DU; ++u)
            if (j0 + u < n) s = fma(a[u], bb[u], s);
    };
    T s = T(0);
    load(0, a0, b0);
    for (int j0 = 0; j0 < n; j0 += 2 * DU) {
        if (j0 + DU < n) load(j0 + DU, a1, b1);
        chain(j0, s, a0, b0);
        if (j0 + DU >= n) break;
        if (j0 + 2 * DU < n) load(j0 + 2 * DU, a0, b0);
        chain(j0 + DU, s, a1, b1);
    }
    y[(i64)i * nv + k] = s;
}

void dense_gemv(Prec p, int nv, int n, const void *AinvT, const void *b, void *y, cudaStream_t s) {
    i64 tot = (i64)n * nv;
    if (tot <= 0) return;
    note_launch();
    unsigned g = (unsigned)((tot + 255) / 256);
    if (p == Prec::F64) k_dense<double><<<g, 256, 0, s>>>(n, nv, (const double *)AinvT, (const double *)b, (double *)y);
    else k_dense<float><<<g, 256, 0, s>>>(n, nv, (const float *)AinvT, (const float *)b, (float *)y);
}

// ---------------------------------------------------------------- dots
// Stage 1: one warp per 256-row chunk; lane l accumulates rows l, l+32, ...,
// l+224 (fma, FP64), then a xor-butterfly over the 32 lanes (off = 16..1),
// whose lane-0 value equals the pairwise tree s[l] += s[l+off].
// Partials are stored dot-major: part[(d*nv + k) * nchunks + c].
template <class TI>
struct DotPairs {
    const TI *a[4];
    const TI *b[4];
};
template <class TI, int NV, int ND>
__global__ void __launch_bounds__(256) k_dot1(i64 n, i64 nch, DotPairs<TI> pr, double *__restrict__ part) {
    const int lane = threadIdx.x & 31;
    const i64 c = (i64)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (c >= nch) return;
    const TI *__restrict__ A[ND];
    const TI *__restrict__ B[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) { A[d] = pr.a[d]; B[d] = pr.b[d]; }
    double acc[ND][NV];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[d][k] = 0.0;
    constexpr int V = Shape<TI, NV>::V;
#pragma unroll 1
    for (int m = 0; m < 8; ++m) {
        i64 i = c * 256 + 32 * m + lane;
        if (i < n) {
#pragma unroll
            for (int d = 0; d < ND; ++d) {
#pragma unroll
                for (int k0 = 0; k0 < NV; k0 += V) {
                    TI xa[V], xb[V];
                    ld<TI, V>(A[d] + i * NV + k0, xa);
                    ld<TI, V>(B[d] + i * NV + k0, xb);
#pragma unroll
                    for (int e = 0; e < V; ++e)
                        acc[d][k0 + e] = fma((double)xa[e], (double)xb[e], acc[d][k0 + e]);
                }
            }
        }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double v = acc[d][k];
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, off));
            if (lane == 0) part[((i64)d * NV + k) * nch + c] = v;
        }
}

// Stage 2: block (d,k): slot t sums chunks t, t+256, ... in order from 0, then
// the 256 slots fold pairwise (off = 128..1).
__global__ void __launch_bounds__(256) k_dot2(i64 nch, const double *__restrict__ part,
                                              double *__restrict__ out) {
    __shared__ double q[256];
    const double *p = part + (i64)blockIdx.x * nch;
    double a = 0.0;
    for (i64 c = threadIdx.x; c < nch; c += 256) a = dadd(a, p[c]);
    q[threadIdx.x] = a;
    __syncthreads();
    for (int off = 128; off >= 32; off >>= 1) {
        if (threadIdx.x < off) q[threadIdx.x] = dadd(q[threadIdx.x], q[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        double v = q[threadIdx.x];
        for (int off = 16; off >= 1; off >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (threadIdx.x == 0) out[blockIdx.x] = v;
    }
}

// Inner products in the reference's single-core order (blas.inl:561-576):
// per column k, res = 0; res += a_i * b_i for i = 0 .. n-1, the product and
// the sum each rounded (no fma).  A sum in that order is one dependent chain
// per column.  Block d serves pair d: warps 1-7 load tiles of SEQ_TILE rows
// and store their products (each rounded) in a shared-memory double buffer
// while lane k of warp 0 adds the previous tile's products of column k in
// row order, so the chain waits on shared memory, not on HBM.  The sum is
// stored as the partial of chunk 0, and the remaining blocks zero the pair's
// other chunk partials, so the reduction stage (k_dot2, k_dot2_epi: +0 plus
// the chunk partials in order, then a pairwise fold with zeros) returns it
// unchanged.
constexpr int SEQ_TILE = 256;
// products a_i * b_i (rounded) of rows [t*SEQ_TILE, ...) into buf, by the
// block's threads 32..255
template <class TI, int NV>
__device__ __forceinline__ void seq_fill(const TI *__restrict__ a, const TI *__restrict__ b, i64 n, i64 t,
                                         double *buf) {
    const i64 r0 = t * SEQ_TILE;
    const int cnt = (int)(n - r0 < SEQ_TILE ? n - r0 : SEQ_TILE) * NV;
    const TI *__restrict__ at = a + r0 * NV;
    const TI *__restrict__ bt = b + r0 * NV;
    int q = (int)threadIdx.x - 32;
    // eight loads of each operand in flight before the products are stored
    for (; q + 7 * 224 < cnt; q += 8 * 224) {
        double xa[8], xb[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) { xa[e] = (double)at[q + e * 224]; xb[e] = (double)bt[q + e * 224]; }
#pragma unroll
        for (int e = 0; e < 8; ++e) buf[q + e * 224] = dmul(xa[e], xb[e]);
    }
    for (; q < cnt; q += 224) buf[q] = dmul((double)at[q], (double)bt[q]);
}
template <class TI, int NV>
__global__ void __launch_bounds__(256) k_dot_seq(i64 n, i64 nch, int nd, DotPairs<TI> pr,
                                                 double *__restrict__ part) {
    if ((int)blockIdx.x >= nd) {
        const i64 per = nch - 1;
        const i64 tot = (i64)nd * NV * per;
        const i64 stride = (i64)(gridDim.x - nd) * blockDim.x;
        for (i64 q = (i64)(blockIdx.x - nd) * blockDim.x + threadIdx.x; q < tot; q += stride)
            part[(q / per) * nch + 1 + q % per] = 0.0;
        return;
    }
    // products of one tile, row-major [row][column]
    extern __shared__ double prod[];  // 2 * SEQ_TILE * NV
    const int d = blockIdx.x;
    // constant indices keep the parameter struct out of local memory
    const TI *__restrict__ a = d == 0 ? pr.a[0] : d == 1 ? pr.a[1] : d == 2 ? pr.a[2] : pr.a[3];
    const TI *__restrict__ b = d == 0 ? pr.b[0] : d == 1 ? pr.b[1] : d == 2 ? pr.b[2] : pr.b[3];
    const i64 ntiles = (n + SEQ_TILE - 1) / SEQ_TILE;
    const int tid = threadIdx.x;
    const bool loader = tid >= 32;
    if (loader && ntiles > 0) seq_fill<TI, NV>(a, b, n, 0, prod);
    __syncthreads();
    double s = 0.0;
    for (i64 t = 0; t < ntiles; ++t) {
        double *cur = prod + (t & 1) * (SEQ_TILE * NV);
        if (loader) {
            if (t + 1 < ntiles) seq_fill<TI, NV>(a, b, n, t + 1, prod + ((t + 1) & 1) * (SEQ_TILE * NV));
        } else if (tid < NV) {
            const int rows = (int)(n - t * SEQ_TILE < SEQ_TILE ? n - t * SEQ_TILE : SEQ_TILE);
            int r = 0;
            // eight products read ahead of their adds (same order)
            for (; r + 8 <= rows; r += 8) {
                double q[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) q[e] = cur[(r + e) * NV + tid];
#pragma unroll
                for (int e = 0; e < 8; ++e) s = dadd(s, q[e]);
            }
            for (; r < rows; ++r) s = dadd(s, cur[r * NV + tid]);
        }
        __syncthreads();
    }
    if (tid < NV) part[((i64)d * NV + tid) * nch] = s;
}

static thread_local bool t_dot_seq = false;
void set_dot_sequential(bool on) { t_dot_seq = on; }
bool dot_sequential() { return t_dot_seq; }

i64 dot_part_size(i64 n, int nd, int nv) { return ((n + 255) / 256) * nd * nv; }

template <class TI, int NV>
static void dots_t(i64 n, int nd, const void *const *a, const void *const *b, double *part,
                   double *out, cudaStream_t s, bool reduce = true) {
    i64 nch = (n + 255) / 256;
    if (nch == 0) {
        if (reduce) cudaMemsetAsync(out, 0, sizeof(double) * nd * NV, s);
        return;
    }
    unsigned g = (unsigned)((nch + 7) / 8);
    DotPairs<TI> pr;
    for (int d = 0; d < 4; ++d) {
        pr.a[d] = (const TI *)a[d < nd ? d : 0];
        pr.b[d] = (const TI *)b[d < nd ? d : 0];
    }
    if (t_dot_seq) {
        // one block per pair plus blocks that zero the other chunk partials
        const unsigned zb = (unsigned)std::min<i64>(4 * 148, std::max<i64>(1, (nd * NV * (nch - 1) + 255) / 256));
        note_launch(reduce ? 2 : 1);
        const size_t smem = sizeof(double) * 2 * SEQ_TILE * NV;  // 128 KB at NV = 32
        cudaFuncSetAttribute(k_dot_seq<TI, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_dot_seq<TI, NV><<<(unsigned)nd + zb, 256, smem, s>>>(n, nch, nd, pr, part);
        if (reduce) k_dot2<<<nd * NV, 256, 0, s>>>(nch, part, out);
        return;
    }
    note_launch(2);
    if (nd == 1) k_dot1<TI, NV, 1><<<g, 256, 0, s>>>(n, nch, pr, part);
    else if (nd == 2) k_dot1<TI, NV, 2><<<g, 256, 0, s>>>(n, nch, pr, part);
    else if (nd == 3) k_dot1<TI, NV, 3><<<g, 256, 0, s>>>(n, nch, pr, part);
    else if constexpr (NV <= 8) k_dot1<TI, NV, 4><<<g, 256, 0, s>>>(n, nch, pr, part);
    else {
        // four pairs at wide NV: two passes of two pairs (register budget);
        // each pair's partials are the same as in one pass
        DotPairs<TI> hi;
        for (int d = 0; d < 2; ++d) { hi.a[d] = pr.a[d + 2]; hi.b[d] = pr.b[d + 2]; hi.a[d + 2] = hi.a[d]; hi.b[d + 2] = hi.b[d]; }
        note_launch();
        k_dot1<TI, NV, 2><<<g, 256, 0, s>>>(n, nch, pr, part);
        k_dot1<TI, NV, 2><<<g, 256, 0, s>>>(n, nch, hi, part + (i64)2 * NV * nch);
    }
    if (!reduce) {
        note_launch(-1);
        return;
    }
    k_dot2<<<nd * NV, 256, 0, s>>>(nch, part, out);
}

void dots(Prec in, int nv, i64 n, int nd, const void *const *a, const void *const *b,
          double *part, double *out, cudaStream_t s) {
    if (in == Prec::F64) {
#define F(NV) dots_t<double, NV>(n, nd, a, b, part, out, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) dots_t<float, NV>(n, nd, a, b, part, out, s)
        NV_DISPATCH(nv, F)
#undef F
    }
}

// ---------------------------------------------------------------- BLAS-1
// Literal evaluation in FP64 with every product rounded (no contraction); FP32
// storage is widened on load and rounded once on store.
template <class T, int NV, int OP>
__global__ void __launch_bounds__(256) k_blas(i64 total, const double *__restrict__ a,
                                              const T *__restrict__ x,
                                              const double *__restrict__ b,
                                              const T *__restrict__ y,
                                              const double *__restrict__ c, T *__restrict__ z) {
    i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q >= total) return;
    int k = (int)(q % NV);
    double r;
    if (OP == (int)Op::AXPBY_Z) {
        r = dadd(dmul(a[k], (double)x[q]), dmul(b[k], (double)y[q]));
    } else if (OP == (int)Op::AXPBYPCZ) {
        r = dadd(dadd(dmul(a[k], (double)x[q]), dmul(b[k], (double)y[q])), dmul(c[k], (double)z[q]));
    } else if (OP == (int)Op::AX_Y) {
        r = dmul(a[k], (double)x[q]);
    } else if (OP == (int)Op::COPY) {
        r = (double)x[q];
    } else if (OP == (int)Op::SET) {
        r = a[k];
    } else if (OP == (int)Op::SCAL_XY) {
        r = dmul((double)z[q], (double)x[q]);
    } else {  // ROW_SCAL: x holds one value per row
        r = dmul((double)z[q], (double)x[q / NV]);
    }
    z[q] = (T)r;
}

template <class T, int NV>
static void blas_t(i64 n, Op op, const double *a, const T *x, const double *b, const T *y,
                   const double *c, T *z, cudaStream_t s) {
    i64 tot = n * NV;
    if (tot <= 0) return;
    note_launch();
    unsigned g = (unsigned)((tot + 255) / 256);
    switch (op) {
    case Op::AXPBY_Z: k_blas<T, NV, 0><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    case Op::AXPBYPCZ: k_blas<T, NV, 1><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    case Op::AX_Y: k_blas<T, NV, 2><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    case Op::COPY: k_blas<T, NV, 3><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    case Op::SET: k_blas<T, NV, 4><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    case Op::SCAL_XY: k_blas<T, NV, 5><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    case Op::ROW_SCAL: k_blas<T, NV, 6><<<g, 256, 0, s>>>(tot, a, x, b, y, c, z); break;
    }
}

void blas(Prec p, int nv, i64 n, Op op, const double *a, const void *x, const double *b,
          const void *y, const double *c, void *z, cudaStream_t s) {
    if (p == Prec::F64) {
#define F(NV) blas_t<double, NV>(n, op, a, (const double *)x, b, (const double *)y, c, (double *)z, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) blas_t<float, NV>(n, op, a, (const float *)x, b, (const float *)y, c, (float *)z, s)
        NV_DISPATCH(nv, F)
#undef F
    }
}

template <class T>
__global__ void k_fill(i64 cnt, T v, T *z) {
    i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q < cnt) z[q] = v;
}
void fill(Prec p, i64 count, double v, void *z, cudaStream_t s) {
    if (count <= 0) return;
    note_launch();
    unsigned g = (unsigned)((count + 255) / 256);
    if (p == Prec::F64) k_fill<double><<<g, 256, 0, s>>>(count, v, (double *)z);
    else k_fill<float><<<g, 256, 0, s>>>(count, (float)v, (float *)z);
}

template <class A, class B>
__global__ void k_conv(i64 cnt, const A *x, B *y) {
    i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q < cnt) y[q] = (B)x[q];
}
void convert(Prec from, Prec to, i64 count, const void *x, void *y, cudaStream_t s) {
    if (count <= 0) return;
    note_launch();
    unsigned g = (unsigned)((count + 255) / 256);
    if (from == Prec::F64 && to == Prec::F32) k_conv<double, float><<<g, 256, 0, s>>>(count, (const double *)x, (float *)y);
    else if (from == Prec::F32 && to == Prec::F64) k_conv<float, double><<<g, 256, 0, s>>>(count, (const float *)x, (double *)y);
    else if (from == Prec::F64) k_conv<double, double><<<g, 256, 0, s>>>(count, (const double *)x, (double *)y);
    else k_conv<float, float><<<g, 256, 0, s>>>(count, (const float *)x, (float *)y);
}

// ---------------------------------------------------------------- scalars
__global__ void k_alpha(int nv, const double *rho, const double *s1, double *alpha) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nv) alpha[k] = __ddiv_rn(rho[k], s1[k]);
}
// one thread per column; nv may exceed a warp (batched systems: nsys * nv columns)
static unsigned sblocks(int nv) { return (unsigned)((nv + 127) / 128); }
void bicg_alpha(int nv, const double *rho, const double *s1, double *alpha, cudaStream_t s) {
    note_launch();
    k_alpha<<<sblocks(nv), 128, 0, s>>>(nv, rho, s1, alpha);
}
__global__ void k_omega(int nv, const double *s2, const double *s3, const double *s4,
                        const double *alpha, const double *iconv, double *omega, double *res,
                        double *ac, double *oc) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double w = __ddiv_rn(s2[k], s3[k]);
    omega[k] = w;
    ac[k] = dmul(iconv[k], alpha[k]);
    oc[k] = dmul(iconv[k], w);
    double rr = dmul(w, s2[k]);
    res[k] = dadd(dmul(1.0, s4[k]), dmul(-1.0, rr));
}
void bicg_omega(int nv, const double *s2, const double *s3, const double *s4,
                const double *alpha, const double *iconv, double *omega, double *res,
                double *ac, double *oc, cudaStream_t s) {
    note_launch();
    k_omega<<<sblocks(nv), 128, 0, s>>>(nv, s2, s3, s4, alpha, iconv, omega, res, ac, oc);
}
__global__ void k_beta(int nv, const double *s1, double *rho, const double *alpha,
                       const double *omega, double *beta, double *c1) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double a2 = __ddiv_rn(s1[k], rho[k]);
    double a3 = __ddiv_rn(alpha[k], omega[k]);
    double bt = dmul(a2, a3);
    beta[k] = bt;
    rho[k] = s1[k];
    c1[k] = dmul(-1.0, dmul(omega[k], bt));
}
void bicg_beta(int nv, const double *s1, double *rho, const double *alpha, const double *omega,
               double *beta, double *c1, cudaStream_t s) {
    note_launch();
    k_beta<<<sblocks(nv), 128, 0, s>>>(nv, s1, rho, alpha, omega, beta, c1);
}
// PCG step length (pcg.inl:125-134): alpha = s1/s2; ac = iconv*alpha; nalpha = -1*alpha
__global__ void k_pcg_alpha(int nv, const double *s1, const double *s2, const double *iconv, double *alpha,
                            double *ac, double *nalpha) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double a = __ddiv_rn(s1[k], s2[k]);
    alpha[k] = a;
    ac[k] = dmul(iconv[k], a);
    nalpha[k] = dmul(-1.0, a);
}
void pcg_alpha(int nv, const double *s1, const double *s2, const double *iconv, double *alpha, double *ac,
               double *nalpha, cudaStream_t s) {
    note_launch();
    k_pcg_alpha<<<sblocks(nv), 128, 0, s>>>(nv, s1, s2, iconv, alpha, ac, nalpha);
}
// RBiCGStab recurrences (rbicgstab.inl:130-134 and 193-211)
__global__ void k_ralpha(int nv, const double *rho, const double *delta, double *alpha,
                         double *nalpha) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double a = __ddiv_rn(rho[k], delta[k]);
    alpha[k] = a;
    nalpha[k] = dmul(-1.0, a);
}
void rbicg_alpha(int nv, const double *rho, const double *delta, double *alpha, double *nalpha,
                 cudaStream_t s) {
    note_launch();
    k_ralpha<<<sblocks(nv), 128, 0, s>>>(nv, rho, delta, alpha, nalpha);
}
__global__ void k_rbeta(int nv, const double *omega, const double *psi, double *delta, double *rho,
                        double *beta, double *nomega) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double w = omega[k];
    double r = dmul(-1.0, dmul(w, psi[k]));
    double bt = __ddiv_rn(r, dmul(delta[k], w));
    double nw = dmul(-1.0, w);
    rho[k] = r;
    beta[k] = bt;
    nomega[k] = nw;
    delta[k] = dmul(nw, bt);
}
void rbicg_beta(int nv, const double *omega, const double *psi, double *delta, double *rho,
                double *beta, double *nomega, cudaStream_t s) {
    note_launch();
    k_rbeta<<<sblocks(nv), 128, 0, s>>>(nv, omega, psi, delta, rho, beta, nomega);
}
__global__ void k_neg(int nv, const double *in, double *out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nv) out[k] = dmul(-1.0, in[k]);
}
void negate(int nv, const double *in, double *out, cudaStream_t s) {
    note_launch();
    k_neg<<<sblocks(nv), 128, 0, s>>>(nv, in, out);
}


// ---------------------------------------------------------------- fused BiCGStab groups
// The merged groups of the reference's MergedBiCGStab / MergedPBiCGStab
// (blas_merged_bicgstab.inl: group 2 `s = r - alpha v`, group 4 `r = s -
// omega t, rho = (r, r0)`, group 5 `x += alpha p + omega s, p = r + beta p -
// beta omega v`) as single passes, with the scalar recurrences folded into the
// reduction stage of the inner products.  Every element and every partial sum
// is computed exactly as by the separate BLAS-1, dot and scalar kernels above
// (same expressions, same chunk/lane/slot tree), so the fused iteration gives
// the same bits.

// s = 1*r + (-alpha)*v; sz (the preconditioned copy about to be formed) = 0
template <class T, int NV>
__global__ void __launch_bounds__(256) k_bicg_s(i64 total, const double *__restrict__ alpha,
                                                const T *__restrict__ r, const T *__restrict__ v,
                                                T *__restrict__ s, T *__restrict__ sz) {
    i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q >= total) return;
    int k = (int)(q % NV);
    double na = dmul(-1.0, alpha[k]);
    s[q] = (T)dadd(dmul(1.0, (double)r[q]), dmul(na, (double)v[q]));
    if (sz) sz[q] = T(0);
}

// p = 1*r + c1*v + beta*p; pz = 0
template <class T, int NV>
__global__ void __launch_bounds__(256) k_bicg_p(i64 total, const double *__restrict__ c1,
                                                const double *__restrict__ beta, const T *__restrict__ r,
                                                const T *__restrict__ v, T *__restrict__ p, T *__restrict__ pz) {
    i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q >= total) return;
    int k = (int)(q % NV);
    p[q] = (T)dadd(dadd(dmul(1.0, (double)r[q]), dmul(c1[k], (double)v[q])), dmul(beta[k], (double)p[q]));
    if (pz) pz[q] = T(0);
}

// x = ac*pp + oc*ss + 1*x;  r = 1*s + (-omega)*t;  chunk partials of (r, r0)
// in the layout of k_dot1 (warp = chunk of 256 rows, lane l sums rows
// l + 32m, m = 0..7, then the lanes fold 16..1).
template <class T, int NV>
__global__ void __launch_bounds__(256) k_bicg_xr(i64 n, i64 nch, const double *__restrict__ ac,
                                                 const double *__restrict__ oc, const double *__restrict__ omega,
                                                 const T *__restrict__ pp, const T *__restrict__ ss,
                                                 T *__restrict__ x, const T *__restrict__ s,
                                                 const T *__restrict__ t, T *__restrict__ r,
                                                 const T *__restrict__ r0, double *__restrict__ part) {
    const int lane = threadIdx.x & 31;
    const i64 c = (i64)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (c >= nch) return;
    constexpr int V = Shape<T, NV>::V;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
#pragma unroll 1
    for (int m = 0; m < 8; ++m) {
        i64 i = c * 256 + 32 * m + lane;
        if (i >= n) continue;
#pragma unroll
        for (int k0 = 0; k0 < NV; k0 += V) {
            const i64 o = i * NV + k0;
            T a[V], b[V], xx[V], sv[V], tv[V], z[V], xo[V], ro[V];
            ld<T, V>(pp + o, a);
            ld<T, V>(ss + o, b);
            ld_cg<T, V>(x + o, xx);
            ld<T, V>(s + o, sv);
            ld<T, V>(t + o, tv);
            ld<T, V>(r0 + o, z);
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const int k = k0 + e;
                xo[e] = (T)dadd(dadd(dmul(__ldg(ac + k), (double)a[e]), dmul(__ldg(oc + k), (double)b[e])),
                                dmul(1.0, (double)xx[e]));
                const double nw = dmul(-1.0, __ldg(omega + k));
                ro[e] = (T)dadd(dmul(1.0, (double)sv[e]), dmul(nw, (double)tv[e]));
                acc[k] = fma((double)ro[e], (double)z[e], acc[k]);
            }
            st<T, V>(x + o, xo);
            st<T, V>(r + o, ro);
        }
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double v = acc[k];
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (lane == 0) part[(i64)k * nch + c] = v;
    }
}

// Stage 2 of the inner products (the k_dot2 tree) for all nd pairs of one
// column k per block, then that column's scalar recurrence.
enum { EPI_ALPHA = 0, EPI_OMEGA = 1, EPI_BETA = 2 };
template <int EPI>
__device__ __forceinline__ void bicg_epi_col(int k, const double *val, const BicgScalars &sc);
template <int EPI>
__global__ void __launch_bounds__(256) k_dot2_epi(i64 nch, int nd, int nv, const double *__restrict__ part,
                                                  double *__restrict__ out, BicgScalars sc) {
    __shared__ double q[256];
    __shared__ double val[4];
    const int k = blockIdx.x;
    for (int d = 0; d < nd; ++d) {
        const double *p = part + ((i64)d * nv + k) * nch;
        double a = 0.0;
        for (i64 c = threadIdx.x; c < nch; c += 256) a = dadd(a, p[c]);
        q[threadIdx.x] = a;
        __syncthreads();
        for (int off = 128; off >= 32; off >>= 1) {
            if (threadIdx.x < off) q[threadIdx.x] = dadd(q[threadIdx.x], q[threadIdx.x + off]);
            __syncthreads();
        }
        if (threadIdx.x < 32) {
            double v = q[threadIdx.x];
            for (int off = 16; off >= 1; off >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, off));
            if (threadIdx.x == 0) {
                val[d] = v;
                out[(i64)d * nv + k] = v;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    bicg_epi_col<EPI>(k, val, sc);
}

// the recurrence alone, from reduced values vals[d*nv + k] (one thread per column)
template <int EPI>
__global__ void k_bicg_epi(int nv, const double *__restrict__ vals, BicgScalars sc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    double val[3];
    for (int d = 0; d < (EPI == EPI_OMEGA ? 3 : 1); ++d) val[d] = vals[(i64)d * nv + k];
    bicg_epi_col<EPI>(k, val, sc);
}

template <int EPI>
__device__ __forceinline__ void bicg_epi_col(int k, const double *val, const BicgScalars &sc) {
    if (EPI == EPI_ALPHA) {  // alpha = rho / (v, r0)
        sc.alpha[k] = __ddiv_rn(sc.rho[k], val[0]);
    } else if (EPI == EPI_OMEGA) {  // omega = (t,s)/(t,t); res = (s,s) - omega (t,s)
        const double s2 = val[0], s3 = val[1], s4 = val[2];
        const double w = __ddiv_rn(s2, s3);
        sc.omega[k] = w;
        const double ic = sc.iconv[k];
        sc.ac[k] = dmul(ic, sc.alpha[k]);
        sc.oc[k] = dmul(ic, w);
        const double rr = dmul(w, s2);
        const double res = dadd(dmul(1.0, s4), dmul(-1.0, rr));
        sc.res[k] = res;
        // the host's convergence rule (sqrt(res) > tol: not converged; a
        // column once converged stays frozen), evaluated here so that the next
        // iteration's masks are ready without a host round trip
        if (sc.check && sc.status[k] == 0.0 && !(__dsqrt_rn(res) > sc.tol[k])) sc.status[k] = 1.0;
        sc.iconv[k] = sc.status[k] != 0.0 ? 0.0 : 1.0;
    } else {  // beta = (rho'/rho)(alpha/omega); rho = rho'; c1 = -(omega beta)
        const double s1 = val[0];
        const double a2 = __ddiv_rn(s1, sc.rho[k]);
        const double a3 = __ddiv_rn(sc.alpha[k], sc.omega[k]);
        const double bt = dmul(a2, a3);
        sc.beta[k] = bt;
        sc.rho[k] = s1;
        sc.c1[k] = dmul(-1.0, dmul(sc.omega[k], bt));
    }
}

template <class T, int NV>
static void bicg_groups_t(int grp, i64 n, const BicgScalars &sc, const void *a0, const void *a1, void *a2,
                          const void *a3, const void *a4, void *a5, const void *a6, double *part, cudaStream_t s) {
    const i64 tot = n * NV;
    if (tot <= 0) return;
    const unsigned g = (unsigned)((tot + 255) / 256);
    note_launch();
    if (grp == 0) {
        k_bicg_s<T, NV><<<g, 256, 0, s>>>(tot, sc.alpha, (const T *)a0, (const T *)a1, (T *)a2, (T *)a5);
    } else if (grp == 1) {
        k_bicg_p<T, NV><<<g, 256, 0, s>>>(tot, sc.c1, sc.beta, (const T *)a0, (const T *)a1, (T *)a2, (T *)a5);
    } else {
        const i64 nch = (n + 255) / 256;
        k_bicg_xr<T, NV><<<(unsigned)((nch + 7) / 8), 256, 0, s>>>(
            n, nch, sc.ac, sc.oc, sc.omega, (const T *)a0, (const T *)a1, (T *)a2, (const T *)a3, (const T *)a4,
            (T *)a5, (const T *)a6, part);
    }
}

void bicg_s(Prec p, int nv, i64 n, const BicgScalars &sc, const void *r, const void *v, void *s_out, void *sz,
            cudaStream_t s) {
    if (p == Prec::F64) {
#define F(NV) bicg_groups_t<double, NV>(0, n, sc, r, v, s_out, nullptr, nullptr, sz, nullptr, nullptr, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) bicg_groups_t<float, NV>(0, n, sc, r, v, s_out, nullptr, nullptr, sz, nullptr, nullptr, s)
        NV_DISPATCH(nv, F)
#undef F
    }
}

void bicg_p(Prec p, int nv, i64 n, const BicgScalars &sc, const void *r, const void *v, void *pv, void *pz,
            cudaStream_t s) {
    if (p == Prec::F64) {
#define F(NV) bicg_groups_t<double, NV>(1, n, sc, r, v, pv, nullptr, nullptr, pz, nullptr, nullptr, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) bicg_groups_t<float, NV>(1, n, sc, r, v, pv, nullptr, nullptr, pz, nullptr, nullptr, s)
        NV_DISPATCH(nv, F)
#undef F
    }
}

void bicg_xr(Prec p, int nv, i64 n, const BicgScalars &sc, const void *pp, const void *ss, void *x, const void *sv,
             const void *t, void *r, const void *r0, double *part, cudaStream_t s) {
    if (p == Prec::F64) {
#define F(NV) bicg_groups_t<double, NV>(2, n, sc, pp, ss, x, sv, t, r, r0, part, s)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) bicg_groups_t<float, NV>(2, n, sc, pp, ss, x, sv, t, r, r0, part, s)
        NV_DISPATCH(nv, F)
#undef F
    }
}

void dot_reduce_epi(int epi, i64 n, int nd, int nv, const double *part, double *out, const BicgScalars &sc,
                    cudaStream_t s) {
    const i64 nch = (n + 255) / 256;
    note_launch();
    if (epi == EPI_ALPHA) k_dot2_epi<EPI_ALPHA><<<nv, 256, 0, s>>>(nch, nd, nv, part, out, sc);
    else if (epi == EPI_OMEGA) k_dot2_epi<EPI_OMEGA><<<nv, 256, 0, s>>>(nch, nd, nv, part, out, sc);
    else k_dot2_epi<EPI_BETA><<<nv, 256, 0, s>>>(nch, nd, nv, part, out, sc);
}

void bicg_epi(int epi, int nv, const double *vals, const BicgScalars &sc, cudaStream_t s) {
    note_launch();
    const unsigned g = (unsigned)((nv + 127) / 128);
    if (epi == EPI_ALPHA) k_bicg_epi<EPI_ALPHA><<<g, 128, 0, s>>>(nv, vals, sc);
    else if (epi == EPI_OMEGA) k_bicg_epi<EPI_OMEGA><<<g, 128, 0, s>>>(nv, vals, sc);
    else k_bicg_epi<EPI_BETA><<<g, 128, 0, s>>>(nv, vals, sc);
}

void dot_reduce(i64 n, int nd, int nv, const double *part, double *out, cudaStream_t s) {
    const i64 nch = (n + 255) / 256;
    if (nch == 0) {
        cudaMemsetAsync(out, 0, sizeof(double) * nd * nv, s);
        return;
    }
    note_launch();
    k_dot2<<<nd * nv, 256, 0, s>>>(nch, part, out);
}

// dst row q = src row idx[q] of block vectors (W: 16- or 4-byte words)
template <class W>
__global__ void k_gather_rows(i64 cnt, int wpr, const int *__restrict__ idx, const W *__restrict__ src,
                              W *__restrict__ dst) {
    const i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q >= cnt * wpr) return;
    const i64 r = q / wpr;
    dst[q] = src[(i64)idx[r] * wpr + q % wpr];
}
void gather_rows(Prec p, int nv, i64 cnt, const int *idx, const void *src, void *dst, cudaStream_t s) {
    if (cnt <= 0) return;
    note_launch();
    const int bytes = nv * (p == Prec::F64 ? 8 : 4);
    if (bytes % 16 == 0) {
        const int wpr = bytes / 16;
        k_gather_rows<float4><<<(unsigned)((cnt * wpr + 255) / 256), 256, 0, s>>>(cnt, wpr, idx, (const float4 *)src,
                                                                                (float4 *)dst);
    } else {
        const int wpr = bytes / 4;
        k_gather_rows<float><<<(unsigned)((cnt * wpr + 255) / 256), 256, 0, s>>>(cnt, wpr, idx, (const float *)src,
                                                                               (float *)dst);
    }
}

void dot_partials(Prec in, int nv, i64 n, int nd, const void *const *a, const void *const *b, double *part,
                  cudaStream_t s) {
    if (in == Prec::F64) {
#define F(NV) dots_t<double, NV>(n, nd, a, b, part, nullptr, s, false)
        NV_DISPATCH(nv, F)
#undef F
    } else {
#define F(NV) dots_t<float, NV>(n, nd, a, b, part, nullptr, s, false)
        NV_DISPATCH(nv, F)
#undef F
    }
}

}  // namespace xk
