// Kernels of the batching form: many independent systems solved together as
// one block-diagonal system whose row segments carry their own Krylov scalars
// (sm_100a).  Per-(segment, column) scalars live at [s*nv + k]; the vectors
// are FP64 block vectors (row-major n x nv) of the concatenated systems.
#include "kernels.cuh"
#include <cuda_runtime.h>

namespace xk {

namespace {

__device__ __forceinline__ double dmul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd_(double a, double b) { return __dadd_rn(a, b); }

// segment of row i: the last s with segoff[s] <= i (segoff ascending, nseg+1 entries)
__device__ __forceinline__ int seg_of(const i64 *segoff, int nseg, i64 i) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segoff[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Stage 1 of the per-segment canonical inner products: one warp per chunk of
// 256 rows of one segment (chunks counted from the segment's first row), the
// same lane/row assignment and butterfly as the whole-vector dots.
template <class TI, int NV, int ND>
__global__ void __launch_bounds__(256) k_segdot1(int nseg, const i64 *__restrict__ segoff,
                                                 const i64 *__restrict__ cstart, i64 nch,
                                                 const TI *__restrict__ a0, const TI *__restrict__ b0,
                                                 const TI *__restrict__ a1, const TI *__restrict__ b1,
                                                 const TI *__restrict__ a2, const TI *__restrict__ b2,
                                                 double *__restrict__ part) {
    const int lane = threadIdx.x & 31;
    const i64 g = (i64)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (g >= nch) return;
    const int s = seg_of(cstart, nseg, g);
    const i64 c = g - cstart[s];
    const i64 r0 = segoff[s], r1 = segoff[s + 1];
    const TI *A[3] = {a0, a1, a2};
    const TI *B[3] = {b0, b1, b2};
    double acc[ND][NV];
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[d][k] = 0.0;
#pragma unroll 1
    for (int m = 0; m < 8; ++m) {
        const i64 i = r0 + c * 256 + 32 * m + lane;
        if (i < r1) {
#pragma unroll
            for (int d = 0; d < ND; ++d)
#pragma unroll
                for (int k = 0; k < NV; ++k)
                    acc[d][k] = fma((double)A[d][i * NV + k], (double)B[d][i * NV + k], acc[d][k]);
        }
    }
#pragma unroll
    for (int d = 0; d < ND; ++d)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double v = acc[d][k];
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) v = dadd_(v, __shfl_xor_sync(0xffffffffu, v, off));
            if (lane == 0) part[((i64)d * NV + k) * nch + g] = v;
        }
}

// Stage 2: block (segment s, dot d, column k) folds the segment's chunks with
// the slot/fold order of the whole-vector dots.
__global__ void __launch_bounds__(256) k_segdot2(int nseg, int ndk, int nv, const i64 *__restrict__ cstart,
                                                 i64 nch, const double *__restrict__ part,
                                                 double *__restrict__ out) {
    __shared__ double q[256];
    const int s = blockIdx.x / ndk, dk = blockIdx.x % ndk;
    const i64 c0 = cstart[s], cn = cstart[s + 1] - c0;
    const double *p = part + (i64)dk * nch + c0;
    double a = 0.0;
    for (i64 c = threadIdx.x; c < cn; c += 256) a = dadd_(a, p[c]);
    q[threadIdx.x] = a;
    __syncthreads();
    for (int off = 128; off >= 32; off >>= 1) {
        if (threadIdx.x < off) q[threadIdx.x] = dadd_(q[threadIdx.x], q[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        double v = q[threadIdx.x];
        for (int off = 16; off >= 1; off >>= 1) v = dadd_(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (threadIdx.x == 0) {
            const int d = dk / nv, k = dk % nv;
            out[(i64)d * nseg * nv + (i64)s * nv + k] = v;
        }
    }
}

// z = a x + b y (OP 0) or z = a x + b y + c z (OP 1), scalars of the row's segment
template <int OP>
__global__ void __launch_bounds__(256) k_segblas(int nv, int nseg, const i64 *__restrict__ segoff,
                                                 i64 total, const double *__restrict__ a,
                                                 const double *__restrict__ x,
                                                 const double *__restrict__ b,
                                                 const double *__restrict__ y,
                                                 const double *__restrict__ c, double *z) {
    const i64 q = (i64)blockIdx.x * 256 + threadIdx.x;
    if (q >= total) return;
    const i64 i = q / nv;
    const int k = (int)(q % nv);
    const int s = seg_of(segoff, nseg, i);
    const int j = s * nv + k;
    double r = dadd_(dmul_(a[j], x[q]), dmul_(b[j], y[q]));
    if (OP == 1) r = dadd_(r, dmul_(c[j], z[q]));
    z[q] = r;
}

__global__ void k_binit(int nsc, const double *res0, double rel, double abs_tol, double *tol2,
                        double *iconv, int *conv_it, int *ctr) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < nsc; k += blockDim.x) {
        const double t = fmax(abs_tol, rel * sqrt(res0[k]));
        tol2[k] = t * t;
        const bool act = sqrt(res0[k]) > t;
        iconv[k] = act ? 1.0 : 0.0;
        conv_it[k] = 0;
        if (act) atomicAdd(&cnt, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctr[0] = 0;
        ctr[1] = cnt;
    }
}

__global__ void k_bomega(int nsc, const double *s2, const double *s3, const double *s4,
                         const double *alpha, const double *iconv, double *omega, double *res,
                         double *ac, double *oc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsc) return;
    const double w = __ddiv_rn(s2[k], s3[k]);
    omega[k] = w;
    const bool act = iconv[k] != 0.0;
    ac[k] = act ? alpha[k] : 0.0;
    oc[k] = act ? w : 0.0;
    res[k] = dadd_(dmul_(1.0, s4[k]), dmul_(-1.0, dmul_(w, s2[k])));
}

__global__ void k_bcheck(int nsc, const double *res, const double *tol2, double *iconv, int *conv_it,
                         double *res_last, int *ctr, int max_iters,
                         cudaGraphConditionalHandle handle, int use_graph) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    const int it = ctr[0] + 1;
    for (int k = threadIdx.x; k < nsc; k += blockDim.x) {
        if (iconv[k] == 0.0) continue;
        res_last[k] = res[k];
        if (res[k] <= tol2[k]) {
            iconv[k] = 0.0;
            conv_it[k] = it;
        } else {
            atomicAdd(&cnt, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctr[0] = it;
        ctr[1] = cnt;
        if (use_graph) cudaGraphSetConditional(handle, (cnt > 0 && it < max_iters) ? 1u : 0u);
    }
}

}  // namespace

template <class TI, int NV>
static void segdots_t(int nseg, const i64 *segoff, const i64 *cstart, i64 nch, int nd,
                      const void *const *a, const void *const *b, double *part, double *out,
                      cudaStream_t s) {
    note_launch(nch > 0 ? 2 : 1);
    if (nch > 0) {
        const unsigned g = (unsigned)((nch + 7) / 8);
        const TI *A0 = (const TI *)a[0], *B0 = (const TI *)b[0];
        const TI *A1 = nd > 1 ? (const TI *)a[1] : A0, *B1 = nd > 1 ? (const TI *)b[1] : B0;
        const TI *A2 = nd > 2 ? (const TI *)a[2] : A0, *B2 = nd > 2 ? (const TI *)b[2] : B0;
        if (nd == 1) k_segdot1<TI, NV, 1><<<g, 256, 0, s>>>(nseg, segoff, cstart, nch, A0, B0, A1, B1, A2, B2, part);
        else if (nd == 2) k_segdot1<TI, NV, 2><<<g, 256, 0, s>>>(nseg, segoff, cstart, nch, A0, B0, A1, B1, A2, B2, part);
        else k_segdot1<TI, NV, 3><<<g, 256, 0, s>>>(nseg, segoff, cstart, nch, A0, B0, A1, B1, A2, B2, part);
    }
    k_segdot2<<<(unsigned)(nseg * nd * NV), 256, 0, s>>>(nseg, nd * NV, NV, cstart, nch, part, out);
}

void seg_dots(Prec in, int nv, int nseg, const i64 *segoff, const i64 *cstart, i64 nchunks, int nd,
              const void *const *a, const void *const *b, double *part, double *out, cudaStream_t s) {
    if (in == Prec::F64) {
#define F(NV) segdots_t<double, NV>(nseg, segoff, cstart, nchunks, nd, a, b, part, out, s)
        switch (nv) {
        case 1: F(1); break;
        case 2: F(2); break;
        case 4: F(4); break;
        case 8: F(8); break;
        case 16: F(16); break;
        case 32: F(32); break;
        default: break;
        }
#undef F
    } else {
#define F(NV) segdots_t<float, NV>(nseg, segoff, cstart, nchunks, nd, a, b, part, out, s)
        switch (nv) {
        case 1: F(1); break;
        case 2: F(2); break;
        case 4: F(4); break;
        case 8: F(8); break;
        case 16: F(16); break;
        case 32: F(32); break;
        default: break;
        }
#undef F
    }
}

void seg_blas(int nv, int nseg, const i64 *segoff, i64 n, int op, const double *a, const double *x,
              const double *b, const double *y, const double *c, double *z, cudaStream_t s) {
    const i64 total = n * nv;
    if (total <= 0) return;
    const unsigned g = (unsigned)((total + 255) / 256);
    note_launch();
    if (op == 0) k_segblas<0><<<g, 256, 0, s>>>(nv, nseg, segoff, total, a, x, b, y, c, z);
    else k_segblas<1><<<g, 256, 0, s>>>(nv, nseg, segoff, total, a, x, b, y, c, z);
}

void batch_init(int nsc, const double *res0, double rel, double abs_tol, double *tol2, double *iconv,
                int *conv_it, int *ctr, cudaStream_t s) {
    note_launch();
    k_binit<<<1, 1024, 0, s>>>(nsc, res0, rel, abs_tol, tol2, iconv, conv_it, ctr);
}

void batch_omega(int nsc, const double *s2, const double *s3, const double *s4, const double *alpha,
                 const double *iconv, double *omega, double *res, double *ac, double *oc, cudaStream_t s) {
    note_launch();
    k_bomega<<<(unsigned)((nsc + 127) / 128), 128, 0, s>>>(nsc, s2, s3, s4, alpha, iconv, omega, res, ac, oc);
}

void batch_check(int nsc, const double *res, const double *tol2, double *iconv, int *conv_it,
                 double *res_last, int *ctr, int max_iters, unsigned long long handle, int use_graph,
                 cudaStream_t s) {
    note_launch();
    k_bcheck<<<1, 1024, 0, s>>>(nsc, res, tol2, iconv, conv_it, res_last, ctr, max_iters,
                                (cudaGraphConditionalHandle)handle, use_graph);
}

}  // namespace xk
