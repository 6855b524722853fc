// Kernels of the learned initial guess: a 3-D convolutional encoder-decoder
// trained and evaluated on the GPU (sm_100a).
//
// Tensors are channels-last BF16 volumes [nb][d][h][w][cs] addressed through a
// channel window (c0, c) of a buffer with cs channels per voxel, so that the
// decoder's concatenations are plain channel offsets.  Channel counts and
// offsets are multiples of 16.  Weights are [cout][27][cin] BF16 (tap t =
// (dz+1)*9 + (dy+1)*3 + (dx+1)), biases FP32; every product is accumulated in
// FP32 on the tensor cores (mma.sync m16n8k16 BF16).
//
//   conv3d   : implicit GEMM, M = voxels (tiles of 128), N = cout (tiles of 16,
//              32 or 64), K = 27 taps x cin in chunks of 16 channels; A and B
//              chunks are staged in shared memory by cp.async (4-stage ring,
//              zero fill outside the volume), fragments by ldmatrix.  The
//              epilogue adds the bias, applies ReLU and stores BF16 (or adds
//              to the stored value, for gradients that meet at a skip).
//   wgrad    : dW[co][t][ci] += sum_p g[p][co] * in[p + off(t)][ci], one CTA
//              per (voxel slice, tap, 16-channel chunk of ci), operands loaded
//              transposed by ldmatrix.trans, FP32 atomics into dW.
//   backward data = conv3d of the gradient with the flipped, transposed
//              weights (weight_flip).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "kernels.cuh"
#include <cstdint>
#include <cstdio>

typedef __nv_bfloat16 bf16;

namespace {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

// 16-byte async copy global -> shared; src_bytes = 0 fills zeros
__device__ __forceinline__ void cp16(void *dst, const void *src, unsigned src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldm_x4(unsigned (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldm_x2(unsigned (&r)[2], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldm_x4_t(unsigned (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

// D = A (16x16, row) * B (16x8, col) + D, BF16 inputs, FP32 accumulate
__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared-memory rows of 16 channels (32 bytes): the two 16-byte halves of
// row r are swapped when bit 2 of r is set, so that 8 consecutive rows read by
// one ldmatrix hit 8 distinct bank groups.
__device__ __forceinline__ int sw32(int r, int h) { return r * 32 + ((h ^ ((r >> 2) & 1)) << 4); }

// Rows of nch 16-byte chunks (nch a power of two, >= 2): chunk index XOR a
// function of the row that spreads 8 consecutive rows over 8 bank groups.
__device__ __forceinline__ int swn(int r, int ch, int nch) {
    const int g = nch >= 8 ? 8 : nch;
    const int per = 8 / g;
    return r * nch * 16 + ((ch ^ ((r / per) & (g - 1))) << 4);
}

struct Vol {
    int nb, d, h, w;
    __host__ __device__ __forceinline__ i64 count() const { return (i64)nb * d * h * w; }
};

// neighbour of linear voxel v at tap t; -1 outside the volume
__device__ __forceinline__ i64 nbr(const Vol &g, i64 v, int t) {
    const int x = (int)(v % g.w);
    const i64 q = v / g.w;
    const int y = (int)(q % g.h);
    const i64 q2 = q / g.h;
    const int z = (int)(q2 % g.d);
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    const int zz = z + dz, yy = y + dy, xx = x + dx;
    if (zz < 0 || zz >= g.d || yy < 0 || yy >= g.h || xx < 0 || xx >= g.w) return -1;
    return v + ((i64)dz * g.h + dy) * g.w + dx;
}

constexpr int BM = 128;  // voxels per CTA tile
constexpr int NS = 4;    // pipeline stages

// conv3d: out[v][oc0 + n] (+)= act(bias[n] + sum_t sum_c in[v+off(t)][ic0 + c] w[n][t][c]);
// flags: 1 ReLU, 2 accumulate, 4 FP32 output (out is then a float buffer)
template <int BN>
__global__ void __launch_bounds__(128) k_conv3d(const bf16 *__restrict__ in, int ics, int ic0,
                                                int cin, const bf16 *__restrict__ w,
                                                const float *__restrict__ bias, bf16 *out, int ocs,
                                                int oc0, int cout, Vol g, int flags) {
    __shared__ __align__(128) unsigned char sa[NS][BM * 32];
    __shared__ __align__(128) unsigned char sb[NS][BN * 32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const i64 nvox = g.count();
    const i64 v0 = (i64)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int kc = cin / 16;          // channel chunks per tap
    const int nk = 27 * kc;           // K chunks
    const i64 myv = v0 + tid;         // the voxel whose A row this thread stages
    const bool vin = myv < nvox;
    int vx = 0, vy = 0, vz = 0;
    if (vin) {
        vx = (int)(myv % g.w);
        vy = (int)((myv / g.w) % g.h);
        vz = (int)((myv / ((i64)g.w * g.h)) % g.d);
    }

    auto stage = [&](int k, int s) {
        const int t = k / kc, cb = (k % kc) * 16;
        // A: 128 rows of 16 channels, two 16-byte halves each
        const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
        const bool inside = vin && (unsigned)(vz + dz) < (unsigned)g.d &&
                            (unsigned)(vy + dy) < (unsigned)g.h && (unsigned)(vx + dx) < (unsigned)g.w;
        const i64 src = inside ? myv + ((i64)dz * g.h + dy) * g.w + dx : -1;
        const bf16 *pa = in + (src < 0 ? 0 : src) * ics + ic0 + cb;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh)
            cp16(&sa[s][sw32(tid, hh)], pa + hh * 8, src < 0 ? 0u : 16u);
        // B: BN rows (output channels) of 16 k values
        for (int q = tid; q < BN * 2; q += 128) {
            const int r = q >> 1, hh = q & 1;
            const bf16 *pb = w + ((i64)(n0 + r) * 27 + t) * cin + cb + hh * 8;
            cp16(&sb[s][sw32(r, hh)], pb, 16u);
        }
    };

    float acc[2][BN / 8][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < BN / 8; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

#pragma unroll
    for (int s = 0; s < NS - 1; ++s) {
        if (s < nk) stage(s, s);
        cp_commit();
    }
    for (int k = 0; k < nk; ++k) {
        cp_wait<NS - 2>();
        __syncthreads();
        if (k + NS - 1 < nk) stage(k + NS - 1, (k + NS - 1) % NS);
        cp_commit();
        const int s = k % NS;
        unsigned a[2][4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = warp * 32 + i * 16 + (lane & 15);
            ldm_x4(a[i], &sa[s][sw32(r, lane >> 4)]);
        }
#pragma unroll
        for (int j = 0; j < BN / 16; ++j) {
            // two n8 tiles: lanes 0-7 rows n 0-7 k0, 8-15 n 0-7 k8, 16-23 n 8-15 k0, 24-31 n 8-15 k8
            const int r = j * 16 + (lane & 7) + ((lane >> 4) << 3);
            unsigned bq[4];
            ldm_x4(bq, &sb[s][sw32(r, (lane >> 3) & 1)]);
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                mma16816(acc[i][2 * j], a[i], bq[0], bq[1]);
                mma16816(acc[i][2 * j + 1], a[i], bq[2], bq[3]);
            }
        }
        if (BN % 16) {
            const int j = BN / 16;
            const int r = j * 16 + (lane & 7);
            unsigned bq[2];
            ldm_x2(bq, &sb[s][sw32(r, (lane >> 3) & 1)]);
#pragma unroll
            for (int i = 0; i < 2; ++i) mma16816(acc[i][2 * j], a[i], bq[0], bq[1]);
        }
    }
    cp_wait<0>();
    // epilogue: rows g = lane/4 (+8), columns 2*(lane%4) (+1)
    const bool relu = flags & 1, accum = flags & 2, f32out = flags & 4;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < BN / 8; ++j)
#pragma unroll
            for (int hr = 0; hr < 2; ++hr) {
                const i64 v = v0 + warp * 32 + i * 16 + (lane >> 2) + hr * 8;
                if (v >= nvox) continue;
                const int n = n0 + j * 8 + 2 * (lane & 3);
                float y0 = acc[i][j][2 * hr], y1 = acc[i][j][2 * hr + 1];
                if (bias) {
                    y0 += bias[n];
                    y1 += bias[n + 1];
                }
                if (relu) {
                    y0 = fmaxf(y0, 0.f);
                    y1 = fmaxf(y1, 0.f);
                }
                if (f32out) {
                    float2 *pf = reinterpret_cast<float2 *>(reinterpret_cast<float *>(out) + v * ocs + oc0 + n);
                    if (accum) {
                        const float2 o = *pf;
                        y0 += o.x;
                        y1 += o.y;
                    }
                    *pf = make_float2(y0, y1);
                    continue;
                }
                __nv_bfloat162 *po = reinterpret_cast<__nv_bfloat162 *>(out + v * ocs + oc0 + n);
                if (accum) {
                    const float2 o = __bfloat1622float2(*po);
                    y0 += o.x;
                    y1 += o.y;
                }
                *po = __floats2bfloat162_rn(y0, y1);
            }
}

// conv3d on boxes: the CTA's 128 output voxels form a bz x by x bx box (the
// volume's sides are multiples of it); for every 16-channel chunk the box's
// halo ((bz+2)(by+2)(bx+2) voxels) and the chunk's weights for all 27 taps are
// staged once in shared memory, and the A operand of tap t is read by
// ldmatrix straight from the halo with per-lane row addresses, so each input
// voxel is fetched once per chunk instead of once per tap.  Same result
// definition as k_conv3d (the FP32 summation runs chunk-major).
template <int BN>
__global__ void __launch_bounds__(128) k_conv3d_box(const bf16 *__restrict__ in, int ics, int ic0,
                                                    int cin, const bf16 *__restrict__ w,
                                                    const float *__restrict__ bias, bf16 *out, int ocs,
                                                    int oc0, int cout, Vol g, int bz, int by, int bx,
                                                    int flags) {
    extern __shared__ __align__(128) unsigned char dyn[];
    const int hz = bz + 2, hy = by + 2, hx = bx + 2, nh = hz * hy * hx;
    unsigned char *sa = dyn;                 // nh rows of 32 bytes
    unsigned char *sb = dyn + nh * 32;       // 27 * BN rows of 32 bytes
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // box origin
    const int nbx = g.w / bx, nby = g.h / by, nbz = g.d / bz;
    int q = blockIdx.x;
    const int ix = q % nbx; q /= nbx;
    const int iy = q % nby; q /= nby;
    const int iz = q % nbz;
    const int b = q / nbz;
    const int x0 = ix * bx, y0 = iy * by, z0 = iz * bz;
    const int n0 = blockIdx.y * BN;
    const int kc = cin / 16;

    float acc[2][BN / 8][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < BN / 8; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    // halo row of this lane's A rows, relative to the tap offset (0,0,0)
    int hrow[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int m = warp * 32 + i * 16 + (lane & 15);
        const int mx = m % bx, my = (m / bx) % by, mz = m / (bx * by);
        hrow[i] = (mz * hy + my) * hx + mx;
    }
    for (int c = 0; c < kc; ++c) {
        const int cb = c * 16;
        __syncthreads();  // the previous chunk's reads are done
        for (int r = tid; r < nh * 2; r += 128) {
            const int hrw = r >> 1, hh = r & 1;
            const int lx = hrw % hx, ly = (hrw / hx) % hy, lz = hrw / (hx * hy);
            const int gx = x0 + lx - 1, gy = y0 + ly - 1, gz = z0 + lz - 1;
            const bool inside = (unsigned)gx < (unsigned)g.w && (unsigned)gy < (unsigned)g.h &&
                                (unsigned)gz < (unsigned)g.d;
            const i64 v = inside ? (((i64)b * g.d + gz) * g.h + gy) * g.w + gx : 0;
            cp16(sa + sw32(hrw, hh), in + v * ics + ic0 + cb + hh * 8, inside ? 16u : 0u);
        }
        for (int r = tid; r < 27 * BN * 2; r += 128) {
            const int row = r >> 1, hh = r & 1;  // row = t * BN + n
            const int t = row / BN, nn = row % BN;
            cp16(sb + sw32(row, hh), w + ((i64)(n0 + nn) * 27 + t) * cin + cb + hh * 8, 16u);
        }
        cp_commit();
        cp_wait<0>();
        __syncthreads();
#pragma unroll 1
        for (int t = 0; t < 27; ++t) {
            const int toff = ((t / 9) * hy + (t / 3) % 3) * hx + t % 3;
            unsigned a[2][4];
#pragma unroll
            for (int i = 0; i < 2; ++i) ldm_x4(a[i], sa + sw32(hrow[i] + toff, lane >> 4));
#pragma unroll
            for (int j = 0; j < BN / 16; ++j) {
                const int r = t * BN + j * 16 + (lane & 7) + ((lane >> 4) << 3);
                unsigned bq[4];
                ldm_x4(bq, sb + sw32(r, (lane >> 3) & 1));
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    mma16816(acc[i][2 * j], a[i], bq[0], bq[1]);
                    mma16816(acc[i][2 * j + 1], a[i], bq[2], bq[3]);
                }
            }
        }
    }
    const bool relu = flags & 1, accum = flags & 2, f32out = flags & 4;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < BN / 8; ++j)
#pragma unroll
            for (int hr = 0; hr < 2; ++hr) {
                const int m = warp * 32 + i * 16 + (lane >> 2) + hr * 8;
                const int mx = m % bx, my = (m / bx) % by, mz = m / (bx * by);
                const i64 v = (((i64)b * g.d + z0 + mz) * g.h + y0 + my) * g.w + x0 + mx;
                const int n = n0 + j * 8 + 2 * (lane & 3);
                float y0v = acc[i][j][2 * hr], y1v = acc[i][j][2 * hr + 1];
                if (bias) {
                    y0v += bias[n];
                    y1v += bias[n + 1];
                }
                if (relu) {
                    y0v = fmaxf(y0v, 0.f);
                    y1v = fmaxf(y1v, 0.f);
                }
                if (f32out) {
                    float2 *pf = reinterpret_cast<float2 *>(reinterpret_cast<float *>(out) + v * ocs + oc0 + n);
                    if (accum) {
                        const float2 o = *pf;
                        y0v += o.x;
                        y1v += o.y;
                    }
                    *pf = make_float2(y0v, y1v);
                    continue;
                }
                __nv_bfloat162 *po = reinterpret_cast<__nv_bfloat162 *>(out + v * ocs + oc0 + n);
                if (accum) {
                    const float2 o = __bfloat1622float2(*po);
                    y0v += o.x;
                    y1v += o.y;
                }
                *po = __floats2bfloat162_rn(y0v, y1v);
            }
}

// wgrad: dw[co][t][ci] += sum over the CTA's voxel slice of g[p][co] * in[p + off(t)][ci]
// grid (slices, 27, cin/16); 4 warps split the slice, then reduce in shared memory.
template <int CO>
__global__ void __launch_bounds__(128) k_wgrad(const bf16 *__restrict__ in, int ics, int ic0,
                                               int cin, const bf16 *__restrict__ gr, int gcs,
                                               int gc0, float *dw, Vol g, int slice) {
    constexpr int KS = 64;             // voxels per staged step (16 per warp)
    constexpr int NCH = CO / 8;        // 16-byte chunks per gradient row
    __shared__ __align__(128) unsigned char sg[2][KS * CO * 2];
    __shared__ __align__(128) unsigned char si[2][KS * 32];
    __shared__ float red[4][256];  // partial sums of warps 1..3, one 16-row group at a time
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t = blockIdx.y, cb = blockIdx.z * 16;
    const i64 nvox = g.count();
    const i64 p0 = (i64)blockIdx.x * slice, p1 = min(nvox, p0 + slice);
    const int nsteps = (int)((p1 - p0 + KS - 1) / KS);

    auto stage = [&](int st, int s) {
        const i64 pb = p0 + (i64)st * KS;
        for (int q = tid; q < KS * NCH; q += 128) {
            const int r = q / NCH, ch = q % NCH;
            const i64 p = pb + r;
            const bool ok = p < p1;
            cp16(&sg[s][swn(r, ch, NCH)], gr + (ok ? p : 0) * gcs + gc0 + ch * 8, ok ? 16u : 0u);
        }
        for (int q = tid; q < KS * 2; q += 128) {
            const int r = q >> 1, hh = q & 1;
            const i64 p = pb + r;
            const i64 src = p < p1 ? nbr(g, p, t) : -1;
            cp16(&si[s][sw32(r, hh)], in + (src < 0 ? 0 : src) * ics + ic0 + cb + hh * 8,
                 src < 0 ? 0u : 16u);
        }
    };

    float acc[CO / 16][2][4];
#pragma unroll
    for (int m = 0; m < CO / 16; ++m)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.f;

    if (nsteps > 0) stage(0, 0);
    cp_commit();
    for (int st = 0; st < nsteps; ++st) {
        if (st + 1 < nsteps) stage(st + 1, (st + 1) & 1);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        const int s = st & 1;
        const int rb = warp * 16;  // this warp's 16 voxels of the step
        // B fragments (k = voxels, n = ci): trans loads of [p][ci]
        unsigned bq[4];
        {
            const int r = rb + (lane & 7) + (((lane >> 3) & 1) << 3);
            ldm_x4_t(bq, &si[s][sw32(r, lane >> 4)]);
        }
#pragma unroll
        for (int m = 0; m < CO / 16; ++m) {
            // A fragment (m = co, k = voxels): trans loads of [p][co]
            unsigned a[4];
            const int r = rb + (lane & 7) + ((lane >> 4) << 3);
            const int ch = m * 2 + ((lane >> 3) & 1);
            ldm_x4_t(a, &sg[s][swn(r, ch, NCH)]);
            mma16816(acc[m][0], a, bq[0], bq[1]);
            mma16816(acc[m][1], a, bq[2], bq[3]);
        }
        __syncthreads();
    }
    cp_wait<0>();
    // reduce the 4 warps' partial sums: warps 1..3 write, warp 0 adds, 16 co rows at a time
    float *dwt = dw + (i64)t * cin + cb;  // dw[co][t][ci] = dwt[co*27*cin + ci]
#pragma unroll
    for (int m = 0; m < CO / 16; ++m) {
        __syncthreads();
        if (warp > 0)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) red[warp][(j * 4 + e) * 32 + lane] = acc[m][j][e];
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    float v = acc[m][j][e] + red[1][(j * 4 + e) * 32 + lane] +
                              red[2][(j * 4 + e) * 32 + lane] + red[3][(j * 4 + e) * 32 + lane];
                    const int co = m * 16 + (lane >> 2) + (e >> 1) * 8;
                    const int ci = j * 8 + 2 * (lane & 3) + (e & 1);
                    atomicAdd(dwt + (i64)co * 27 * cin + ci, v);
                }
        }
    }
}

// w [cout][27][cin] -> wt [cin][27][cout] with taps reversed (backward data)
__global__ void k_weight_flip(const bf16 *__restrict__ w, bf16 *__restrict__ wt, int cout, int cin) {
    const i64 total = (i64)cout * 27 * cin;
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (i64)gridDim.x * blockDim.x) {
        const int ci = (int)(q % cin);
        const i64 r = q / cin;
        const int t = (int)(r % 27), co = (int)(r / 27);
        wt[((i64)ci * 27 + (26 - t)) * cout + co] = w[q];
    }
}

// g[p][gc0 + c] *= (act[p][ac0 + c] > 0)
__global__ void k_relu_bwd(bf16 *g, int gcs, int gc0, const bf16 *__restrict__ act, int acs, int ac0,
                           int c, i64 nvox) {
    const i64 total = nvox * c;
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (i64)gridDim.x * blockDim.x) {
        const i64 p = q / c;
        const int k = (int)(q % c);
        if (!(__bfloat162float(act[p * acs + ac0 + k]) > 0.f)) g[p * gcs + gc0 + k] = __float2bfloat16(0.f);
    }
}

// db[c] += sum_p g[p][gc0 + c]; one thread per channel and voxel slice
__global__ void k_bias_grad(const bf16 *__restrict__ g, int gcs, int gc0, int c, i64 nvox,
                            i64 slice, float *db) {
    const int k = threadIdx.x % c;
    const int lanes = blockDim.x / c;
    const i64 p0 = (i64)blockIdx.x * slice, p1 = min(nvox, p0 + slice);
    float s = 0.f;
    for (i64 p = p0 + threadIdx.x / c; p < p1; p += lanes) s += __bfloat162float(g[p * gcs + gc0 + k]);
    atomicAdd(db + k, s);
}

// Elementwise volume kernels work on groups of 8 channels (16 bytes), which
// every channel count and offset here allows (multiples of 16).
struct Oct {
    float v[8];
};
__device__ __forceinline__ Oct ld8(const bf16 *p) {
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
    Oct o;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 f = __bfloat1622float2(h[k]);
        o.v[2 * k] = f.x;
        o.v[2 * k + 1] = f.y;
    }
    return o;
}
__device__ __forceinline__ void st8(bf16 *p, const Oct &o) {
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(o.v[2 * k], o.v[2 * k + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}

// 2x2x2 average pooling of volume g (even sides): one thread per coarse voxel
// and 8 channels
__global__ void k_pool2(const bf16 *__restrict__ in, int ics, int ic0, bf16 *out, int ocs, int oc0,
                        int c, Vol g) {
    const int D = g.d / 2, H = g.h / 2, W = g.w / 2, c8 = c / 8;
    const i64 total = (i64)g.nb * D * H * W * c8;
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (i64)gridDim.x * blockDim.x) {
        const int k = (int)(q % c8) * 8;
        const i64 cv = q / c8;
        i64 r = cv;
        const int x = (int)(r % W); r /= W;
        const int y = (int)(r % H); r /= H;
        const int z = (int)(r % D);
        const i64 b = r / D;
        Oct s;
#pragma unroll
        for (int e = 0; e < 8; ++e) s.v[e] = 0.f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const i64 v = ((b * g.d + 2 * z + (o >> 2)) * g.h + 2 * y + ((o >> 1) & 1)) * g.w + 2 * x + (o & 1);
            const Oct t = ld8(in + v * ics + ic0 + k);
#pragma unroll
            for (int e = 0; e < 8; ++e) s.v[e] += t.v[e];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) s.v[e] *= 0.125f;
        st8(out + cv * ocs + oc0 + k, s);
    }
}

// nearest upsampling of a (d/2, h/2, w/2) volume to g; mode 1 adds the
// pooled-gradient share (x 1/8) for the pooling backward, mode 0 copies.
// One thread per coarse voxel and 8 channels writes its 8 fine voxels.
__global__ void k_up2(const bf16 *__restrict__ in, int ics, int ic0, bf16 *out, int ocs, int oc0,
                      int c, Vol g, int mode) {
    const int D = g.d / 2, H = g.h / 2, W = g.w / 2, c8 = c / 8;
    const i64 total = (i64)g.nb * D * H * W * c8;
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (i64)gridDim.x * blockDim.x) {
        const int k = (int)(q % c8) * 8;
        const i64 cv = q / c8;
        i64 r = cv;
        const int x = (int)(r % W); r /= W;
        const int y = (int)(r % H); r /= H;
        const int z = (int)(r % D);
        const i64 b = r / D;
        const Oct src = ld8(in + cv * ics + ic0 + k);
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const i64 v = ((b * g.d + 2 * z + (o >> 2)) * g.h + 2 * y + ((o >> 1) & 1)) * g.w + 2 * x + (o & 1);
            bf16 *po = out + v * ocs + oc0 + k;
            if (mode == 1) {
                Oct t = ld8(po);
#pragma unroll
                for (int e = 0; e < 8; ++e) t.v[e] += src.v[e] * 0.125f;
                st8(po, t);
            } else {
                st8(po, src);
            }
        }
    }
}

// backward of nearest upsampling: dIn[coarse] = sum of the 8 fine gradients
__global__ void k_up2_bwd(const bf16 *__restrict__ gfine, int gcs, int gc0, bf16 *gin, int ics,
                          int ic0, int c, Vol g) {
    const int D = g.d / 2, H = g.h / 2, W = g.w / 2, c8 = c / 8;
    const i64 total = (i64)g.nb * D * H * W * c8;
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (i64)gridDim.x * blockDim.x) {
        const int k = (int)(q % c8) * 8;
        const i64 cv = q / c8;
        i64 r = cv;
        const int x = (int)(r % W); r /= W;
        const int y = (int)(r % H); r /= H;
        const int z = (int)(r % D);
        const i64 b = r / D;
        Oct s;
#pragma unroll
        for (int e = 0; e < 8; ++e) s.v[e] = 0.f;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            const i64 v = ((b * g.d + 2 * z + (o >> 2)) * g.h + 2 * y + ((o >> 1) & 1)) * g.w + 2 * x + (o & 1);
            const Oct t = ld8(gfine + v * gcs + gc0 + k);
#pragma unroll
            for (int e = 0; e < 8; ++e) s.v[e] += t.v[e];
        }
        st8(gin + cv * ics + ic0 + k, s);
    }
}

// loss = mean (pred - target)^2 over nvox voxels (pred = channel pc0 of an
// FP32 volume); grad[p][0] = 2 (pred - target) / nvox, other grad channels 0
__global__ void k_mse(const float *__restrict__ pred, int pcs, int pc0, const float *__restrict__ tgt,
                      bf16 *grad, int gcs, i64 nvox, float *loss) {
    float s = 0.f;
    for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < nvox; p += (i64)gridDim.x * blockDim.x) {
        const float d = pred[p * pcs + pc0] - tgt[p];
        s += d * d;
        if (grad) {
            for (int k = 0; k < gcs; ++k) grad[p * gcs + k] = __float2bfloat16(0.f);
            grad[p * gcs] = __float2bfloat16(2.f * d / (float)nvox);
        }
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / (float)nvox);
}

// Adam on FP32 master weights; refreshes the BF16 copy
__global__ void k_adam(float *w, const float *__restrict__ gw, float *m, float *v, bf16 *wb, i64 n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (i64)gridDim.x * blockDim.x) {
        const float gq = gw[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float wq = w[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
        w[q] = wq;
        if (wb) wb[q] = __float2bfloat16(wq);
    }
}

// network input: channel 0 = a[p], channel 1 = b[p], channels 2..15 = 0
__global__ void k_pack2(const float *__restrict__ a, const float *__restrict__ b, bf16 *out, i64 nvox) {
    for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < nvox; p += (i64)gridDim.x * blockDim.x) {
        uint4 u0 = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<__nv_bfloat162 *>(&u0.x) = __floats2bfloat162_rn(a[p], b[p]);
        uint4 *po = reinterpret_cast<uint4 *>(out + p * 16);
        po[0] = u0;
        po[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// f32 out[p] = scale[p / per] * bf16 in[p][c0]
__global__ void k_unpack(const float *__restrict__ in, int cs, int c0, const float *__restrict__ scale,
                         i64 per, float *out, i64 nvox) {
    for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < nvox; p += (i64)gridDim.x * blockDim.x)
        out[p] = in[p * cs + c0] * (scale ? scale[p / per] : 1.f);
}

// x0 in the solver's block-vector layout: x[v * nv + s] = scale[s] * in[s * per + v][c0]
__global__ void k_unpack_x0(const float *__restrict__ in, int cs, int c0, const float *__restrict__ scale,
                            int nv, i64 per, double *x) {
    const i64 total = per * nv;
    for (i64 q = (i64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (i64)gridDim.x * blockDim.x) {
        const i64 v = q / nv;
        const int sidx = (int)(q % nv);
        x[q] = (double)in[(sidx * per + v) * cs + c0] * (double)scale[sidx];
    }
}

// ---------------------------------------------------------------- tcgen05 conv3d
// The same convolution on the 5th-generation tensor cores: implicit GEMM with
// M = 128 voxels, N = BN output channels, K = 16 channels of one tap per
// step.  The 128 threads stage A (the tap's shifted voxel rows) and B (the
// weights) by cp.async exactly as k_conv3d does: 32-byte rows with the
// 16-byte halves swapped on bit 2 of the row, which is the canonical K-major
// SWIZZLE_32B layout of the UMMA shared-memory descriptors (8-row groups 256
// bytes apart).  One thread issues tcgen05.mma (kind::f16, BF16 x BF16 ->
// FP32) into a TMEM accumulator of BN columns and commits each step to the
// stage's mbarrier, which tells the producers when the stage may be
// refilled.  The epilogue reads TMEM with tcgen05.ld (warp w: lanes 32w ..
// 32w+31 = its voxels).  Every mbarrier wait is bounded; on expiry the error
// word is set, the CTA stops issuing and frees its TMEM after the tensor
// pipe has drained (bounded as well).
__device__ int g_tc_err;

__device__ __forceinline__ unsigned long long tc_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void tc_mbar_init(unsigned long long *b) {
    asm volatile("mbarrier.init.shared.b64 [%0], 1;" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool tc_mbar_try(unsigned long long *b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool tc_mbar_wait(unsigned long long *b, unsigned parity) {
    if (tc_mbar_try(b, parity)) return true;
    const unsigned long long t0 = tc_now();
    while (!tc_mbar_try(b, parity))
        if (tc_now() - t0 > 1000000000ull) return false;
    return true;
}
// K-major SWIZZLE_32B shared-memory matrix descriptor: start address, leading
// byte offset 1 (unused within one swizzle atom), stride between 8-row groups
// 256 bytes, descriptor version 1, layout type 6
__device__ __forceinline__ unsigned long long tc_desc(const void *p) {
    const unsigned long long a = (smem_u32(p) & 0x3FFFFu) >> 4;
    return a | (1ull << 16) | ((unsigned long long)(256 >> 4) << 32) | (1ull << 46) | (6ull << 61);
}

template <int BN>
__global__ void __launch_bounds__(128) k_conv3d_tc(const bf16 *__restrict__ in, int ics, int ic0, int cin,
                                                   const bf16 *__restrict__ w, const float *__restrict__ bias,
                                                   bf16 *out, int ocs, int oc0, int cout, Vol g, int flags) {
    constexpr int TCOLS = BN < 32 ? 32 : BN;  // TMEM columns (a power of two >= 32)
    __shared__ __align__(1024) unsigned char sa[NS][BM * 32];
    __shared__ __align__(1024) unsigned char sb[NS][BN * 32 < 1024 ? 1024 : BN * 32];
    __shared__ __align__(8) unsigned long long mbar[NS];
    __shared__ unsigned s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const i64 nvox = g.count();
    const i64 v0 = (i64)blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    const int kc = cin / 16;
    const int nk = 27 * kc;
    const i64 myv = v0 + tid;
    const bool vin = myv < nvox;
    int vx = 0, vy = 0, vz = 0;
    if (vin) {
        vx = (int)(myv % g.w);
        vy = (int)((myv / g.w) % g.h);
        vz = (int)((myv / ((i64)g.w * g.h)) % g.d);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int q = 0; q < NS; ++q) tc_mbar_init(&mbar[q]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = s_tmem;
    // instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
    // N = BN, M = 128
    const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(BN >> 3) << 17) | ((128u >> 4) << 24);

    auto stage = [&](int k, int st) {
        const int t = k / kc, cb = (k % kc) * 16;
        const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
        const bool inside = vin && (unsigned)(vz + dz) < (unsigned)g.d && (unsigned)(vy + dy) < (unsigned)g.h &&
                            (unsigned)(vx + dx) < (unsigned)g.w;
        const i64 src = inside ? myv + ((i64)dz * g.h + dy) * g.w + dx : -1;
        const bf16 *pa = in + (src < 0 ? 0 : src) * ics + ic0 + cb;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) cp16(&sa[st][sw32(tid, hh)], pa + hh * 8, src < 0 ? 0u : 16u);
        for (int q = tid; q < BN * 2; q += 128) {
            const int r = q >> 1, hh = q & 1;
            const bf16 *pb = w + ((i64)(n0 + r) * 27 + t) * cin + cb + hh * 8;
            cp16(&sb[st][sw32(r, hh)], pb, 16u);
        }
    };
    unsigned uses[NS] = {0u, 0u, 0u, 0u};  // completed MMA phases awaited per stage
    bool ok = true;
#pragma unroll
    for (int q = 0; q < NS - 1; ++q) {
        if (q < nk) stage(q, q);
        cp_commit();
    }
    for (int k = 0; k < nk; ++k) {
        // refill the stage that step k-1 read once its MMA has completed
        const int kn = k + NS - 1;
        if (kn < nk) {
            const int st = kn % NS;
            if (k >= 1) {
                if (ok && !tc_mbar_wait(&mbar[st], uses[st] & 1u)) ok = false;
                uses[st]++;
            }
            stage(kn, st);
        }
        cp_commit();
        cp_wait<NS - 2>();
        // the copies of step k are complete: publish them to the tensor core
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        ok = __syncthreads_and(ok) != 0;
        if (!ok) break;
        if (tid == 0) {
            const int st = k % NS;
            const unsigned long long da = tc_desc(&sa[st][0]), db = tc_desc(&sb[st][0]);
            const unsigned acc = k > 0 ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
                "l"(da), "l"(db), "r"(idesc), "r"(acc)
                : "memory");
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar[st]))
                         : "memory");
        }
    }
    cp_wait<0>();
    // the last step's commit completes after every earlier MMA
    if (ok && nk > 0) {
        const int st = (nk - 1) % NS;
        // phases of this stage awaited so far, plus the ones not awaited
        unsigned ph = uses[st];
        for (int k = st; k < nk; k += NS) {
            if ((unsigned)(k / NS) < ph) continue;
            if (!tc_mbar_wait(&mbar[st], (unsigned)(k / NS) & 1u)) { ok = false; break; }
        }
    }
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        const bool relu = flags & 1, accum = flags & 2, f32out = flags & 4;
        const i64 v = v0 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
            unsigned r[16];
            const unsigned ta = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(ta));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (v >= nvox) continue;
#pragma unroll
            for (int e = 0; e < 16; e += 2) {
                const int n = n0 + c0 + e;
                float y0 = __uint_as_float(r[e]), y1 = __uint_as_float(r[e + 1]);
                if (bias) {
                    y0 += bias[n];
                    y1 += bias[n + 1];
                }
                if (relu) {
                    y0 = fmaxf(y0, 0.f);
                    y1 = fmaxf(y1, 0.f);
                }
                if (f32out) {
                    float2 *pf = reinterpret_cast<float2 *>(reinterpret_cast<float *>(out) + v * ocs + oc0 + n);
                    if (accum) {
                        const float2 o = *pf;
                        y0 += o.x;
                        y1 += o.y;
                    }
                    *pf = make_float2(y0, y1);
                } else {
                    __nv_bfloat162 *po = reinterpret_cast<__nv_bfloat162 *>(out + v * ocs + oc0 + n);
                    if (accum) {
                        const float2 o = __bfloat1622float2(*po);
                        y0 += o.x;
                        y1 += o.y;
                    }
                    *po = __floats2bfloat162_rn(y0, y1);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(&g_tc_err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
    }
}

// the tcgen05 kernel is used when switched on (xcnn_set_tc_conv(1))
int g_tc_conv = 0;

// the box kernel is the default; xcnn_set_box_conv(0) selects the
// voxel-tile kernel (both compute the same convolution)
int g_box_conv = 1;
bool box_conv_enabled() { return g_box_conv != 0; }

int grid_for(i64 n) {
    i64 g = (n + 255) / 256;
    return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

int last_err() {
    xk::note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "xcnn: %s\n", cudaGetErrorString(e));
        return 3;
    }
    return 0;
}

bool ch_ok(int c) { return c > 0 && c % 16 == 0; }

}  // namespace

extern "C" {

int xcnn_conv3d(const void *in, int ics, int ic0, int cin, const void *w, const float *bias, void *out,
                int ocs, int oc0, int cout, int nb, int d, int h, int wd, int flags, void *stream) {
    if (!ch_ok(cin) || !ch_ok(cout) || ic0 % 16 || oc0 % 16 || ics % 16 || ocs % 16 ||
        ic0 + cin > ics || oc0 + cout > ocs || nb <= 0 || d <= 0 || h <= 0 || wd <= 0)
        return 2;
    Vol g{nb, d, h, wd};
    const i64 nvox = (i64)nb * d * h * wd;
    cudaStream_t s = (cudaStream_t)stream;
    const int bn = cout % 64 == 0 ? 64 : (cout % 32 == 0 ? 32 : 16);
    const bf16 *pi = (const bf16 *)in;
    const bf16 *pw = (const bf16 *)w;
    bf16 *po = (bf16 *)out;
    if (g_tc_conv) {
        dim3 grid((unsigned)((nvox + BM - 1) / BM), (unsigned)(cout / bn));
        if (bn == 64) k_conv3d_tc<64><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, flags);
        else if (bn == 32) k_conv3d_tc<32><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, flags);
        else k_conv3d_tc<16><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, flags);
        return last_err();
    }
    // box kernel when the volume tiles into 128-voxel boxes of at least 8 x 8
    // in (y, x): sides multiples of 8 and a depth that is a multiple of 2
    const int bx = 8, by = 8, bz = 2;
    if (box_conv_enabled() && wd % bx == 0 && h % by == 0 && d % bz == 0) {
        dim3 gb((unsigned)((i64)nb * (d / bz) * (h / by) * (wd / bx)), (unsigned)(cout / bn));
        const int sm = (bz + 2) * (by + 2) * (bx + 2) * 32 + 27 * bn * 32;
#define LB(BN)                                                                                     \
    {                                                                                              \
        auto k = k_conv3d_box<BN>;                                                                 \
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);                 \
        k<<<gb, 128, sm, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, bz, by, bx, flags); \
    }
        if (bn == 64) LB(64) else if (bn == 32) LB(32) else LB(16)
#undef LB
        return last_err();
    }
    dim3 grid((unsigned)((nvox + BM - 1) / BM), (unsigned)(cout / bn));
    if (bn == 64) k_conv3d<64><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, flags);
    else if (bn == 32) k_conv3d<32><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, flags);
    else k_conv3d<16><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pw, bias, po, ocs, oc0, cout, g, flags);
    return last_err();
}

int xcnn_conv3d_wgrad(const void *in, int ics, int ic0, int cin, const void *grad, int gcs, int gc0,
                      int cout, float *dw, int nb, int d, int h, int wd, void *stream) {
    if (!ch_ok(cin) || ic0 % 16 || ics % 16 || gc0 % 16 || gcs % 16 || ic0 + cin > ics ||
        gc0 + cout > gcs || !(cout == 16 || cout == 32 || cout == 64 || cout == 128))
        return 2;
    Vol g{nb, d, h, wd};
    const i64 nvox = (i64)nb * d * h * wd;
    // slices of at least 512 voxels, about 4 CTAs per SM in total
    const i64 want = (i64)148 * 4 / (27 * (cin / 16));
    i64 slice = (nvox + (want > 1 ? want : 1) - 1) / (want > 1 ? want : 1);
    slice = ((slice < 512 ? 512 : slice) + 63) / 64 * 64;
    dim3 grid((unsigned)((nvox + slice - 1) / slice), 27, (unsigned)(cin / 16));
    cudaStream_t s = (cudaStream_t)stream;
    const bf16 *pi = (const bf16 *)in;
    const bf16 *pg = (const bf16 *)grad;
    switch (cout) {
    case 16: k_wgrad<16><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pg, gcs, gc0, dw, g, (int)slice); break;
    case 32: k_wgrad<32><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pg, gcs, gc0, dw, g, (int)slice); break;
    case 64: k_wgrad<64><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pg, gcs, gc0, dw, g, (int)slice); break;
    default: k_wgrad<128><<<grid, 128, 0, s>>>(pi, ics, ic0, cin, pg, gcs, gc0, dw, g, (int)slice); break;
    }
    return last_err();
}

int xcnn_weight_flip(const void *w, void *wt, int cout, int cin, void *stream) {
    const i64 n = (i64)cout * 27 * cin;
    k_weight_flip<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const bf16 *)w, (bf16 *)wt, cout, cin);
    return last_err();
}

int xcnn_relu_bwd(void *g, int gcs, int gc0, const void *act, int acs, int ac0, int c, int64_t nvox,
                  void *stream) {
    k_relu_bwd<<<grid_for(nvox * c), 256, 0, (cudaStream_t)stream>>>((bf16 *)g, gcs, gc0, (const bf16 *)act,
                                                                        acs, ac0, c, nvox);
    return last_err();
}

int xcnn_bias_grad(const void *g, int gcs, int gc0, int c, int64_t nvox, float *db, void *stream) {
    if (c <= 0 || c > 256 || 256 % c) return 2;
    const i64 slice = 4096;
    k_bias_grad<<<(unsigned)((nvox + slice - 1) / slice), 256, 0, (cudaStream_t)stream>>>(
        (const bf16 *)g, gcs, gc0, c, nvox, slice, db);
    return last_err();
}

int xcnn_pool2(const void *in, int ics, int ic0, void *out, int ocs, int oc0, int c, int nb, int d, int h,
               int w, void *stream) {
    if (d % 2 || h % 2 || w % 2 || c % 8 || ic0 % 8 || ics % 8 || oc0 % 8 || ocs % 8) return 2;
    Vol g{nb, d, h, w};
    k_pool2<<<grid_for(g.count() / 8 * (c / 8)), 256, 0, (cudaStream_t)stream>>>((const bf16 *)in, ics, ic0,
                                                                              (bf16 *)out, ocs, oc0, c, g);
    return last_err();
}

// fine volume (nb, d, h, w): mode 0 out = up(in); mode 1 out += up(in) / 8
int xcnn_up2(const void *in, int ics, int ic0, void *out, int ocs, int oc0, int c, int nb, int d, int h,
             int w, int mode, void *stream) {
    if (d % 2 || h % 2 || w % 2 || c % 8 || ic0 % 8 || ics % 8 || oc0 % 8 || ocs % 8) return 2;
    Vol g{nb, d, h, w};
    k_up2<<<grid_for(g.count() / 8 * (c / 8)), 256, 0, (cudaStream_t)stream>>>((const bf16 *)in, ics, ic0,
                                                                                 (bf16 *)out, ocs, oc0, c, g, mode);
    return last_err();
}

int xcnn_up2_bwd(const void *gfine, int gcs, int gc0, void *gin, int ics, int ic0, int c, int nb, int d,
                 int h, int w, void *stream) {
    if (d % 2 || h % 2 || w % 2 || c % 8 || gc0 % 8 || gcs % 8 || ic0 % 8 || ics % 8) return 2;
    Vol g{nb, d, h, w};
    k_up2_bwd<<<grid_for(g.count() / 8 * (c / 8)), 256, 0, (cudaStream_t)stream>>>(
        (const bf16 *)gfine, gcs, gc0, (bf16 *)gin, ics, ic0, c, g);
    return last_err();
}

int xcnn_mse(const void *pred, int pcs, int pc0, const float *tgt, void *grad, int gcs, int64_t nvox,
             float *loss, void *stream) {
    k_mse<<<grid_for(nvox), 256, 0, (cudaStream_t)stream>>>((const float *)pred, pcs, pc0, tgt, (bf16 *)grad,
                                                            gcs, nvox, loss);
    return last_err();
}

int xcnn_adam(float *w, const float *g, float *m, float *v, void *wb, int64_t n, float lr, float b1,
              float b2, float eps, int step, void *stream) {
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (bf16 *)wb, n, lr, b1, b2, eps, c1, c2);
    return last_err();
}

int xcnn_pack2(const float *a, const float *b, void *out, int64_t nvox, void *stream) {
    k_pack2<<<grid_for(nvox), 256, 0, (cudaStream_t)stream>>>(a, b, (bf16 *)out, nvox);
    return last_err();
}

int xcnn_unpack(const void *in, int cs, int c0, const float *scale, int64_t per, float *out, int64_t nvox,
                void *stream) {
    k_unpack<<<grid_for(nvox), 256, 0, (cudaStream_t)stream>>>((const float *)in, cs, c0, scale, per, out, nvox);
    return last_err();
}

int xcnn_unpack_x0(const void *in, int cs, int c0, const float *scale, int nv, int64_t per, double *x,
                   void *stream) {
    if (nv <= 0 || per <= 0 || !scale) return 2;
    k_unpack_x0<<<grid_for(per * nv), 256, 0, (cudaStream_t)stream>>>((const float *)in, cs, c0, scale, nv, per, x);
    return last_err();
}

int xcnn_set_tc_conv(int on) {
    const int old = g_tc_conv;
    g_tc_conv = on != 0;
    return old;
}
// 1 when a tcgen05 convolution gave up waiting on its tensor pipe since the
// last call (then cleared)
int xcnn_tc_error() {
    int h = 0;
    if (cudaMemcpyFromSymbol(&h, g_tc_err, sizeof(int)) != cudaSuccess) return -1;
    const int z = 0;
    if (h) cudaMemcpyToSymbol(g_tc_err, &z, sizeof(int));
    return h;
}
int xcnn_set_box_conv(int on) {
    const int old = g_box_conv;
    g_box_conv = on != 0;
    return old;
}

}  // extern "C"
