// Hybrid Gauss-Seidel sweep, one warp per hybrid block (sm_100a).
//
// The hybrid smoother (Gauss-Seidel inside each row block, Jacobi across the
// blocks; blas2.h:184-281 of the reference) runs one block as a chain of
// wavefront levels of a few tens of rows each.  Here one warp owns one block
// and each lane owns whole rows of a level (NV <= 16: all NV columns of its
// row; NV = 32: half a row), so a level needs no CTA barrier at all: the
// lanes' updates of the block's x values are made visible to the next level
// by __syncwarp.  A lane's row is NV independent FMA chains (CSR order, as in
// the oracle), which the warp issues back to back.
//
// Everything a level reads comes from shared memory:
//   * the level's record (column indices, values, row offsets, row ids,
//     inverse diagonals, and with the slot window the rows' slots and the
//     level's window load list) is copied by cp.async three levels ahead into
//     one of four fixed-size stage slots;
//   * the rows' t values are copied into the same record two levels ahead,
//     once the record's row ids are in;
//   * x: the block's whole x tile (XM 1), the slot window of the rows live at
//     once (XM 2; first-use rows copied kGsSlotAhead levels ahead), or a
//     per-level gather of the level's x values (XM 0; the rows' old x are
//     staged with t).
// Every copy is a 16-byte piece (4 or 8 bytes for rows narrower than 16
// bytes) on a 16-byte boundary; there is no spin-wait anywhere (cp.async
// groups complete by themselves).
//
// Padding entries (column -1 at a row's tail, rows padded to 4 entries, value
// +0) read a row of zeros: fma(-0, 0, s) == s exactly for every s, signed
// zeros included, so every sum equals the oracle's bit for bit.
#include "kernels.cuh"
#include <algorithm>

namespace xk {

template <int WB> struct WordT;
template <> struct WordT<16> { typedef int4 t; };
template <> struct WordT<8> { typedef int2 t; };
template <> struct WordT<4> { typedef int t; };

namespace {

__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// one B-byte global -> shared copy (B = 4, 8 or 16, naturally aligned)
template <int B> __device__ __forceinline__ void cpa(void *dst, const void *src) {
    static_assert(B == 4 || B == 8 || B == 16, "cp.async copies 4, 8 or 16 bytes");
    if (B == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(su32(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(su32(dst)), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ double mulrn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mulrn(float a, float b) { return __fmul_rn(a, b); }

// a lane's piece of a row: CW contiguous elements, moved as 16-byte words
// (or one 8- or 4-byte word when narrower)
template <class T, int CW> struct RowW {
    static constexpr int BYTES = CW * (int)sizeof(T);
    static constexpr int WB = BYTES >= 16 ? 16 : BYTES;
    static constexpr int NW = BYTES / WB;
};

// Rows in shared memory are stored as 16-byte chunks whose order is XOR-ed
// with the row's low bits (mask SWM): chunk j of row r sits at chunk
// position j ^ (r & SWM).  Lanes that read the same chunk of different rows
// then spread over the banks instead of queueing on the same four.  Rows
// narrower than 16 bytes are not swizzled (SWM = 0).
// ldrow/strow move the lane's CW elements of row r (lane part sub) between a
// row base in shared memory and registers; gstrow stores them to global
// memory (no swizzle).
template <class T, int CW, int SWM>
__device__ __forceinline__ void ldrow(const T *row, int r, int sub, T (&v)[CW]) {
    typedef RowW<T, CW> R;
    typedef typename WordT<R::WB>::t W;
#pragma unroll
    for (int k = 0; k < R::NW; ++k) {
        const int j = sub * R::NW + k;
        const W w = reinterpret_cast<const W *>(row)[R::WB == 16 ? (j ^ (r & SWM)) : j];
        memcpy(reinterpret_cast<char *>(v) + k * R::WB, &w, R::WB);
    }
}
template <class T, int CW, int SWM>
__device__ __forceinline__ void strow(T *row, int r, int sub, const T (&v)[CW]) {
    typedef RowW<T, CW> R;
    typedef typename WordT<R::WB>::t W;
#pragma unroll
    for (int k = 0; k < R::NW; ++k) {
        const int j = sub * R::NW + k;
        W w;
        memcpy(&w, reinterpret_cast<const char *>(v) + k * R::WB, R::WB);
        reinterpret_cast<W *>(row)[R::WB == 16 ? (j ^ (r & SWM)) : j] = w;
    }
}
template <class T, int CW> __device__ __forceinline__ void gstrow(T *p, const T (&v)[CW]) {
    typedef RowW<T, CW> R;
    typedef typename WordT<R::WB>::t W;
#pragma unroll
    for (int k = 0; k < R::NW; ++k) {
        W w;
        memcpy(&w, reinterpret_cast<const char *>(v) + k * R::WB, R::WB);
        reinterpret_cast<W *>(p)[k] = w;
    }
}

}  // namespace

// Byte offsets of the pieces of one level's record (ci at 0).  ne = entries
// (a multiple of 4), nr = rows rounded out to 4-row boundaries, nl = window
// load list length (even); every piece is a multiple of 16 bytes.
struct GswLay {
    int va, rp, row, di, sl, ld, t, xo, size;
};
__host__ __device__ __forceinline__ GswLay gsw_lay(int ne, int nr, int nl, int s, int nv, int xm) {
    GswLay y;
    int o = ne * 4;
    y.va = o;
    o += ne * s;
    y.rp = o;
    o += (nr + 4) * 4;
    y.row = o;
    o += nr * 4;
    y.di = o;
    o += nr * s;
    y.sl = o;
    if (xm == 2) o += nr * 4;
    y.ld = o;
    if (xm == 2) o += nl * 8;
    y.t = o;
    o += nr * nv * s;
    y.xo = o;
    if (xm == 0) o += nr * nv * s;
    y.size = o;
    return y;
}

// Record stages: a block's levels cycle through 4 stage slots; records are
// copied 3 levels ahead, t rows 2 levels ahead.
constexpr int kGswStages = 4;

// XM: 0 = per-level x gather, 1 = x tile of the block, 2 = slot window.
// One CTA (one warp) per hybrid block b: levels blev[b] .. blev[b + 1] of the
// level-ordered copy, descriptors desc[blev[b] + l] = {r0, r1, e0, e1}.
// Dynamic shared memory: x region (xoff bytes: the tile or window plus one
// zero row, or the gather buffer), the block's descriptor and window-range
// tables (lmax levels), then kGswStages record stages of recb bytes.
// Padding entries carry the value +0 and read the zero row (the gather
// writes zeros for them), so fma(-0, 0, s) == s leaves every sum unchanged.
template <class T, int NV, int XM>
__global__ void __launch_bounds__(32) k_gsw(const int4 *__restrict__ desc, const int *__restrict__ blev,
                                            const int *__restrict__ lrp, const int *__restrict__ lci,
                                            const T *__restrict__ lva, const int *__restrict__ lrow,
                                            const T *__restrict__ linvd, const T *__restrict__ t, T *x,
                                            const T *__restrict__ relax, i64 brows, i64 n, GsSlotWin sw, int recb,
                                            int lmax, int xoff) {
    constexpr int S = (int)sizeof(T);
    constexpr int CW = NV < 16 ? NV : 16;  // columns of a lane
    constexpr int TPR = NV / CW;           // lanes per row
    constexpr int RPP = 32 / TPR;          // rows per pass
    constexpr int PB = NV * S >= 16 ? 16 : NV * S;  // copy piece of an x / t row
    constexpr int PPR = NV * S / PB;                // pieces per row
    constexpr int PE = PB / S;                      // elements per piece
    constexpr int U = S == 8 ? 2 : 4;               // entries in flight per lane
    constexpr int CPR = NV * S / 16;                // 16-byte chunks per row (0: narrower)
    constexpr int SWM = PB == 16 ? (CPR >= 8 ? 7 : CPR - 1) : 0;
    constexpr int NS = kGswStages, DR = NS - 1, DT = 2;
    typedef typename WordT<PB>::t PW;
    extern __shared__ __align__(128) unsigned char dyn[];
    __shared__ GswLay s_lay[NS];  // layout of the record in each stage slot
    T *xs = reinterpret_cast<T *>(dyn);
    int4 *sdesc = reinterpret_cast<int4 *>(dyn + xoff);
    int2 *sldd = reinterpret_cast<int2 *>(dyn + xoff + lmax * 16);
    unsigned char *ring = dyn + xoff + ((lmax * 24 + 127) & ~127);

    const int lane = threadIdx.x, b = blockIdx.x;
    const int dbase = __ldg(blev + b), nlv = __ldg(blev + b + 1) - dbase;
    const i64 xbase = XM == 2 ? 0 : (i64)b * brows;
    const i64 zr = XM == 1 ? brows : XM == 2 ? (i64)sw.nslots : 0;  // the zero row
    for (int k = lane; k < nlv; k += 32) {
        sdesc[k] = __ldg(desc + dbase + k);
        if (XM == 2) sldd[k] = __ldg(sw.ldd + dbase + k);
    }
    if (XM != 0)
        for (int e = lane; e < NV; e += 32) xs[zr * NV + e] = T(0);
    const int sub = lane % TPR;
    // element offset of piece j of row r in shared memory (swizzled chunks)
    auto swz = [&](i64 r, int j) { return (j ^ ((int)r & SWM)) * PE; };
    // the block's x tile by cp.async (it joins the first group)
    const i64 xrows = XM == 1 ? min((i64)brows, n - xbase) : 0;
    if (XM == 1)
        for (i64 w = lane; w < xrows * PPR; w += 32)
            cpa<PB>(xs + (w / PPR) * NV + swz(w / PPR, (int)(w % PPR)), x + (xbase + w / PPR) * NV + (w % PPR) * PE);
    T rl[CW];
#pragma unroll
    for (int e = 0; e < CW; ++e) rl[e] = relax[sub * CW + e];
    __syncwarp();

    auto nlist = [&](int k) { return XM == 2 ? sldd[k].y - sldd[k].x : 0; };
    auto rec = [&](int k) { return ring + (k & (NS - 1)) * recb; };
    // level k's arrays, 16-byte pieces spread over the lanes; lane 0 records
    // the layout for the later readers of the stage slot
    auto stage_record = [&](int k) {
        const int4 d = sdesc[k];
        const int ne = d.w - d.z, ra = d.x & ~3, nr = ((d.y + 3) & ~3) - ra, nl = nlist(k);
        const GswLay y = gsw_lay(ne, nr, nl, S, NV, XM);
        if (lane == 0) s_lay[k & (NS - 1)] = y;
        unsigned char *a = rec(k);
        auto seg = [&](unsigned char *dst, const void *src, int bytes) {
            const unsigned char *s8 = reinterpret_cast<const unsigned char *>(src);
            for (int p = lane; p < bytes / 16; p += 32) cpa<16>(dst + p * 16, s8 + p * 16);
        };
        seg(a, lci + d.z, ne * 4);
        seg(a + y.va, lva + d.z, ne * S);
        seg(a + y.rp, lrp + ra, (nr + 4) * 4);
        seg(a + y.row, lrow + ra, nr * 4);
        seg(a + y.di, linvd + ra, nr * S);
        if (XM == 2) {
            seg(a + y.sl, sw.lslot + ra, nr * 4);
            seg(a + y.ld, sw.ld + sldd[k].x, nl * 8);
        }
    };
    // level k's t rows (and without x in shared memory the rows' old x) into
    // its record; needs the record's row ids
    auto stage_rows = [&](int k) {
        const int4 d = sdesc[k];
        const int ra = d.x & ~3;
        const GswLay y = s_lay[k & (NS - 1)];
        unsigned char *a = rec(k);
        const int *rows = reinterpret_cast<const int *>(a + y.row);
        T *ts = reinterpret_cast<T *>(a + y.t);
        T *xos = reinterpret_cast<T *>(a + y.xo);
        for (int w = lane; w < (d.y - d.x) * PPR; w += 32) {
            const int i = d.x - ra + w / PPR, j = w % PPR;
            const int row = rows[i];
            if (row >= 0) {
                cpa<PB>(ts + i * NV + swz(i, j), t + (i64)row * NV + j * PE);
                if (XM == 0) cpa<PB>(xos + i * NV + swz(i, j), x + (i64)row * NV + j * PE);
            }
        }
    };
    // slot window: the old x of the listed rows into their slots
    auto load_rows = [&](const int2 *lst, int cnt) {
        for (int w = lane; w < cnt * PPR; w += 32) {
            const int2 e = lst[w / PPR];
            const int j = w % PPR;
            if (e.x >= 0) cpa<PB>(xs + (i64)e.y * NV + swz(e.y, j), x + (i64)e.x * NV + j * PE);
        }
    };

    // cp.async groups: iteration l (from -DR) commits one group with level
    // l + DR's record, level l + DT's t rows and (window) the rows first used
    // at level l + kGsSlotAhead; the window rows of the first kGsSlotAhead
    // levels join the first group.  Before staging level l + DT's rows its
    // record (DR - DT groups back) must be in; before computing level l its t
    // rows (DT groups back), its record and its window rows (older) must be.
    static_assert(DR - DT - 1 == 0 && kGsSlotAhead >= DT, "group bookkeeping below assumes these");
    if (XM == 2) {
        const int2 pr = __ldg(sw.ldpre + b);
        if (pr.y > pr.x) load_rows(sw.ld + pr.x, pr.y - pr.x);
    }
    for (int l = -DR; l < nlv; ++l) {
        cpa_wait<DR - DT - 1>();
        __syncwarp();
        if (l + DR < nlv) stage_record(l + DR);
        if (l + DT >= 0 && l + DT < nlv) stage_rows(l + DT);
        if (XM == 2 && l >= 0) load_rows(reinterpret_cast<const int2 *>(rec(l) + s_lay[l & (NS - 1)].ld), nlist(l));
        cpa_commit();
        if (l < 0) continue;
        cpa_wait<DT>();
        __syncwarp();

        const int4 d = sdesc[l];
        const int ra = d.x & ~3;
        const GswLay y = s_lay[l & (NS - 1)];
        const unsigned char *a = rec(l);
        const int *sci = reinterpret_cast<const int *>(a);
        const T *sva = reinterpret_cast<const T *>(a + y.va);
        const int *srp = reinterpret_cast<const int *>(a + y.rp);
        const int *srow = reinterpret_cast<const int *>(a + y.row);
        const T *sdi = reinterpret_cast<const T *>(a + y.di);
        const int *ssl = reinterpret_cast<const int *>(a + y.sl);
        const T *sts = reinterpret_cast<const T *>(a + y.t);
        const T *sxo = reinterpret_cast<const T *>(a + y.xo);
        if (XM == 0) {
            // the x rows of the level's entries, entry k's at xs[k * NV];
            // padding entries get zeros.  Their own group, waited for at once
            // (an extra complete group only makes the later waits stricter).
            const int ne = d.w - d.z;
            for (int w = lane; w < ne * PPR; w += 32) {
                const int c = sci[w / PPR], j = w % PPR;
                T *dst = xs + (i64)(w / PPR) * NV + swz(w / PPR, j);
                if (c >= 0) cpa<PB>(dst, x + (i64)c * NV + j * PE);
                else *reinterpret_cast<PW *>(dst) = PW{};
            }
            cpa_commit();
            cpa_wait<0>();
            __syncwarp();
        }
        const int nrow = d.y - d.x;
        for (int p = lane / TPR; p < nrow; p += RPP) {
            const int i = d.x - ra + p;
            const int row = srow[i];
            if (row < 0) continue;
            T sum[CW], xo[CW];
            ldrow<T, CW, SWM>(sts + i * NV, i, sub, sum);
            i64 xr = 0;
            if (XM == 1) xr = (i64)row - xbase;
            if (XM == 2) xr = ssl[i];
            if (XM == 0) ldrow<T, CW, SWM>(sxo + i * NV, i, sub, xo);
            else ldrow<T, CW, SWM>(xs + xr * NV, (int)xr, sub, xo);
            const T di = sdi[i];
            const int j0 = srp[i] - d.z, j1 = srp[i + 1] - d.z;
            for (int j = j0; j < j1; j += U) {
                int c[U];
                T av[U], xv[U][CW];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    c[u] = sci[j + u];
                    av[u] = sva[j + u];
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    i64 q;
                    if (XM == 0) q = j + u;
                    else if (XM == 1) q = c[u] >= 0 ? (i64)c[u] - xbase : zr;
                    else q = c[u] >= 0 ? (i64)c[u] : zr;
                    ldrow<T, CW, SWM>(xs + q * NV, (int)q, sub, xv[u]);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int e = 0; e < CW; ++e) sum[e] = fma(-av[u], xv[u][e], sum[e]);
            }
#pragma unroll
            for (int e = 0; e < CW; ++e) xo[e] = fma(mulrn(rl[e], di), sum[e], xo[e]);
            if (XM != 0) strow<T, CW, SWM>(xs + xr * NV, (int)xr, sub, xo);
            if (XM != 1) gstrow<T, CW>(x + (i64)row * NV + sub * CW, xo);
        }
        // the gather reads x through L2 (cp.async.cg): the level's new values
        // must be there before another lane copies them (a warp barrier
        // orders them only for loads through this SM's L1)
        if (XM == 0) __threadfence();
        __syncwarp();
    }
    cpa_wait<0>();
    __syncwarp();
    if (XM == 1) {
        for (i64 w = lane; w < xrows * PPR; w += 32)
            *reinterpret_cast<PW *>(x + (xbase + w / PPR) * NV + (w % PPR) * PE) =
                *reinterpret_cast<const PW *>(xs + (w / PPR) * NV + swz(w / PPR, (int)(w % PPR)));
    }
}

// Launch shape: the x form that fits, with kGswStages record stages, the
// shared memory of one CTA when all blocks are resident at once (228 KB per
// SM shared by ceil(blocks / SMs) CTAs, 1 KB of it reserved per CTA).
// Preference: x tile, then slot window, then the per-level gather.  xm = -1:
// none fits.
GswShape gsw_shape(int s, int nv, int nblocks, int sms, i64 brows, int nslots, int emax, int rmax, int lmax,
                   int nlmax) {
    const long per_sm = std::min<long>(32, std::max<long>(1, (nblocks + sms - 1) / std::max(sms, 1)));
    const long budget = std::min<long>(227l * 1024, (228l * 1024) / per_sm - 1024);
    const long tables = ((long)lmax * 24 + 127) & ~127l;
    GswShape z;
    auto fits = [&](int xm) {
        if (xm == 2 && nslots <= 0) return false;
        const long xbytes = xm == 1   ? (long)(brows + 1) * nv * s
                            : xm == 2 ? (long)(nslots + 1) * nv * s
                                      : (long)((emax + 3) & ~3) * nv * s;
        const long xoff = (xbytes + 127) & ~127l;
        const long recb = ((long)gsw_lay((emax + 3) & ~3, (rmax + 3) & ~3, (nlmax + 1) & ~1, s, nv, xm).size + 15) & ~15l;
        if (recb <= 0 || budget - xoff - tables < kGswStages * recb) return false;
        z.xm = xm;
        z.ns = kGswStages;
        z.recb = (int)recb;
        z.xoff = (int)xoff;
        z.smem = (size_t)(xoff + tables + kGswStages * recb);
        return true;
    };
    if (fits(1) || fits(2) || fits(0)) return z;
    return GswShape{};
}

template <class T, int NV, int XM>
static cudaError_t gsw_launch(const GswShape &z, int nblocks, const int *desc, const int *blev, const int *lrp,
                              const int *lci, const void *lva, const int *lrow, const void *invd, const void *t,
                              void *x, const void *relax, i64 brows, i64 n, const GsSlotWin *win, int lmax,
                              cudaStream_t s) {
    auto k = k_gsw<T, NV, XM>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)z.smem);
    if (e != cudaSuccess) return e;
    GsSlotWin w = win ? *win : GsSlotWin{};
    note_launch();
    k<<<nblocks, 32, z.smem, s>>>((const int4 *)desc, blev, lrp, lci, (const T *)lva, lrow, (const T *)invd,
                                  (const T *)t, (T *)x, (const T *)relax, brows, n, w, z.recb, lmax, z.xoff);
    return cudaGetLastError();
}

template <class T, int NV>
static cudaError_t gsw_nv(const GswShape &z, int nblocks, const int *desc, const int *blev, const int *lrp,
                          const int *lci, const void *lva, const int *lrow, const void *invd, const void *t, void *x,
                          const void *relax, i64 brows, i64 n, const GsSlotWin *win, int lmax, cudaStream_t s) {
    switch (z.xm) {
    case 0: return gsw_launch<T, NV, 0>(z, nblocks, desc, blev, lrp, lci, lva, lrow, invd, t, x, relax, brows, n, win, lmax, s);
    case 1: return gsw_launch<T, NV, 1>(z, nblocks, desc, blev, lrp, lci, lva, lrow, invd, t, x, relax, brows, n, win, lmax, s);
    case 2: return gsw_launch<T, NV, 2>(z, nblocks, desc, blev, lrp, lci, lva, lrow, invd, t, x, relax, brows, n, win, lmax, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t gs_sweep_warp(Prec p, int nv, const GswShape &z, int nblocks, const int *desc, const int *blev,
                          const int *lrp, const int *lci, const void *lva, const int *lrow, const void *invd,
                          const void *t, void *x, const void *relax, i64 brows, i64 n, const GsSlotWin *win,
                          int lmax, cudaStream_t s) {
    if (z.xm < 0 || z.ns != kGswStages || (z.xm == 2 && !win)) return cudaErrorInvalidValue;
#define GSW_ARGS z, nblocks, desc, blev, lrp, lci, lva, lrow, invd, t, x, relax, brows, n, win, lmax, s
    if (p == Prec::F64) {
        switch (nv) {
        case 1: return gsw_nv<double, 1>(GSW_ARGS);
        case 2: return gsw_nv<double, 2>(GSW_ARGS);
        case 4: return gsw_nv<double, 4>(GSW_ARGS);
        case 8: return gsw_nv<double, 8>(GSW_ARGS);
        case 16: return gsw_nv<double, 16>(GSW_ARGS);
        case 32: return gsw_nv<double, 32>(GSW_ARGS);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (nv) {
    case 1: return gsw_nv<float, 1>(GSW_ARGS);
    case 2: return gsw_nv<float, 2>(GSW_ARGS);
    case 4: return gsw_nv<float, 4>(GSW_ARGS);
    case 8: return gsw_nv<float, 8>(GSW_ARGS);
    case 16: return gsw_nv<float, 16>(GSW_ARGS);
    case 32: return gsw_nv<float, 32>(GSW_ARGS);
    default: return cudaErrorInvalidValue;
    }
#undef GSW_ARGS
}

}  // namespace xk
