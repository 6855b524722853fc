// Gauss-Seidel sweeps over a level-ordered copy of the matrix (sm_100a).
//
// The sweep's rows are stored in schedule order (level by level, and block by
// block for hybrid plans); each row keeps its entries in the original CSR
// order and is padded to a multiple of 4 entries with column -1, so any
// contiguous row range starts on a 16-byte boundary and spans a multiple of 16
// bytes.  A CTA processes one contiguous row range per level, and the entries
// of its NEXT level are fetched into shared memory by a 1-D TMA bulk copy
// (cp.async.bulk + mbarrier) while the current level computes; the dependent
// chain of a level is then shared-memory reads, the x gathers and one barrier.
//
//   GRID   : all CTAs cooperate on every level (cooperative launch), with a
//            bounded grid barrier between levels; x lives in global memory and
//            is read through L2 (ld.cg) because other CTAs write it.
//   BLOCKS : CTA b owns hybrid block b; CTA barriers only.  The block's x tile
//            is held in shared memory when it fits (XS = true); otherwise,
//            when the rows live at once fit, in a slot window (SL = true): every
//            row has a shared-memory slot for its live range, entries carry slot
//            numbers, and the old x of a row is copied into its slot
//            kGsSlotAhead levels before its first use (cp.async, off the
//            level's critical path); new values go to the slot and to global
//            memory.  Failing both, each level gathers its x values.
//
// Every wait (grid barrier, mbarrier) is bounded by a wall-clock limit; on
// expiry the error word is set, the CTA waits (bounded) for its own copies in
// flight and returns.
#include "kernels.cuh"
#include <algorithm>
#include <cstdio>
#include <vector>

namespace xk {

namespace {

constexpr unsigned long long kLimitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned cnt) {
    asm volatile("mbarrier.init.shared.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(cnt) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 16-byte global -> shared copy through L2 only (other CTAs' and this CTA's
// earlier stores are visible to it), tracked per thread
__device__ __forceinline__ void cp_async16_cg(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait on an mbarrier phase; false on timeout
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity,
                                          unsigned long long limit = kLimitNs) {
    if (mbar_try(bar, parity)) return true;
    unsigned long long t0 = now_ns();
    while (!mbar_try(bar, parity))
        if (now_ns() - t0 > limit) return false;
    return true;
}

// Grid barrier on two words that the launcher zeroes before the launch, on
// separate 128-byte lines so that arrivals and polls do not queue on one L2
// line: words[0] counts arrivals, words[16] is the release word.  Barrier k
// is complete when the counter reaches target = (k + 1) * gridDim.x; the CTA
// whose arrival completes it publishes target in the release word, the others
// poll that word (bounded: on timeout *err is set).  Thread 0's fences order
// the whole CTA's stores (they follow the CTA barrier).
__device__ __forceinline__ bool grid_barrier(unsigned long long *words, unsigned long long target,
                                             int *err, unsigned long long limit = kLimitNs) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        volatile unsigned long long *rel = words + 16;
        if (atomicAdd(words, 1ull) + 1 == target) {
            __threadfence();
            *rel = target;
        } else {
            unsigned long long t0 = now_ns();
            unsigned spins = 0;
            while (*rel < target) {
                if ((++spins & 63) == 0) {
                    if (*(volatile int *)err) break;
                    if (now_ns() - t0 > limit) {
                        atomicExch(err, 1);
                        break;
                    }
                }
            }
        }
        __threadfence();
    }
    // one verdict for the whole CTA (thread 0 reads the error word after its
    // fence), so that no thread leaves a loop its neighbours stay in
    return __syncthreads_and(threadIdx.x != 0 || *(volatile int *)err == 0) != 0;
}

__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }

template <class T, int V> struct VW;
template <> struct VW<double, 1> { typedef double t; };
template <> struct VW<double, 2> { typedef double2 t; };
template <> struct VW<float, 1> { typedef float t; };
template <> struct VW<float, 2> { typedef float2 t; };
template <> struct VW<float, 4> { typedef float4 t; };

template <class T, int NV> struct Sh {
    static constexpr int V = (NV * (int)sizeof(T) >= 16) ? 16 / (int)sizeof(T) : NV;
    static constexpr int TPR = NV / V;
};

template <class T, int V, bool CG>
__device__ __forceinline__ void gld(const T *p, T (&r)[V]) {
    typedef typename VW<T, V>::t W;
    W w = CG ? __ldcg(reinterpret_cast<const W *>(p)) : *reinterpret_cast<const W *>(p);
    memcpy(r, &w, sizeof(W));
}
template <class T, int V, bool CG>
__device__ __forceinline__ void gst(T *p, const T (&r)[V]) {
    typedef typename VW<T, V>::t W;
    W w;
    memcpy(&w, r, sizeof(W));
    if (CG) __stcg(reinterpret_cast<W *>(p), w);
    else *reinterpret_cast<W *>(p) = w;
}

}  // namespace

// Staging buffers: three levels in flight, each with up to E entries and RB
// rows (column indices, values, row offsets, row ids, inverse diagonals).
// 256-thread CTAs (two per SM) stage larger levels than 128-thread CTAs (four
// per SM, about 25 KB of static shared memory each).
template <class T, int NT = 256> struct GsBuf {
    static constexpr int E = NT == 256 ? (sizeof(T) == 8 ? 1024 : 1536) : (sizeof(T) == 8 ? 512 : 768);
    static constexpr int RB = NT == 256 ? 128 : 64;
    // slot-window loads staged per level (int2 each)
    static constexpr int LB = NT == 256 ? (sizeof(T) == 8 ? 160 : 192) : (sizeof(T) == 8 ? 96 : 128);
};

// One level of one CTA: rows [r0, r1) and entries [e0, e1) of the
// level-ordered copy.  e0 and e1 are multiples of 4 (rows are padded to 4
// entries); r0 and r1 are arbitrary, and the per-row arrays are staged from
// r0 rounded down to the 4-row boundary (level groups are padded to 4 rows, so
// the rounded range stays inside the arrays).
struct Desc {
    int r0, r1, e0, e1;
};
__device__ __forceinline__ int rlo(const Desc &d) { return d.r0 & ~3; }
__device__ __forceinline__ int rspan(const Desc &d) { return ((d.r1 + 3) & ~3) - (d.r0 & ~3); }

// MODE 0 = GRID, 1 = BLOCKS.  XS: x tile of the block in shared memory; SL:
// slot window (lci then holds slot numbers).
// desc: GRID -> desc[l*gridDim.x + b]; BLOCKS -> desc[blev[b] + (l - l0)].
template <class T, int NV, int MODE, bool XS, bool SL = false, int NT = 256>
__global__ void __launch_bounds__(NT, MODE == 1 ? 512 / NT : 1) k_gs3(int nlev, const int4 *__restrict__ desc,
                                             const int *__restrict__ blev,
                                             const int *__restrict__ lrp,
                                             const int *__restrict__ lci,
                                             const T *__restrict__ lva,
                                             const int *__restrict__ lrow,
                                             const T *__restrict__ linvd,
                                             const T *__restrict__ t, T *x,
                                             const T *__restrict__ relax, i64 brows, i64 n,
                                             int eg, unsigned *gbar, int *err, GsSlotWin sw, GsDeps gd) {
    constexpr int V = Sh<T, NV>::V, TPR = Sh<T, NV>::TPR, E = GsBuf<T, NT>::E, RB = GsBuf<T, NT>::RB;
    static_assert(NT == 256 || (NT == 128 && MODE == 1), "128-thread CTAs serve hybrid blocks only");
    constexpr int NB = 3;
    constexpr int LB = SL ? GsBuf<T, NT>::LB : 2;
    constexpr bool CG = (MODE == 0);
    constexpr bool TILE = XS || SL;  // every x value is read from shared memory
    constexpr int AH = kGsSlotAhead;
    extern __shared__ __align__(128) unsigned char dyn[];
    __shared__ __align__(16) int s_ci[NB][E];
    __shared__ __align__(16) T s_va[NB][E];
    __shared__ __align__(16) int s_rp[NB][RB + 4];
    __shared__ __align__(16) int s_row[NB][RB];
    __shared__ __align__(16) int s_sl[NB][SL ? RB : 4];
    __shared__ __align__(16) int2 s_ld[NB][LB];
    __shared__ __align__(16) T s_di[NB][RB];
    __shared__ __align__(8) unsigned long long mbar[NB];
    __shared__ int s_stage[NB];
    __shared__ int s_ldn[NB];
    T *xs = reinterpret_cast<T *>(dyn);

    const int b = blockIdx.x, tid = threadIdx.x;
    int l0 = 0, l1 = nlev, dbase = 0;
    i64 xbase = 0;
    if (MODE == 1) {
        dbase = __ldg(blev + b);
        l1 = __ldg(blev + b + 1) - dbase;
        xbase = SL ? 0 : (i64)b * brows;
    }
    auto dget = [&](int l) -> Desc {
        int4 v = MODE == 0 ? __ldg(desc + (i64)l * gridDim.x + b) : __ldg(desc + dbase + l);
        return Desc{v.x, v.y, v.z, v.w};
    };
    if (tid == 0) {
        for (int q = 0; q < NB; ++q) mbar_init(&mbar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const i64 xrows = MODE == 1 && XS ? min((i64)brows, n - xbase) : 0;
    if (XS) {
        const T *xg = x + xbase * NV;
        for (i64 q = tid; q < xrows * NV; q += NT) xs[q] = xg[q];
    }
    // the row of zeros that padding entries (column -1, value +0) read after
    // the x tile or the slot window: fma(-0, 0, s) == s for every s
    const i64 zrow = XS ? (i64)brows : SL ? (i64)sw.nslots : 0;
    // shared-memory row indices fit in 32 bits (a tile or window of at most
    // 227 KB); the block's first row does too (rows < 2^31)
    const int zr32 = (int)zrow, xb32 = (int)xbase;
    if (TILE)
        for (int q = tid; q < NV; q += NT) xs[zrow * NV + q] = T(0);
    T rl[V];  // this thread's relaxation factors (its columns never change)
#pragma unroll
    for (int e = 0; e < V; ++e) rl[e] = relax[(tid % TPR) * V + e];
    __syncthreads();
    unsigned par = 0u;  // bit q: phase parity of staging buffer q's next wait
    // issuer: the last thread, which rarely owns a row of a level
    const bool issuer = tid == NT - 1;
    // the slot window's load range of level l (loaded with the level's
    // descriptor, one iteration before it is needed)
    auto lget = [&](int l) { return SL ? __ldg(sw.ldd + dbase + l) : make_int2(0, 0); };
    auto issue = [&](int l, const Desc &d, int2 lr) {
        int q = l % NB;
        int nr = rspan(d), ne = d.e1 - d.e0, ra = rlo(d);
        const int nl = lr.y - lr.x;
        if (d.r1 > d.r0 && nr <= RB && ne <= E && nl <= LB) {
            unsigned bytes = (unsigned)ne * (4u + (unsigned)sizeof(T)) + (unsigned)(nr + 4) * 4u +
                             (unsigned)nr * 4u + (unsigned)nr * (unsigned)sizeof(T);
            if (SL) bytes += (unsigned)nr * 4u + (unsigned)nl * 8u;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&mbar[q], bytes);
            if (ne > 0) {
                bulk_g2s(&s_ci[q][0], lci + d.e0, (unsigned)ne * 4u, &mbar[q]);
                bulk_g2s(&s_va[q][0], lva + d.e0, (unsigned)ne * (unsigned)sizeof(T), &mbar[q]);
            }
            bulk_g2s(&s_rp[q][0], lrp + ra, (unsigned)(nr + 4) * 4u, &mbar[q]);
            bulk_g2s(&s_row[q][0], lrow + ra, (unsigned)nr * 4u, &mbar[q]);
            bulk_g2s(&s_di[q][0], linvd + ra, (unsigned)nr * (unsigned)sizeof(T), &mbar[q]);
            if (SL) {
                bulk_g2s(&s_sl[q][0], sw.lslot + ra, (unsigned)nr * 4u, &mbar[q]);
                if (nl > 0) bulk_g2s(&s_ld[q][0], sw.ld + lr.x, (unsigned)nl * 8u, &mbar[q]);
            }
            s_stage[q] = 1;
        } else {
            s_stage[q] = 0;
        }
        s_ldn[q] = nl;
    };
    // slot window: copy the old x of the listed rows into their slots, one
    // 16-byte piece per thread and pass (entries {-1, -1} are padding)
    auto load_rows = [&](const int2 *lst, int cnt) {
        for (int w = tid; w < cnt * TPR; w += NT) {
            const int2 e = lst[w / TPR];
            if (e.x >= 0) cp_async16_cg(xs + (i64)e.y * NV + (w % TPR) * V, x + (i64)e.x * NV + (w % TPR) * V);
        }
    };
    Desc dn1{0, 0, 0, 0}, dn2{0, 0, 0, 0};
    int2 ln2 = make_int2(0, 0);
    if (issuer) {
        if (l0 < l1) issue(l0, dget(l0), lget(l0));
        if (l0 + 1 < l1) { dn1 = dget(l0 + 1); issue(l0 + 1, dn1, lget(l0 + 1)); }
        if (l0 + 2 < l1) { dn2 = dget(l0 + 2); ln2 = lget(l0 + 2); }
    }
    __syncthreads();
    bool ok = true;
    // register prefetch of this thread's first row of a level: row index, t
    // and (without the x tile) the row's old x.  Neither changes during the
    // sweep before the row's own level (one launch per sweep direction, every
    // row updated once), so level l+1's are loaded at the start of level l
    // and arrive while level l computes.
    bool pv = false, nf = false;
    int pr = 0, nr = 0;
    T pt[V], px[V], nt[V], nx[V];
    auto wait_q = [&](int q) {
        if (s_stage[q]) {
            if (!mbar_wait(&mbar[q], (par >> q) & 1u)) {
                atomicExch(err, 1);
                ok = false;
            }
            par ^= 1u << q;
        }
    };
    auto prefetch = [&](int l, const Desc &d) {  // into nf, nr, nt, nx
        int q = l % NB;
        nf = false;
        if (!ok) return;  // staging buffers are not trustworthy after a timeout
        int items = (d.r1 - d.r0) * TPR;
        if (tid < items) {
            int r = d.r0 + tid / TPR, lane = tid % TPR;
            int row = s_stage[q] ? s_row[q][r - rlo(d)] : __ldg(lrow + r);
            if (row >= 0) {
                nf = true;
                nr = row;
                gld<T, V, CG>(t + (i64)row * NV + lane * V, nt);
                if (!TILE) gld<T, V, CG>(x + (i64)row * NV + lane * V, nx);
            }
        }
    };
    auto rotate = [&]() {
        pv = nf;
        pr = nr;
#pragma unroll
        for (int e = 0; e < V; ++e) {
            pt[e] = nt[e];
            px[e] = nx[e];
        }
    };
    Desc dc = l0 < l1 ? dget(l0) : Desc{0, 0, 0, 0};
    Desc dq1 = l0 + 1 < l1 ? dget(l0 + 1) : Desc{0, 0, 0, 0};
    Desc dq2 = l0 + 2 < l1 ? dget(l0 + 2) : Desc{0, 0, 0, 0};
    int dfirst = 0, dcnt = 0;
    int2 dn = make_int2(0, 0);
    if (MODE == 0 && gd.dptr && l0 + 1 < l1) {
        dfirst = __ldg(gd.dptr + (i64)(l0 + 1) * gridDim.x + b);
        dcnt = __ldg(gd.dptr + (i64)(l0 + 1) * gridDim.x + b + 1) - dfirst;
        if (tid < 32 && tid < dcnt) dn = __ldg(gd.deps + dfirst + tid);
    }
    if (SL) {
        // rows first used in the first AH levels, then AH - 1 empty groups:
        // the rows first used at level l >= AH are in the group iteration
        // l - AH commits, which the wait at the end of iteration l - 1
        // (all but the newest AH - 1 groups) completes
        const int2 pr2 = __ldg(sw.ldpre + b);
        if (pr2.y > pr2.x) load_rows(sw.ld + pr2.x, pr2.y - pr2.x);
        cp_async_commit();
#pragma unroll
        for (int g = 1; g < AH; ++g) cp_async_commit();
        // the rows of the first level are in before it starts; from then on
        // each level's end barrier publishes the next level's (below)
        cp_async_wait_group<AH - 1>();
        __syncthreads();
    }
    if (l0 < l1) {
        wait_q(l0 % NB);
        prefetch(l0, dc);
        rotate();
    }
    for (int l = l0; ok && l < l1; ++l) {
        const int q = l % NB;
        if (issuer && l + 2 < l1) {
            issue(l + 2, dn2, ln2);
            if (l + 3 < l1) { dn2 = dget(l + 3); ln2 = lget(l + 3); }
        }
        if (SL) {
            // the rows first used AH levels from now (list staged with this level)
            if (s_stage[q]) {
                load_rows(&s_ld[q][0], s_ldn[q]);
            } else {
                const int2 lr = __ldg(sw.ldd + dbase + l);
                if (lr.y > lr.x) load_rows(sw.ld + lr.x, lr.y - lr.x);
            }
            cp_async_commit();
        }
        // descriptors come through a two-level register queue: level l+3's
        // is loaded now and used two levels later, off the critical path
        const Desc dnx = dq1;
        dq1 = dq2;
        if (l + 3 < l1) dq2 = dget(l + 3);
        if (l + 1 < l1) {
            wait_q((l + 1) % NB);
            prefetch(l + 1, dnx);
        }
        const bool staged = s_stage[q] != 0;
        const int items = (dc.r1 - dc.r0) * TPR;
        // without the block's x tile in shared memory (GRID, or BLOCKS whose
        // tile is too large): gather every x value this level's entries need
        // into shared memory in one parallel round trip (xs: eg entries x NV)
        const bool gath = !TILE && ok && staged && (dc.e1 - dc.e0) <= eg;
        if (MODE == 0 && gd.dptr && l > l0) {
            // point-to-point: wait until every CTA whose rows this level
            // depends on has finished the levels it must have (bounded; the
            // list was loaded during the previous level), then make their
            // stores visible to the whole CTA
            if (tid < 32) {
                for (int k = 0; k < dcnt; k += 32) {
                    int2 e = dn;
                    if (k > 0) e = tid + k < dcnt ? __ldg(gd.deps + dfirst + tid + k) : make_int2(0, 0);
                    if (tid + k >= dcnt) continue;
                    volatile unsigned *pw = gd.prog + (size_t)e.x * 8;
                    if (*pw >= (unsigned)e.y) continue;
                    const unsigned long long t0 = now_ns();
                    unsigned spins = 0;
                    while (*pw < (unsigned)e.y) {
                        if ((++spins & 63) == 0) {
                            if (*(volatile int *)err) break;
                            if (now_ns() - t0 > kLimitNs) {
                                atomicExch(err, 1);
                                break;
                            }
                        }
                    }
                }
                __threadfence();
            }
            ok = __syncthreads_and(ok && (tid != 0 || *(volatile int *)err == 0)) != 0;
        }
        if (MODE == 0 && gd.dptr && ok && l + 1 < l1) {
            // the next level's list: its range and this lane's first entry
            dfirst = __ldg(gd.dptr + (i64)(l + 1) * gridDim.x + b);
            dcnt = __ldg(gd.dptr + (i64)(l + 1) * gridDim.x + b + 1) - dfirst;
            if (tid < 32 && tid < dcnt) dn = __ldg(gd.deps + dfirst + tid);
        }
        if (!TILE) {
            if (gath && V * (int)sizeof(T) == 16) {
                // 16-byte pieces: every piece is copied by cp.async straight
                // into shared memory, all in flight together (one L2 round
                // trip, no registers held); padding entries (column -1) get
                // zeros
                const int tot = (dc.e1 - dc.e0) * TPR;
                for (int w = tid; w < tot; w += NT) {
                    const int c = s_ci[q][w / TPR];
                    if (c >= 0) cp_async16_cg(xs + (i64)w * V, x + (i64)c * NV + (w % TPR) * V);
                    else *reinterpret_cast<int4 *>(xs + (i64)w * V) = make_int4(0, 0, 0, 0);
                }
                cp_async_wait_all();
            } else if (gath) {
                // every thread issues up to GU independent loads before it
                // stores any, so the gather costs one or two L2 round trips
                constexpr int GU = 8;
                const int tot = (dc.e1 - dc.e0) * TPR;
                for (int w0 = tid; w0 < tot; w0 += NT * GU) {
                    int c[GU];
                    T tmp[GU][V];
#pragma unroll
                    for (int u = 0; u < GU; ++u) {
                        const int w = w0 + u * NT;
                        c[u] = w < tot ? s_ci[q][w / TPR] : -2;  // -1: padding (zeros), -2: past the end
                        if (c[u] >= 0) gld<T, V, CG>(x + (i64)c[u] * NV + (w % TPR) * V, tmp[u]);
                    }
#pragma unroll
                    for (int u = 0; u < GU; ++u)
                        if (c[u] != -2) {
                            T *p = xs + (i64)(w0 + u * NT) * V;
#pragma unroll
                            for (int e = 0; e < V; ++e) p[e] = c[u] >= 0 ? tmp[u][e] : T(0);
                        }
                }
            }
            __syncthreads();
        }
        const int ra = rlo(dc);
        for (int it = tid; ok && it < items; it += NT) {
            const int r = dc.r0 + it / TPR, lane = it % TPR;
            const int row = it == tid ? (pv ? pr : -1) : (staged ? s_row[q][r - ra] : __ldg(lrow + r));
            if (row < 0) continue;
            T sum[V], xo[V];
            if (it == tid) {
#pragma unroll
                for (int e = 0; e < V; ++e) sum[e] = pt[e];
            } else {
                gld<T, V, CG>(t + (i64)row * NV + lane * V, sum);
            }
            const int xrow = SL ? (staged ? s_sl[q][r - ra] : __ldg(sw.lslot + r)) : row - xb32;
            if (TILE) {
                gld<T, V, false>(xs + xrow * NV + lane * V, xo);
            } else if (it == tid) {
#pragma unroll
                for (int e = 0; e < V; ++e) xo[e] = px[e];
            } else {
                gld<T, V, CG>(x + (i64)row * NV + lane * V, xo);
            }
            const T di = staged ? s_di[q][r - ra] : __ldg(linvd + r);
            const int j0 = staged ? s_rp[q][r - ra] : __ldg(lrp + r);
            const int j1 = staged ? s_rp[q][r - ra + 1] : __ldg(lrp + r + 1);
            if (staged && (TILE || gath)) {
                // every operand is in shared memory: a loop over the row's
                // entries four at a time (rows are padded to 4 entries; the
                // padding, value +0, reads zeros)
                const int o = j0 - dc.e0, m = j1 - j0;
                const T *vr = &s_va[q][o];
                if (TILE) {
                    const int *cr = &s_ci[q][o];
                    for (int k = 0; k < m; k += 4) {
                        T xv[4][V];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int c = cr[k + u];
                            gld<T, V, false>(xs + (c >= 0 ? c - xb32 : zr32) * NV + lane * V, xv[u]);
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const T a = vr[k + u];
#pragma unroll
                            for (int e = 0; e < V; ++e) sum[e] = fma(-a, xv[u][e], sum[e]);
                        }
                    }
                } else {
                    const T *xr = xs + (i64)o * NV + lane * V;
                    for (int k = 0; k < m; k += 4) {
                        T xv[4][V];
#pragma unroll
                        for (int u = 0; u < 4; ++u) gld<T, V, false>(xr + (i64)(k + u) * NV, xv[u]);
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const T a = vr[k + u];
#pragma unroll
                            for (int e = 0; e < V; ++e) sum[e] = fma(-a, xv[u][e], sum[e]);
                        }
                    }
                }
            } else
            // fallback for levels too large for the staging buffers: entries
            // and x read from global memory, 4 gathers at a time
            for (int j = j0; j < j1; j += 4) {
                constexpr int GB = 4;
                int c[GB];
                T v[GB];
#pragma unroll
                for (int k = 0; k < GB; ++k) {
                    const bool in = j + k < j1;
                    c[k] = in ? (staged ? s_ci[q][j + k - dc.e0] : __ldg(lci + j + k)) : -1;
                    v[k] = in ? (staged ? s_va[q][j + k - dc.e0] : __ldg(lva + j + k)) : T(0);
                }
                T xv[GB][V];
#pragma unroll
                for (int k = 0; k < GB; ++k) {
                    if (c[k] >= 0) {
                        if (TILE) {
                            const T *p = xs + ((i64)c[k] - xbase) * NV + lane * V;
#pragma unroll
                            for (int e = 0; e < V; ++e) xv[k][e] = p[e];
                        } else if (gath) {
                            const T *p = xs + ((i64)(j + k - dc.e0) * TPR + lane) * V;
#pragma unroll
                            for (int e = 0; e < V; ++e) xv[k][e] = p[e];
                        } else {
                            gld<T, V, CG>(x + (i64)c[k] * NV + lane * V, xv[k]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < GB; ++k)
                    if (c[k] >= 0) {
#pragma unroll
                        for (int e = 0; e < V; ++e) sum[e] = fma(-v[k], xv[k][e], sum[e]);
                    }
            }
#pragma unroll
            for (int e = 0; e < V; ++e) {
                T cf = rmul(rl[e], di);
                xo[e] = fma(cf, sum[e], xo[e]);
            }
            if (TILE) {
                gst<T, V, false>(xs + xrow * NV + lane * V, xo);
            }
            if (!XS) gst<T, V, CG>(x + (i64)row * NV + lane * V, xo);
        }
        // next level: its row, t and x were prefetched at the start of this one
        if (l + 1 < l1) {
            dc = dnx;
            rotate();
        }
        // the next level's window rows (committed kGsSlotAhead - 1 groups ago)
        // are in this thread's slots; the barrier below makes every thread's
        // visible, so the next level needs no barrier of its own for them
        if (SL) cp_async_wait_group<AH - 1>();
        // every thread agrees on ok before the loop test (a wait that gave up
        // in one thread ends the sweep for the whole CTA)
        ok = __syncthreads_and(ok) != 0;
        if (MODE == 0 && gd.dptr) {
            // publish: this CTA has finished level l
            if (ok && tid == 0) {
                __threadfence();
                *(volatile unsigned *)(gd.prog + (size_t)b * 8) = (unsigned)(l + 1);
            }
        } else if (MODE == 0) {
            if (ok && l + 1 < l1 &&
                !grid_barrier(reinterpret_cast<unsigned long long *>(gbar),
                              (unsigned long long)(l + 1) * gridDim.x, err))
                ok = false;
        }
    }
    // after an early exit, wait (bounded) for staging copies still in flight;
    // window copies of this thread complete by themselves
    if (SL) cp_async_wait_all();
    __syncthreads();
    if (!ok && tid == 0) {
        for (int q = 0; q < NB; ++q)
            if (s_stage[q]) mbar_wait(&mbar[q], (par >> q) & 1u);
    }
    __syncthreads();
    if (XS && ok) {
        T *xg = x + xbase * NV;
        for (i64 q = tid; q < xrows * NV; q += NT) xg[q] = xs[q];
    }
}

// entries of the per-level x gather buffer: the largest level of any CTA
// (emax, from the plan; <= 0 = unknown), capped by the staging buffer and by
// 176 KB of shared memory
template <class T> static int gather_entries(int nv, int emax) {
    int eg = (int)std::min<long>(GsBuf<T>::E, (176l * 1024) / ((long)nv * (long)sizeof(T)));
    if (emax > 0) eg = std::min(eg, (emax + 3) & ~3);
    return std::max(eg, 4);
}

static int device_sms() {
    thread_local int dev = -1, sms = 0;
    int d = 0;
    cudaGetDevice(&d);
    if (d != dev) {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
        dev = d;
    }
    return sms > 0 ? sms : 1;
}

// One hybrid-block sweep launch: 256-thread CTAs, or 128-thread CTAs (smaller
// staging buffers) when the blocks outnumber what the 256-thread kernel keeps
// resident and more of the 128-thread one fit an SM (one wave instead of
// two).  The choice is cached per (dynamic shared memory, blocks).
template <class T, int NV, bool XSV, bool SLV>
static cudaError_t gs3_blocks(size_t sm, int ncta, int nlev, const int4 *lev_row, const int *blev, const int *lrp,
                              const int *lci, const T *va, const int *lrow, const T *di, const T *tt, T *xx,
                              const T *rl, i64 brows, i64 n, int eg, unsigned *gbar, int *err, GsSlotWin w,
                              cudaStream_t s) {
    auto k2 = k_gs3<T, NV, 1, XSV, SLV, 256>;
    auto k1 = k_gs3<T, NV, 1, XSV, SLV, 128>;
    struct Choice {
        size_t sm;
        int ncta;
        bool small;
    };
    thread_local std::vector<Choice> cache;
    bool small = false, found = false;
    for (auto &c : cache)
        if (c.sm == sm && c.ncta == ncta) small = c.small, found = true;
    cudaError_t e;
    if (!found) {
        int o2 = 0, o1 = 0;
        if (cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) == cudaSuccess &&
            cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k1, 128, sm) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k2, 256, sm) == cudaSuccess)
            small = (long)o2 * device_sms() < ncta && o1 > o2;
        cudaGetLastError();  // a refused query only rules the 128-thread kernel out
        cache.push_back({sm, ncta, small});
    }
    // the dynamic shared-memory limit is a property of the kernel: set it for
    // this launch's size every time (another plan may have set a smaller one)
    GsDeps nodeps{nullptr, nullptr, nullptr};
    if (small) {
        if ((e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) != cudaSuccess)
            return e;
        k1<<<ncta, 128, sm, s>>>(nlev, lev_row, blev, lrp, lci, va, lrow, di, tt, xx, rl, brows, n, eg, gbar, err, w,
                                 nodeps);
    } else {
        if ((e = cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) != cudaSuccess)
            return e;
        k2<<<ncta, 256, sm, s>>>(nlev, lev_row, blev, lrp, lci, va, lrow, di, tt, xx, rl, brows, n, eg, gbar, err, w,
                                 nodeps);
    }
    return cudaGetLastError();
}

template <class T, int NV>
static cudaError_t gs3_t(int mode, int xs, int nlev, int ncta, const int *descp, const int *blev,
                         const int *lrp, const int *lci, const void *lva, const int *lrow,
                         const void *invd, const void *t, void *x, const void *relax, i64 brows,
                         i64 n, unsigned *gbar, int *err, int emax, const GsSlotWin *win, const GsDeps *deps,
                         cudaStream_t s) {
    const T *va = (const T *)lva;
    const int4 *lev_row = (const int4 *)descp;
    const T *di = (const T *)invd;
    const T *tt = (const T *)t;
    T *xx = (T *)x;
    const T *rl = (const T *)relax;
    GsSlotWin none{};
    GsDeps nodeps{nullptr, nullptr, nullptr};
    note_launch();
    if (mode == 1) {
#define GS3B(XSV, SLV, SM, EG, W)                                                                              \
    gs3_blocks<T, NV, XSV, SLV>(SM, ncta, nlev, lev_row, blev, lrp, lci, va, lrow, di, tt, xx, rl, brows, n, EG, \
                                gbar, err, W, s)
        if (xs) return GS3B(true, false, (size_t)(brows + 1) * NV * sizeof(T), 0, none);  // + the zero row
        if (win && win->nslots > 0 && Sh<T, NV>::V * (int)sizeof(T) == 16 &&
            (size_t)win->nslots * NV * sizeof(T) <= (size_t)gs_slot_window_bytes())
            // lci holds slot numbers (the plan's slot-mapped copy); + the zero slot
            return GS3B(false, true, (size_t)(win->nslots + 1) * NV * sizeof(T), 0, *win);
        const int eg = gather_entries<T>(NV, emax);
        return GS3B(false, false, (size_t)eg * NV * sizeof(T), eg, none);
#undef GS3B
    }
    // the grid must match the per-(level, CTA) descriptors built on the host;
    // dynamic shared memory holds the per-level x gather buffer (eg entries)
    int nblk = ncta;
    int eg = gather_entries<T>(NV, emax);
    size_t sm = (size_t)eg * NV * sizeof(T);
    auto k = k_gs3<T, NV, 0, false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    // the grid barrier's arrival counter and release word start from zero,
    // and so do the per-CTA level counts of the point-to-point waits
    e = cudaMemsetAsync(gbar, 0, 256, s);
    if (e != cudaSuccess) return e;
    GsDeps gdv = deps ? *deps : nodeps;
    if (gdv.dptr) {
        e = cudaMemsetAsync(gdv.prog, 0, (size_t)nblk * 32, s);
        if (e != cudaSuccess) return e;
    }
    void *args[] = {&nlev, &lev_row, &blev, &lrp, &lci, &va, &lrow, &di, &tt, &xx, &rl, &brows, &n, &eg, &gbar, &err,
                    &none, &gdv};
    return cudaLaunchCooperativeKernel((const void *)k, dim3(nblk), dim3(256), args, sm, s);
}

#define NV_SWITCH(nv, FN)                                                                         \
    switch (nv) {                                                                                  \
    case 1: return FN(1);                                                                          \
    case 2: return FN(2);                                                                          \
    case 4: return FN(4);                                                                          \
    case 8: return FN(8);                                                                          \
    case 16: return FN(16);                                                                        \
    case 32: return FN(32);                                                                        \
    default: return cudaErrorInvalidValue;                                                         \
    }

cudaError_t gs_sweep_lcsr(Prec p, int nv, int mode, int xs, int nlev, int ncta, const int *lev_row,
                          const int *blev, const int *lrp, const int *lci, const void *lva,
                          const int *lrow, const void *invd, const void *t, void *x,
                          const void *relax, i64 brows, i64 n, unsigned *gbar, int *err,
                          int emax, const GsSlotWin *win, const GsDeps *deps, cudaStream_t s) {
    if (p == Prec::F64) {
#define F(NV) gs3_t<double, NV>(mode, xs, nlev, ncta, lev_row, blev, lrp, lci, lva, lrow, invd, t, x, relax, brows, n, gbar, err, emax, win, deps, s)
        NV_SWITCH(nv, F)
#undef F
    } else {
#define F(NV) gs3_t<float, NV>(mode, xs, nlev, ncta, lev_row, blev, lrp, lci, lva, lrow, invd, t, x, relax, brows, n, gbar, err, emax, win, deps, s)
        NV_SWITCH(nv, F)
#undef F
    }
}

// dynamic shared memory of a slot window that still leaves two CTAs per SM
int gs_slot_window_bytes() { return 64 * 1024; }

// dynamic shared memory available for the x tile next to the two staging buffers
int gs_lcsr_max_xs_bytes() { return 170 * 1024; }
// an x tile this small leaves room for two CTAs per SM next to the staging
// buffers (about 43 KB of static shared memory each)
int gs_lcsr_xs_bytes_two_per_sm() { return 64 * 1024; }


// ---------------------------------------------------------------- wait self-test
// The bounded waits above, made to run out on purpose with a short limit:
// which = 0: a cooperative grid of ncta CTAs meets at the grid barrier but
// CTA 0 never arrives, so the others give up after `limit` ns and set *err;
// which = 1: one CTA waits on an mbarrier phase that nothing completes and
// records the expiry in *err.  Every thread returns; nothing is left in
// flight.  Used by the tests to check that an expired wait surfaces as an
// error status instead of a hang.
__global__ void k_wait_selftest(int which, unsigned long long limit, unsigned long long *words, int *err) {
    if (which == 0) {
        if (blockIdx.x == 0) return;  // the missing arrival
        grid_barrier(words, (unsigned long long)gridDim.x, err, limit);
        return;
    }
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait(&bar, 0u, limit)) atomicExch(err, 2);
    __syncthreads();
}

cudaError_t wait_selftest(int which, int ncta, unsigned long long limit_ns, unsigned *words, int *err,
                          cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(words, 0, 256, s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    note_launch();
    unsigned long long *w = reinterpret_cast<unsigned long long *>(words);
    if (which == 0) {
        void *args[] = {&which, &limit_ns, &w, &err};
        return cudaLaunchCooperativeKernel((const void *)k_wait_selftest, dim3(ncta), dim3(128), args, 0, s);
    }
    k_wait_selftest<<<1, 128, 0, s>>>(which, limit_ns, w, err);
    return cudaGetLastError();
}

}  // namespace xk
