"""ctypes loader of the CPU oracle (liboracle.so) — test infrastructure only.

Only the tests, the smoke check and the CPU-baseline leg of bench.py use this
module, always as the checker; the product library never imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(PATH):
            import subprocess
            import sys
            subprocess.check_call([sys.executable, os.path.join(os.path.dirname(HERE), "xamg-test_b200", "build.py")])
        L = C.CDLL(PATH)
        P = C.c_void_p
        i64 = C.c_int64
        sig = {
            "orc_spmv_d": (None, [i64, P, P, P, P, P, C.c_int, C.c_int]),
            "orc_spmv_f": (None, [i64, P, P, P, P, P, C.c_int, C.c_int]),
            "orc_hsgs_d": (None, [i64, P, P, P, P, P, P, P, C.c_int, C.c_int, P]),
            "orc_hsgs_f": (None, [i64, P, P, P, P, P, P, P, C.c_int, C.c_int, P]),
            "orc_jacobi_d": (None, [i64, P, P, P, P, P, P, P, P, C.c_int]),
            "orc_jacobi_f": (None, [i64, P, P, P, P, P, P, P, P, C.c_int]),
            "orc_dot_d": (None, [i64, C.c_int, P, P, P]),
            "orc_dot_fd": (None, [i64, C.c_int, P, P, P]),
            "orc_dot_seq_d": (None, [i64, C.c_int, P, P, P]),
            "orc_dense_inverse": (None, [C.c_int, P, P]),
            "orc_dense_gemv_d": (None, [C.c_int, P, P, P, C.c_int]),
            "orc_dense_gemv_f": (None, [C.c_int, P, P, P, C.c_int]),
            "orc_transpose": (None, [i64, i64, P, P, P, P, P, P]),
            "orc_gs_levels": (None, [i64, P, P, P, P]),
            "orc_mg_create": (P, [C.c_int]),
            "orc_mg_destroy": (None, [P]),
            "orc_mg_set_A": (None, [P, C.c_int, i64, P, P, P]),
            "orc_mg_set_P": (None, [P, C.c_int, i64, i64, P, P, P]),
            "orc_mg_set_blocks": (None, [P, C.c_int, C.c_int, P]),
            "orc_mg_set_smoothers": (None, [P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double]),
            "orc_mg_set_cheb": (None, [P, C.c_int, C.c_double, P, P]),
            "orc_mg_finalize": (None, [P, C.c_int]),
            "orc_mg_set_cycle": (None, [P, C.c_int]),
            "orc_mg_set_reduced": (None, [P, C.c_int]),
            "orc_chebyshev_d": (None, [C.c_int64, P, P, P, P, P, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double]),
            "orc_mg_get_coarse_inverse": (None, [P, P]),
            "orc_mg_get_R": (None, [P, C.c_int, P, P, P]),
            "orc_mg_apply_d": (None, [P, P, P, C.c_int]),
            "orc_mg_apply_f": (None, [P, P, P, C.c_int]),
            "orc_pbicgstab_d": (C.c_int, [i64, P, P, P, P, P, P, C.c_int, C.c_int, C.c_double, C.c_double, P, C.c_int, P, P]),
            "orc_rbicgstab_d": (C.c_int, [i64, P, P, P, P, P, P, C.c_int, C.c_int, C.c_double, C.c_double, P, C.c_int, P, P]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
            "orc_pcg_d": (C.c_int, [i64, P, P, P, P, P, P, C.c_int, C.c_int, C.c_double, C.c_double, P, C.c_int, P, P]),
            "orc_gen27_size": (None, [i64, P, P]),
            "orc_gen27": (None, [i64, C.c_double, C.c_double, C.c_double, P, P, P]),
            "orc_amg_setup": (P, [i64, P, P, P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                  C.c_int]),
            "orc_amg_num_levels": (C.c_int, [P]),
            "orc_amg_level_info": (None, [P, C.c_int, P]),
            "orc_amg_level_export": (None, [P, C.c_int, P, P, P, P, P, P]),
            "orc_amg_destroy": (None, [P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def spmv(rp, ci, v, x, nv, y=None, acc=False):
    n = len(rp) - 1
    f = lib().orc_spmv_d if v.dtype == np.float64 else lib().orc_spmv_f
    y = np.zeros((n, nv), dtype=v.dtype) if y is None else y
    f(n, p(rp), p(ci), p(v), p(x), p(y), nv, int(acc))
    return y


def dot(x, y):
    n, nv = x.shape
    out = np.zeros(nv)
    if x.dtype == np.float64:
        lib().orc_dot_d(n, nv, p(x), p(y), p(out))
    else:
        lib().orc_dot_fd(n, nv, p(x), p(y), p(out))
    return out


def dot_sequential(x, y):
    n, nv = x.shape
    out = np.zeros(nv)
    lib().orc_dot_seq_d(n, nv, p(x), p(y), p(out))
    return out


def hsgs(rp, ci, v, invd, b, x, relax, block_rows=0):
    n, nv = b.shape
    if block_rows and block_rows < n:
        bp = np.arange(0, n, block_rows, dtype=np.int64)
        bp = np.append(bp, n).astype(np.int64)
    else:
        bp = np.array([0, n], dtype=np.int64)
    f = lib().orc_hsgs_d if v.dtype == np.float64 else lib().orc_hsgs_f
    f(n, p(rp), p(ci), p(v), p(invd), p(b), p(x), p(relax), nv, len(bp) - 1, p(bp))
    return x


def jacobi(rp, ci, v, invd, b, x, relax):
    n, nv = b.shape
    r = np.zeros_like(b)
    f = lib().orc_jacobi_d if v.dtype == np.float64 else lib().orc_jacobi_f
    f(n, p(rp), p(ci), p(v), p(invd), p(b), p(x), p(r), p(relax), nv)
    return x


def dense_inverse(A):
    n = A.shape[0]
    A = np.ascontiguousarray(A, dtype=np.float64)
    out = np.zeros_like(A)
    lib().orc_dense_inverse(n, p(A), p(out))
    return out


def dense_gemv(Ainv, b):
    n = Ainv.shape[0]
    nv = b.shape[1]
    y = np.zeros_like(b)
    f = lib().orc_dense_gemv_d if b.dtype == np.float64 else lib().orc_dense_gemv_f
    f(n, p(np.ascontiguousarray(Ainv, dtype=b.dtype)), p(b), p(y), nv)
    return y


def gs_levels(rp, ci):
    n = len(rp) - 1
    lf = np.zeros(n, np.int32)
    lb = np.zeros(n, np.int32)
    lib().orc_gs_levels(n, p(rp), p(ci), p(lf), p(lb))
    return lf, lb


def transpose(rp, ci, v, ncols):
    n = len(rp) - 1
    rrp = np.zeros(ncols + 1, np.int32)
    rci = np.zeros(len(ci), np.int32)
    rv = np.zeros(len(ci))
    lib().orc_transpose(n, ncols, p(rp), p(ci), p(v), p(rrp), p(rci), p(rv))
    return rrp, rci, rv


SM_JACOBI, SM_HSGS, SM_CHEB = 0, 1, 2


class MG:
    """Oracle multigrid hierarchy (levels exported from the product's setup)."""

    def __init__(self, levels, fp32=False, pre=(SM_HSGS, 1, 0.99), post=(SM_HSGS, 1, 0.99), block_rows=None,
                 cheb=None, cycle=0, reduced=False):
        """cheb = (order, spectrum_fraction, [(min_eig, max_eig) per level])
        for the Chebyshev smoother (method SM_CHEB); cycle = mg_cycle (0 V,
        1 F, 2 W); reduced = mg_reduced_precision (level 0 in FP64, the
        coarser levels in FP32, an FP64 solve's preconditioner)."""
        self.h = lib().orc_mg_create(len(levels))
        self.keep = []
        for l, lv in enumerate(levels):
            rp, ci, v = lv["A"]
            n = len(rp) - 1
            lib().orc_mg_set_A(self.h, l, n, p(rp), p(ci), p(v))
            if lv.get("P") is not None:
                prp, pci, pv = lv["P"]
                lib().orc_mg_set_P(self.h, l, n, lv["ncP"], p(prp), p(pci), p(pv))
            br = (block_rows[l] if isinstance(block_rows, (list, tuple)) else block_rows) if block_rows else 0
            if br and br < n:
                bp = np.append(np.arange(0, n, br, dtype=np.int64), n).astype(np.int64)
                self.keep.append(bp)
                lib().orc_mg_set_blocks(self.h, l, len(bp) - 1, p(bp))
            self.keep.append(lv)
        lib().orc_mg_set_smoothers(self.h, pre[0], pre[1], pre[2], post[0], post[1], post[2])
        if cheb is not None:
            order, frac, eig = cheb
            mn = np.array([e[0] for e in eig], np.float64)
            mx = np.array([e[1] for e in eig], np.float64)
            self.keep += [mn, mx]
            lib().orc_mg_set_cheb(self.h, int(order), float(frac), p(mn), p(mx))
        lib().orc_mg_set_cycle(self.h, int(cycle))  # mg_cycle: 0 V, 1 F, 2 W
        lib().orc_mg_set_reduced(self.h, int(bool(reduced)))
        lib().orc_mg_finalize(self.h, int(fp32))
        self.nc = len(levels[-1]["A"][0]) - 1

    def coarse_inverse(self):
        out = np.zeros((self.nc, self.nc))
        lib().orc_mg_get_coarse_inverse(self.h, p(out))
        return out

    def apply(self, b):
        x = np.zeros_like(b)
        if b.dtype == np.float64:
            lib().orc_mg_apply_d(self.h, p(b), p(x), b.shape[1])
        else:
            lib().orc_mg_apply_f(self.h, p(b), p(x), b.shape[1])
        return x

    def __del__(self):
        try:
            lib().orc_mg_destroy(self.h)
        except Exception:
            pass


def pbicgstab(rp, ci, v, b, x0, mg=None, max_iters=1000, abs_tol=0.0, rel_tol=1e-8):
    """FP64 (P)BiCGStab; returns (x, iters, history[iters+1, nv], status, res0)."""
    n, nv = b.shape
    x = np.array(x0, dtype=np.float64, copy=True)
    cap = max_iters + 2
    hist = np.zeros((cap, nv))
    status = np.zeros(nv, np.int32)
    res0 = np.zeros(nv)
    it = lib().orc_pbicgstab_d(n, p(rp), p(ci), p(v), mg.h if mg is not None else None, p(b), p(x), nv,
                               max_iters, abs_tol, rel_tol, p(hist), cap, p(status), p(res0))
    return x, it, hist[: it + 1], status, res0


def set_seq_dot(on):
    """Krylov inner products in the reference's single-core order (FP64) instead
    of the fixed tree the GPU shares; used only to compare whole solves with the
    reference's loops compiled unchanged (oracle/ref_loops)."""
    lib().orc_set_seq_dot(int(bool(on)))


def chebyshev(rp, ci, v, b, x, order, fraction, min_eig, max_eig):
    """One Chebyshev smoothing of x (in place) with the given spectrum bounds."""
    n, nv = b.shape
    lib().orc_chebyshev_d(n, p(rp), p(ci), p(v), p(b), p(x), nv, order, fraction, min_eig, max_eig)
    return x


def set_merged_bicgstab(on):
    """Unpreconditioned solves with the direction update of the reference's
    MergedBiCGStab (p = r + beta p - (beta omega) v, left to right) instead of
    BiCGStab's (r + (-omega beta) v + beta p)."""
    lib().orc_set_merged_bicgstab(int(bool(on)))


def num_threads():
    """Host threads of the oracle's parallel loops."""
    return int(lib().orc_num_threads())


def set_num_threads(t):
    lib().orc_set_num_threads(int(t))


def pcg(rp, ci, v, b, x0, mg=None, max_iters=1000, abs_tol=0.0, rel_tol=1e-8):
    """FP64 PCG (mg=None: identity preconditioner); returns as pbicgstab."""
    n, nv = b.shape
    x = np.array(x0, dtype=np.float64, copy=True)
    cap = max_iters + 2
    hist = np.zeros((cap, nv))
    status = np.zeros(nv, np.int32)
    res0 = np.zeros(nv)
    it = lib().orc_pcg_d(n, p(rp), p(ci), p(v), mg.h if mg is not None else None, p(b), p(x), nv,
                         max_iters, abs_tol, rel_tol, p(hist), cap, p(status), p(res0))
    return x, it, hist[: it + 1], status, res0


def rbicgstab(rp, ci, v, b, x0, mg=None, max_iters=1000, abs_tol=0.0, rel_tol=1e-8):
    """FP64 RBiCGStab (mg=None: identity preconditioner); returns as pbicgstab."""
    n, nv = b.shape
    x = np.array(x0, dtype=np.float64, copy=True)
    cap = max_iters + 2
    hist = np.zeros((cap, nv))
    status = np.zeros(nv, np.int32)
    res0 = np.zeros(nv)
    it = lib().orc_rbicgstab_d(n, p(rp), p(ci), p(v), mg.h if mg is not None else None, p(b), p(x), nv,
                               max_iters, abs_tol, rel_tol, p(hist), cap, p(status), p(res0))
    return x, it, hist[: it + 1], status, res0


def ir_pbicgstab(rp, ci, v, b, x0, mg, max_outer=20, max_inner=200, abs_tol=0.0, rel_tol=1e-8,
                 inner_rel=1e-4):
    """Precision form: FP64 refinement around FP32 PBiCGStab + FP32 V-cycle
    (mg built with fp32=True).  Returns (x, outer_iters, history, status, sub_iters)."""
    n, nv = b.shape
    x = np.array(x0, dtype=np.float64, copy=True)
    cap = max_outer + 2
    hist = np.zeros((cap, nv))
    status = np.zeros(nv, np.int32)
    sub = np.zeros(1, np.int32)
    f = lib().orc_ir_pbicgstab
    f.restype = C.c_int
    f.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                  C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    it = f(n, p(rp), p(ci), p(v), mg.h, p(b), p(x), nv, max_outer, max_inner, abs_tol, rel_tol, inner_rel,
           p(hist), cap, p(status), p(sub))
    return x, it, hist[: it + 1], status, int(sub[0])


def gen27(n, kx=1.0, ky=1.0, kz=1e-3):
    """The 27-point anisotropic operator on an n^3 grid: (rp, ci, v)."""
    rows = np.zeros(1, np.int64)
    nnz = np.zeros(1, np.int64)
    lib().orc_gen27_size(n, p(rows), p(nnz))
    rp = np.zeros(int(rows[0]) + 1, np.int32)
    ci = np.zeros(int(nnz[0]), np.int32)
    v = np.zeros(int(nnz[0]))
    lib().orc_gen27(n, kx, ky, kz, p(rp), p(ci), p(v))
    return rp, ci, v


# defaults of the reference's MultiGrid parameter family
# (src/param/xamg_params_details.h:244-267) for the keys this setup reads
AMG_DEFAULTS = dict(mg_max_levels=25, mg_coarse_matrix_size=100, mg_strength_threshold=0.5, mg_trunc_factor=0.25,
                    mg_Pmax_elements=4, mg_max_row_sum=0.9, mg_coarsening_type=6)


def amg_setup(rp, ci, v, **prm):
    """Oracle AMG hierarchy (classical strength, Ruge-Stueben first pass [+
    second pass for coarsening types 1/3/6], extended+i interpolation with
    truncation, Galerkin products) from the reference's parameter keys.
    Returns the level list in the form MG() takes."""
    q = dict(AMG_DEFAULTS, **prm)
    rp = np.ascontiguousarray(rp, np.int32)
    ci = np.ascontiguousarray(ci, np.int32)
    v = np.ascontiguousarray(v, np.float64)
    h = lib().orc_amg_setup(len(rp) - 1, p(rp), p(ci), p(v), int(q["mg_max_levels"]), int(q["mg_coarse_matrix_size"]),
                            float(q["mg_strength_threshold"]), float(q["mg_trunc_factor"]), int(q["mg_Pmax_elements"]),
                            float(q["mg_max_row_sum"]), int(q["mg_coarsening_type"]))
    out = []
    try:
        for l in range(lib().orc_amg_num_levels(h)):
            info = np.zeros(4, np.int64)
            lib().orc_amg_level_info(h, l, p(info))
            n, nnz, ncP, nnzP = (int(t) for t in info)
            A = (np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz))
            P = (np.zeros(n + 1, np.int32), np.zeros(nnzP, np.int32), np.zeros(nnzP)) if nnzP else None
            lib().orc_amg_level_export(h, l, p(A[0]), p(A[1]), p(A[2]), p(P[0]) if P else None,
                                       p(P[1]) if P else None, p(P[2]) if P else None)
            out.append(dict(n=n, A=A, P=P, ncP=ncP))
    finally:
        lib().orc_amg_destroy(h)
    return out
