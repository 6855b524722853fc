"""ctypes binding of the reference-loop libraries (oracle/_ref/
libxamg_ref_loops_{generic,haswell,contract}.so, built by
oracle/build_ref_loops.py from the reference's own loop files): test and
benchmark-baseline infrastructure, never part of the product.

lib(kind) loads one build (None when it was not built: the reference tree
was absent and no prebuilt library travelled with the repository); solver()
runs one of the reference's own Krylov solver classes over its compiled
loops, the generators and the reader return the reference's problems (see
ref_loops.h)."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")
_libs = {}


def path(kind):
    return os.path.join(REF, "libxamg_ref_loops_%s.so" % kind)


def lib(kind, build=True):
    if kind in _libs:
        return _libs[kind]
    if not os.path.exists(path(kind)) and build:
        import build_ref_loops

        build_ref_loops.build()
    if not os.path.exists(path(kind)):
        return None
    L = C.CDLL(path(kind))
    i64, vp, ci_, cd = C.c_int64, C.c_void_p, C.c_int, C.c_double
    PP = C.POINTER(C.c_void_p)
    for name in ("ref_csr_ax_y_d", "ref_csr_ax_y_f", "ref_csr_axpy_d", "ref_csr_axpy_f"):
        getattr(L, name).argtypes = [i64, vp, vp, vp, vp, vp, ci_]
    for name in ("ref_hsgs_d", "ref_hsgs_f"):
        getattr(L, name).argtypes = [i64, vp, vp, vp, vp, vp, vp, vp, ci_, ci_, vp]
    for name in ("ref_dense_ax_y_d", "ref_dense_ax_y_f"):
        getattr(L, name).argtypes = [i64, i64, vp, vp, vp, ci_]
    L.ref_dot_d.argtypes = [i64, ci_, vp, vp, vp]
    L.ref_axpby_d.argtypes = [i64, ci_, vp, vp, vp, vp]
    L.ref_axpby_z_d.argtypes = [i64, ci_, vp, vp, vp, vp, vp]
    L.ref_axpbypcz_d.argtypes = [i64, ci_, vp, vp, vp, vp, vp, vp]
    L.ref_xdivy_z_d.argtypes = [i64, ci_, vp, vp, vp]
    L.ref_ax_y_d.argtypes = [i64, ci_, vp, vp, vp]
    L.ref_scal_d.argtypes = [i64, ci_, vp, vp]
    L.ref_dense_inverse_d.argtypes = [i64, vp, vp]
    L.ref_jacobi_d.argtypes = [i64, vp, vp, vp, vp, vp, vp, vp, ci_, ci_]
    L.ref_hier_create.restype = vp
    L.ref_hier_create.argtypes = [ci_, vp, PP, PP, PP, PP, PP, PP, PP, PP, PP, vp, PP, cd, ci_, ci_, ci_]
    L.ref_hier_apply_d.argtypes = [vp, vp, vp, ci_]
    L.ref_hier_destroy.argtypes = [vp]
    L.ref_mg_create.restype = vp
    L.ref_mg_create.argtypes = [ci_, ci_, vp, PP, PP, PP, PP, PP, PP, PP, PP, PP, vp, PP, cd, ci_, ci_, ci_]
    L.ref_mg_apply_d.argtypes = [vp, vp, vp]
    L.ref_mg_destroy.argtypes = [vp]
    L.ref_mg_set_chebyshev.argtypes = [vp, ci_, cd, vp, vp]
    L.ref_solver_d.argtypes = [ci_, vp, i64, vp, vp, vp, vp, vp, ci_, ci_, cd, cd, vp, ci_]
    L.ref_chebyshev_d.argtypes = [i64, vp, vp, vp, vp, vp, ci_, ci_, cd, cd, cd]
    L.ref_channel_cube_d.restype = C.c_int64
    L.ref_channel_cube_d.argtypes = [ci_, ci_, ci_, vp, vp, vp, vp, vp]
    L.ref_read_system_d.restype = C.c_int64
    L.ref_read_system_d.argtypes = [C.c_char_p, ci_, vp, vp, vp, vp, vp, vp]
    L.ref_cube_d.restype = C.c_int64
    L.ref_cube_d.argtypes = [i64, i64, i64, ci_, vp, vp, vp, vp]
    _libs[kind] = L
    return L


def p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def transpose(rp, ci, v, ncols):
    """R = P^T with each row's entries in increasing column order."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
    order = np.lexsort((rows, ci))
    rrp = np.zeros(ncols + 1, np.int32)
    np.cumsum(np.bincount(ci, minlength=ncols), out=rrp[1:])
    return rrp, np.ascontiguousarray(rows[order]), np.ascontiguousarray(v[order])


def _ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data if a is not None else None for a in arrs])


def _hier_args(levels, blocks):
    nrows = np.array([lv["n"] for lv in levels], np.int64)
    R = [transpose(*lv["P"], lv["ncP"]) if lv.get("P") is not None else None for lv in levels]
    cols = []
    for k in range(3):
        cols.append([np.ascontiguousarray(lv["A"][k]) for lv in levels])
        cols.append([np.ascontiguousarray(lv["P"][k]) if lv.get("P") is not None else None for lv in levels])
        cols.append([r[k] if r is not None else None for r in R])
    arp, prp, rrp, aci, pci, rci, av, pv, rv = cols
    if blocks is None:
        blocks = [np.array([0, lv["n"]], np.int64) for lv in levels]
    blocks = [np.ascontiguousarray(b, np.int64) for b in blocks]
    nb = np.array([len(b) - 1 for b in blocks], np.int32)
    PP = C.POINTER(C.c_void_p)
    tabs = [_ptrs(x) for x in (arp, aci, av, prp, pci, pv, rrp, rci, rv, blocks)]
    cast = [C.cast(t, PP) for t in tabs]
    keep = (nrows, R, cols, blocks, nb, tabs)
    return nrows, cast, nb, keep


def channel_cube(L, scale, nv, const_rhs=False):
    """The reference's channel-with-cube problem: (rp, ci, v, B)."""
    nnz = np.zeros(1, np.int64)
    n = L.ref_channel_cube_d(scale, int(const_rhs), nv, p(nnz), None, None, None, None)
    if n < 0:
        raise ValueError("unsupported scale or nv")
    rp = np.zeros(n + 1, np.int32)
    ci = np.zeros(int(nnz[0]), np.int32)
    v = np.zeros(int(nnz[0]))
    B = np.zeros((n, nv))
    L.ref_channel_cube_d(scale, int(const_rhs), nv, None, p(rp), p(ci), p(v), p(B))
    return rp, ci, v, B


def cube(L, nx, ny, nz, config=0):
    """The reference's cube generator (configurations 0-4): (rp, ci, v)."""
    nnz = np.zeros(1, np.int64)
    n = L.ref_cube_d(nx, ny, nz, config, p(nnz), None, None, None)
    if n < 0:
        raise ValueError("unsupported configuration")
    rp = np.zeros(n + 1, np.int32)
    ci = np.zeros(int(nnz[0]), np.int32)
    v = np.zeros(int(nnz[0]))
    L.ref_cube_d(nx, ny, nz, config, None, p(rp), p(ci), p(v))
    return rp, ci, v


def read_system(L, path, nv=1):
    """The reference's binary system reader: (rp, ci, v, B, X)."""
    nnz = np.zeros(1, np.int64)
    n = L.ref_read_system_d(path.encode(), nv, p(nnz), None, None, None, None, None)
    if n < 0:
        raise ValueError("unsupported nv")
    rp = np.zeros(n + 1, np.int32)
    ci = np.zeros(int(nnz[0]), np.int32)
    v = np.zeros(int(nnz[0]))
    B = np.zeros((n, nv))
    X = np.zeros((n, nv))
    L.ref_read_system_d(path.encode(), nv, None, p(rp), p(ci), p(v), p(B), p(X))
    return rp, ci, v, B, X


SOLVERS = {"BiCGStab": 0, "PBiCGStab": 1, "PCG": 2, "RBiCGStab": 3, "MergedBiCGStab": 4, "MergedPBiCGStab": 5}


def solver(L, method, rp, ci, v, B, levels=None, max_iters=1000, rel_tol=1e-8, relax=0.99, cycle="V",
           smoother="HSGS", sweeps=1, reduced=False, blocks=None, mg_class=True, cheb=None):
    """The reference's own solver class `method` (one of SOLVERS, compiled
    unchanged) from x = 0 on (rp, ci, v).  With `levels` (dicts with n, A, P,
    ncP as the oracle's setup or the library's hierarchy export gives them)
    the preconditioned methods apply the reference's MultiGrid class with
    its HSGS / Jacobi smoother classes (mg_class; else the cycle restated
    over its loops): `cycle` "V", "F" or "W", `smoother` "HSGS"
    (on the hybrid blocks `blocks[l]`, default one block per level) or
    "Jacobi" with `sweeps` before and after, `reduced` for
    mg_reduced_precision (FP32 below the first level, HSGS only).  Without
    levels PCG and RBiCGStab use the identity.  Returns (x, iterations,
    history of the checked squared residual norms)."""
    n, nv = B.shape
    B = np.ascontiguousarray(B, np.float64)
    h = None
    keep = None
    if levels is not None:
        nrows, cast, nb, keep = _hier_args(levels, blocks)
        code = {"HSGS": 0, "Jacobi": 1}[smoother] | ({"V": 0, "F": 1, "W": 2}[cycle] << 4) | (int(reduced) << 8)
        if mg_class:
            h = L.ref_mg_create(nv, len(levels), p(nrows), *cast[:9], p(nb), cast[9], relax, sweeps, sweeps, code)
            if cheb is not None:  # (order, spectrum_fraction, [(min_eig, max_eig) per level])
                mn = np.array([e[0] for e in cheb[2]], np.float64)
                mx = np.array([e[1] for e in cheb[2]], np.float64)
                L.ref_mg_set_chebyshev(h, int(cheb[0]), float(cheb[1]), p(mn), p(mx))
        else:
            h = L.ref_hier_create(len(levels), p(nrows), *cast[:9], p(nb), cast[9], relax, sweeps, sweeps, code)
    try:
        x = np.zeros_like(B)
        hist = np.zeros((max_iters + 2, nv))
        it = L.ref_solver_d(SOLVERS[method] | (16 if (mg_class and h) else 0), h, n, p(rp), p(ci), p(v), p(B),
                            p(x), nv, max_iters, 0.0, rel_tol, p(hist), max_iters + 2)
    finally:
        if h:
            (L.ref_mg_destroy if mg_class else L.ref_hier_destroy)(h)
    if it < 0:
        raise ValueError("unsupported nv or method")
    return x, it, hist[: it + 1]
