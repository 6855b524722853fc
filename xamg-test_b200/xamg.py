"""ctypes binding of libxamg_b200.so (the XAMG C API and the kernel interface).

The classes mirror the reference's C API objects (api/c/xamg_c_api.h): Params,
CsrMatrix, Matrix, Vector and Solver own one handle each.  The library must be
built (build.py); importing this module on a machine with a GPU and no built
library raises instead of falling back to anything else.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxamg_b200.so")

_lib = None

F64, F32 = 0, 1
MEM_LOCAL, MEM_SHARED, MEM_DISTRIBUTED = 0, 1, 2


class XamgError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise XamgError("libxamg_b200.so is not built; run xamg-test_b200/build.py")
        L = C.CDLL(LIB_PATH)
        sz = C.c_size_t
        P = C.c_void_p
        i64 = C.c_int64
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        sig = {
            "XAMG_init": (C.c_int, [C.c_int, P, C.c_char_p]),
            "XAMG_finalize": (C.c_int, []),
            "XAMG_get_nv": (C.c_int, []),
            "XAMG_param_create": (C.c_int, [C.POINTER(sz)]),
            "XAMG_param_add_value_s": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, sz]),
            "XAMG_param_add_value_i": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint32, sz]),
            "XAMG_param_add_value_d": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, sz]),
            "XAMG_param_add_value_b": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint8, sz]),
            "XAMG_param_change_value_d": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, sz]),
            "XAMG_param_change_value_i": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint32, sz]),
            "XAMG_param_override_create": (C.c_int, [C.POINTER(sz)]),
            "XAMG_param_override_add_value": (C.c_int, [C.c_char_p, C.c_char_p, sz]),
            "XAMG_param_override_apply": (C.c_int, [C.c_char_p, sz, sz]),
            "XAMG_param_override_destroy": (C.c_int, [sz]),
            "XAMG_param_set_default": (None, [sz]),
            "XAMG_param_print": (C.c_int, [sz]),
            "XAMG_param_destroy": (C.c_int, [sz]),
            "XAMG_part_create": (C.c_int, [C.POINTER(sz)]),
            "XAMG_part_construct": (C.c_int, [C.c_int, sz]),
            "XAMG_part_get_numa_size": (C.c_int, [sz]),
            "XAMG_vector_create": (C.c_int, [C.POINTER(sz), C.c_int]),
            "XAMG_vector_offset": (C.c_int, [C.c_uint64, sz]),
            "XAMG_vector_alloc_d": (C.c_int, [C.c_int, C.c_uint16, sz]),
            "XAMG_vector_set_part": (C.c_int, [sz, sz]),
            "XAMG_vector_set_val_d": (C.c_int, [C.c_double, sz]),
            "XAMG_vector_download_d": (C.c_int, [P, C.c_uint64, C.c_uint64, C.c_uint16, sz]),
            "XAMG_vector_upload_v": (C.c_int, [sz, sz]),
            "XAMG_vector_upload_d": (C.c_int, [P, C.c_uint64, C.c_uint64, C.c_uint16, sz]),
            "XAMG_vector_destroy": (C.c_int, [sz]),
            "XAMG_csr_matrix_create": (C.c_int, [C.POINTER(sz)]),
            "XAMG_csr_matrix_alloc": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64, sz]),
            "XAMG_csr_matrix_fill": (C.c_int, [P, P, P, sz]),
            "XAMG_csr_matrix_get_nrows": (C.c_uint32, [sz]),
            "XAMG_csr_matrix_destroy": (C.c_int, [sz]),
            "XAMG_matrix_create": (C.c_int, [C.POINTER(sz)]),
            "XAMG_matrix_set_part": (C.c_int, [sz, sz]),
            "XAMG_matrix_construct": (C.c_int, [sz, sz]),
            "XAMG_matrix_destroy": (C.c_int, [sz]),
            "XAMG_solver_create1": (C.c_int, [sz, sz, C.POINTER(sz)]),
            "XAMG_solver_create2": (C.c_int, [sz, sz, sz, sz, C.POINTER(sz)]),
            "XAMG_solver_renew_params": (C.c_int, [sz, sz]),
            "XAMG_solver_solve1": (C.c_int, [C.c_uint16, sz]),
            "XAMG_solver_solve2": (C.c_int, [C.c_uint16, sz, sz, sz]),
            "XAMG_solver_print_info": (C.c_int, [sz]),
            "XAMG_solver_get_convergence_info": (C.c_int, [ip, C.c_uint16, sz]),
            "XAMG_solver_get_iter_info": (C.c_int, [ip, sz]),
            "XAMG_solver_destroy": (C.c_int, [sz]),
            "XAMG_timer": (C.c_double, []),
            "XAMG_barrier": (C.c_int, []),
            "XAMG_b200_set_nv": (C.c_int, [C.c_int]),
            "XAMG_b200_last_error": (C.c_char_p, []),
            "XAMG_b200_synchronize": (C.c_int, []),
            "XAMG_b200_vector_device_ptr": (P, [sz]),
            "XAMG_b200_solver_get_residual_history": (C.c_int, [dp, C.c_int, sz]),
            "XAMG_b200_solver_get_res0": (C.c_int, [dp, sz]),
            "XAMG_b200_solver_last_solve_ms": (C.c_double, [sz]),
            "XAMG_b200_solver_num_levels": (C.c_int, [sz]),
            "XAMG_b200_solver_level_info": (C.c_int, [C.POINTER(i64), C.c_int, sz]),
            "XAMG_b200_solver_export_level": (C.c_int, [P, P, P, P, P, P, C.c_int, sz]),
            "XAMG_b200_solver_export_gs_levels": (C.c_int, [P, P, C.c_int, sz]),
            "XAMG_b200_solver_export_coarse_inverse": (C.c_int, [P, sz]),
            "XAMG_b200_solver_info": (C.c_int, [C.c_char_p, C.c_int, sz]),
            "XAMG_b200_solver_level_eig": (C.c_int, [P, C.c_int, sz]),
            "XAMG_b200_csr_matrix_generate": (C.c_int, [C.c_int, P, P, P, sz]),
            "XAMG_b200_csr_matrix_get_nnz": (i64, [sz]),
            "XAMG_b200_channel_cube_rows": (i64, [C.c_int]),
            "XAMG_b200_generate_channel_cube": (C.c_int, [C.c_int, C.c_int, C.c_int, P, sz]),
            "XAMG_b200_csr_matrix_export": (C.c_int, [P, P, P, sz]),
            "XAMG_b200_csr_matrix_read_bin": (C.c_int, [C.c_char_p, P, P, sz]),
            "XAMG_b200_csr_matrix_write_bin": (C.c_int, [C.c_char_p, P, P, sz]),
            "XAMG_b200_amg_host_create": (C.c_int, [sz, sz, C.POINTER(sz)]),
            "XAMG_b200_amg_host_num_levels": (C.c_int, [sz]),
            "XAMG_b200_amg_host_level_info": (C.c_int, [C.POINTER(i64), C.c_int, sz]),
            "XAMG_b200_amg_host_export_level": (C.c_int, [P, P, P, P, P, P, C.c_int, sz]),
            "XAMG_b200_amg_host_destroy": (C.c_int, [sz]),
            "XAMG_b200_gs_levels_host": (C.c_int, [i64, P, P, i64, P, P, P]),
            "xamg_csr_spmv": (C.c_int, [C.c_int, C.c_int, i64, P, P, P, P, P, C.c_int, P, P]),
            "xamg_spmv_set_variant": (C.c_int, [C.c_int]),
            "xamg_spmv_set_run_rows": (C.c_int, [C.c_int]),
            "xamg_spmv_set_run_form": (C.c_int, [C.c_int]),
            "xamg_spmv_runs_plan_create": (P, [i64, P, P, P, C.c_int, C.c_int]),
            "xamg_spmv_runs_plan_info": (C.c_int, [P, P, P, P, P]),
            "xamg_spmv_runs_analyze": (C.c_int, [i64, P, P, C.c_int, P, P, P]),
            "XAMG_b200_rowpart_create": (C.c_int, [i64, P, P, C.c_int, C.c_int, P]),
            "XAMG_b200_rowpart_info": (C.c_int, [C.c_size_t, P]),
            "XAMG_b200_rowpart_local_csr": (C.c_int, [C.c_size_t, P, P, P]),
            "XAMG_b200_rowpart_halo": (C.c_int, [C.c_size_t, P, P]),
            "XAMG_b200_rowpart_sends": (C.c_int, [C.c_size_t, C.c_int, P, P]),
            "XAMG_b200_rowpart_destroy": (C.c_int, [C.c_size_t]),
            "XAMG_b200_dist_unique_id": (C.c_int, [P]),
            "XAMG_b200_dist_create": (C.c_int, [P, sz, P, sz, C.c_int, C.POINTER(sz)]),
            "XAMG_b200_dist_solve": (C.c_int, [sz, P, P]),
            "XAMG_b200_dist_info": (C.c_int, [sz, P]),
            "XAMG_b200_dist_history": (C.c_int, [sz, P, i64]),
            "XAMG_b200_dist_destroy": (C.c_int, [sz]),
            "xamg_spmv_runs": (C.c_int, [P, C.c_int, C.c_int, P, P, C.c_int, P, P]),
            "xamg_spmv_runs_plan_destroy": (C.c_int, [P]),
            "xamg_gs_plan_create": (P, [i64, P, P, i64, C.c_int]),
            "xamg_gs_plan_levels": (C.c_int, [P, P, P, P]),
            "xamg_gs_plan_set_values": (C.c_int, [P, P, C.c_int]),
            "xamg_gs_plan_error": (C.c_int, [P]),
            "xamg_gs_plan_slots": (C.c_int, [P, P]),
            "XAMG_b200_wait_selftest": (C.c_int, [C.c_int, C.c_int, C.c_double]),
            "xamg_gs_plan_destroy": (None, [P]),
            "xamg_hsgs": (C.c_int, [P, C.c_int, C.c_int, P, P, P, P, P, P, P, P, P]),
            "xamg_jacobi": (C.c_int, [C.c_int, C.c_int, i64, P, P, P, P, P, P, P, P, P]),
            "xamg_dot_part_size": (i64, [i64, C.c_int, C.c_int]),
            "xamg_dot": (C.c_int, [C.c_int, C.c_int, i64, C.c_int, P, P, P, P, P]),
            "xamg_seg_dot": (C.c_int, [C.c_int, C.c_int, C.c_int, P, C.c_int, P, P, P, P]),
            "xamg_dot_noalloc": (C.c_int, [C.c_int, C.c_int, i64, C.c_int, P, P, P, P]),
            "xamg_blas": (C.c_int, [C.c_int, C.c_int, i64, C.c_int, P, P, P, P, P, P, P]),
            "xamg_dense_gemv": (C.c_int, [C.c_int, C.c_int, C.c_int, P, P, P, P]),
            "XAMG_b200_batch_create": (C.c_int, [C.c_int, P, P, P, P, P, sz, C.POINTER(sz)]),
            "XAMG_b200_batch_upload": (C.c_int, [sz, C.c_int, P, P]),
            "XAMG_b200_batch_set_graph": (C.c_int, [sz, C.c_int]),
            "XAMG_b200_batch_solve": (C.c_int, [sz]),
            "XAMG_b200_batch_download": (C.c_int, [sz, C.c_int, P]),
            "XAMG_b200_batch_stats": (C.c_int, [sz, C.c_int, P, P]),
            "XAMG_b200_batch_last_ms": (C.c_double, [sz]),
            "XAMG_b200_batch_last_kernels": (C.c_longlong, [sz]),
            "XAMG_b200_kernel_launches": (C.c_longlong, []),
            "XAMG_b200_kernel_timing": (C.c_int, [C.c_int]),
            "XAMG_b200_gs_sweep_kernel": (C.c_int, []),
            "XAMG_b200_kernel_timing_read": (C.c_int, [C.c_int, P, P, P, P, P]),
            "XAMG_b200_batch_groups": (C.c_int, [sz, P, C.c_int]),
            "XAMG_b200_batch_destroy": (C.c_int, [sz]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise XamgError("xamg error %d: %s" % (rc, lib().XAMG_b200_last_error().decode()))
    return rc


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def kernel_launches():
    """Kernels launched by the library so far (its own launch counter)."""
    return lib().XAMG_b200_kernel_launches()


KCLASS = {0: "gs", 1: "spmv", 2: "gs_grid", 3: "gs_tile", 4: "gs_window", 5: "gs_gather",
          6: "gsw_tile", 7: "gsw_window", 8: "gsw_gather"}


def gs_sweep_kernel():
    """'warp' or 'cta': the kernel of this process's hybrid Gauss-Seidel sweeps."""
    return "warp" if lib().XAMG_b200_gs_sweep_kernel() else "cta"


def kernel_timing(on):
    """Start (True) or stop and discard (False) the CUDA-event timing of the
    Gauss-Seidel sweeps and sparse products inside solves."""
    return bool(lib().XAMG_b200_kernel_timing(int(bool(on))))


def kernel_timing_read(cap=256):
    """Per (kernel class, operator rows): launches, total ms and total
    algorithmic bytes of the timed launches so far; clears the records."""
    kc = np.zeros(cap, np.int32)
    rows = np.zeros(cap, np.int64)
    nl = np.zeros(cap, np.int64)
    ms = np.zeros(cap)
    by = np.zeros(cap)
    g = lib().XAMG_b200_kernel_timing_read(cap, _ptr(kc), _ptr(rows), _ptr(nl), _ptr(ms), _ptr(by))
    if g < 0:
        check(-g)
    return [dict(kernel=KCLASS[int(kc[i])], rows=int(rows[i]), launches=int(nl[i]), ms=float(ms[i]),
                 bytes=float(by[i])) for i in range(g)]


def init(nv=1):
    check(lib().XAMG_init(0, None, b""))
    check(lib().XAMG_b200_set_nv(nv))


def set_nv(nv):
    check(lib().XAMG_b200_set_nv(nv))


class Params:
    """Parameter dictionary (roles/keys of the reference)."""

    def __init__(self, spec=None, overrides=None):
        h = C.c_size_t()
        check(lib().XAMG_param_create(C.byref(h)))
        self.h = h.value
        for role, kv in (spec or {}).items():
            for k, v in kv.items():
                self.add(role, k, v)
        for role, kv in (overrides or {}).items():
            o = C.c_size_t()
            check(lib().XAMG_param_override_create(C.byref(o)))
            for k, v in kv.items():
                check(lib().XAMG_param_override_add_value(k.encode(), str(v).encode(), o.value))
            check(lib().XAMG_param_override_apply(role.encode(), self.h, o.value))
            check(lib().XAMG_param_override_destroy(o.value))
        lib().XAMG_param_set_default(self.h)

    def add(self, role, key, v):
        r, k = role.encode(), key.encode()
        if isinstance(v, bool):
            check(lib().XAMG_param_add_value_b(r, k, int(v), self.h))
        elif isinstance(v, int):
            check(lib().XAMG_param_add_value_i(r, k, v, self.h))
        elif isinstance(v, float):
            check(lib().XAMG_param_add_value_d(r, k, v, self.h))
        else:
            check(lib().XAMG_param_add_value_s(r, k, str(v).encode(), self.h))

    def change(self, role, key, v):
        if isinstance(v, float):
            check(lib().XAMG_param_change_value_d(role.encode(), key.encode(), v, self.h))
        else:
            check(lib().XAMG_param_change_value_i(role.encode(), key.encode(), int(v), self.h))


class CsrMatrix:
    """Host CSR matrix object (XAMG_csr_matrix_*)."""

    def __init__(self):
        h = C.c_size_t()
        check(lib().XAMG_csr_matrix_create(C.byref(h)))
        self.h = h.value

    @classmethod
    def from_arrays(cls, rp, ci, v):
        m = cls()
        rp = np.ascontiguousarray(rp, dtype=np.int32)
        ci = np.ascontiguousarray(ci, dtype=np.int32)
        v = np.ascontiguousarray(v, dtype=np.float64)
        n = len(rp) - 1
        check(lib().XAMG_csr_matrix_alloc(n, n, len(ci), m.h))
        check(lib().XAMG_csr_matrix_fill(_ptr(rp), _ptr(ci), _ptr(v), m.h))
        return m

    @classmethod
    def cube(cls, nx, ny, nz, config=0):
        m = cls()
        ia = np.array([nx, ny, nz, config], dtype=np.int64)
        check(lib().XAMG_b200_csr_matrix_generate(0, _ptr(ia), None, None, m.h))
        return m

    @classmethod
    def channel_cube(cls, scale=1, nv=1, const_rhs=False):
        """The reference's channel-with-cube system: (matrix, B[rows, nv])."""
        rows = lib().XAMG_b200_channel_cube_rows(scale)
        if rows < 0:
            raise XamgError("channel_cube: scale must be 1, 2 or 3")
        m = cls()
        B = np.zeros((rows, nv))
        check(lib().XAMG_b200_generate_channel_cube(scale, int(const_rhs), nv, _ptr(B), m.h))
        return m, B

    @classmethod
    def aniso27(cls, n, kx=1.0, ky=1.0, kz=1e-3):
        m = cls()
        ia = np.array([n], dtype=np.int64)
        da = np.array([kx, ky, kz], dtype=np.float64)
        check(lib().XAMG_b200_csr_matrix_generate(1, _ptr(ia), _ptr(da), None, m.h))
        return m

    @classmethod
    def faces7(cls, nx, ny, nz, kx, ky, kz):
        m = cls()
        ia = np.array([nx, ny, nz], dtype=np.int64)
        f = np.ascontiguousarray(np.concatenate([np.ravel(kx), np.ravel(ky), np.ravel(kz)]), dtype=np.float64)
        assert f.size == (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
        check(lib().XAMG_b200_csr_matrix_generate(2, _ptr(ia), None, _ptr(f), m.h))
        return m

    @classmethod
    def read_bin(cls, path):
        m = cls()
        check(lib().XAMG_b200_csr_matrix_read_bin(path.encode(), None, None, m.h))
        n = m.nrows
        b = np.zeros(n)
        x = np.zeros(n)
        check(lib().XAMG_b200_csr_matrix_read_bin(path.encode(), _ptr(b), _ptr(x), m.h))
        return m, b, x

    @property
    def nrows(self):
        return lib().XAMG_csr_matrix_get_nrows(self.h)

    @property
    def nnz(self):
        return lib().XAMG_b200_csr_matrix_get_nnz(self.h)

    def arrays(self):
        n, nnz = self.nrows, self.nnz
        rp = np.zeros(n + 1, np.int32)
        ci = np.zeros(nnz, np.int32)
        v = np.zeros(nnz, np.float64)
        check(lib().XAMG_b200_csr_matrix_export(_ptr(rp), _ptr(ci), _ptr(v), self.h))
        return rp, ci, v

    def __del__(self):
        try:
            lib().XAMG_csr_matrix_destroy(self.h)
        except Exception:
            pass


class Matrix:
    """Device matrix (XAMG_matrix_*), built from a CsrMatrix."""

    def __init__(self, csr):
        h = C.c_size_t()
        check(lib().XAMG_matrix_create(C.byref(h)))
        self.h = h.value
        check(lib().XAMG_matrix_construct(csr.h, self.h))
        self.n = csr.nrows

    def __del__(self):
        try:
            lib().XAMG_matrix_destroy(self.h)
        except Exception:
            pass


class Vector:
    """Block vector n x nv (device-resident unless mode == MEM_LOCAL)."""

    def __init__(self, n, nv, mode=MEM_DISTRIBUTED):
        h = C.c_size_t()
        check(lib().XAMG_vector_create(C.byref(h), mode))
        self.h = h.value
        self.n, self.nv = n, nv
        check(lib().XAMG_vector_alloc_d(n, nv, self.h))

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.n, self.nv)
        check(lib().XAMG_vector_upload_d(_ptr(a), self.n, 0, self.nv, self.h))

    def download(self, out=None):
        out = np.empty((self.n, self.nv)) if out is None else out
        check(lib().XAMG_vector_download_d(_ptr(out), self.n, 0, self.nv, self.h))
        return out

    def set(self, v):
        check(lib().XAMG_vector_set_val_d(float(v), self.h))

    @property
    def device_ptr(self):
        return lib().XAMG_b200_vector_device_ptr(self.h)

    def __del__(self):
        try:
            lib().XAMG_vector_destroy(self.h)
        except Exception:
            pass


class Solver:
    """Solver tree (XAMG_solver_create2 / solve / stats)."""

    def __init__(self, A, params, x=None, b=None):
        h = C.c_size_t()
        if x is None:
            check(lib().XAMG_solver_create1(A.h, params.h, C.byref(h)))
        else:
            check(lib().XAMG_solver_create2(A.h, params.h, x.h, b.h, C.byref(h)))
        self.h = h.value
        self.A, self.params, self.x, self.b = A, params, x, b

    def solve(self, x=None, b=None):
        nv = lib().XAMG_get_nv()
        if x is None:
            check(lib().XAMG_solver_solve1(nv, self.h))
        else:
            check(lib().XAMG_solver_solve2(nv, x.h, b.h, self.h))

    def renew(self, params):
        check(lib().XAMG_solver_renew_params(params.h, self.h))

    def iters(self):
        it = (C.c_int * 2)()
        check(lib().XAMG_solver_get_iter_info(it, self.h))
        return it[0], it[1]

    def converged(self):
        nv = lib().XAMG_get_nv()
        c = (C.c_int * nv)()
        check(lib().XAMG_solver_get_convergence_info(c, nv, self.h))
        return [bool(v) for v in c]

    def history(self):
        nv = lib().XAMG_get_nv()
        cap = 100000
        buf = np.zeros(cap * nv)
        cnt = lib().XAMG_b200_solver_get_residual_history(buf.ctypes.data_as(C.POINTER(C.c_double)), cap, self.h)
        return buf[: cnt * nv].reshape(cnt, nv)

    def last_ms(self):
        return lib().XAMG_b200_solver_last_solve_ms(self.h)

    def info(self):
        buf = C.create_string_buffer(4096)
        check(lib().XAMG_b200_solver_info(buf, 4096, self.h))
        return buf.value.decode()

    def num_levels(self):
        return lib().XAMG_b200_solver_num_levels(self.h)

    def level_eig(self, l):
        out = np.zeros(2)
        check(lib().XAMG_b200_solver_level_eig(_ptr(out), l, self.h))
        return float(out[0]), float(out[1])

    def level(self, l):
        info = (C.c_int64 * 6)()
        check(lib().XAMG_b200_solver_level_info(info, l, self.h))
        n, nnz, ncP, nnzP, nlf, nlb = list(info)
        rpA = np.zeros(n + 1, np.int32)
        ciA = np.zeros(nnz, np.int32)
        vA = np.zeros(nnz)
        rpP = np.zeros(n + 1, np.int32) if nnzP else None
        ciP = np.zeros(nnzP, np.int32) if nnzP else None
        vP = np.zeros(nnzP) if nnzP else None
        check(lib().XAMG_b200_solver_export_level(_ptr(rpA), _ptr(ciA), _ptr(vA), _ptr(rpP), _ptr(ciP), _ptr(vP), l, self.h))
        return dict(n=n, A=(rpA, ciA, vA), P=(rpP, ciP, vP) if nnzP else None, ncP=ncP, nlev=(nlf, nlb))

    def gs_levels(self, l):
        n = self.level(l)["n"]
        lf = np.zeros(n, np.int32)
        lb = np.zeros(n, np.int32)
        check(lib().XAMG_b200_solver_export_gs_levels(_ptr(lf), _ptr(lb), l, self.h))
        return lf, lb

    def coarse_inverse(self):
        L = self.num_levels()
        n = self.level(L - 1)["n"]
        out = np.zeros((n, n))
        check(lib().XAMG_b200_solver_export_coarse_inverse(_ptr(out), self.h))
        return out

    def __del__(self):
        try:
            lib().XAMG_solver_destroy(self.h)
        except Exception:
            pass


def amg_host(csr, params):
    """Host-only AMG setup; returns the level list (A, P arrays) like Solver.level."""
    h = C.c_size_t()
    check(lib().XAMG_b200_amg_host_create(csr.h, params.h, C.byref(h)))
    out = []
    try:
        for l in range(lib().XAMG_b200_amg_host_num_levels(h.value)):
            info = (C.c_int64 * 4)()
            check(lib().XAMG_b200_amg_host_level_info(info, l, h.value))
            n, nnz, ncP, nnzP = list(info)
            rpA, ciA, vA = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
            rpP = np.zeros(n + 1, np.int32) if nnzP else None
            ciP = np.zeros(nnzP, np.int32) if nnzP else None
            vP = np.zeros(nnzP) if nnzP else None
            check(lib().XAMG_b200_amg_host_export_level(_ptr(rpA), _ptr(ciA), _ptr(vA), _ptr(rpP), _ptr(ciP), _ptr(vP), l, h.value))
            out.append(dict(n=n, A=(rpA, ciA, vA), P=(rpP, ciP, vP) if nnzP else None, ncP=ncP))
    finally:
        lib().XAMG_b200_amg_host_destroy(h.value)
    return out


class RowPart:
    """One rank's rows of a system for a multi-GPU solve: the local matrix with
    columns renumbered [owned | halo], the halo slots and the per-peer send
    lists (host arrays; see XAMG_b200_rowpart_* in include/xamg_b200.h)."""

    def __init__(self, rp, ci, nranks, rank):
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        self.h = C.c_size_t()
        check(lib().XAMG_b200_rowpart_create(len(rp) - 1, _ptr(rp), _ptr(ci), nranks, rank, C.byref(self.h)))
        info = np.zeros(4, np.int64)
        check(lib().XAMG_b200_rowpart_info(self.h.value, _ptr(info)))
        self.first, self.nrows, nnz, nhalo = (int(v) for v in info)
        self.rp = np.zeros(self.nrows + 1, np.int32)
        self.ci = np.zeros(nnz, np.int32)
        self.src = np.zeros(nnz, np.int64)
        check(lib().XAMG_b200_rowpart_local_csr(self.h.value, _ptr(self.rp), _ptr(self.ci), _ptr(self.src)))
        self.halo = np.zeros(nhalo, np.int64)
        self.owner = np.zeros(nhalo, np.int32)
        check(lib().XAMG_b200_rowpart_halo(self.h.value, _ptr(self.halo), _ptr(self.owner)))
        self.sends = {}
        for peer in range(nranks):
            if peer == rank:
                continue
            cnt = np.zeros(1, np.int64)
            check(lib().XAMG_b200_rowpart_sends(self.h.value, peer, None, _ptr(cnt)))
            rows = np.zeros(int(cnt[0]), np.int64)
            check(lib().XAMG_b200_rowpart_sends(self.h.value, peer, _ptr(rows), _ptr(cnt)))
            self.sends[peer] = rows

    def __del__(self):
        try:
            lib().XAMG_b200_rowpart_destroy(self.h.value)
        except Exception:
            pass


def gs_levels_host(rp, ci, block_rows=0):
    n = len(rp) - 1
    lf = np.zeros(n, np.int32)
    lb = np.zeros(n, np.int32)
    nl = np.zeros(2, np.int32)
    check(lib().XAMG_b200_gs_levels_host(n, _ptr(np.ascontiguousarray(rp, np.int32)), _ptr(np.ascontiguousarray(ci, np.int32)), block_rows, _ptr(lf), _ptr(lb), _ptr(nl)))
    return lf, lb, tuple(nl)


def device_ptr(t):
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else C.c_void_p(t.data_ptr())


class Batch:
    """Independent systems solved together (XAMG_b200_batch_*): systems is a
    list of (CsrMatrix, nv); params supplies the solver and preconditioner."""

    def __init__(self, systems, params):
        arrs = [m.arrays() for m, _ in systems]
        self._keep = [(np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                       np.ascontiguousarray(v, np.float64)) for rp, ci, v in arrs]
        ns = len(systems)
        self.n = [len(k[0]) - 1 for k in self._keep]
        self.nv = [int(nv) for _, nv in systems]
        n = np.array(self.n, np.int64)
        nv = np.array(self.nv, np.int32)
        rp = (C.c_void_p * ns)(*[k[0].ctypes.data for k in self._keep])
        ci = (C.c_void_p * ns)(*[k[1].ctypes.data for k in self._keep])
        v = (C.c_void_p * ns)(*[k[2].ctypes.data for k in self._keep])
        h = C.c_size_t()
        check(lib().XAMG_b200_batch_create(ns, _ptr(n), rp, ci, v, _ptr(nv), params.h, C.byref(h)))
        self.h = h.value
        self.params = params

    def upload(self, sys, b, x0=None):
        b = np.ascontiguousarray(b, np.float64).reshape(self.n[sys], self.nv[sys])
        x0 = None if x0 is None else np.ascontiguousarray(x0, np.float64).reshape(self.n[sys], self.nv[sys])
        check(lib().XAMG_b200_batch_upload(self.h, sys, _ptr(b), None if x0 is None else _ptr(x0)))

    def set_graph(self, on):
        check(lib().XAMG_b200_batch_set_graph(self.h, int(bool(on))))

    def solve(self):
        check(lib().XAMG_b200_batch_solve(self.h))

    def download(self, sys):
        out = np.empty((self.n[sys], self.nv[sys]))
        check(lib().XAMG_b200_batch_download(self.h, sys, _ptr(out)))
        return out

    def stats(self, sys):
        it = np.zeros(self.nv[sys], np.int32)
        rr = np.zeros(self.nv[sys])
        check(lib().XAMG_b200_batch_stats(self.h, sys, _ptr(it), _ptr(rr)))
        return it, rr

    def last_ms(self):
        return lib().XAMG_b200_batch_last_ms(self.h)

    def last_kernels(self):
        return lib().XAMG_b200_batch_last_kernels(self.h)

    def groups(self):
        out = np.zeros(4 * 64, np.int32)
        g = lib().XAMG_b200_batch_groups(self.h, _ptr(out), out.size)
        return [tuple(int(v) for v in out[4 * i:4 * i + 4]) for i in range(g)]

    def __del__(self):
        try:
            lib().XAMG_b200_batch_destroy(self.h)
        except Exception:
            pass


def dist_unique_id():
    """A new NCCL unique id (128 bytes) for DistSolver."""
    buf = (C.c_char * 128)()
    check(lib().XAMG_b200_dist_unique_id(buf))
    return bytes(buf)


class DistSolver:
    """This rank's part of a row-partitioned (P)BiCGStab solve of one system
    over several GPUs (XAMG_b200_dist_*).  rp, ci, v: the GLOBAL host CSR
    arrays; uid: the same 128-byte NCCL id on every rank."""

    def __init__(self, rp, ci, v, nranks, rank, params, nv, uid):
        self.part = RowPart(rp, ci, nranks, rank)
        v = np.ascontiguousarray(v, np.float64)
        ub = (C.c_char * 128).from_buffer_copy(uid)
        h = C.c_size_t()
        check(lib().XAMG_b200_dist_create(ub, self.part.h.value, _ptr(v), params.h, nv, C.byref(h)))
        self.h = h.value
        self.nv = nv
        self.params = params

    def solve(self, b_ptr, x_ptr):
        """b, x: device pointers of this rank's rows (rows x nv FP64)."""
        check(lib().XAMG_b200_dist_solve(self.h, C.c_void_p(b_ptr), C.c_void_p(x_ptr)))

    def info(self):
        out = np.zeros(4, np.int64)
        check(lib().XAMG_b200_dist_info(self.h, _ptr(out)))
        return dict(iters=int(out[0]), converged=bool(out[1]), rows=int(out[2]), hist=int(out[3]))

    def history(self):
        n = self.info()["hist"]
        out = np.zeros(max(n, 1))
        check(lib().XAMG_b200_dist_history(self.h, _ptr(out), n))
        return out[:n].reshape(-1, self.nv)

    def __del__(self):
        try:
            lib().XAMG_b200_dist_destroy(self.h)
        except Exception:
            pass
