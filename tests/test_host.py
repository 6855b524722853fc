"""Host-side logic of the library: C ABI exports, parameters, generators, AMG
setup and Gauss-Seidel schedules (no GPU needed)."""
import os
import re

import numpy as np
import pytest

import oracle as orc
import util
import xamg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("xamg_c_api.h", "xamg_b200.h", "xamg_learned.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b((?:XAMG|xamg|xcnn)_\w+)\s*\(", src):
            if m.group(1) != "XAMG_id_get_comm":
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    import ctypes
    lib = ctypes.CDLL(xamg.LIB_PATH)
    names = declared_symbols()
    assert len(names) > 90
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_api_surface_is_complete():
    # every function of the reference's api/c/xamg_c_api.h:43-122
    ref = """XAMG_init XAMG_finalize XAMG_get_nv XAMG_id_get_proc XAMG_id_get_nprocs
    XAMG_id_get_comm_ptr XAMG_param_create XAMG_param_add_value_s XAMG_param_add_value_i
    XAMG_param_add_value_d XAMG_param_add_value_b XAMG_param_forced_change_value_s
    XAMG_param_forced_change_value_i XAMG_param_forced_change_value_d
    XAMG_param_forced_change_value_b XAMG_param_change_value_s XAMG_param_change_value_i
    XAMG_param_change_value_d XAMG_param_change_value_b XAMG_param_override_create
    XAMG_param_override_add_value XAMG_param_override_apply XAMG_param_override_destroy
    XAMG_param_set_default XAMG_param_print XAMG_param_destroy XAMG_part_create
    XAMG_part_construct XAMG_part_get_numa_size XAMG_part_destroy XAMG_vector_create
    XAMG_vector_offset XAMG_vector_alloc_d XAMG_vector_set_part XAMG_vector_set_val_d
    XAMG_vector_download_d XAMG_vector_upload_v XAMG_vector_upload_d XAMG_vector_destroy
    XAMG_csr_matrix_create XAMG_csr_matrix_alloc XAMG_csr_matrix_fill XAMG_csr_matrix_offset
    XAMG_csr_matrix_get_nrows XAMG_csr_matrix_destroy XAMG_matrix_create XAMG_matrix_set_part
    XAMG_matrix_construct XAMG_matrix_destroy XAMG_solver_create1 XAMG_solver_create2
    XAMG_solver_renew_params XAMG_solver_solve1 XAMG_solver_solve2 XAMG_solver_print_info
    XAMG_solver_get_convergence_info XAMG_solver_get_iter_info XAMG_solver_destroy
    XAMG_timer XAMG_barrier""".split()
    assert set(ref) <= declared_symbols()


def test_params_defaults_and_overrides():
    L = xamg.lib()
    p = xamg.Params({"solver": {"method": "PBiCGStab"}, "preconditioner": {"method": "MultiGrid"}},
                    overrides={"preconditioner": {"mg_coarsening_type": "8@lev0-1"}})
    assert p.h >= 0
    # unknown key and wrong type are refused with code 2
    assert L.XAMG_param_add_value_i(b"solver", b"no_such_key", 1, p.h) == 2
    assert L.XAMG_param_add_value_s(b"solver", b"max_iters", b"x", p.h) == 2
    assert L.XAMG_param_change_value_d(b"solver", b"rel_tolerance", 1e-6, p.h) == 0
    assert L.XAMG_param_print(12345) == 2
    assert b"invalid param handle" in L.XAMG_b200_last_error()


def test_nv_mismatch_and_bad_handles_return_codes():
    L = xamg.lib()
    xamg.check(L.XAMG_b200_set_nv(4))
    h = xamg.C.c_size_t()
    xamg.check(L.XAMG_vector_create(xamg.C.byref(h), xamg.MEM_LOCAL))
    assert L.XAMG_vector_alloc_d(10, 2, h.value) == 2
    assert L.XAMG_vector_alloc_d(10, 4, h.value) == 0
    a = np.arange(40, dtype=np.float64)
    assert L.XAMG_vector_upload_d(xamg._ptr(a), 10, 0, 4, h.value) == 0
    out = np.zeros(40)
    assert L.XAMG_vector_download_d(xamg._ptr(out), 10, 0, 4, h.value) == 0
    assert np.all(out == a)
    assert L.XAMG_vector_download_d(xamg._ptr(out), 11, 0, 4, h.value) == 2
    assert L.XAMG_b200_set_nv(3) == 2
    assert L.XAMG_solver_solve1(4, 999) == 2
    xamg.check(L.XAMG_b200_set_nv(1))


def test_cube_generator_matches_reference_layout():
    m = xamg.CsrMatrix.cube(32, 32, 32, 0)
    assert m.nrows == 32768 and m.nnz == 223232
    rp, ci, v = m.arrays()
    # row order: diagonal first, then ascending (b, s, w, e, n, t); row sums
    # zero inside, positive (Dirichlet) on the boundary
    for r in (0, 1000, 16912, 32767):
        cols = ci[rp[r]:rp[r + 1]]
        assert cols[0] == r and np.all(np.diff(cols[1:]) > 0)
    inner = 16912
    assert abs(v[rp[inner]:rp[inner + 1]].sum()) < 1e-9 * v[rp[inner]]
    assert v[rp[inner]] == 6 * 32 * 32


def test_27pt_generator():
    m = xamg.CsrMatrix.aniso27(8)
    rp, ci, v = m.arrays()
    assert m.nnz == (3 * 8 - 2) ** 3
    import scipy.sparse as sp
    A = sp.csr_matrix((v, ci, rp), copy=True)
    assert abs(A - A.T).max() < 1e-15
    assert np.all(v[rp[:-1]] > 0) and np.all(np.delete(v, rp[:-1]) < 0)


def test_amg_setup_structure():
    m = xamg.CsrMatrix.aniso27(20)
    prm = xamg.Params(util.amg_params(max_levels=6))
    lv = xamg.amg_host(m, prm)
    assert 2 <= len(lv) <= 6
    for l in range(len(lv) - 1):
        n, nc = lv[l]["n"], lv[l]["ncP"]
        assert nc == lv[l + 1]["n"] and nc < n
        prp, pci, pv = lv[l]["P"]
        assert np.all(np.diff(prp) <= 4)  # P_max_elmts = 4
        # coarse operator rows: diagonal first, then ascending
        rp, ci, v = lv[l + 1]["A"]
        for r in range(0, lv[l + 1]["n"], 7):
            assert ci[rp[r]] == r and np.all(np.diff(ci[rp[r] + 1:rp[r + 1]]) > 0)
        # Galerkin: A_c == P^T A P
        import scipy.sparse as sp
        A = sp.csr_matrix((lv[l]["A"][2], lv[l]["A"][1], lv[l]["A"][0]), shape=(n, n), copy=True)
        P = sp.csr_matrix((pv, pci, prp), shape=(n, nc), copy=True)
        Ac = sp.csr_matrix((v, ci, rp), shape=(nc, nc), copy=True)
        D = (P.T @ A @ P - Ac)
        assert abs(D).max() <= 1e-12 * abs(Ac).max()
    # the setup is deterministic
    lv2 = xamg.amg_host(m, prm)
    for a, b in zip(lv, lv2):
        for q in range(3):
            assert np.array_equal(a["A"][q], b["A"][q])


def test_amg_preconditioner_quality():
    rng = np.random.default_rng(7)
    m = xamg.CsrMatrix.aniso27(16)
    rp, ci, v = m.arrays()
    mg = orc.MG(xamg.amg_host(m, xamg.Params(util.amg_params(max_levels=6))))
    b = rng.uniform(-1, 1, (m.nrows, 2))
    x, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, b, np.zeros_like(b), mg=mg, max_iters=50, rel_tol=1e-8)
    assert st.all() and it <= 10


@pytest.mark.parametrize("brows", [0, 1, 7, 64])
def test_gs_levels_host_match_oracle(brows):
    rng = np.random.default_rng(8)
    rp, ci, v = util.random_csr(400, 400, rng, max_nnz=7)
    lf, lb, nl = xamg.gs_levels_host(rp, ci, brows)
    if brows == 0:
        of, ob = orc.gs_levels(rp, ci)
        assert np.array_equal(lf, of) and np.array_equal(lb, ob)
    for i in range(400):
        for j in ci[rp[i]:rp[i + 1]]:
            if brows and j // brows != i // brows:
                continue
            if j < i:
                assert lf[j] < lf[i]
            elif j > i:
                assert lf[j] > lf[i] and lb[j] < lb[i]
    assert nl[0] == lf.max() + 1 and nl[1] == lb.max() + 1


def test_gs_levels_27pt_count():
    m = xamg.CsrMatrix.aniso27(16)
    rp, ci, v = m.arrays()
    lf, lb, nl = xamg.gs_levels_host(rp, ci, 0)
    # lexicographic 27-point: level(i,j,k) = i + 2j + 4k
    assert nl == (7 * 16 - 6, 7 * 16 - 6)


def _run_model(rp, ci, R=8):
    """Independent model of the run detection: chunks of up to R consecutive
    rows with equal entry counts whose columns are the previous row's plus
    one; segments = runs of at most 3 consecutive columns of a chunk's first row."""
    n = len(rp) - 1
    chunks = segs = full = 0
    r = 0
    while r < n:
        m = rp[r + 1] - rp[r]
        cnt = 1
        while cnt < R and r + cnt < n:
            a, b = rp[r + cnt - 1], rp[r + cnt]
            if rp[r + cnt + 1] - b != m or not np.array_equal(ci[b:b + m], ci[a:a + m] + 1):
                break
            cnt += 1
        cols = ci[rp[r]:rp[r] + m]
        e = 0
        while e < m:
            ln = 1
            while ln < 3 and e + ln < m and cols[e + ln] == cols[e + ln - 1] + 1:
                ln += 1
            segs += 1
            e += ln
        chunks += 1
        if cnt == R:
            full += cnt * m
        r += cnt
    return chunks, (full / len(ci) if len(ci) else 0.0), segs


def test_run_detection_matches_model():
    rng = np.random.default_rng(4)
    cases = [xamg.CsrMatrix.aniso27(9).arrays()[:2], xamg.CsrMatrix.cube(7, 5, 3, 0).arrays()[:2],
             util.random_csr(300, 300, rng, max_nnz=9, empty_rows=(0, 5))[:2]]
    # a band matrix: every row a shifted copy, runs cut only by the chunk size
    n = 100
    rp = np.arange(0, 3 * n + 1, 3, dtype=np.int32)
    ci = (np.arange(n)[:, None] + np.arange(3)[None, :]).ravel().astype(np.int32) % n
    cases.append((rp, ci))
    L = xamg.lib()
    for rp, ci in cases:
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        out = np.zeros(2, np.int64)
        cov = np.zeros(1)
        xamg.check(L.xamg_spmv_runs_analyze(len(rp) - 1, xamg._ptr(rp), xamg._ptr(ci), 8, xamg._ptr(out[0:]),
                                            xamg._ptr(cov), xamg._ptr(out[1:])))
        chunks, coverage, segs = _run_model(rp, ci)
        assert (out[0], out[1]) == (chunks, segs)
        assert cov[0] == pytest.approx(coverage, abs=1e-15)
    assert L.xamg_spmv_runs_analyze(len(rp) - 1, xamg._ptr(rp), xamg._ptr(ci), 4, xamg._ptr(out[0:]),
                                    xamg._ptr(cov), xamg._ptr(out[1:])) == 2


@pytest.mark.parametrize("seed", range(6))
def test_run_detection_random_stencils(seed):
    """Random stencil-like matrices (a shifted pattern per row with random
    breaks: changed entry counts, perturbed columns, empty rows) against the
    independent model of the run detection."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(50, 400))
    offs = np.sort(rng.choice(np.arange(-40, 41), size=int(rng.integers(1, 12)), replace=False))
    rp, ci = [0], []
    for r in range(n):
        cols = [r + o for o in offs if 0 <= r + o < n]
        u = rng.random()
        if u < 0.05:
            cols = []
        elif u < 0.12 and cols:
            cols[int(rng.integers(len(cols)))] = int(rng.integers(n))
        elif u < 0.18:
            cols = cols + [int(rng.integers(n))]
        ci += cols
        rp.append(len(ci))
    rp = np.array(rp, np.int32)
    ci = np.array(ci, np.int32)
    out = np.zeros(2, np.int64)
    cov = np.zeros(1)
    xamg.check(xamg.lib().xamg_spmv_runs_analyze(n, xamg._ptr(rp), xamg._ptr(ci), 8, xamg._ptr(out[0:]),
                                                 xamg._ptr(cov), xamg._ptr(out[1:])))
    chunks, coverage, segs = _run_model(rp, ci)
    assert (out[0], out[1]) == (chunks, segs)
    assert cov[0] == pytest.approx(coverage, abs=1e-15)


def test_run_plan_of_the_benchmark_operator():
    # the 128^3 27-point operator of the benchmark: 94.2 % of its entries in
    # full chunks of 8 rows, 9 segments of 3 columns per interior row
    rp, ci, v = xamg.CsrMatrix.aniso27(128).arrays()
    out = np.zeros(2, np.int64)
    cov = np.zeros(1)
    xamg.check(xamg.lib().xamg_spmv_runs_analyze(len(rp) - 1, xamg._ptr(rp), xamg._ptr(ci), 8, xamg._ptr(out[0:]),
                                                 xamg._ptr(cov), xamg._ptr(out[1:])))
    assert out[0] == 294912 and out[1] == 3183687
    assert cov[0] == pytest.approx(0.9424083769633508, abs=1e-12)


REF_EXAMPLES = os.path.join(os.environ.get("XAMG_REFERENCE_ROOT", "/root/reference"), "examples", "c")


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference sources not present")
@pytest.mark.parametrize("name", ["example", "example_ir"])
def test_reference_c_examples_build_unchanged(name, tmp_path):
    """The reference's own C callers compile against include/xamg_c_api.h and
    link against the library with no source change (the drop-in claim)."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    obj, exe = str(tmp_path / (name + ".o")), str(tmp_path / name)
    subprocess.run(["gcc", "-O1", "-c", os.path.join(REF_EXAMPLES, name + ".c"), "-I",
                    os.path.join(root, "include"), "-o", obj], check=True)
    libdir = os.path.join(root, "xamg-test_b200")
    subprocess.run(["gcc", obj, "-L", libdir, "-lxamg_b200", "-Wl,-rpath," + libdir, "-lm", "-o", exe], check=True)
    assert os.path.exists(exe)
