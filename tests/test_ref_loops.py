"""The oracle against the reference's own loops, compiled unchanged from its
source tree (oracle/build_ref_loops.py): sparse and dense products, the hybrid
symmetric Gauss-Seidel call, the BLAS-1 updates, the single-core inner product
the coarse-grid dense inverse and a whole BiCGStab solve in the reference's
step order.

Three builds of the same loop files (see oracle/build_ref_loops.py):
  contract  row loops fused (FMA), BLAS-1 literal: the oracle's arithmetic
            contract, so everything must be bit-identical;
  haswell   the Haswell machine configuration with contraction everywhere:
            row loops bit-identical, BLAS-1 within one rounding per product;
  generic   the generic release flags, no FMA: row loops within a few
            roundings, BLAS-1 and the inner product bit-identical.
The libraries are built from the reference tree in this container; where it
is absent (and no prebuilt library travelled) the tests skip."""
import numpy as np
import pytest

import oracle as orc
import reference_loops
import util

EPS = np.finfo(np.float64).eps
EPS32 = np.finfo(np.float32).eps
p = orc.p


def _load(kind):
    L = reference_loops.lib(kind)
    if L is None:
        pytest.skip("reference loop library not built (reference tree absent)")
    return L


@pytest.fixture(scope="module")
def libs():
    return {k: _load(k) for k in ("contract", "haswell", "generic")}


def poisson7(m):
    """7-point Poisson operator on an m^3 grid with Dirichlet boundary,
    diagonal first in every row (the cube generator's row layout)."""
    idx = np.arange(m ** 3).reshape(m, m, m)
    rp, ci, v = [0], [], []
    for z in range(m):
        for y in range(m):
            for x in range(m):
                ci.append(idx[z, y, x])
                v.append(6.0)
                for dz, dy, dx in ((-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1), (0, 1, 0), (1, 0, 0)):
                    if 0 <= z + dz < m and 0 <= y + dy < m and 0 <= x + dx < m:
                        ci.append(idx[z + dz, y + dy, x + dx])
                        v.append(-1.0)
                rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v)


def operators():
    rng = np.random.default_rng(5)
    yield "aniso27_12", orc.gen27(12)
    yield "dd_random_700", util.dd_csr(700, rng)


def inv_diag(rp, ci, v):
    n = len(rp) - 1
    d = np.zeros(n)
    for i in range(n):
        for j in range(rp[i], rp[i + 1]):
            if ci[j] == i:
                d[i] = v[j]
    return 1.0 / d


def abs_spmv(rp, ci, v, x):
    return orc.spmv(rp, ci, np.abs(v), np.abs(x), x.shape[1])


@pytest.mark.parametrize("nv", [1, 2, 4, 8, 16, 32])
def test_spmv_matches_reference_loops(libs, nv):
    rng = np.random.default_rng(nv)
    for name, (rp, ci, v) in operators():
        n = len(rp) - 1
        x = rng.uniform(-1, 1, (n, nv))
        yo = orc.spmv(rp, ci, v, x, nv)
        y0 = rng.uniform(-1, 1, (n, nv))
        yao = orc.spmv(rp, ci, v, x, nv, y=y0.copy(), acc=True)
        for kind, L in libs.items():
            y = np.zeros((n, nv))
            assert L.ref_csr_ax_y_d(n, p(rp), p(ci), p(v), p(x), p(y), nv) == 0
            ya = y0.copy()
            assert L.ref_csr_axpy_d(n, p(rp), p(ci), p(v), p(x), p(ya), nv) == 0
            if kind == "generic":  # no FMA: within the rounding of each product
                bound = 2 * 32 * EPS * abs_spmv(rp, ci, v, x)
                assert np.all(np.abs(y - yo) <= bound), (name, kind)
                assert np.all(np.abs(ya - yao) <= bound + 2 * EPS * np.abs(y0)), (name, kind)
            else:
                assert np.array_equal(y, yo), (name, kind)
                assert np.array_equal(ya, yao), (name, kind)
        # FP32 values and vectors
        v32, x32 = v.astype(np.float32), x.astype(np.float32)
        y32o = orc.spmv(rp, ci, v32, x32, nv)
        y32 = np.zeros((n, nv), np.float32)
        assert libs["contract"].ref_csr_ax_y_f(n, p(rp), p(ci), p(v32), p(x32), p(y32), nv) == 0
        assert np.array_equal(y32, y32o), name


@pytest.mark.parametrize("nv", [1, 4, 16])
@pytest.mark.parametrize("nblocks", [1, 3, 8])
def test_hybrid_gauss_seidel_matches_reference_loops(libs, nv, nblocks):
    rng = np.random.default_rng(10 * nv + nblocks)
    for name, (rp, ci, v) in operators():
        n = len(rp) - 1
        invd = inv_diag(rp, ci, v)
        b = rng.uniform(-1, 1, (n, nv))
        x0 = rng.uniform(-1, 1, (n, nv))
        relax = rng.uniform(0.5, 1.0, nv)
        block_rows = -(-n // nblocks) if nblocks > 1 else 0
        xo = orc.hsgs(rp, ci, v, invd, b, x0.copy(), relax, block_rows=block_rows)
        bp = (np.append(np.arange(0, n, block_rows), n) if block_rows else np.array([0, n])).astype(np.int64)
        for kind in ("contract", "haswell"):
            x = x0.copy()
            assert libs[kind].ref_hsgs_d(n, p(rp), p(ci), p(v), p(invd), p(b), p(x), p(relax), nv, len(bp) - 1,
                                         p(bp)) == 0
            assert np.array_equal(x, xo), (name, kind)
        x = x0.copy()
        libs["generic"].ref_hsgs_d(n, p(rp), p(ci), p(v), p(invd), p(b), p(x), p(relax), nv, len(bp) - 1, p(bp))
        np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-13 * np.abs(xo).max(), err_msg=name)
        # FP32
        v32, d32, b32, x32 = (a.astype(np.float32) for a in (v, invd, b, x0))
        r32 = relax.astype(np.float32)
        xo32 = orc.hsgs(rp, ci, v32, d32, b32, x32.copy(), r32, block_rows=block_rows)
        xr32 = x32.copy()
        libs["contract"].ref_hsgs_f(n, p(rp), p(ci), p(v32), p(d32), p(b32), p(xr32), p(r32), nv, len(bp) - 1,
                                    p(bp))
        assert np.array_equal(xr32, xo32), name


@pytest.mark.parametrize("nv", [1, 4, 16])
def test_jacobi_matches_reference_loops(libs, nv):
    """Two Jacobi sweeps (the smoother's no-check path, merged update
    x += relax*invd*(b - Ax)): the oracle fuses the update, as the Haswell
    build compiles the reference's loop; the generic build rounds the product
    apart (within a rounding per sweep)."""
    rng = np.random.default_rng(70 + nv)
    for name, (rp, ci, v) in operators():
        n = len(rp) - 1
        invd = inv_diag(rp, ci, v)
        b = rng.uniform(-1, 1, (n, nv))
        x0 = rng.uniform(-1, 1, (n, nv))
        relax = rng.uniform(0.5, 1.0, nv)
        xo = x0.copy()
        for _ in range(2):
            orc.jacobi(rp, ci, v, invd, b, xo, relax)
        x = x0.copy()
        assert libs["haswell"].ref_jacobi_d(n, p(rp), p(ci), p(v), p(invd), p(b), p(x), p(relax), nv, 2) == 0
        assert np.array_equal(x, xo), name
        x = x0.copy()
        libs["generic"].ref_jacobi_d(n, p(rp), p(ci), p(v), p(invd), p(b), p(x), p(relax), nv, 2)
        np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max(), err_msg=name)


@pytest.mark.parametrize("nv", [1, 4, 16])
def test_dense_product_matches_reference_loops(libs, nv):
    rng = np.random.default_rng(40 + nv)
    nc = 57
    A = rng.uniform(-1, 1, (nc, nc))
    b = rng.uniform(-1, 1, (nc, nv))
    yo = orc.dense_gemv(A, b)
    for kind in ("contract", "haswell"):
        y = np.zeros((nc, nv))
        assert libs[kind].ref_dense_ax_y_d(nc, nc, p(A), p(b), p(y), nv) == 0
        assert np.array_equal(y, yo), kind
    A32, b32 = A.astype(np.float32), b.astype(np.float32)
    y32 = np.zeros((nc, nv), np.float32)
    libs["contract"].ref_dense_ax_y_f(nc, nc, p(A32), p(b32), p(y32), nv)
    assert np.array_equal(y32, orc.dense_gemv(A32, b32))


@pytest.mark.parametrize("n", [1, 7, 64, 100])
def test_dense_inverse_matches_reference_loops(libs, n):
    """The coarse-grid Direct solver's Gauss-Jordan inverse (inverse.inl:31-106):
    the oracle's restatement (and the library's host setup, which the GPU tests
    hold to the oracle bit for bit) against the reference's routine compiled
    unchanged, on a diagonally dominant and on a 27-point coarse-like matrix."""
    rng = np.random.default_rng(n)
    A = rng.uniform(-1, 1, (n, n)) + np.diag(rng.uniform(n, 2 * n, n))
    for kind in ("contract", "generic"):
        R = np.zeros_like(A)
        assert libs[kind].ref_dense_inverse_d(n, p(A), p(R)) == 0
        assert np.array_equal(R, orc.dense_inverse(A)), kind
    R = np.zeros_like(A)
    libs["haswell"].ref_dense_inverse_d(n, p(A), p(R))  # fused eliminations: within rounding
    np.testing.assert_allclose(R, orc.dense_inverse(A), rtol=1e-12, atol=1e-15 * np.abs(R).max())
    if n == 64:
        rp, ci, v = orc.gen27(4)
        D = np.zeros((64, 64))
        for i in range(64):
            D[i, ci[rp[i]:rp[i + 1]]] = v[rp[i]:rp[i + 1]]
        R = np.zeros_like(D)
        libs["contract"].ref_dense_inverse_d(64, p(D), p(R))
        assert np.array_equal(R, orc.dense_inverse(D))


@pytest.mark.parametrize("nv", [1, 4, 16])
def test_blas1_and_inner_product_match_reference_loops(libs, nv):
    """The oracle and the GPU kernels evaluate the vector updates literally
    (every product rounded, sums left to right), as numpy does here; the
    reference's loops give the same bits when compiled without contraction."""
    rng = np.random.default_rng(60 + nv)
    n = 1000
    x, y, z0 = (rng.uniform(-1, 1, (n, nv)) for _ in range(3))
    a, b, c = (rng.uniform(-2, 2, nv) for _ in range(3))
    expect = {
        "axpby": a * x + b * z0,
        "axpby_z": a * x + b * y,
        "axpbypcz": a * x + b * y + c * z0,
        "xdivy_z": x / y,
        "ax_y": a * x,
        "scal": a * z0,
    }
    for kind in ("contract", "generic", "haswell"):
        L = libs[kind]
        got = {}
        z = z0.copy(); L.ref_axpby_d(n, nv, p(a), p(x), p(b), p(z)); got["axpby"] = z
        z = np.zeros_like(z0); L.ref_axpby_z_d(n, nv, p(a), p(x), p(b), p(y), p(z)); got["axpby_z"] = z
        z = z0.copy(); L.ref_axpbypcz_d(n, nv, p(a), p(x), p(b), p(y), p(c), p(z)); got["axpbypcz"] = z
        z = np.zeros_like(z0); L.ref_xdivy_z_d(n, nv, p(x), p(y), p(z)); got["xdivy_z"] = z
        z = np.zeros_like(z0); L.ref_ax_y_d(n, nv, p(a), p(x), p(z)); got["ax_y"] = z
        z = z0.copy(); L.ref_scal_d(n, nv, p(a), p(z)); got["scal"] = z
        for op, e in expect.items():
            if kind == "haswell":  # a product fused into its sum: one rounding less
                mag = np.abs(a * x) + np.abs(b * (y if op == "axpby_z" else z0)) + np.abs(c * z0)
                assert np.all(np.abs(got[op] - e) <= 4 * EPS * mag + 4 * EPS * np.abs(e)), (op, kind)
            else:
                assert np.array_equal(got[op], e), (op, kind)
        d = np.zeros(nv)
        L.ref_dot_d(n, nv, p(x), p(y), p(d))
        if kind == "haswell":
            np.testing.assert_allclose(d, orc.dot_sequential(x, y), rtol=0, atol=n * EPS * np.abs(x * y).sum(0).max())
        else:
            assert np.array_equal(d, orc.dot_sequential(x, y)), kind


@pytest.fixture
def seq_dot():
    orc.set_seq_dot(True)
    yield
    orc.set_seq_dot(False)


def _ref_bicgstab(L, rp, ci, v, B, max_iters=1000, rel_tol=1e-8):
    return reference_loops.solver(L, "BiCGStab", rp, ci, v, B, max_iters=max_iters, rel_tol=rel_tol)


@pytest.mark.parametrize("nv", [1, 4])
def test_bicgstab_solve_matches_reference_loops(libs, seq_dot, nv):
    """A whole BiCGStab solve (the first configuration: 7-point Poisson on 32^3,
    RHS uniform[-1,1], 1e-8) in the reference's step order over its own loops
    equals the oracle bit for bit once the oracle sums its inner products in
    the reference's single-core order: same iterations, residual history and x."""
    rp, ci, v = poisson7(32)
    B = np.random.default_rng(1234).uniform(-1, 1, (len(rp) - 1, nv))
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), None, 1000, 0.0, 1e-8)
    for kind in ("contract", "generic"):  # this operator's products are exact either way
        x, itr, h = _ref_bicgstab(libs[kind], rp, ci, v, B)
        assert itr == it, kind
        assert np.array_equal(h, hist), kind
        assert np.array_equal(x, xo), kind
    rp, ci, v = orc.gen27(14)
    B = np.random.default_rng(99).uniform(-1, 1, (len(rp) - 1, nv))
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), None, 1000, 0.0, 1e-8)
    x, itr, h = _ref_bicgstab(libs["contract"], rp, ci, v, B)
    assert itr == it and np.array_equal(h, hist) and np.array_equal(x, xo)


def test_bicgstab_inner_product_order_changes_iterations(libs):
    """What the order of the inner products does to a whole solve: the tree
    order shared by the oracle and the GPU kernels and the reference's
    single-core order start from the same residual and end at the same
    tolerance, but BiCGStab's iteration count on this system moves with the
    rounding (recorded here, so that a parity claim for the tree order is made
    against the sequential order with this in view)."""
    rp, ci, v = poisson7(32)
    B = np.random.default_rng(1234).uniform(-1, 1, (len(rp) - 1, 1))
    _, it_tree, h_tree, _, _ = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), None, 1000, 0.0, 1e-8)
    _, it_ref, h_ref = _ref_bicgstab(libs["contract"], rp, ci, v, B)
    k = min(it_tree, it_ref) + 1
    rel = np.abs(h_tree[:k] - h_ref[:k]) / h_ref[:k]
    assert rel[0] < 1e-14
    assert rel[:10].max() < 1e-12  # the histories agree to rounding at first ...
    assert rel.max() > 1e-3        # ... and drift apart over ~90 iterations
    assert (it_tree, it_ref) == (90, 88)


@pytest.mark.parametrize("block_rows", [0, 300])
def test_amg_pbicgstab_solve_matches_reference_loops(libs, seq_dot, block_rows):
    """The benchmark's method (AMG-PBiCGStab: HMIS / extended+i hierarchy,
    HSGS 1+1, Direct coarse solve) on a 27-point 16^3 system, NV = 4: the
    reference's loops in the step order of pbicgstab.inl and mg.inl, its own
    Gauss-Jordan inverse on the coarsest level, against the oracle with the
    reference's inner-product order on the same hierarchy: same iterations,
    residual history and x, bit for bit; single-process sweeps and hybrid
    blocks of 300 rows on every level."""
    rp, ci, v = orc.gen27(16)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
    assert len(levels) >= 3
    B = np.random.default_rng(2024).uniform(-1, 1, (len(rp) - 1, 4))
    mg = orc.MG(levels, block_rows=block_rows or None)
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    blocks = []
    for lv in levels:
        n = lv["n"]
        br = block_rows if block_rows and block_rows < n else 0
        blocks.append((np.append(np.arange(0, n, br), n) if br else np.array([0, n])).astype(np.int64))
    x, itr, h = reference_loops.solver(libs["contract"], "PBiCGStab", rp, ci, v, B, levels=levels, blocks=blocks,
                                       max_iters=200)
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("method", ["PCG", "RBiCGStab"])
@pytest.mark.parametrize("precond", [False, True])
def test_pcg_and_rbicgstab_solves_match_reference_loops(libs, seq_dot, method, precond):
    """PCG (pcg.inl) and RBiCGStab (rbicgstab.inl) in the reference's step
    order over its compiled loops, with the identity or one AMG V-cycle as
    the preconditioner, against the oracle's solvers in the reference's
    inner-product order: same iterations, residual history and x, bit for bit
    (27-point 14^3 system, NV = 4)."""
    rp, ci, v = orc.gen27(14)
    B = np.random.default_rng(31).uniform(-1, 1, (len(rp) - 1, 4))
    if precond:
        levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                               mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
        mg = orc.MG(levels)
    else:
        levels = [dict(n=len(rp) - 1, A=(rp, ci, v), P=None, ncP=0)]
        mg = None
    fn = orc.pcg if method == "PCG" else orc.rbicgstab
    xo, it, hist, st, r0 = fn(rp, ci, v, B, np.zeros_like(B), mg, 500, 0.0, 1e-8)
    x, itr, h = reference_loops.solver(libs["contract"], method, rp, ci, v, B, levels=levels if precond else None,
                                       max_iters=500)
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


def test_amg_pbicgstab_jacobi_smoothing_matches_reference_loops(libs, seq_dot):
    """AMG-PBiCGStab with two Jacobi sweeps before and after (the no-check
    path of jacobi.inl with the merged update) on a 27-point 16^3 system,
    NV = 4, bit for bit against the oracle on the same hierarchy."""
    rp, ci, v = orc.gen27(16)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
    B = np.random.default_rng(2025).uniform(-1, 1, (len(rp) - 1, 4))
    mg = orc.MG(levels, pre=(orc.SM_JACOBI, 2, 0.99), post=(orc.SM_JACOBI, 2, 0.99))
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    x, itr, h = reference_loops.solver(libs["contract"], "PBiCGStab", rp, ci, v, B, levels=levels, max_iters=200,
                                       smoother="Jacobi", sweeps=2)
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("config", [0, 1, 2, 3, 4])
def test_cube_generator_matches_reference_generator(libs, config):
    """The library's cube generator (configurations 0-4: isotropic,
    anisotropic, coefficient jumps, core) against the reference's cube.inl
    compiled unchanged: row pointers, entry order and values identical on a
    non-cubic grid and on the first configuration's 32^3 grid."""
    import xamg

    for dims in ((10, 12, 14), (32, 32, 32)):
        ref = reference_loops.cube(libs["generic"], *dims, config)
        got = xamg.CsrMatrix.cube(*dims, config).arrays()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), (config, dims)


def test_binary_reader_matches_reference_reader(libs):
    """The reference's read_system (io/detail/reader.inl) compiled unchanged,
    on its own fixture (examples/test/mtx_Paus.bin): the library's reader
    returns the same matrix and right-hand side, bit for bit.  The initial
    guess differs on purpose: the reference seeks to an absolute offset that
    is zero on one process before reading x (reader.inl:148-151), so its x is
    the file's first bytes reinterpreted; its test driver overwrites x before
    every solve (tst_solver.h:90-93).  The library reads the x section."""
    import os
    import xamg

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mtx_Paus_n5.bin")
    rp, ci, v, B, X = reference_loops.read_system(libs["generic"], path, 1)
    m, b, x = xamg.CsrMatrix.read_bin(path)
    got = m.arrays()
    assert np.array_equal(got[0], rp) and np.array_equal(got[1], ci) and np.array_equal(got[2], v)
    assert np.array_equal(b, B[:, 0])
    raw = open(path, "rb").read()
    assert np.array_equal(X[:, 0], np.frombuffer(raw[: 8 * len(X)], np.float64))
    n, nnz = len(rp) - 1, len(ci)
    x_section = np.frombuffer(raw, np.float64, count=n, offset=8 + 4 * (n + 1) + 4 * nnz + 8 * nnz + 8 * n)
    assert np.array_equal(x, x_section)


@pytest.mark.parametrize("cycle", ["F", "W"])
def test_amg_pbicgstab_f_and_w_cycles_match_reference_loops(libs, seq_dot, cycle):
    """F- and W-cycle preconditioning (mg_cycle 1 and 2 of mg.inl:186-280: the
    F-cycle skips pre-smoothing on its level and follows its coarse F-cycle
    with a V-cycle, the W-cycle recurses twice) in AMG-PBiCGStab, 27-point
    16^3, NV = 4: bit for bit against the oracle's cycles; W through the
    reference's MultiGrid class itself, F through the cycle restated over its
    loops (the class's F-cycle reuses stale coarse vectors, see the next
    test)."""
    rp, ci, v = orc.gen27(16)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
    B = np.random.default_rng(2026).uniform(-1, 1, (len(rp) - 1, 4))
    mg = orc.MG(levels, cycle={"F": 1, "W": 2}[cycle])
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    x, itr, h = reference_loops.solver(libs["contract"], "PBiCGStab", rp, ci, v, B, levels=levels, max_iters=200,
                                       cycle=cycle, mg_class=(cycle == "W"))
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("cycle", ["V", "W"])
def test_amg_pbicgstab_reduced_precision_matches_reference_loops(libs, seq_dot, cycle):
    """mg_reduced_precision (mg.inl:147-149, 320-321): the first level and its
    smoothers in FP64, the residual converted to FP32 for R_0, every coarser
    level (operators, inverse diagonals, HSGS, the coarse Direct solver with
    its Gauss-Jordan inverse computed in FP32) in FP32, the correction
    converted back and added.  The oracle's reduced cycle against the
    reference's loops in FP64 and FP32 (convert.inl for the conversions):
    AMG-PBiCGStab on 27-point 16^3, NV = 4, bit for bit."""
    rp, ci, v = orc.gen27(16)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
    B = np.random.default_rng(2027).uniform(-1, 1, (len(rp) - 1, 4))
    mg = orc.MG(levels, cycle={"V": 0, "W": 2}[cycle], reduced=True)
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    x, itr, h = reference_loops.solver(libs["contract"], "PBiCGStab", rp, ci, v, B, levels=levels, max_iters=200,
                                       cycle=cycle, reduced=True)
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("order", [1, 2, 3, 4])
@pytest.mark.parametrize("nv", [1, 4])
def test_chebyshev_smoother_matches_reference_solver(libs, order, nv):
    """The reference's Chebyshev smoother class (chebyshev.inl: coefficient
    table of orders 1-4, the polynomial applied in D^-1/2 A D^-1/2 from the
    residual b - A x) compiled unchanged, against the oracle's smoother with
    the same spectrum bounds: bit for bit."""
    rng = np.random.default_rng(10 * order + nv)
    rp, ci, v = orc.gen27(10)
    n = len(rp) - 1
    b = rng.uniform(-1, 1, (n, nv))
    x0 = rng.uniform(-1, 1, (n, nv))
    lo, hi, frac = 0.013, 1.97, 0.3
    xo = orc.chebyshev(rp, ci, v, b, x0.copy(), order, frac, lo, hi)
    x = x0.copy()
    assert libs["contract"].ref_chebyshev_d(n, p(rp), p(ci), p(v), p(b), p(x), nv, order, frac, lo, hi) == 0
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("method", ["BiCGStab", "MergedBiCGStab"])
@pytest.mark.parametrize("nv", [1, 4])
def test_reference_bicgstab_classes_match_oracle(libs, seq_dot, method, nv):
    """The reference's BiCGStab and MergedBiCGStab solver classes themselves
    (bicgstab.inl, merged/merged_bicgstab.inl with the merged BLAS groups),
    compiled unchanged against stand-ins for the solver framework, on the C1
    system: the same iterations, residual history and x as the oracle, bit for
    bit.  MergedBiCGStab forms the new direction as r + beta p - (beta omega) v
    (blas_merged_bicgstab.inl), which rounds differently from BiCGStab's
    r + (-omega beta) v + beta p: the oracle follows it under
    set_merged_bicgstab, and the iteration counts of the two classes differ."""
    rp, ci, v = poisson7(32)
    B = np.random.default_rng(1234).uniform(-1, 1, (len(rp) - 1, nv))
    orc.set_merged_bicgstab(method == "MergedBiCGStab")
    try:
        xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), None, 1000, 0.0, 1e-8)
    finally:
        orc.set_merged_bicgstab(False)
    x, itr, h = reference_loops.solver(libs["contract"], method, rp, ci, v, B)
    assert itr == it
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


@pytest.mark.parametrize("method", ["PBiCGStab", "MergedPBiCGStab", "PCG", "RBiCGStab"])
def test_reference_preconditioned_solver_classes_match_oracle(libs, seq_dot, method):
    """The reference's PBiCGStab, MergedPBiCGStab, PCG and RBiCGStab classes
    compiled unchanged, preconditioned by one V-cycle of its loops on the
    oracle's AMG hierarchy (27-point 16^3, NV = 4): bit for bit the oracle's
    solvers (MergedPBiCGStab forms its direction as PBiCGStab does)."""
    rp, ci, v = orc.gen27(16)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
    B = np.random.default_rng(4).uniform(-1, 1, (len(rp) - 1, 4))
    mg = orc.MG(levels)
    fn = {"PBiCGStab": orc.pbicgstab, "MergedPBiCGStab": orc.pbicgstab, "PCG": orc.pcg,
          "RBiCGStab": orc.rbicgstab}[method]
    xo, it, hist, st, r0 = fn(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    x, itr, h = reference_loops.solver(libs["contract"], method, rp, ci, v, B, levels=levels, max_iters=200)
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)


def test_reference_f_cycle_reuses_stale_coarse_vectors(libs):
    """The reference's MultiGrid class with mg_cycle = F: its first application
    equals the F-cycle of the oracle and of the restated cycle, the second does
    not.  MG_cycle clears the coarse vector x_H by flag only
    (set_const without force, mg.inl:226), an F-cycle skips the pre-smoother
    that would clear it (mg.inl:218), and csr_Axpy adds the prolongated
    correction into its previous contents (csr_matvec.inl:32-144), so from the
    second application on the coarse levels start from the last cycle's x_H.
    The oracle and the library start every coarse level from zero."""
    rp, ci, v = orc.gen27(12)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=4, mg_coarse_matrix_size=10)
    b = np.random.default_rng(1).uniform(-1, 1, (len(rp) - 1, 1))
    L = libs["contract"]
    nrows, cast, nb, keep = reference_loops._hier_args(levels, None)
    h = L.ref_mg_create(1, len(levels), p(nrows), *cast[:9], p(nb), cast[9], 0.99, 1, 1, 1 << 4)
    try:
        mg = orc.MG(levels, cycle=1)
        expect = mg.apply(b)
        first, second = np.zeros_like(b), np.zeros_like(b)
        L.ref_mg_apply_d(h, p(b), p(first))
        L.ref_mg_apply_d(h, p(b), p(second))
    finally:
        L.ref_mg_destroy(h)
    assert np.array_equal(first, expect)
    assert not np.array_equal(second, expect)


@pytest.mark.parametrize("order", [2, 3])
def test_amg_pbicgstab_chebyshev_smoothing_matches_reference_classes(libs, seq_dot, order):
    """AMG-PBiCGStab with Chebyshev smoothing: the reference's PBiCGStab,
    MultiGrid and Chebyshev classes against the oracle with the same spectrum
    bounds per level (27-point 16^3, NV = 4), bit for bit."""
    rp, ci, v = orc.gen27(16)
    levels = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_interpolation_type=6,
                           mg_strength_threshold=0.25, mg_max_levels=6, mg_coarse_matrix_size=100)
    B = np.random.default_rng(2028).uniform(-1, 1, (len(rp) - 1, 4))
    eig = [(0.02 + 0.01 * l, 1.9 - 0.05 * l) for l in range(len(levels))]
    cheb = (order, 0.3, eig)
    mg = orc.MG(levels, pre=(orc.SM_CHEB, 1, 0.99), post=(orc.SM_CHEB, 1, 0.99), cheb=cheb)
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    x, itr, h = reference_loops.solver(libs["contract"], "PBiCGStab", rp, ci, v, B, levels=levels, max_iters=200,
                                       cheb=cheb)
    assert itr == it and it > 0
    assert np.array_equal(h, hist)
    assert np.array_equal(x, xo)
