"""Solver-level parity: the GPU solve through the XAMG C API against the CPU
oracle on the same inputs and the same (exported) multigrid hierarchy.  In
plain FP64 the iteration counts and residual histories must be identical; the
tolerance written into each assertion is 1e-12 relative, and the runs are in
fact bit-identical."""
import json
import os

import numpy as np
import pytest

import oracle as orc
import reference_loops
import util
import xamg

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def solve_api(csr, spec, B, X0=None):
    n, nv = B.shape
    xamg.set_nv(nv)
    A = xamg.Matrix(csr)
    x = xamg.Vector(n, nv)
    b = xamg.Vector(n, nv)
    x.upload(np.zeros((n, nv)) if X0 is None else X0)
    b.upload(B)
    s = xamg.Solver(A, xamg.Params(spec), x, b)
    s.solve()
    return s, x.download(), (A, x, b)


def oracle_mg(s, spec):
    levels = [s.level(l) for l in range(s.num_levels())]
    sm = spec.get("pre_smoother", {})
    kind = orc.SM_HSGS if sm.get("method", "HSGS") == "HSGS" else orc.SM_JACOBI
    it = sm.get("max_iters", 1)
    br = sm.get("hybrid_block_rows", 0)
    return orc.MG(levels, pre=(kind, it, 0.99), post=(kind, it, 0.99), block_rows=br)


def assert_same_history(h_gpu, h_orc):
    assert h_gpu.shape == h_orc.shape, (h_gpu.shape, h_orc.shape)
    np.testing.assert_allclose(h_gpu, h_orc, rtol=1e-12, atol=0)


@pytest.mark.parametrize("nv", [1, 4])
def test_bicgstab_c1_parity(gpu, nv):
    # 7-point Poisson (cube generator config 0), BiCGStab to 1e-8 rel.
    csr = xamg.CsrMatrix.cube(32, 32, 32, 0)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(1234)
    B = rng.uniform(-1, 1, (csr.nrows, nv))
    spec = util.amg_params(precond_mg=False, max_iters=1000)
    s, X, keep = solve_api(csr, spec, B)
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), None, 1000, 0.0, 1e-8)
    assert s.iters()[0] == it
    assert_same_history(s.history(), hist)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())
    assert all(s.converged())


def _oracle_seq(fn, *args):
    orc.set_seq_dot(True)
    try:
        return fn(*args)
    finally:
        orc.set_seq_dot(False)


@pytest.mark.parametrize("nv", [1, 4])
def test_bicgstab_c1_sequential_dot_matches_reference_order(gpu, nv):
    """dot_order = sequential: the inner products run in the reference's
    single-core order (one dependent chain per column), and the whole C1
    solve (7-point Poisson on 32^3, BiCGStab to 1e-8) is bit for bit the
    oracle's in that order, itself bit for bit the reference's own loops
    compiled unchanged (tests/test_ref_loops.py); where that library travelled
    with the repository the GPU is compared with it directly as well.  The
    tree order gives a different iteration count on this system."""
    csr = xamg.CsrMatrix.cube(32, 32, 32, 0)
    rp, ci, v = csr.arrays()
    B = np.random.default_rng(1234).uniform(-1, 1, (csr.nrows, nv))
    spec = util.amg_params(precond_mg=False, max_iters=1000)
    spec["solver"]["dot_order"] = "sequential"
    s, X, keep = solve_api(csr, spec, B)
    xo, it, hist, st, r0 = _oracle_seq(orc.pbicgstab, rp, ci, v, B, np.zeros_like(B), None, 1000, 0.0, 1e-8)
    assert s.iters()[0] == it
    assert np.array_equal(s.history(), hist)
    assert np.array_equal(X, xo)
    L = reference_loops.lib("contract", build=False)
    if L is not None:
        xr, itr, hr = reference_loops.solver(L, "BiCGStab", rp, ci, v, B, max_iters=1000, rel_tol=1e-8)
        assert itr == s.iters()[0]
        assert np.array_equal(hr, s.history())
        assert np.array_equal(xr, X)


def test_pbicgstab_amg_sequential_dot_parity(gpu):
    """AMG-PBiCGStab (27-point 24^3, HSGS) with the reference's single-core
    inner-product order, bit for bit against the oracle in that order."""
    csr = xamg.CsrMatrix.aniso27(24)
    rp, ci, v = csr.arrays()
    B = np.random.default_rng(78).uniform(-1, 1, (csr.nrows, 4))
    spec = util.amg_params(max_levels=6)
    spec["solver"]["dot_order"] = "sequential"
    s, X, keep = solve_api(csr, spec, B)
    mg = oracle_mg(s, spec)
    xo, it, hist, st, r0 = _oracle_seq(orc.pbicgstab, rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    assert s.iters()[0] == it and it > 0
    assert np.array_equal(s.history(), hist)
    assert np.array_equal(X, xo)
    # the tree order reaches the same solution to rounding
    spec["solver"]["dot_order"] = "tree"
    s2, X2, keep2 = solve_api(csr, spec, B)
    np.testing.assert_allclose(X2, X, rtol=1e-6, atol=1e-9 * np.abs(X).max())


@pytest.mark.parametrize("grid,nv", [(11, 32), (13, 1), (23, 8)])
def test_sequential_dot_ragged_sizes(gpu, grid, nv):
    """The sequential inner products on row counts that end in a partial tile
    (1331, 2197 and 12167 rows) and on the widest block (NV = 32, the largest
    shared-memory stage): 40 BiCGStab iterations, converged or not, bit for
    bit against the oracle in the same order."""
    csr = xamg.CsrMatrix.aniso27(grid)
    rp, ci, v = csr.arrays()
    B = np.random.default_rng(grid).uniform(-1, 1, (csr.nrows, nv))
    spec = util.amg_params(precond_mg=False, max_iters=40, rel=1e-14)
    spec["solver"]["dot_order"] = "sequential"
    s, X, keep = solve_api(csr, spec, B)
    xo, it, hist, st, r0 = _oracle_seq(orc.pbicgstab, rp, ci, v, B, np.zeros_like(B), None, 40, 0.0, 1e-14)
    assert s.iters()[0] == it
    assert np.array_equal(s.history(), hist)
    assert np.array_equal(X, xo)


def test_dot_order_rejects_unknown_value(gpu):
    csr = xamg.CsrMatrix.aniso27(8)
    B = np.ones((csr.nrows, 1))
    spec = util.amg_params(precond_mg=False)
    spec["solver"]["dot_order"] = "pairwise"
    with pytest.raises(Exception, match="dot_order"):
        solve_api(csr, spec, B)


@pytest.mark.parametrize("smoother,block_rows", [("HSGS", 0), ("HSGS", 512), ("Jacobi", 0)])
def test_pbicgstab_amg_parity(gpu, smoother, block_rows):
    csr = xamg.CsrMatrix.aniso27(24)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(77)
    B = rng.uniform(-1, 1, (csr.nrows, 4))
    spec = util.amg_params(max_levels=6, smoother=smoother, sweeps=1 if smoother == "HSGS" else 2,
                           block_rows=block_rows)
    s, X, keep = solve_api(csr, spec, B)
    mg = oracle_mg(s, spec)
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    assert s.iters()[0] == it and it > 0
    assert_same_history(s.history(), hist)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())
    # bit-exact indexing: GS wavefront levels and coarse inverse agree with the oracle
    if smoother == "HSGS" and block_rows == 0:
        lf, lb = s.gs_levels(0)
        of, ob = orc.gs_levels(rp, ci)
        assert np.array_equal(lf, of) and np.array_equal(lb, ob)
    assert np.array_equal(s.coarse_inverse(), mg.coarse_inverse())


@pytest.mark.parametrize("order,nv", [(2, 4), (3, 1), (4, 2)])
def test_pbicgstab_chebyshev_parity(gpu, order, nv):
    """Chebyshev smoothing (chebyshev.inl) in the V-cycle: the oracle is given
    the library's spectrum estimates and must reproduce the iterations and
    the residual history."""
    csr = xamg.CsrMatrix.aniso27(20)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(order)
    B = rng.uniform(-1, 1, (csr.nrows, nv))
    spec = util.amg_params(max_levels=6)
    for role in ("pre_smoother", "post_smoother"):
        spec[role] = {"method": "Chebyshev", "polynomial_order": order, "spectrum_fraction": 0.3}
    s, X, keep = solve_api(csr, spec, B)
    levels = [s.level(l) for l in range(s.num_levels())]
    eig = [s.level_eig(l) for l in range(s.num_levels())]
    for mn, mx in eig[:-1]:
        assert 0 < mn < mx < 4.0, eig
    mg = orc.MG(levels, pre=(orc.SM_CHEB, 1, 0.0), post=(orc.SM_CHEB, 1, 0.0), cheb=(order, 0.3, eig))
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    assert s.iters()[0] == it and it > 0 and all(s.converged())
    assert_same_history(s.history(), hist)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())


@pytest.mark.parametrize("method,with_mg,nv", [("RBiCGStab", True, 4), ("RBiCGStab", False, 1),
                                               ("MergedRBiCGStab", True, 2), ("RBiCGStab", True, 16)])
def test_rbicgstab_parity(gpu, method, with_mg, nv):
    """RBiCGStab (rbicgstab.inl): identical iterations, residual history and
    solution to the oracle's restatement, with the AMG preconditioner and with
    none (identity)."""
    csr = xamg.CsrMatrix.aniso27(24) if with_mg else xamg.CsrMatrix.cube(24, 24, 24, 0)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(11 + nv)
    B = rng.uniform(-1, 1, (csr.nrows, nv))
    spec = util.amg_params(precond_mg=with_mg, max_levels=6, max_iters=1000)
    spec["solver"]["method"] = method
    s, X, keep = solve_api(csr, spec, B)
    mg = oracle_mg(s, spec) if with_mg else None
    xo, it, hist, st, r0 = orc.rbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 1000, 0.0, 1e-8)
    assert s.iters()[0] == it and it > 0 and all(s.converged())
    assert_same_history(s.history(), hist)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())


@pytest.mark.parametrize("with_mg,nv", [(True, 4), (False, 1), (True, 16)])
def test_pcg_parity(gpu, with_mg, nv):
    """PCG (pcg.inl) on the symmetric 7-point operator: identical iterations,
    residual history and solution to the oracle's restatement."""
    csr = xamg.CsrMatrix.cube(24, 24, 24, 0)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(5 + nv)
    B = rng.uniform(-1, 1, (csr.nrows, nv))
    spec = util.amg_params(precond_mg=with_mg, max_levels=6, max_iters=1000)
    spec["solver"]["method"] = "PCG"
    s, X, keep = solve_api(csr, spec, B)
    mg = oracle_mg(s, spec) if with_mg else None
    xo, it, hist, st, r0 = orc.pcg(rp, ci, v, B, np.zeros_like(B), mg, 1000, 0.0, 1e-8)
    assert s.iters()[0] == it and it > 0 and all(s.converged())
    assert_same_history(s.history(), hist)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())


def test_recorded_2d_problem_through_api(gpu):
    rec = json.load(open(os.path.join(GOLD, "recorded.json")))
    rp, ci, v, b, u = util.gen2d(100)
    csr = xamg.CsrMatrix.from_arrays(rp, ci, v)
    spec = util.amg_params(max_levels=25)
    s, X, keep = solve_api(csr, spec, b.reshape(-1, 1))
    h = s.history()
    assert np.sqrt(h[0, 0]) == pytest.approx(rec["initial_residual"], rel=4e-15)
    assert abs(np.linalg.norm(X) - rec["X_norm"]) / rec["X_norm"] < 1e-7
    assert np.linalg.norm(X[:, 0] - u) / np.sqrt(len(u)) < 1e-5


def test_repeated_solves_identical(gpu):
    # tst_solver.h:141-155: identical residuals on repeated solve() calls
    csr = xamg.CsrMatrix.aniso27(20)
    rng = np.random.default_rng(3)
    B = rng.uniform(-1, 1, (csr.nrows, 8))
    spec = util.amg_params(max_levels=6)
    xamg.set_nv(8)
    A = xamg.Matrix(csr)
    x, b = xamg.Vector(csr.nrows, 8), xamg.Vector(csr.nrows, 8)
    b.upload(B)
    s = xamg.Solver(A, xamg.Params(spec), x, b)
    hs = []
    xs = []
    for _ in range(3):
        x.set(0.0)
        s.solve()
        hs.append(s.history())
        xs.append(x.download())
    for q in range(1, 3):
        assert np.array_equal(hs[0], hs[q]) and np.array_equal(xs[0], xs[q])


def test_large_27pt_true_residual(gpu):
    """A larger anisotropic case checked by a size-independent property: the
    true residual ||b - A x|| computed independently (torch, FP64) meets the
    tolerance for every column."""
    import torch
    n = 64
    csr = xamg.CsrMatrix.aniso27(n)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(9)
    B = rng.uniform(-1, 1, (csr.nrows, 16))
    spec = util.amg_params(max_levels=6)
    s, X, keep = solve_api(csr, spec, B)
    assert all(s.converged())
    At = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)), torch.from_numpy(ci.astype(np.int64)),
                                 torch.from_numpy(v), size=(csr.nrows, csr.nrows)).cuda()
    R = torch.from_numpy(B).cuda() - At @ torch.from_numpy(X).cuda()
    rel = (R.norm(dim=0) / torch.from_numpy(B).cuda().norm(dim=0)).cpu().numpy()
    assert np.all(rel <= 1e-8 * 1.05), rel


def test_nonconvergence_and_bad_input_report(gpu):
    csr = xamg.CsrMatrix.cube(16, 16, 16, 0)
    rng = np.random.default_rng(4)
    B = rng.uniform(-1, 1, (csr.nrows, 1))
    spec = util.amg_params(precond_mg=False, max_iters=3)
    s, X, keep = solve_api(csr, spec, B)
    assert s.iters()[0] == 3 and not any(s.converged())
    L = xamg.lib()
    assert L.XAMG_solver_solve1(2, s.h) == 2  # nv mismatch is an error code, not an abort


@pytest.mark.parametrize("block_rows", [0, 576])
def test_precision_form_parity(gpu, block_rows):
    """FP64 refinement around the FP32 PBiCGStab / FP32 V-cycle: identical
    outer and inner iteration counts and residual history as the oracle."""
    csr = xamg.CsrMatrix.aniso27(24)
    rp, ci, v = csr.arrays()
    rng = np.random.default_rng(5)
    B = rng.uniform(-1, 1, (csr.nrows, 4))
    spec = util.amg_params(max_levels=6, block_rows=block_rows, max_iters=200,
                           meta={"method": "IterativeRefinement", "max_iters": 20, "abs_tolerance": 0.0,
                                 "rel_tolerance": 1e-8, "subsolver_reduced_precision": True,
                                 "inner_rel_tolerance": 1e-4, "convergence_details": "check-L2,noprint"})
    s, X, keep = solve_api(csr, spec, B)
    levels = [s.level(l) for l in range(s.num_levels())]
    mg = orc.MG(levels, fp32=True, block_rows=block_rows)
    xo, it, hist, st, sub = orc.ir_pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 20, 200, 0.0, 1e-8, 1e-4)
    assert s.iters() == (it, sub)
    assert_same_history(s.history(), hist)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())
    assert st.all() and all(s.converged())
    # error against an FP64 solve of the same system
    xp, _, _, _, _ = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), orc.MG(levels), 200, 0.0, 1e-10)
    assert np.linalg.norm(X - xp) / np.linalg.norm(xp) < 1e-6
