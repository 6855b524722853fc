"""The CPU oracle pinned against the reference's own fixtures and recorded
values (no GPU needed)."""
import json
import os

import numpy as np
import pytest

import oracle as orc
import util
import xamg

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REC = json.load(open(os.path.join(GOLD, "recorded.json")))


def test_fixture_n5_reads_like_reference():
    # examples/test/mtx_gen.cpp: identity boundary rows, 4/h^2 and -1/h^2 inside
    m, b, x = xamg.CsrMatrix.read_bin(os.path.join(GOLD, "mtx_Paus_n5.bin"))
    assert m.nrows == REC["fixture_n5"]["nrows"] and m.nnz == REC["fixture_n5"]["nonzeros"]
    rp, ci, v = m.arrays()
    n = 5
    h = np.pi / n / 2
    assert np.all(x == 1.0)
    # b of mtx_gen.cpp: cos(hi) sin(hj), doubled inside
    for r in range(m.nrows):
        i, j = r // (n + 1), r % (n + 1)
        f = 1.0 if (i * j == 0 or i == n or j == n) else 2.0
        assert b[r] == np.cos(h * i) * np.sin(h * j) * f
    inner = [r for r in range(m.nrows) if rp[r + 1] - rp[r] == 5]
    assert len(inner) == (n - 1) ** 2
    for r in inner:
        row = dict(zip(ci[rp[r]:rp[r + 1]], v[rp[r]:rp[r + 1]]))
        assert row[r] == 4.0 / h / h
    # a fixture round trip through the writer keeps every byte
    out = os.path.join(GOLD, "..", "_tmp_roundtrip.bin")
    try:
        assert xamg.lib().XAMG_b200_csr_matrix_write_bin(out.encode(), xamg._ptr(b), xamg._ptr(x), m.h) == 0
        assert open(out, "rb").read() == open(os.path.join(GOLD, "mtx_Paus_n5.bin"), "rb").read()
    finally:
        if os.path.exists(out):
            os.remove(out)


def test_recorded_rhs_norm():
    rp, ci, v, b, u = util.gen2d(100)
    assert len(rp) - 1 == REC["nrows"] and len(ci) == REC["nonzeros"]
    nb = np.sqrt(orc.dot(b.reshape(-1, 1), b.reshape(-1, 1))[0])
    nbs = np.sqrt(orc.dot_sequential(b.reshape(-1, 1), b.reshape(-1, 1))[0])
    # the reference summed on 4 ranks; both orders agree to rounding
    assert abs(nb - REC["Y_norm"]) / REC["Y_norm"] < 4e-15
    assert abs(nbs - REC["Y_norm"]) / REC["Y_norm"] < 4e-15


def test_recorded_solution_norm_and_analytic_check():
    rp, ci, v, b, u = util.gen2d(100)
    csr = xamg.CsrMatrix.from_arrays(rp, ci, v)
    prm = xamg.Params(util.amg_params(max_levels=25))
    mg = orc.MG(xamg.amg_host(csr, prm))
    x, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, b.reshape(-1, 1), np.zeros((len(b), 1)), mg=mg,
                                        max_iters=100, rel_tol=1e-8)
    assert st[0] == 1
    assert np.sqrt(r0[0]) == pytest.approx(REC["initial_residual"], rel=4e-15)
    # recorded solve stopped at rel. residual 9.39e-9; solutions agree to that level
    assert abs(np.linalg.norm(x) - REC["X_norm"]) / REC["X_norm"] < 1e-7
    # xamg_test.cpp:162-177: difference to cos(hi) sin(hj)
    assert np.linalg.norm(x[:, 0] - u) / np.sqrt(len(u)) < 1e-5


@pytest.mark.parametrize("with_mg", [True, False])
def test_rbicgstab_restatement_solves_recorded_problem(with_mg):
    # rbicgstab.inl on the recorded 2-D problem: same solution as the recorded
    # PBiCGStab run, and its recurrence residual is the true residual
    rp, ci, v, b, u = util.gen2d(100 if with_mg else 40)
    B = b.reshape(-1, 1)
    mg = None
    if with_mg:
        csr = xamg.CsrMatrix.from_arrays(rp, ci, v)
        mg = orc.MG(xamg.amg_host(csr, xamg.Params(util.amg_params(max_levels=25))))
    x, it, hist, st, r0 = orc.rbicgstab(rp, ci, v, B, np.zeros_like(B), mg=mg, max_iters=2000, rel_tol=1e-8)
    assert st[0] == 1 and it > 0 and hist.shape == (it + 1, 1)
    true = B - orc.spmv(rp, ci, v, x, 1)
    assert np.sqrt(orc.dot(true, true)[0]) <= 1.01e-8 * np.sqrt(r0[0])
    assert abs(np.sqrt(hist[-1, 0]) - np.linalg.norm(true)) <= 1e-3 * np.sqrt(r0[0]) * 1e-8 + 1e-12
    if with_mg:
        assert abs(np.linalg.norm(x) - REC["X_norm"]) / REC["X_norm"] < 1e-7
        xp, itp, _, _, _ = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg=mg, max_iters=100, rel_tol=1e-8)
        assert abs(it - itp) <= 2


@pytest.mark.parametrize("with_mg", [True, False])
def test_pcg_restatement_solves_recorded_problem(with_mg):
    # pcg.inl: with AMG on the recorded 2-D problem, without a preconditioner
    # on the symmetric positive definite 7-point operator
    if with_mg:
        rp, ci, v, b, u = util.gen2d(100)
        B = b.reshape(-1, 1)
    else:
        rp, ci, v = xamg.CsrMatrix.cube(12, 12, 12, 0).arrays()
        B = np.random.default_rng(9).uniform(-1, 1, (len(rp) - 1, 1))
    mg = None
    if with_mg:
        csr = xamg.CsrMatrix.from_arrays(rp, ci, v)
        mg = orc.MG(xamg.amg_host(csr, xamg.Params(util.amg_params(max_levels=25))))
    x, it, hist, st, r0 = orc.pcg(rp, ci, v, B, np.zeros_like(B), mg=mg, max_iters=2000, rel_tol=1e-8)
    assert st[0] == 1 and it > 0 and hist.shape == (it + 1, 1)
    true = B - orc.spmv(rp, ci, v, x, 1)
    # the recurrence residual tracks the true one to rounding
    assert np.sqrt(orc.dot(true, true)[0]) <= 1.05e-8 * np.sqrt(r0[0])
    if with_mg:
        assert abs(np.linalg.norm(x) - REC["X_norm"]) / REC["X_norm"] < 1e-7


def test_dot_orders_agree_to_rounding():
    rng = np.random.default_rng(1)
    for n, nv in [(1, 1), (255, 2), (257, 4), (70000, 16), (1000, 32)]:
        a = rng.uniform(-1, 1, (n, nv))
        c = rng.uniform(-1, 1, (n, nv))
        d1 = orc.dot(a, c)
        d2 = orc.dot_sequential(a, c)
        ref = np.einsum("ik,ik->k", a.astype(np.longdouble), c.astype(np.longdouble))
        assert np.all(np.abs(d1 - ref) <= 1e-13 * np.sqrt(n) * np.abs(a * c).sum(0))
        assert np.all(np.abs(d2 - ref) <= 1e-13 * n * np.abs(a * c).sum(0))


def test_spmv_matches_numpy():
    rng = np.random.default_rng(2)
    rp, ci, v = util.random_csr(500, 300, rng, empty_rows=(3, 17))
    import scipy.sparse as sp
    A = sp.csr_matrix((v, ci, rp), shape=(500, 300))
    for nv in (1, 4, 16):
        x = rng.uniform(-1, 1, (300, nv))
        y = orc.spmv(rp, ci, v, x, nv)
        assert np.allclose(y, A @ x, rtol=1e-13, atol=1e-13)
        y0 = rng.uniform(-1, 1, (500, nv))
        y1 = orc.spmv(rp, ci, v, x, nv, y=y0.copy(), acc=True)
        assert np.allclose(y1, y0 + A @ x, rtol=1e-13, atol=1e-13)


def test_sgs_single_block_is_sequential_gauss_seidel():
    rng = np.random.default_rng(3)
    rp, ci, v = util.dd_csr(60, rng)
    n = 60
    invd = np.array([1.0 / v[rp[i]] for i in range(n)])
    b = rng.uniform(-1, 1, (n, 2))
    x0 = rng.uniform(-1, 1, (n, 2))
    relax = np.array([0.99, 0.99])
    x = orc.hsgs(rp, ci, v, invd, b, x0.copy(), relax)
    # plain python restatement of csr_gs.inl:75-130
    xr = x0.copy()
    for order in (range(n), range(n - 1, -1, -1)):
        for i in order:
            for k in range(2):
                s = b[i, k]
                for j in range(rp[i], rp[i + 1]):
                    s = s - v[j] * xr[ci[j], k]
                xr[i, k] += relax[k] * invd[i] * s
    assert np.allclose(x, xr, rtol=1e-13, atol=1e-13)


def test_dense_inverse_and_transpose():
    rng = np.random.default_rng(4)
    A = rng.uniform(-1, 1, (40, 40)) + 40 * np.eye(40)
    Ai = orc.dense_inverse(A)
    assert np.allclose(Ai @ A, np.eye(40), atol=1e-12)
    rp, ci, v = util.random_csr(50, 20, rng, diag=False)
    trp, tci, tv = orc.transpose(rp, ci, v, 20)
    import scipy.sparse as sp
    P = sp.csr_matrix((v, ci, rp), shape=(50, 20))
    R = sp.csr_matrix((tv, tci, trp), shape=(20, 50))
    assert (abs(P.T - R)).max() == 0
    for r in range(20):
        assert np.all(np.diff(tci[trp[r]:trp[r + 1]]) > 0)


def test_gs_levels_respect_sequential_order():
    rng = np.random.default_rng(5)
    rp, ci, v = util.random_csr(300, 300, rng, max_nnz=6)
    lf, lb = orc.gs_levels(rp, ci)
    for i in range(300):
        for j in ci[rp[i]:rp[i + 1]]:
            if j < i:
                assert lf[j] < lf[i]
            elif j > i:
                assert lf[j] > lf[i] and lb[j] < lb[i]


def test_threaded_oracle_is_bit_identical():
    """The oracle's parallel loops write disjoint outputs: one thread and all
    threads give the same bits (products, inner products, a preconditioned
    solve with its hybrid smoother)."""
    rp, ci, v = xamg.CsrMatrix.aniso27(14).arrays()
    rng = np.random.default_rng(21)
    B = rng.uniform(-1, 1, (len(rp) - 1, 4))
    csr = xamg.CsrMatrix.from_arrays(rp, ci, v)
    lv = xamg.amg_host(csr, xamg.Params(util.amg_params(max_levels=4)))
    full = orc.num_threads()
    out = []
    try:
        for t in (1, max(full, 2)):
            orc.set_num_threads(t)
            mg = orc.MG(lv, block_rows=300)
            x, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 100, 0.0, 1e-8)
            out.append((orc.spmv(rp, ci, v, B, 4), orc.dot(B, B), x, hist))
    finally:
        orc.set_num_threads(full)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
