"""Kernel-level parity through the C ABI: every result is compared with the CPU
oracle bit for bit (same operation order, same rounding)."""
import ctypes as C

import numpy as np
import pytest

import oracle as orc
import util
import xamg

pytestmark = pytest.mark.gpu

NVS = [1, 2, 4, 8, 16, 32]


_alive = []


def D(a):
    """Device copy of a host array.  Every copy is kept alive until the next
    test starts, so a pointer handed to the library never dangles."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    _alive.append(t)
    return t


@pytest.fixture(autouse=True)
def _release_device_copies():
    yield
    sync()
    _alive.clear()


def P(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def sync():
    import torch
    torch.cuda.synchronize()
    xamg.check(xamg.lib().XAMG_b200_synchronize())
    torch.cuda.synchronize()


def H(t):
    sync()
    return t.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("nv", NVS)
def test_spmv_bit_exact(gpu, dtype, nv):
    rng = np.random.default_rng(nv)
    n, ncols = 1500, 1300
    rp, ci, v = util.random_csr(n, ncols, rng, max_nnz=30, empty_rows=(0, 5, 1499))
    v = v.astype(dtype)
    x = rng.uniform(-1, 1, (ncols, nv)).astype(dtype)
    y0 = rng.uniform(-1, 1, (n, nv)).astype(dtype)
    b = rng.uniform(-1, 1, (n, nv)).astype(dtype)
    prec = 0 if dtype == np.float64 else 1
    drp, dci, dv, dx, db = D(rp), D(ci), D(v), D(x), D(b)
    L = xamg.lib()
    old = L.xamg_spmv_set_variant(-1)
    try:
        for variant in (0, -1, 1, 2, 3, 4, 5, 6, 11, 13):
            L.xamg_spmv_set_variant(variant)
            for mode in (0, 1, 2):
                dy = D(y0)
                sync()
                xamg.check(L.xamg_csr_spmv(prec, nv, n, P(drp), P(dci), P(dv), P(dx), P(dy), mode, P(db), None))
                got = H(dy)
                if mode == 0:
                    ref = orc.spmv(rp, ci, v, x, nv)
                elif mode == 1:
                    ref = orc.spmv(rp, ci, v, x, nv, y=y0.copy(), acc=True)
                else:
                    ref = orc.spmv(rp, ci, v, x, nv)
                    ref = (dtype(1) * b + dtype(-1) * ref).astype(dtype)
                assert np.array_equal(got, ref), (variant, mode, np.abs(got - ref).max())
    finally:
        L.xamg_spmv_set_variant(old)


def _run_matrices():
    """Square test operators for the shifted-row run kernel: stencils (runs
    along the grid lines), a ragged random matrix (every row a chunk of one,
    unsorted columns, empty rows) and a block-diagonal mix of both with one
    long row, so chunks of every length and tiles with unequal entry counts
    occur."""
    import scipy.sparse as sp
    rng = np.random.default_rng(42)
    out = [xamg.CsrMatrix.aniso27(13).arrays(), xamg.CsrMatrix.cube(11, 7, 5, 0).arrays(),
           util.random_csr(1200, 1200, rng, max_nnz=30, empty_rows=(0, 7, 1199))]
    arp, aci, av = xamg.CsrMatrix.aniso27(9).arrays()
    a = sp.csr_matrix((av, aci, arp), shape=(len(arp) - 1,) * 2)
    rp, ci, v = util.random_csr(301, 301, rng, max_nnz=9, empty_rows=(3,))
    r = sp.csr_matrix((v, ci, rp), shape=(301, 301))
    blk = sp.block_diag([a, r, sp.identity(5), a], format="lil")
    blk[7, :200] = rng.uniform(-1, 1, 200)  # one long row
    blk = blk.tocsr()
    blk.sort_indices()
    out.append((blk.indptr.astype(np.int32), blk.indices.astype(np.int32), blk.data.astype(np.float64)))
    return out


@pytest.mark.parametrize("form", [0, 1], ids=["x_in_registers", "x_staged"])
@pytest.mark.parametrize("dtype,nv", [(np.float64, 8), (np.float64, 16), (np.float64, 32),
                                      (np.float32, 16), (np.float32, 32)])
def test_spmv_runs_bit_exact(gpu, dtype, nv, form):
    """Shifted-row run kernel, both forms (x rows gathered into registers, or
    copied into shared memory a segment ahead): identical bits to the
    oracle's CSR product in all three modes, on stencil, irregular and mixed
    operators."""
    L = xamg.lib()
    old_form = L.xamg_spmv_set_run_form(form)
    prec = 0 if dtype == np.float64 else 1
    for mi, (rp, ci, v) in enumerate(_run_matrices()):
        n = len(rp) - 1
        plan = L.xamg_spmv_runs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), xamg._ptr(v), 8, 1)
        assert plan, xamg.lib().XAMG_b200_last_error()
        try:
            nch = np.zeros(1, np.int64)
            cov = np.zeros(1)
            ns = np.zeros(1, np.int64)
            xamg.check(L.xamg_spmv_runs_plan_info(plan, xamg._ptr(nch), xamg._ptr(cov), xamg._ptr(ns), None))
            assert ns[0] <= len(ci)
            if mi == 0:
                assert ns[0] < len(ci) / 6  # 27-point rows: 9 segments of 3, chunks of several rows
            if mi == 0:
                assert cov[0] > 0.6 and nch[0] < n / 2, (cov, nch, n)
            if mi == 2:
                assert cov[0] == 0.0 and nch[0] == n
            vv = v.astype(dtype)
            rng = np.random.default_rng(nv + mi)
            x = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            y0 = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            b = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            dx, db = D(x), D(b)
            for mode in (0, 1, 2):
                dy = D(y0)
                sync()
                xamg.check(L.xamg_spmv_runs(plan, prec, nv, P(dx), P(dy), mode, P(db), None))
                got = H(dy)
                ref = orc.spmv(rp, ci, vv, x, nv, y=y0.copy() if mode == 1 else None, acc=mode == 1)
                if mode == 2:
                    ref = (dtype(1) * b + dtype(-1) * ref).astype(dtype)
                assert np.array_equal(got, ref), (mi, mode, np.abs(got - ref).max())
        finally:
            L.xamg_spmv_runs_plan_destroy(plan)
    L.xamg_spmv_set_run_form(old_form)


def test_spmv_runs_rejects_narrow_shapes(gpu):
    rp, ci, v = xamg.CsrMatrix.aniso27(6).arrays()
    L = xamg.lib()
    plan = L.xamg_spmv_runs_plan_create(len(rp) - 1, xamg._ptr(rp), xamg._ptr(ci), xamg._ptr(v), 8, 0)
    try:
        n = len(rp) - 1
        dx, dy = D(np.zeros((n, 4))), D(np.zeros((n, 4)))
        assert L.xamg_spmv_runs(plan, 0, 4, P(dx), P(dy), 0, None, None) == 2   # nv 4: not a run shape
        assert L.xamg_spmv_runs(plan, 1, 16, P(dx), P(dy), 0, None, None) == 2  # no FP32 values
    finally:
        L.xamg_spmv_runs_plan_destroy(plan)
    assert L.xamg_spmv_runs_plan_create(len(rp) - 1, xamg._ptr(rp), xamg._ptr(ci), xamg._ptr(v), 4, 0) is None


def test_spmv_large_checksum(gpu):
    """Full-size product through a size-independent property: y = A x for
    x = e_k columns reproduces the CSR columns, checked by a bxor-style
    checksum of the result bits (tst_spmv.h:63-91)."""
    m = xamg.CsrMatrix.aniso27(64)
    rp, ci, v = m.arrays()
    n = m.nrows
    nv = 16
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (n, nv))
    dy = D(np.zeros((n, nv)))
    L = xamg.lib()
    xamg.check(L.xamg_csr_spmv(0, nv, n, P(D(rp)), P(D(ci)), P(D(v)), P(D(x)), P(dy), 0, None, None))
    got = H(dy)
    ref = orc.spmv(rp, ci, v, x, nv)
    xor = np.bitwise_xor.reduce(got.view(np.uint64), axis=0)
    xref = np.bitwise_xor.reduce(ref.view(np.uint64), axis=0)
    assert np.array_equal(xor, xref)


@pytest.mark.parametrize("nv", NVS)
@pytest.mark.parametrize("n", [1, 200, 256, 257, 70001])
def test_dot_bit_exact(gpu, nv, n):
    rng = np.random.default_rng(n + nv)
    L = xamg.lib()
    for dtype, prec in ((np.float64, 0), (np.float32, 1)):
        vs = [rng.uniform(-1, 1, (n, nv)).astype(dtype) for _ in range(3)]
        dvs = [D(a) for a in vs]
        # three pairs, and the four of RBiCGStab's step 13 (one pass up to
        # nv 8, two passes of two pairs above)
        for pairs in ([(0, 1), (1, 1), (2, 0)], [(0, 1), (0, 0), (0, 2), (1, 1)]):
            nd = len(pairs)
            A = (C.c_void_p * nd)(*[P(dvs[i]) for i, _ in pairs])
            B = (C.c_void_p * nd)(*[P(dvs[j]) for _, j in pairs])
            part = D(np.zeros(max(L.xamg_dot_part_size(n, nd, nv), 1)))
            out = D(np.zeros(nd * nv))
            xamg.check(L.xamg_dot(prec, nv, n, nd, A, B, P(part), P(out), None))
            got = H(out).reshape(nd, nv)
            for d, (i, j) in enumerate(pairs):
                assert np.array_equal(got[d], orc.dot(vs[i], vs[j])), (d, nd, dtype)


@pytest.mark.parametrize("nv", [1, 4, 16, 32])
def test_blas_bit_exact(gpu, nv):
    rng = np.random.default_rng(11)
    n = 3001
    L = xamg.lib()
    a, b, c = (rng.uniform(-2, 2, nv) for _ in range(3))
    da, db, dc = D(a), D(b), D(c)
    for dtype, prec in ((np.float64, 0), (np.float32, 1)):
        x, y, z = (rng.uniform(-1, 1, (n, nv)).astype(dtype) for _ in range(3))
        x64, y64, z64 = (q.astype(np.float64) for q in (x, y, z))
        refs = {
            0: a * x64 + b * y64,
            1: (a * x64 + b * y64) + c * z64,
            2: a * x64,
            3: x64,
            4: np.broadcast_to(a, (n, nv)),
            5: z64 * x64,
        }
        for op, ref in refs.items():
            dz = D(z)
            xamg.check(L.xamg_blas(prec, nv, n, op, P(da), P(D(x)), P(db), P(D(y)), P(dc), P(dz), None))
            assert np.array_equal(H(dz), ref.astype(dtype)), (op, dtype)


def _gs_case(rng, kind, n=500):
    if kind == "dd":
        return util.dd_csr(n, rng)
    m = xamg.CsrMatrix.aniso27(9)
    return m.arrays()


@pytest.mark.parametrize("kind", ["dd", "27pt"])
@pytest.mark.parametrize("block_rows", [0, 64])
@pytest.mark.parametrize("schedule", [0, 1, 2])
@pytest.mark.parametrize("lcsr", [False, True])
@pytest.mark.parametrize("nv", [1, 4, 16])
def test_hsgs_bit_exact(gpu, kind, block_rows, schedule, lcsr, nv):
    rng = np.random.default_rng(21)
    rp, ci, v = _gs_case(rng, kind)
    n = len(rp) - 1
    L = xamg.lib()
    plan = L.xamg_gs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), block_rows, schedule)
    assert plan
    try:
        for dtype, prec in ((np.float64, 0), (np.float32, 1)):
            if lcsr:
                xamg.check(L.xamg_gs_plan_set_values(plan, xamg._ptr(np.ascontiguousarray(v, np.float64)), prec))
            vv = v.astype(dtype)
            invd = np.zeros(n, dtype)
            for i in range(n):
                for j in range(rp[i], rp[i + 1]):
                    if ci[j] == i:
                        invd[i] = dtype(1.0 / np.float64(vv[j]))
            b = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            x0 = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            relax = np.full(nv, 0.99, dtype)
            dx = D(x0)
            t = D(np.zeros((n, nv), dtype))
            xamg.check(L.xamg_hsgs(plan, prec, nv, P(D(rp)), P(D(ci)), P(D(vv)), P(D(invd)), P(D(b)),
                                   P(dx), P(D(relax)), P(t), None))
            got = H(dx)
            ref = orc.hsgs(rp, ci, vv, invd, b, x0.copy(), relax, block_rows=block_rows)
            assert np.array_equal(got, ref), (dtype, np.abs(got - ref).max())
        assert L.xamg_gs_plan_error(plan) == 0
    finally:
        L.xamg_gs_plan_destroy(plan)


@pytest.mark.parametrize("nv", [4, 16])
def test_hsgs_blocks_without_shared_tile_bit_exact(gpu, nv):
    """Hybrid blocks too large for a shared-memory x tile (x gathered per
    level instead): same results as the oracle."""
    rng = np.random.default_rng(23)
    n, brows = 7000, 3000
    rp, ci, v = util.dd_csr(n, rng)
    L = xamg.lib()
    plan = L.xamg_gs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), brows, 1)
    assert plan
    try:
        for dtype, prec in ((np.float64, 0), (np.float32, 1)):
            assert brows * nv * np.dtype(dtype).itemsize > 170 * 1024 or nv == 4
            xamg.check(L.xamg_gs_plan_set_values(plan, xamg._ptr(np.ascontiguousarray(v, np.float64)), prec))
            vv = v.astype(dtype)
            invd = np.array([dtype(1.0 / np.float64(vv[rp[i]])) for i in range(n)], dtype)
            b = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            x0 = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            relax = np.full(nv, 0.99, dtype)
            dx = D(x0)
            t = D(np.zeros((n, nv), dtype))
            xamg.check(L.xamg_hsgs(plan, prec, nv, P(D(rp)), P(D(ci)), P(D(vv)), P(D(invd)), P(D(b)),
                                   P(dx), P(D(relax)), P(t), None))
            got = H(dx)
            ref = orc.hsgs(rp, ci, vv, invd, b, x0.copy(), relax, block_rows=brows)
            assert np.array_equal(got, ref), (dtype, np.abs(got - ref).max())
        assert L.xamg_gs_plan_error(plan) == 0
    finally:
        L.xamg_gs_plan_destroy(plan)


@pytest.mark.parametrize("nv", [8, 16, 32])
def test_hsgs_blocks_slot_window_bit_exact(gpu, nv):
    """Hybrid blocks of one 56x56 plane of the 27-point operator (56^3): the
    block's x tile is too large for shared memory, but the rows live at once
    fit a slot window, so every x value is read from shared memory and
    first-use rows are loaded ahead.  Same results as the oracle, and the
    window really is the path taken."""
    rng = np.random.default_rng(29)
    n3 = 56
    rp, ci, v = xamg.CsrMatrix.aniso27(n3).arrays()
    n = len(rp) - 1
    brows = n3 * n3
    L = xamg.lib()
    plan = L.xamg_gs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), brows, 1)
    assert plan
    try:
        for dtype, prec in ((np.float64, 0), (np.float32, 1)):
            xamg.check(L.xamg_gs_plan_set_values(plan, xamg._ptr(np.ascontiguousarray(v, np.float64)), prec))
            sz = np.dtype(dtype).itemsize
            ns = np.zeros(2, np.int32)
            xamg.check(L.xamg_gs_plan_slots(plan, xamg._ptr(ns)))
            if brows * nv * sz <= 170 * 1024 or ns.max() * nv * sz > 64 * 1024:
                continue  # the tile or the gather form applies at this width
            assert 0 < ns.max() < brows // 4
            vv = v.astype(dtype)
            invd = np.array([dtype(1.0 / np.float64(vv[rp[i]])) for i in range(n)], dtype)
            b = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            x0 = rng.uniform(-1, 1, (n, nv)).astype(dtype)
            relax = np.full(nv, 0.99, dtype)
            for rep in range(2):  # two calls in a row on the same plan
                dx = D(x0)
                t = D(np.zeros((n, nv), dtype))
                xamg.check(L.xamg_hsgs(plan, prec, nv, P(D(rp)), P(D(ci)), P(D(vv)), P(D(invd)), P(D(b)),
                                       P(dx), P(D(relax)), P(t), None))
                got = H(dx)
                ref = orc.hsgs(rp, ci, vv, invd, b, x0.copy(), relax, block_rows=brows)
                assert np.array_equal(got, ref), (dtype, rep, np.abs(got - ref).max())
        assert L.xamg_gs_plan_error(plan) == 0
    finally:
        L.xamg_gs_plan_destroy(plan)


@pytest.mark.parametrize("nv", [1, 8, 32])
def test_jacobi_and_dense_bit_exact(gpu, nv):
    rng = np.random.default_rng(31)
    rp, ci, v = util.dd_csr(700, rng)
    n = 700
    L = xamg.lib()
    invd = np.array([1.0 / v[rp[i]] for i in range(n)])
    b = rng.uniform(-1, 1, (n, nv))
    x0 = rng.uniform(-1, 1, (n, nv))
    relax = np.full(nv, 0.99)
    dxo = D(np.zeros((n, nv)))
    xamg.check(L.xamg_jacobi(0, nv, n, P(D(rp)), P(D(ci)), P(D(v)), P(D(invd)), P(D(b)), P(D(x0)), P(dxo), P(D(relax)), None))
    ref = orc.jacobi(rp, ci, v, invd, b, x0.copy(), relax)
    assert np.array_equal(H(dxo), ref)
    nc = 123
    Ai = rng.uniform(-1, 1, (nc, nc))
    bb = rng.uniform(-1, 1, (nc, nv))
    dy = D(np.zeros((nc, nv)))
    xamg.check(L.xamg_dense_gemv(0, nv, nc, P(D(np.ascontiguousarray(Ai.T))), P(D(bb)), P(dy), None))
    assert np.array_equal(H(dy), orc.dense_gemv(Ai, bb))
