"""Batching form: independent systems of uneven size and nv solved together in
one CUDA-graph launch; every system must reach 1e-8 and agree with an FP64
solve of that system alone."""
import numpy as np
import pytest
import scipy.sparse as sp

import families
import xamg

pytestmark = pytest.mark.gpu


def _plain_fp64(A, B, nv):
    spec = {
        "solver": {"method": "PBiCGStab", "max_iters": 300, "abs_tolerance": 0.0, "rel_tolerance": 1e-12,
                   "convergence_details": "check-L2,noprint"},
        "preconditioner": {"method": "MultiGrid", "mg_coarsening_type": 10, "mg_interpolation_type": 6,
                           "mg_strength_threshold": 0.25, "mg_max_levels": 6, "mg_agg_num_levels": 0},
        "pre_smoother": {"method": "HSGS", "max_iters": 1},
        "post_smoother": {"method": "HSGS", "max_iters": 1},
        "coarse_grid_solver": {"method": "Direct"},
    }
    xamg.set_nv(nv)
    M = xamg.Matrix(A)
    x, b = xamg.Vector(A.nrows, nv), xamg.Vector(A.nrows, nv)
    b.upload(B)
    s = xamg.Solver(M, xamg.Params(spec), x, b)
    s.solve()
    assert all(s.converged())
    return x.download()


def _members(seeds, lo, hi):
    return [families.batch_member(s, lo, hi) for s in seeds]


def test_batch_matches_single_system_solves(gpu):
    mem = _members(range(11, 21), 6, 18)
    batch = xamg.Batch([(A, nv) for A, nv, _ in mem], xamg.Params(families.batch_spec(block_rows=64)))
    assert {g[0] for g in batch.groups()} == {nv for _, nv, _ in mem}
    for q, (A, nv, B) in enumerate(mem):
        batch.upload(q, B)
    batch.solve()
    X_graph = [batch.download(q) for q in range(len(mem))]
    for q, (A, nv, B) in enumerate(mem):
        rp, ci, v = A.arrays()
        M = sp.csr_matrix((v, ci, rp), shape=(A.nrows, A.nrows))
        X = X_graph[q]
        it, rr = batch.stats(q)
        assert np.all(it > 0) and np.all(rr <= 1e-8), (q, it, rr)
        res = np.linalg.norm(B - M @ X, axis=0) / np.linalg.norm(B, axis=0)
        assert np.all(res <= 3e-8), (q, res)
        ref = _plain_fp64(A, B, nv)
        err = np.linalg.norm(X - ref) / np.linalg.norm(ref)
        assert err <= 1e-6, (q, err)
    # the same steps launched from the host give the same answer, bit for bit
    batch.set_graph(False)
    for q, (A, nv, B) in enumerate(mem):
        batch.upload(q, B)
    batch.solve()
    for q in range(len(mem)):
        assert np.array_equal(batch.download(q), X_graph[q])


def test_batch_repeated_solves_are_identical(gpu):
    mem = _members(range(31, 37), 8, 20)
    batch = xamg.Batch([(A, nv) for A, nv, _ in mem], xamg.Params(families.batch_spec(block_rows=128)))
    outs = []
    for _ in range(3):
        for q, (A, nv, B) in enumerate(mem):
            batch.upload(q, B)
        batch.solve()
        outs.append([batch.download(q) for q in range(len(mem))])
    for q in range(len(mem)):
        assert np.array_equal(outs[0][q], outs[1][q]) and np.array_equal(outs[0][q], outs[2][q])
    assert batch.last_ms() > 0


def test_batch_reports_unconverged_columns(gpu):
    """An iteration cap below what the systems need leaves columns marked
    not converged (-1) and the graph loop still ends."""
    mem = _members(range(41, 45), 10, 16)
    batch = xamg.Batch([(A, nv) for A, nv, _ in mem], xamg.Params(families.batch_spec(max_iters=1, block_rows=64)))
    for q, (A, nv, B) in enumerate(mem):
        batch.upload(q, B)
    batch.solve()
    its = np.concatenate([batch.stats(q)[0] for q in range(len(mem))])
    assert np.all(its == -1)


def test_segmented_dots_equal_oracle_per_segment(gpu):
    """The batching form's per-system inner products (k_segdot1/2) over
    concatenated vectors of uneven segments (empty, under one 256-row chunk,
    ragged) equal the oracle's canonical tree (orc.dot, the reference's
    blas.inl:488-612 with the fixed chunk tree) run on each segment alone,
    bit for bit, FP64 and FP32 inputs, NV 1, 4 and 16, one to three pairs."""
    import ctypes as C
    import torch
    import oracle as orc
    L = xamg.lib()
    rng = np.random.default_rng(77)
    sizes = [1000, 1, 0, 4000, 70000, 123, 256]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    n, nseg = int(off[-1]), len(sizes)
    for dtype, prec in ((np.float64, 0), (np.float32, 1)):
        for nv in (1, 4, 16):
            vs = [rng.uniform(-1, 1, (n, nv)).astype(dtype) for _ in range(3)]
            dv = [torch.from_numpy(a).cuda() for a in vs]
            for pairs in ([(0, 1)], [(0, 1), (2, 2)], [(0, 1), (1, 1), (2, 0)]):
                nd = len(pairs)
                A = (C.c_void_p * nd)(*[C.c_void_p(dv[i].data_ptr()) for i, _ in pairs])
                B = (C.c_void_p * nd)(*[C.c_void_p(dv[j].data_ptr()) for _, j in pairs])
                out = torch.zeros(nd * nseg * nv, dtype=torch.float64, device="cuda")
                xamg.check(L.xamg_seg_dot(prec, nv, nseg, off.ctypes.data, nd, A, B,
                                          C.c_void_p(out.data_ptr()), None))
                got = out.cpu().numpy().reshape(nd, nseg, nv)
                for d, (i, j) in enumerate(pairs):
                    for s in range(nseg):
                        a, b = vs[i][off[s]:off[s + 1]], vs[j][off[s]:off[s + 1]]
                        ref = orc.dot(np.ascontiguousarray(a), np.ascontiguousarray(b)) if len(a) else np.zeros(nv)
                        assert np.array_equal(got[d, s], ref), (dtype, nv, nd, d, s)
