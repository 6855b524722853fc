"""Row-partitioned solve of one system (XAMG_b200_dist_*), on the one GPU a
test has: with a single rank the halo is empty and the allreduce sums one
value, so every iteration must equal the single-GPU solver's bit for bit
(iteration count, residual history and solution).  This runs the whole
device path of the distributed solver (local operator with renumbered
columns, NCCL communicator, allreduce of every step's inner products, the
preconditioner on the rank's diagonal block, the fused update kernels); the
halo exchange between ranks is checked on the host (tests/test_rowpart.py)."""
import numpy as np
import pytest

import util
import xamg


def _single(csr, spec, B):
    n, nv = B.shape
    xamg.set_nv(nv)
    A = xamg.Matrix(csr)
    x, b = xamg.Vector(n, nv), xamg.Vector(n, nv)
    b.upload(B)
    s = xamg.Solver(A, xamg.Params(spec), x, b)
    x.set(0.0)
    s.solve()
    return s.iters()[0], s.history(), x.download()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["bicgstab_7pt", "pbicgstab_amg_27pt", "pbicgstab_amg_hybrid"])
def test_dist_one_rank_equals_single_gpu(gpu, case):
    import torch
    nv = 4
    if case == "bicgstab_7pt":
        csr = xamg.CsrMatrix.cube(20, 20, 20, 0)
        spec = util.amg_params(precond_mg=False, max_iters=500)
    else:
        csr = xamg.CsrMatrix.aniso27(24)
        spec = util.amg_params(max_levels=6, block_rows=0 if case == "pbicgstab_amg_27pt" else 300)
    rp, ci, v = csr.arrays()
    B = np.random.default_rng(5).uniform(-1, 1, (csr.nrows, nv))
    it1, h1, X1 = _single(csr, spec, B)
    xamg.set_nv(nv)
    ds = xamg.DistSolver(rp, ci, v, 1, 0, xamg.Params(spec), nv, xamg.dist_unique_id())
    b = torch.from_numpy(B).cuda()
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    ds.solve(b.data_ptr(), x.data_ptr())
    info = ds.info()
    assert info["rows"] == csr.nrows and info["converged"]
    assert info["iters"] == it1 and it1 > 1
    h = ds.history()
    assert h.shape == h1.shape
    np.testing.assert_allclose(h, h1, rtol=1e-12, atol=0)
    X = x.cpu().numpy()
    np.testing.assert_allclose(X, X1, rtol=1e-12, atol=1e-14 * np.abs(X1).max())
    assert np.array_equal(X, X1)


def test_dist_refuses_other_methods_before_any_device_work():
    # the method is checked before NCCL or the device are touched
    rp, ci, v = xamg.CsrMatrix.cube(6, 6, 6, 0).arrays()
    spec = util.amg_params(precond_mg=False)
    spec["solver"]["method"] = "PCG"
    with pytest.raises(xamg.XamgError) as e:
        xamg.DistSolver(rp, ci, v, 1, 0, xamg.Params(spec), 1, bytes(128))
    assert "(P)BiCGStab" in str(e.value)
