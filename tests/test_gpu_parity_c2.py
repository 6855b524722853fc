"""Full-solve parity of the benchmark's solver on the benchmark's operator
family at the benchmark's width: the 27-point anisotropic (1, 1, 1e-3)
operator on a 48^3 grid, 16 right-hand sides uniform[-1,1], FP64
AMG-PBiCGStab (HMIS, extended+i, theta 0.25, 6 levels, HSGS 1+1 sweeps, direct
coarse solve) to 1e-8, through the XAMG C API on the GPU against the oracle on
the same hierarchy: identical iteration count, residual histories within
1e-12 relative (they are in fact identical), solutions within 1e-12.

Two smoother forms: the reference's single-process order (one Gauss-Seidel
sweep over each whole level) and the hybrid split the benchmark's mixed form
uses (every level cut into 296 equal blocks: Gauss-Seidel inside a block,
Jacobi across blocks, the reference's semantics on 296 processes), and 48
blocks, one z-plane each on the finest level, whose x tiles are too large for
shared memory (the slot-window form of the sweep)."""
import numpy as np
import pytest

import oracle as orc
import xamg

pytestmark = pytest.mark.gpu

NV = 16


def _spec(blocks):
    sm = {"method": "HSGS", "max_iters": 1}
    if blocks:
        sm["hybrid_blocks"] = blocks
    return {
        "solver": {"method": "PBiCGStab", "max_iters": 200, "abs_tolerance": 0.0, "rel_tolerance": 1e-8,
                   "convergence_details": "check-L2,noprint"},
        "preconditioner": {"method": "MultiGrid", "mg_coarsening_type": 10, "mg_interpolation_type": 6,
                           "mg_strength_threshold": 0.25, "mg_max_levels": 6, "mg_agg_num_levels": 0},
        "pre_smoother": dict(sm),
        "post_smoother": dict(sm),
        "coarse_grid_solver": {"method": "Direct"},
    }


@pytest.mark.parametrize("blocks", [0, 296, 48], ids=["sequential", "hybrid296", "hybrid48"])
def test_c2_family_full_solve_parity(gpu, blocks):
    n = 48
    csr = xamg.CsrMatrix.aniso27(n, 1.0, 1.0, 1e-3)
    rp, ci, v = csr.arrays()
    B = np.random.default_rng(2024).uniform(-1.0, 1.0, (csr.nrows, NV))
    xamg.set_nv(NV)
    A = xamg.Matrix(csr)
    x, b = xamg.Vector(csr.nrows, NV), xamg.Vector(csr.nrows, NV)
    b.upload(B)
    s = xamg.Solver(A, xamg.Params(_spec(blocks)), x, b)
    x.set(0.0)
    s.solve()
    X = x.download()
    levels = [s.level(l) for l in range(s.num_levels())]
    # the oracle builds the same hierarchy itself (its own setup) ...
    mine = orc.amg_setup(rp, ci, v, mg_coarsening_type=10, mg_strength_threshold=0.25, mg_max_levels=6)
    assert len(mine) == len(levels)
    for a, o in zip(levels, mine):
        assert all(np.array_equal(a["A"][k], o["A"][k]) for k in range(3))
    # ... and solves with it in the same smoother form
    br = [(lv["n"] + blocks - 1) // blocks for lv in mine] if blocks else None
    mg = orc.MG(mine, block_rows=br)
    xo, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), mg, 200, 0.0, 1e-8)
    assert all(s.converged()) and np.all(st > 0)
    assert s.iters()[0] == it and it >= 2
    h = s.history()
    assert h.shape == hist.shape
    np.testing.assert_allclose(h, hist, rtol=1e-12, atol=0)
    np.testing.assert_allclose(X, xo, rtol=1e-12, atol=1e-14 * np.abs(xo).max())
