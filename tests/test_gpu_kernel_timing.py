"""In-solve CUDA-event timing of the hot kernels (XAMG_b200_kernel_timing):
a 48^3 27-point FP64 AMG-PBiCGStab solve with 296- and 48-block hybrid
smoothers and the sequential-order smoother records every level's sweeps
under the form that ran (x tile, slot window, cooperative grid; hybrid
blocks by one warp per block, gsw_*, unless XAMG_GS_CTA_SWEEP selects one CTA
per block, gs_*) and every sparse product, with launch counts, positive times
and the algorithmic bytes of each launch."""
import numpy as np
import pytest

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


@pytest.mark.parametrize("blocks,fine_form", [(296, "tile"), (48, "window"), (0, "grid")],
                         ids=["hybrid296", "hybrid48", "sequential"])
def test_kernel_timing_records_sweep_forms(gpu, blocks, fine_form):
    n = 48
    csr = xamg.CsrMatrix.aniso27(n, 1.0, 1.0, 1e-3)
    B = np.random.default_rng(7).uniform(-1.0, 1.0, (csr.nrows, NV))
    xamg.set_nv(NV)
    A = xamg.Matrix(csr)
    x, b = xamg.Vector(csr.nrows, NV), xamg.Vector(csr.nrows, NV)
    b.upload(B)
    s = xamg.Solver(A, xamg.Params(_spec(blocks)), x, b)
    x.set(0.0)
    xamg.kernel_timing(True)
    try:
        s.solve()
        rec = xamg.kernel_timing_read()
    finally:
        xamg.kernel_timing(False)
    assert s.converged()
    fine = [r for r in rec if r["rows"] == csr.nrows]
    kinds = {r["kernel"] for r in fine}
    assert any(k.startswith("gs") and k.endswith("_" + fine_form) for k in kinds) and "spmv" in kinds
    sweeps = [r for r in rec if r["kernel"].startswith("gs")]
    assert len({r["rows"] for r in sweeps}) >= 3  # every smoothed level
    for r in rec:
        assert r["launches"] > 0 and r["ms"] > 0.0 and r["bytes"] > 0.0
    # the records were cleared by the read
    assert xamg.kernel_timing_read() == []
