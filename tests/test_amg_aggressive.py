"""Aggressive coarsening of the host AMG setup (mg_agg_num_levels > 0, the
reference's default of 10 levels, xamg_params_details.h:261, passed to hypre
at hypre_base.h:168-175): second-stage coarsening over paths of length <= 2
and multipass interpolation (mg_agg_interpolation_type 4, the default).  hypre
is absent, so there are no reference values to compare with; these CPU tests
check what the method guarantees: fewer coarse points and lower operator
complexity than standard coarsening, C rows of P that are unit rows, and an
AMG-PBiCGStab (oracle, on the exported hierarchy) that still reaches 1e-8."""
import numpy as np
import pytest

import oracle as orc
import xamg


def _levels(csr, spec, overrides=None):
    xamg.set_nv(1)
    p = xamg.Params({"solver": {"method": "PBiCGStab"}, "preconditioner": dict(method="MultiGrid", **spec)},
                    overrides)
    return xamg.amg_host(csr, p)


def _opc(lv):
    return sum(int(l["A"][0][-1]) for l in lv) / int(lv[0]["A"][0][-1])


def _solve(csr, lv):
    rp, ci, v = csr.arrays()
    B = np.random.default_rng(5).uniform(-1, 1, (csr.nrows, 2))
    x, it, hist, st, r0 = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), orc.MG(lv), 100, 0.0, 1e-8)
    R = B - _dense_spmv(rp, ci, v, x)
    return it, bool(np.all(st > 0)), float(np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)))


def _dense_spmv(rp, ci, v, x):
    import scipy.sparse as sp
    n = len(rp) - 1
    return sp.csr_matrix((v, ci, rp), shape=(n, n)) @ x


@pytest.mark.parametrize("gen", ["7pt", "27pt"])
def test_default_parameters_coarsen_aggressively_and_converge(gen):
    csr = xamg.CsrMatrix.cube(28, 28, 28, 0) if gen == "7pt" else xamg.CsrMatrix.aniso27(28, 1.0, 1.0, 1e-3)
    agg = _levels(csr, {})                             # reference defaults: 10 aggressive levels
    std = _levels(csr, {"mg_agg_num_levels": 0})
    assert len(agg) >= 3
    assert _opc(agg) < _opc(std)
    assert sum(l["n"] for l in agg[1:]) < sum(l["n"] for l in std[1:])
    for l in agg[:-1]:
        rpP, ciP, vP = l["P"]
        assert np.all(np.isfinite(vP))
        cnt = np.diff(rpP)
        # every coarse column has its C point: a row whose only entry is that
        # column with weight 1
        first = rpP[:-1][cnt == 1]
        unit_cols = np.unique(ciP[first[vP[first] == 1.0]])
        assert len(unit_cols) == l["ncP"]
    it, conv, res = _solve(csr, agg)
    assert conv and it <= 20 and res <= 1.1e-8


def test_multipass_preserves_constants_on_zero_row_sum_rows():
    # 2-D periodic-free Laplacian of the reference's analytic test: interior
    # rows sum to zero, so multipass interpolation reproduces constants there
    import util
    rp, ci, v, b, u = util.gen2d(64)
    csr = xamg.CsrMatrix.from_arrays(rp, ci, v)
    lv = _levels(csr, {"mg_agg_num_levels": 1})
    rpP, ciP, vP = lv[0]["P"]
    n = lv[0]["n"]
    rows = np.repeat(np.arange(n), np.diff(rpP))
    psum = np.bincount(rows, weights=vP, minlength=n)
    arow = np.bincount(np.repeat(np.arange(n), np.diff(rp)), weights=v, minlength=n)
    nbr_ok = np.diff(rpP) > 0
    interior = (np.abs(arow) < 1e-14) & nbr_ok
    # rows whose whole interpolation stencil stays among zero-sum rows
    assert np.count_nonzero(interior) > n // 2
    frac = np.mean(np.abs(psum[interior] - 1.0) < 1e-12)
    assert frac > 0.9


def test_per_level_override_and_unavailable_interpolation():
    csr = xamg.CsrMatrix.cube(16, 16, 16, 0)
    # the reference's example.c style: coarsening/interpolation changed on levels 0-1
    lv = _levels(csr, {}, {"preconditioner": {"mg_coarsening_type": "8@lev0-1", "mg_interpolation_type": "6@lev0-1"}})
    assert len(lv) >= 3
    with pytest.raises(xamg.XamgError) as e:
        _levels(csr, {"mg_agg_interpolation_type": 1})
    assert "error 4" in str(e.value) and "multipass" in str(e.value)
