"""The oracle's own AMG setup and 27-point generator against the product's
host setup (CPU only).

Both are restatements of the algorithms the reference configures hypre with
(hypre_base.h:121-217: classical strength, HMIS / Falgout coarsening,
extended+i interpolation, truncation, Galerkin products).  They are written
independently; on the stated conventions they must give the same hierarchy,
entry for entry and bit for bit.  The oracle's setup is what the benchmark's
reference arm solves with, so that arm loads no product code."""
import numpy as np
import pytest

import families
import oracle as orc
import xamg

HMIS = {"mg_coarsening_type": 10, "mg_interpolation_type": 6, "mg_strength_threshold": 0.25, "mg_max_levels": 6,
        "mg_agg_num_levels": 0}
FALGOUT = {"mg_coarsening_type": 6, "mg_strength_threshold": 0.5, "mg_agg_num_levels": 0}


def _same_levels(lp, lo):
    assert len(lp) == len(lo)
    for l, (a, b) in enumerate(zip(lp, lo)):
        assert a["n"] == b["n"], l
        for k in range(3):
            assert np.array_equal(a["A"][k], b["A"][k]), (l, "A", k)
        assert (a["P"] is None) == (b["P"] is None), l
        if a["P"] is not None:
            assert a["ncP"] == b["ncP"]
            for k in range(3):
                assert np.array_equal(a["P"][k], b["P"][k]), (l, "P", k)


def _product_levels(csr, spec):
    xamg.set_nv(1)
    return xamg.amg_host(csr, xamg.Params({"preconditioner": dict(method="MultiGrid", **spec)}))


@pytest.mark.parametrize("n", [10, 24, 40])
def test_gen27_matches_product_generator(n):
    csr = xamg.CsrMatrix.aniso27(n, 1.0, 1.0, 1e-3)
    got = orc.gen27(n, 1.0, 1.0, 1e-3)
    for a, b in zip(csr.arrays(), got):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("spec", [HMIS, FALGOUT], ids=["hmis", "falgout"])
@pytest.mark.parametrize("n", [16, 40])
def test_oracle_amg_matches_product_27pt(spec, n):
    csr = xamg.CsrMatrix.aniso27(n, 1.0, 1.0, 1e-3)
    rp, ci, v = csr.arrays()
    q = {k: v2 for k, v2 in spec.items() if k in orc.AMG_DEFAULTS}
    lo = orc.amg_setup(rp, ci, v, **q)
    assert len(lo) >= 3
    _same_levels(_product_levels(csr, spec), lo)


@pytest.mark.parametrize("seed", [3, 17])
def test_oracle_amg_matches_product_variable_coefficients(seed):
    # a member of the batching family: 7-point, lognormal cell coefficients,
    # harmonic face averages (unstructured coarse levels)
    A, nv, B = families.batch_member(seed)
    rp, ci, v = A.arrays()
    q = {k: v2 for k, v2 in HMIS.items() if k in orc.AMG_DEFAULTS}
    lo = orc.amg_setup(rp, ci, v, **q)
    _same_levels(_product_levels(A, HMIS), lo)
