"""The reference's channel-with-cube test system
(examples/common/generator/channel_with_cube.inl, geometry lame.inl).

CPU: the properties the generator's construction fixes (sizes, the solid
block's identity rows, symmetry of the finite-volume couplings up to rounding
except the identity last row, zero row sums of interior fluid rows, the
right-hand-side forms), and bit for bit against the reference's own generator
compiled unchanged (oracle/build_ref_loops.py).  GPU: the reference's own
solver configuration for this
case (examples/test/yaml/multi_node/config-channel-cube1.yaml: PBiCGStab, 20
iterations, aggressive-coarsening AMG with HSGS) reduces the residual."""
import numpy as np
import pytest
import scipy.sparse as sp

import reference_loops
import xamg


@pytest.fixture(scope="module")
def channel1():
    xamg.set_nv(1)
    m, B = xamg.CsrMatrix.channel_cube(1, nv=2)
    rp, ci, v = m.arrays()
    return m, (rp, ci, v), B


def test_channel_cube_structure(channel1):
    m, (rp, ci, v), B = channel1
    nx, ny, nz = 144, 112, 144
    n = nx * ny * nz
    assert len(rp) - 1 == n == xamg.lib().XAMG_b200_channel_cube_rows(1)
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    r = np.arange(n)
    i, j, k = r % nx, (r // nx) % ny, r // (nx * ny)
    solid = (i >= 46) & (i < 98) & (j < 48) & (k >= 46) & (k < 98)
    cnt = np.diff(rp)
    assert np.all(cnt[solid] == 1)
    assert np.all(ci[rp[:-1]] == r)                      # diagonal first
    fluid = ~solid
    # 7-point rows away from the block and the walls (x and z periodic)
    assert np.all(cnt[fluid & (j > 0) & (j < ny - 1) & ~np.isin(r, [n - 1])] >= 6)
    # couplings symmetric to rounding, except the identity last row
    D = abs(A - A.T).tocoo()
    keep = (D.row != n - 1) & (D.col != n - 1)
    assert D.data[keep].max() <= 1e-12 * np.abs(v).max()
    # fluid rows whose neighbours are all fluid: zero row sum (to rounding)
    rs = np.asarray(A.sum(axis=1)).ravel()
    d = A.diagonal()
    inner = fluid & (cnt == 7) & (r != n - 1)
    assert np.all(np.abs(rs[inner]) <= 1e-12 * d[inner])
    # last row: identity with the others kept at zero; rhs 0 there
    assert v[rp[n - 1]] > 0 and np.all(v[rp[n - 1] + 1:rp[n]] == 0.0)
    assert np.all(B[n - 1] == 0.0)


def test_channel_cube_rhs_forms(channel1):
    m, (rp, ci, v), B = channel1
    assert np.all(np.isfinite(B)) and B.std() > 0
    # the two columns use different velocity draws
    assert not np.allclose(B[:, 0], B[:, 1])
    m1, B1 = xamg.CsrMatrix.channel_cube(1, nv=1, const_rhs=True)
    assert np.all(B1 == 1.0)
    assert np.array_equal(m1.arrays()[2], v)


@pytest.mark.gpu
def test_channel_cube_reference_config_converges(gpu, channel1):
    m, (rp, ci, v), B = channel1
    nv = 1
    xamg.set_nv(nv)
    B1 = np.ascontiguousarray(B[:, :1])
    spec = {
        "solver": {"method": "PBiCGStab", "abs_tolerance": 0.0, "rel_tolerance": 0.0, "max_iters": 20,
                   "convergence_details": "check-L2,noprint"},
        "preconditioner": {"method": "MultiGrid", "max_iters": 1, "mg_agg_num_levels": 10,
                           "mg_coarse_matrix_size": 500, "mg_num_paths": 2, "mg_trunc_factor": 0.3,
                           "mg_agg_trunc_factor": 0.3, "mg_strength_threshold": 0.25},
        "pre_smoother": {"method": "HSGS", "relax_factor": 0.95, "max_iters": 1},
        "post_smoother": {"method": "HSGS", "relax_factor": 0.95, "max_iters": 1},
        "coarse_grid_solver": {"method": "Direct"},
    }
    A = xamg.Matrix(m)
    x, b = xamg.Vector(len(rp) - 1, nv), xamg.Vector(len(rp) - 1, nv)
    b.upload(B1)
    s = xamg.Solver(A, xamg.Params(spec), x, b)
    x.set(0.0)
    s.solve()
    X = x.download()
    assert s.iters()[0] == 20
    As = sp.csr_matrix((v, ci, rp), shape=(len(rp) - 1,) * 2)
    rel = np.linalg.norm(B1 - As @ X) / np.linalg.norm(B1)
    assert rel < 1e-6, rel
    assert s.num_levels() >= 4


def test_channel_cube_matches_reference_generator(channel1):
    """The reference's generator (channel_with_cube.inl + lame.inl, its
    pseudo-random velocity stream from misc/rand.h) compiled unchanged: grid
    scale 1, divergence right-hand sides, NV = 2.  Row pointers, entry order,
    values and right-hand sides are identical bit for bit."""
    L = reference_loops.lib("generic")
    if L is None:
        pytest.skip("reference loop library not built (reference tree absent)")
    m, (rp, ci, v), B = channel1
    rrp, rci, rv, rB = reference_loops.channel_cube(L, 1, 2, const_rhs=False)
    assert np.array_equal(rp, rrp)
    assert np.array_equal(ci, rci)
    assert np.array_equal(v, rv)
    assert np.array_equal(B, rB)
