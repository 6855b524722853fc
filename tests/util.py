"""Shared test inputs: the reference's analytic 2-D problem, random CSR matrices
and parameter sets of the benchmark configurations."""
import numpy as np


def gen2d(n):
    """examples/test/generate.hpp:188-286: (n+1)^2 grid, identity rows on the
    boundary, [-1,-1,4,-1,-1] inside; b = u on the boundary and 2 u h^2 inside,
    u = cos(h i) sin(h j), h = pi / (2 n)."""
    h = np.pi / n / 2
    N = (n + 1) * (n + 1)
    rp = [0]
    ci = []
    v = []
    for i in range(n + 1):
        for j in range(n + 1):
            r = i * (n + 1) + j
            if i == 0 or j == 0 or i == n or j == n:
                ci.append(r)
                v.append(1.0)
            else:
                ci += [(i - 1) * (n + 1) + j, i * (n + 1) + j - 1, r, i * (n + 1) + j + 1, (i + 1) * (n + 1) + j]
                v += [-1.0, -1.0, 4.0, -1.0, -1.0]
            rp.append(len(ci))
    r = np.arange(N)
    i, j = r // (n + 1), r % (n + 1)
    u = np.cos(h * i) * np.sin(h * j)
    bnd = (i == 0) | (j == 0) | (i == n) | (j == n)
    b = np.where(bnd, u, u * 2.0 * h * h)
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v), b, u


def random_csr(n, ncols, rng, min_nnz=0, max_nnz=12, diag=True, empty_rows=()):
    """Ragged random CSR (unsorted columns inside a row, optional empty rows)."""
    rp = [0]
    ci = []
    for r in range(n):
        k = 0 if r in empty_rows else int(rng.integers(min_nnz, max_nnz + 1))
        cols = list(rng.choice(ncols, size=min(k, ncols), replace=False))
        if diag and r not in empty_rows and r < ncols and r not in cols:
            cols = [r] + cols
        ci += cols
        rp.append(len(ci))
    v = rng.uniform(-1, 1, len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), v


def dd_csr(n, rng, max_off=8):
    """Diagonally dominant random sparse matrix with symmetric pattern."""
    rows = [set() for _ in range(n)]
    for r in range(n):
        for c in rng.choice(n, size=int(rng.integers(0, max_off + 1)), replace=False):
            if c != r:
                rows[r].add(int(c))
                rows[int(c)].add(r)
    rp = [0]
    ci = []
    v = []
    for r in range(n):
        cols = sorted(rows[r])
        vals = list(-rng.uniform(0.1, 1.0, len(cols)))
        d = -sum(vals) + rng.uniform(0.5, 1.5)
        ci += [r] + cols
        v += [d] + vals
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v)


def amg_params(precond_mg=True, max_levels=6, coarse=100, theta=0.25, smoother="HSGS",
               sweeps=1, max_iters=200, rel=1e-8, block_rows=0, schedule="persistent",
               meta=None, mg_reduced=False):
    spec = {"solver": {"method": "PBiCGStab" if precond_mg else "BiCGStab", "max_iters": max_iters,
                       "abs_tolerance": 0.0, "rel_tolerance": rel,
                       "convergence_details": "check-L2,noprint"}}
    if precond_mg:
        spec["preconditioner"] = {"method": "MultiGrid", "mg_coarsening_type": 10,
                                  "mg_interpolation_type": 6, "mg_strength_threshold": theta,
                                  "mg_agg_num_levels": 0, "mg_max_levels": max_levels,
                                  "mg_coarse_matrix_size": coarse, "mg_reduced_precision": mg_reduced}
        sm = {"method": smoother, "max_iters": sweeps}
        if smoother == "HSGS":
            sm["hybrid_block_rows"] = block_rows
            sm["gs_schedule"] = schedule
        spec["pre_smoother"] = dict(sm)
        spec["post_smoother"] = dict(sm)
        spec["coarse_grid_solver"] = {"method": "Direct"}
    if meta:
        spec["meta_solver"] = meta
    return spec
