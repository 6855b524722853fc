"""Synthetic problem families of the batching form and their sharding.

Batch family (one member per seed):
  side  = round(exp(U[ln 16, ln 96])) cells per axis (a cube);
  K     = lognormal(mu = 0, sigma = 1) per cell, harmonic means on interior
          faces and the cell value on the Dirichlet boundary faces;
  nv    = uniform in {1, 2, 4, 8}; right-hand sides uniform in [-1, 1].
The operator is the 7-point finite-volume diffusion matrix of the library's
face-coefficient generator (rows x-fastest, diagonal first).
"""
import numpy as np

import xamg


def faces_from_cells(k):
    """Harmonic means on interior faces, the cell value on boundary faces
    (k indexed [z, y, x])."""
    def hm(a, b):
        return 2.0 * a * b / (a + b)
    kx = np.concatenate([k[:, :, :1], hm(k[:, :, 1:], k[:, :, :-1]), k[:, :, -1:]], axis=2)
    ky = np.concatenate([k[:, :1, :], hm(k[:, 1:, :], k[:, :-1, :]), k[:, -1:, :]], axis=1)
    kz = np.concatenate([k[:1], hm(k[1:], k[:-1]), k[-1:]], axis=0)
    return kx, ky, kz


def batch_member(seed, lo=16, hi=96):
    """(matrix, nv, rhs [n^3, nv]) of family member `seed`."""
    rng = np.random.default_rng(seed)
    side = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
    k = rng.lognormal(0.0, 1.0, (side, side, side))
    A = xamg.CsrMatrix.faces7(side, side, side, *faces_from_cells(k))
    nv = int(rng.choice([1, 2, 4, 8]))
    B = rng.uniform(-1.0, 1.0, (side ** 3, nv))
    return A, nv, B


def shard(weights, world):
    """Greedy longest-processing-time assignment of items (by weight, e.g.
    nnz x nv) to `world` ranks; returns one sorted index list per rank."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += weights[i]
    return [sorted(o) for o in out]


def batch_spec(rel_tol=1e-8, max_iters=200, block_rows=256, blocks=0):
    """PBiCGStab (FP64) + AMG (FP32 inside the batch) with hybrid SGS on
    blocks of block_rows rows, or on `blocks` blocks per level when > 0."""
    hyb = {"hybrid_blocks": blocks} if blocks > 0 else {"hybrid_block_rows": block_rows}
    return {
        "solver": {"method": "PBiCGStab", "max_iters": max_iters, "abs_tolerance": 0.0, "rel_tolerance": rel_tol},
        "preconditioner": {"method": "MultiGrid", "mg_coarsening_type": 10, "mg_interpolation_type": 6,
                           "mg_strength_threshold": 0.25, "mg_max_levels": 6, "mg_agg_num_levels": 0},
        "pre_smoother": dict({"method": "HSGS", "max_iters": 1}, **hyb),
        "post_smoother": dict({"method": "HSGS", "max_iters": 1}, **hyb),
        "coarse_grid_solver": {"method": "Direct"},
    }
