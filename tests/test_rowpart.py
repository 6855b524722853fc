"""Host side of a row-partitioned multi-GPU solve: the reference's block
partition (part.h), the halo plan and the send lists.  A product over
[owned x | halo x] with the renumbered local matrix must give every owned row
the single-system bits; checked in one process for 1..4 ranks and with two
gloo ranks exchanging the halo rows."""
import os

import numpy as np
import pytest

import oracle as orc
import util
import xamg


def _matrices():
    rng = np.random.default_rng(3)
    return [xamg.CsrMatrix.aniso27(9).arrays(), xamg.CsrMatrix.cube(8, 6, 5, 0).arrays(),
            util.random_csr(400, 400, rng, max_nnz=12, empty_rows=(0, 17))]


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_partition_products_match_the_whole_system(world):
    for rp, ci, v in _matrices():
        n = len(rp) - 1
        x = np.random.default_rng(world).uniform(-1, 1, (n, 4))
        ref = orc.spmv(rp, ci, v, x, 4)
        parts = [xamg.RowPart(rp, ci, world, r) for r in range(world)]
        # the reference's equal blocks, the remainder on the last
        bs = n // world
        assert [p.first for p in parts] == [r * bs for r in range(world)]
        assert sum(p.nrows for p in parts) == n
        for r, p in enumerate(parts):
            own = x[p.first:p.first + p.nrows]
            # the halo as the owners send it: each peer's send list, in order
            halo = np.zeros((len(p.halo), 4))
            for q in range(world):
                if q == r:
                    continue
                rows = parts[q].sends[r]
                slots = np.nonzero(p.owner == q)[0]
                assert np.array_equal(rows, p.halo[slots])
                halo[slots] = x[rows]
            assert np.all(np.diff(p.halo) > 0) and np.all((p.halo < p.first) | (p.halo >= p.first + p.nrows))
            xe = np.ascontiguousarray(np.vstack([own, halo]))
            y = orc.spmv(p.rp, p.ci, np.ascontiguousarray(v[p.src]), xe, 4)
            assert np.array_equal(y, ref[p.first:p.first + p.nrows])


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rp, ci, v = xamg.CsrMatrix.aniso27(10).arrays()
        n = len(rp) - 1
        x = np.random.default_rng(11).uniform(-1, 1, (n, 8))  # every rank slices its own rows
        p = xamg.RowPart(rp, ci, world, rank)
        own = x[p.first:p.first + p.nrows]
        reqs, bufs = [], {}
        for peer, rows in p.sends.items():
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(x[rows])), dst=peer))
        for peer in p.sends:
            slots = np.nonzero(p.owner == peer)[0]
            bufs[peer] = (slots, torch.zeros((len(slots), 8), dtype=torch.float64))
            reqs.append(dist.irecv(bufs[peer][1], src=peer))
        for r in reqs:
            r.wait()
        halo = np.zeros((len(p.halo), 8))
        for peer, (slots, t) in bufs.items():
            halo[slots] = t.numpy()
        y = orc.spmv(p.rp, p.ci, np.ascontiguousarray(v[p.src]), np.ascontiguousarray(np.vstack([own, halo])), 8)
        ok = bool(np.array_equal(y, orc.spmv(rp, ci, v, x, 8)[p.first:p.first + p.nrows]))
        q.put((rank, ok, len(p.halo)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_halo_rows():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (ok, nh)) for r, ok, nh in (q.get(timeout=180) for _ in ps))
    for p in ps:
        p.join(timeout=60)
    assert all(ok for ok, _ in res.values()), res
    assert all(nh > 0 for _, nh in res.values())


def _bicgstab_rank(rank, world, port, q):
    """Unpreconditioned BiCGStab (bicgstab.inl step order) over the row
    partition: one halo exchange per product, one allreduce per group of inner
    products (each rank's partial sums in the canonical tree over its rows)."""
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rp, ci, v = xamg.CsrMatrix.cube(12, 12, 12, 0).arrays()
        n, nv = len(rp) - 1, 2
        b_all = np.random.default_rng(5).uniform(-1, 1, (n, nv))
        p = xamg.RowPart(rp, ci, world, rank)
        lv = np.ascontiguousarray(v[p.src])
        sl = slice(p.first, p.first + p.nrows)

        def matvec(xl):
            reqs, bufs = [], {}
            for peer, rows in p.sends.items():
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(xl[rows - p.first])), dst=peer))
            for peer in p.sends:
                slots = np.nonzero(p.owner == peer)[0]
                bufs[peer] = (slots, torch.zeros((len(slots), nv), dtype=torch.float64))
                reqs.append(dist.irecv(bufs[peer][1], src=peer))
            for r in reqs:
                r.wait()
            halo = np.zeros((len(p.halo), nv))
            for slots, t in bufs.values():
                halo[slots] = t.numpy()
            return orc.spmv(p.rp, p.ci, lv, np.ascontiguousarray(np.vstack([xl, halo])), nv)

        def dots(*pairs):
            t = torch.from_numpy(np.concatenate([orc.dot(np.ascontiguousarray(a), np.ascontiguousarray(c))
                                                 for a, c in pairs]))
            dist.all_reduce(t)
            return t.numpy().reshape(len(pairs), nv)

        b = b_all[sl]
        x = np.zeros((p.nrows, nv))
        r0 = b - matvec(x)
        rho = dots((r0, r0))[0]
        tol = 1e-8 * np.sqrt(rho)
        r, pv = r0.copy(), r0.copy()
        it = 0
        while it < 500:
            it += 1
            vv = matvec(pv)
            alpha = rho / dots((vv, r0))[0]
            s = r - alpha * vv
            t = matvec(s)
            ts, tt, ss = dots((t, s), (t, t), (s, s))
            omega = ts / tt
            x = x + alpha * pv + omega * s
            res = ss - omega * ts
            if np.all(np.sqrt(np.maximum(res, 0)) <= tol):
                break
            r = s - omega * t
            s1 = dots((r, r0))[0]
            beta = (s1 / rho) * (alpha / omega)
            rho = s1
            pv = r - omega * beta * vv + beta * pv
        # true residual of the assembled solution, on rank 0
        got = [None] * world
        dist.all_gather_object(got, (p.first, x))
        if rank == 0:
            X = np.zeros((n, nv))
            for f, xl in got:
                X[f:f + len(xl)] = xl
            true = b_all - orc.spmv(rp, ci, v, X, nv)
            rel = np.linalg.norm(true, axis=0) / np.linalg.norm(b_all, axis=0)
            q.put((it, float(rel.max())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_with_bicgstab():
    import multiprocessing as mp
    rp, ci, v = xamg.CsrMatrix.cube(12, 12, 12, 0).arrays()
    B = np.random.default_rng(5).uniform(-1, 1, (len(rp) - 1, 2))
    _, it1, _, _, _ = orc.pbicgstab(rp, ci, v, B, np.zeros_like(B), None, 500, 0.0, 1e-8)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29800 + os.getpid() % 1000
    ps = [ctx.Process(target=_bicgstab_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    it, rel = q.get(timeout=300)
    for p in ps:
        p.join(timeout=60)
    # same method, inner products summed in another order: same convergence
    assert abs(it - it1) <= 1 and rel < 2e-8, (it, it1, rel)
