"""The allocation-free inner product (xamg_dot_noalloc).

Callers that cannot allocate device memory when they need an inner product
(a plug-in handed only its input and output buffers, a latency-critical loop
that must not pay cudaMalloc's implicit synchronisation) use this entry point
instead of xamg_dot: it needs no scratch buffer from them because its partial
sums live in a fixed array inside the library's device image.  These tests
call it through the C ABI and require exactly the results of xamg_dot (the
same bit-for-bit tolerance as every other kernel test), on two calls in a row
(the shared array keeps the previous call's contents, which must not leak
into the next result), and check that sizes beyond its fixed limit are
refused before anything runs.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import xamg

pytestmark = pytest.mark.gpu


def _dev(a, keep):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    keep.append(t)
    return t


def _p(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("prec,dtype", [(0, np.float64), (1, np.float32)])
def test_dot_noalloc_matches_dot_twice(gpu, prec, dtype):
    import torch
    L = xamg.lib()
    keep = []
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)
    # two calls in a row with different sizes (the second must not see the
    # first one's partial sums), then the four-pair form at nv 8 and 16
    for call, (n, nv, nd) in enumerate([(70001, 16, 3), (3000, 4, 3), (50003, 8, 4), (20000, 16, 4)]):
        rng = np.random.default_rng(100 + call)
        vs = [_dev(rng.uniform(-1, 1, (n, nv)).astype(dtype), keep) for _ in range(3)]
        A = (C.c_void_p * 4)(_p(vs[0]), _p(vs[1]), _p(vs[2]), _p(vs[2]))
        B = (C.c_void_p * 4)(_p(vs[1]), _p(vs[1]), _p(vs[0]), _p(vs[2]))
        part = _dev(np.zeros(max(L.xamg_dot_part_size(n, nd, nv), 1)), keep)
        ref = _dev(np.zeros(nd * nv), keep)
        got = _dev(np.full(nd * nv, np.nan), keep)
        torch.cuda.synchronize()
        xamg.check(L.xamg_dot(prec, nv, n, nd, A, B, _p(part), _p(ref), sp))
        xamg.check(L.xamg_dot_noalloc(prec, nv, n, nd, A, B, _p(got), sp))
        stream.synchronize()
        assert np.array_equal(got.cpu().numpy(), ref.cpu().numpy()), call


def test_dot_noalloc_null_stream_is_ordered_after_library_calls(gpu):
    """A NULL stream means the library's own stream for both entry points, so
    an inner product issued right after a BLAS-1 update that writes its input
    sees the update."""
    import torch
    L = xamg.lib()
    keep = []
    n, nv = 1 << 21, 16
    rng = np.random.default_rng(7)
    x = _dev(rng.uniform(-1, 1, (n, nv)), keep)
    y = _dev(rng.uniform(-1, 1, (n, nv)), keep)
    z = _dev(np.full((n, nv), np.nan), keep)
    a = _dev(np.full(nv, 0.5), keep)
    b = _dev(np.full(nv, -2.0), keep)
    got = _dev(np.full(nv, np.nan), keep)
    ref = _dev(np.zeros(nv), keep)
    part = _dev(np.zeros(L.xamg_dot_part_size(n, 1, nv)), keep)
    torch.cuda.synchronize()
    Z = (C.c_void_p * 1)(_p(z))
    xamg.check(L.xamg_blas(0, nv, n, 0, _p(a), _p(x), _p(b), _p(y), None, _p(z), None))
    xamg.check(L.xamg_dot_noalloc(0, nv, n, 1, Z, Z, _p(got), None))
    xamg.check(L.XAMG_b200_synchronize())
    torch.cuda.synchronize()
    xamg.check(L.xamg_dot(0, nv, n, 1, Z, Z, _p(part), _p(ref), None))
    xamg.check(L.XAMG_b200_synchronize())
    g = got.cpu().numpy()
    assert np.all(np.isfinite(g))
    assert np.array_equal(g, ref.cpu().numpy())


def test_dot_noalloc_at_its_exact_limit(gpu):
    """n = 2^28 rows at nv 1 needs exactly 2^20 partial sums: the last chunk
    writes the array's final element.  FP32, one 1 GiB vector."""
    import torch
    L = xamg.lib()
    n = (1 << 20) * 256
    assert L.xamg_dot_part_size(n, 1, 1) == 1 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    v = torch.rand(n, dtype=torch.float32, device="cuda", generator=g) - 0.5
    part = torch.zeros(1 << 20, dtype=torch.float64, device="cuda")
    ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    got = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    V = (C.c_void_p * 1)(_p(v))
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)
    torch.cuda.synchronize()
    for _ in range(2):
        xamg.check(L.xamg_dot(1, 1, n, 1, V, V, _p(part), _p(ref), sp))
        xamg.check(L.xamg_dot_noalloc(1, 1, n, 1, V, V, _p(got), sp))
        stream.synchronize()
        assert got.item() == ref.item() and np.isfinite(got.item())
        v.mul_(-1.5)  # the second call sees other values
        torch.cuda.synchronize()
    del v, part


def test_dot_noalloc_rejects_sizes_beyond_its_limit(gpu):
    L = xamg.lib()
    out = np.zeros(1)
    dummy = (C.c_void_p * 1)(None)
    # 2^20 partial sums fit; one chunk more does not
    n_ok = (1 << 20) * 256
    assert L.xamg_dot_part_size(n_ok, 1, 1) == 1 << 20
    rc = L.xamg_dot_noalloc(0, 1, n_ok + 256, 1, dummy, dummy, C.c_void_p(out.ctypes.data), None)
    assert rc == 2
    assert b"more than the fixed" in L.XAMG_b200_last_error()
