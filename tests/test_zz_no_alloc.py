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
    for call, (n, nv) in enumerate([(70001, 16), (3000, 4)]):
        rng = np.random.default_rng(100 + call)
        vs = [_dev(rng.uniform(-1, 1, (n, nv)).astype(dtype), keep) for _ in range(3)]
        A = (C.c_void_p * 3)(_p(vs[0]), _p(vs[1]), _p(vs[2]))
        B = (C.c_void_p * 3)(_p(vs[1]), _p(vs[1]), _p(vs[0]))
        part = _dev(np.zeros(max(L.xamg_dot_part_size(n, 3, nv), 1)), keep)
        ref = _dev(np.zeros(3 * nv), keep)
        got = _dev(np.full(3 * nv, np.nan), keep)
        torch.cuda.synchronize()
        xamg.check(L.xamg_dot(prec, nv, n, 3, A, B, _p(part), _p(ref), sp))
        xamg.check(L.xamg_dot_noalloc(prec, nv, n, 3, A, B, _p(got), sp))
        stream.synchronize()
        assert np.array_equal(got.cpu().numpy(), ref.cpu().numpy()), call


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
