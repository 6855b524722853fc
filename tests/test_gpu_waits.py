"""Expired device waits come back as an error status, not a hang.

Every spin-wait in the library's kernels (the grid barrier of the cooperative
Gauss-Seidel sweep, the mbarrier waits on its staged copies) is bounded by a
wall-clock limit after which the kernel sets an error word and returns.  The
self-test entry point runs those same wait helpers with a short limit on a
wait that is made to run out on purpose (a barrier one CTA never reaches, an
mbarrier phase nothing completes) and must report code 3 within about the
limit; the device must stay usable afterwards."""
import time

import numpy as np
import pytest

import xamg


@pytest.mark.gpu
@pytest.mark.parametrize("which,ncta", [(0, 8), (1, 2)], ids=["grid_barrier", "mbarrier"])
def test_expired_wait_reports_code_3(gpu, which, ncta):
    L = xamg.lib()
    t0 = time.perf_counter()
    rc = L.XAMG_b200_wait_selftest(which, ncta, 0.2)
    dt = time.perf_counter() - t0
    assert rc == 3, L.XAMG_b200_last_error()
    assert b"bounded wait expired" in L.XAMG_b200_last_error()
    assert 0.15 <= dt < 10.0
    # the context is intact: a library call after the expired wait works
    assert L.XAMG_b200_synchronize() == 0
    import torch
    n, nv = 4096, 4
    x = torch.rand(n, nv, dtype=torch.float64, device="cuda")
    part = torch.zeros(L.xamg_dot_part_size(n, 1, nv), dtype=torch.float64, device="cuda")
    out = torch.zeros(nv, dtype=torch.float64, device="cuda")
    import ctypes as C
    X = (C.c_void_p * 1)(C.c_void_p(x.data_ptr()))
    torch.cuda.synchronize()
    xamg.check(L.xamg_dot(0, nv, n, 1, X, X, C.c_void_p(part.data_ptr()), C.c_void_p(out.data_ptr()), None))
    assert L.XAMG_b200_synchronize() == 0
    np.testing.assert_allclose(out.cpu().numpy(), (x * x).sum(0).cpu().numpy(), rtol=1e-12)


def test_wait_selftest_refuses_bad_arguments():
    L = xamg.lib()
    assert L.XAMG_b200_wait_selftest(7, 8, 0.2) == 2
    assert L.XAMG_b200_wait_selftest(0, 1, 0.2) == 2
    assert L.XAMG_b200_wait_selftest(0, 8, 5.0) == 2
