"""The hybrid Gauss-Seidel sweep's forms, each checked bit for bit against
the oracle (orc.hsgs, the reference's blas2::SGS restated) and identified by
the kernel-timing record of the form that ran: one warp per block with the
block's x tile in shared memory, with the slot window, and with the
per-level x gather (slot window off: XAMG_GS_NO_SLOT_WINDOW); and the
one-CTA-per-block kernel for every case, and as the warp kernel's fallback
when a level is too wide for one warp's record stages.  XAMG_GS_SWEEP
(warp / cta) picks the kernel; the switches are read once per process, so
the other kernel's cases run in child processes."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as orc
import util
import xamg

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


_alive = []


def D(a):
    """Device copy of a host array, kept alive until the next test starts
    (a pointer handed to the library must not dangle)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    _alive.append(t)
    return t


@pytest.fixture(autouse=True)
def _release_device_copies():
    yield
    import torch
    torch.cuda.synchronize()
    _alive.clear()


def H(t):
    return t.cpu().numpy()


def P(t):
    import ctypes as C
    return C.c_void_p(t.data_ptr())


def _run(rp, ci, v, brows, nv, dtype, prec, seed):
    rng = np.random.default_rng(seed)
    n = len(rp) - 1
    L = xamg.lib()
    plan = L.xamg_gs_plan_create(n, xamg._ptr(rp), xamg._ptr(ci), brows, 1)
    assert plan
    try:
        xamg.check(L.xamg_gs_plan_set_values(plan, xamg._ptr(np.ascontiguousarray(v, np.float64)), prec))
        vv = v.astype(dtype)
        rows = np.repeat(np.arange(n), np.diff(rp))
        dg = ci == rows
        invd = np.zeros(n, dtype)
        invd[rows[dg]] = [dtype(1.0 / np.float64(a)) for a in vv[dg]]
        b = rng.uniform(-1, 1, (n, nv)).astype(dtype)
        x0 = rng.uniform(-1, 1, (n, nv)).astype(dtype)
        relax = np.full(nv, 0.99, dtype)
        dx = D(x0)
        t = D(np.zeros((n, nv), dtype))
        xamg.kernel_timing(True)
        try:
            xamg.check(L.xamg_hsgs(plan, prec, nv, P(D(rp)), P(D(ci)), P(D(vv)), P(D(invd)), P(D(b)), P(dx),
                                   P(D(relax)), P(t), None))
            rec = xamg.kernel_timing_read()
        finally:
            xamg.kernel_timing(False)
        got = H(dx)
        ref = orc.hsgs(rp, ci, vv, invd, b, x0.copy(), relax, block_rows=brows)
        assert np.array_equal(got, ref), (dtype, nv, np.abs(got - ref).max())
        assert L.xamg_gs_plan_error(plan) == 0
        return {r["kernel"] for r in rec if r["kernel"].startswith("gs")}
    finally:
        L.xamg_gs_plan_destroy(plan)


def _warp_default():
    import xamg as _x
    return _x.gs_sweep_kernel() == "warp"


SWEEP = os.environ.get("XAMG_GS_SWEEP")
CTA = (SWEEP == "cta") if SWEEP in ("warp", "cta") else not _warp_default()
NOWIN = os.environ.get("XAMG_GS_NO_SLOT_WINDOW") is not None
PRE = "gs_" if CTA else "gsw_"


@pytest.mark.parametrize("nv", [1, 4, 16, 32])
@pytest.mark.parametrize("prec", [0, 1])
def test_tile_form(gpu, nv, prec):
    """27-point 24^3, 48 blocks of 288 rows: the x tile fits."""
    rp, ci, v = xamg.CsrMatrix.aniso27(24).arrays()
    dtype = np.float64 if prec == 0 else np.float32
    kinds = _run(rp, ci, v, 288, nv, dtype, prec, 31)
    assert PRE + "tile" in kinds, kinds


@pytest.mark.parametrize("nv", [8, 16, 32])
@pytest.mark.parametrize("prec", [0, 1])
def test_window_form(gpu, nv, prec):
    """27-point 80^3 in 296 blocks of 1730 rows (more blocks than SMs): from
    NV = 16 in FP32 on the block's x tile no longer fits beside the staging,
    the rows live at once do."""
    rp, ci, v = xamg.CsrMatrix.aniso27(80).arrays()
    dtype = np.float64 if prec == 0 else np.float32
    brows = -(-(len(rp) - 1) // 296)
    kinds = _run(rp, ci, v, brows, nv, dtype, prec, 37)
    row = nv * np.dtype(dtype).itemsize
    assert any(k.startswith("gs") for k in kinds), kinds
    if not NOWIN and row <= 128:  # wider FP64 rows may leave the warp kernel no room: CTA fallback
        assert any(k.startswith(PRE) for k in kinds), kinds
    if not CTA and not NOWIN and 64 <= row <= 128:
        assert PRE + "window" in kinds, kinds


@pytest.mark.parametrize("prec", [0, 1])
def test_gather_form(gpu, prec):
    """27-point 80^3 in 296 blocks, NV = 16: with the slot window switched off
    (XAMG_GS_NO_SLOT_WINDOW, a child process) neither the tile nor a window
    is available and each level gathers its x values."""
    rp, ci, v = xamg.CsrMatrix.aniso27(80).arrays()
    dtype = np.float64 if prec == 0 else np.float32
    brows = -(-(len(rp) - 1) // 296)
    kinds = _run(rp, ci, v, brows, 16, dtype, prec, 43)
    if NOWIN and not CTA:
        assert PRE + "gather" in kinds, kinds
    else:
        assert any(k.startswith(PRE) for k in kinds), kinds


@pytest.mark.parametrize("nv", [4, 16])
def test_falls_back_when_nothing_fits(gpu, nv):
    """Diagonally dominant random pattern, 7000 rows in blocks of 3000: its
    levels are too wide for three record stages of one warp, so the sweep
    runs one CTA per block."""
    rng = np.random.default_rng(41)
    rp, ci, v = util.dd_csr(7000, rng)
    kinds = _run(rp, ci, v, 3000, nv, np.float64, 0, 43)
    assert any(k.startswith("gs_") for k in kinds), kinds


@pytest.mark.parametrize("nv", [4, 16])
@pytest.mark.parametrize("prec", [0, 1])
def test_many_blocks(gpu, nv, prec):
    """27-point 64^3 in 1184 blocks of 222 rows (eight per SM): more blocks
    than two 256-thread CTAs per SM hold, so the CTA kernel runs 128-thread
    CTAs (four per SM); the warp kernel runs one warp per block."""
    rp, ci, v = xamg.CsrMatrix.aniso27(64).arrays()
    dtype = np.float64 if prec == 0 else np.float32
    brows = -(-(len(rp) - 1) // 1184)
    kinds = _run(rp, ci, v, brows, nv, dtype, prec, 47)
    assert any(k.startswith("gs") for k in kinds), kinds


def _child(**env):
    e = dict(os.environ, **env)
    return subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider",
                           os.path.join(HERE, "test_gpu_gs_forms.py"), os.path.join(HERE, "test_gpu_kernels.py"),
                           "-k", "form and not child or hsgs or falls_back or many_blocks"],
                          env=e, capture_output=True, text=True, timeout=900)


CHILD = SWEEP is not None or NOWIN


@pytest.mark.skipif(CHILD, reason="already a child process")
def test_gather_form_in_child_process(gpu):
    r = _child(XAMG_GS_NO_SLOT_WINDOW="1", XAMG_GS_SWEEP="warp")
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]


@pytest.mark.skipif(CHILD, reason="already a child process")
def test_other_sweep_kernel_in_child_process(gpu):
    r = _child(XAMG_GS_SWEEP="cta" if not CTA else "warp")
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
