"""The reference's own C callers, examples/c/example.c (AMG-PBiCGStab) and
example_ir.c (iterative refinement around an FP32 AMG-PBiCGStab), built
unchanged against this library (oracle/build_ref_examples.py) and run on the
GPU: each program solves the reference's 10^3 7-point system twice (to 1e-6,
then, after XAMG_solver_renew_params, to 1e-8) and prints its convergence
lines; the run must exit 0 and its last printed relative residual of the
second solve must meet 1e-8.  Built for XAMG_NV = 1 and 4 (the library takes
its NV from the XAMG_NV environment variable, the programs from the same
compile-time macro)."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref")


def _last_relres(lines, prefix):
    vals = None
    for ln in lines:
        if ln.startswith(prefix):
            vals = [float(t) for t in ln.split()[2:]]
    return vals


@pytest.mark.parametrize("nv", [1, 4])
@pytest.mark.parametrize("name,prefix", [("example", "SOLV"), ("example_ir", "META")])
def test_reference_c_example_runs_and_converges(gpu, name, prefix, nv, tmp_path):
    exe = os.path.join(REF, "%s_nv%d" % (name, nv))
    if not os.path.exists(exe):
        pytest.skip("reference examples not built (oracle/build_ref_examples.py needs the reference tree)")
    env = dict(os.environ, XAMG_NV=str(nv))
    env.pop("XAMG_QUIET", None)
    r = subprocess.run([exe], cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=300)
    out = r.stdout
    assert r.returncode == 0, out[-2000:] + r.stderr[-2000:]
    parts = out.split("Solver time:")
    assert len(parts) == 3, out[-2000:]
    first, second = parts[0].splitlines(), parts[1].splitlines()
    last1 = _last_relres(first, prefix)
    last2 = _last_relres(second, prefix)
    assert last1 is not None and last2 is not None, out[-2000:]
    assert len(last2) == nv
    assert max(last1) <= 1e-6 * 1.0001
    assert max(last2) <= 1e-8 * 1.0001
