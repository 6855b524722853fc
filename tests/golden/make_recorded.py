"""Write recorded.json: the reference's own recorded test values.

Source: examples/test/out.yml:1-21 of the reference (MultiGrid solve of the
analytic 2-D problem of examples/test/generate.hpp:188-286, n = 100, NV = 1,
4 MPI ranks, hypre hierarchy).  Y_norm is ||b||_2 (tst_output.h:54-64), which
depends only on the generator and is reproduced here to rounding; X_norm is
the norm of the converged solution (rel. residual 9.39e-9), reproduced to the
solve tolerance.
"""
import json
import os

REC = {
    "source": "examples/test/out.yml:1-21",
    "problem": "examples/test/generate.hpp:188-286, n=100",
    "nrows": 10201,
    "nonzeros": 49405,
    "Y_norm": 10.000029834533674,
    "X_norm": 50.500156445526947,
    "initial_residual": 10.000029834533674,
    "rel_residual": 9.3910715945348913e-09,
    "fixture_n5": {"file": "mtx_Paus_n5.bin", "nrows": 36, "nonzeros": 100},
}

if __name__ == "__main__":
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "recorded.json"), "w") as f:
        json.dump(REC, f, indent=1)
