"""Compile the reference's own loop files (src/blas/detail/blas.inl,
blas_ext.inl, blas_wrapper.inl, specific/blas_merged_jacobi.inl,
src/blas2/detail/csr_matvec.inl, csr_gs.inl, dense_matvec.inl,
src/primitives/matrix/operations/inverse.inl, src/misc/rand.h), its binary
system reader (src/io/detail/reader.inl) and its cube and channel-with-cube
generators (examples/common/generator/cube.inl, channel_with_cube.inl,
lame.inl) unchanged, where they lie under the reference tree (default
/root/reference, or $XAMG_REFERENCE_ROOT), into CPU libraries under
oracle/_ref/ that the tests use to check the oracle.  Nothing is copied: the
stand-in types of oracle/ref_loops/shim.h replace the reference's runtime
(MPI, shared memory, vector and matrix classes), and the loop files are read
through the include path.  Without the reference tree this step does nothing
and the tests that need the libraries skip.

Three libraries, the same entry points (oracle/ref_loops/ref_loops.h):
  libxamg_ref_loops_generic.so  every file with the reference's generic
      release flags (Make.inc/compilerflags.inc:34,47: -std=c++11 -O3
      -DNDEBUG); x86-64 without FMA, so every product and sum rounds apart;
  libxamg_ref_loops_haswell.so  every file with the instruction set of its
      Haswell machine configuration (compilerflags.inc:86, -march=haswell)
      and FP contraction (-ffp-contract=fast), without that configuration's
      -ffast-math (which lets the compiler reorder sums at will): a product
      feeding a sum becomes one fused multiply-add;
  libxamg_ref_loops_contract.so  the row loops (sparse and dense products,
      Gauss-Seidel, the Jacobi update) as in the Haswell build, the BLAS-1
      loops as in the generic build: the arithmetic contract the oracle and the GPU kernels
      follow (fused row sums, literal vector updates), assembled from the two.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ref_loops")
OUT = os.path.join(HERE, "_ref")
GENERIC = ["-std=c++11", "-O3", "-DNDEBUG", "-fPIC", "-w"]
HASWELL = GENERIC + ["-march=haswell", "-ffp-contract=fast"]
# The row loops mark their loop over a row's entries XAMG_NOVECTOR (Intel's
# "#pragma novector", src/xamg_macros.h:27-31); GCC 13 has no such pragma and
# the macro is empty there, so the row loops are compiled with GCC's loop
# vectoriser off to keep that intent.  The loops over a row's nv columns,
# which the reference does vectorise, are independent lanes: vectorising them
# changes no result.
HASWELL_ROWS = HASWELL + ["-fno-tree-vectorize"]
LIBS = {"generic": (GENERIC, GENERIC), "haswell": (HASWELL_ROWS, HASWELL), "contract": (HASWELL_ROWS, GENERIC)}


def reference_src():
    return os.path.join(os.environ.get("XAMG_REFERENCE_ROOT", "/root/reference"), "src")


def library(kind):
    return os.path.join(OUT, "libxamg_ref_loops_%s.so" % kind)


def build():
    from concurrent.futures import ThreadPoolExecutor

    ref = reference_src()
    if not os.path.isdir(os.path.join(ref, "blas2", "detail")):
        return []
    os.makedirs(OUT, exist_ok=True)
    deps = [os.path.join(d, f) for d in (SRC, os.path.join(SRC, "stub")) for f in sorted(os.listdir(d))
            if os.path.isfile(os.path.join(d, f))] + [os.path.abspath(__file__)]
    todo = {}
    for kind, (rows_flags, vec_flags) in LIBS.items():
        lib = library(kind)
        if os.path.exists(lib) and all(os.path.getmtime(lib) >= os.path.getmtime(d) for d in deps):
            continue
        todo[kind] = []
        for name, flags in (("rows", rows_flags), ("smooth", rows_flags), ("vec", vec_flags),
                            ("gen", GENERIC), ("io", GENERIC), ("cheb", vec_flags),
                            ("krylov", vec_flags), ("mg", rows_flags)):
            obj = os.path.join(OUT, "ref_%s_%s.o" % (name, kind))
            # XAMG renamed per unit: no template instance is shared between units;
            # ref_loops/stub comes first so that its xamg_types.h stands in
            todo[kind].append((obj, ["g++", *flags, "-DXAMG=XAMG_" + name, "-I", os.path.join(SRC, "stub"),
                                     "-I", SRC, "-I", ref, "-I", os.path.join(os.path.dirname(ref), "examples",
                                                                              "common"),
                                     "-c", os.path.join(SRC, name + ".cpp"), "-o", obj]))
    jobs = [cmd for units in todo.values() for _, cmd in units]
    with ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        for r in ex.map(lambda cmd: subprocess.run(cmd).returncode, jobs):
            if r != 0:
                raise RuntimeError("reference loop build failed")
    for kind, units in todo.items():
        objs = [o for o, _ in units]
        subprocess.run(["g++", "-shared", "-o", library(kind), *objs], check=True)
        for o in objs:
            os.remove(o)
    return [library(k) for k in LIBS]


if __name__ == "__main__":
    for b in build():
        sys.stdout.write(b + "\n")
