"""Build the reference's own C callers (examples/c/example.c and
example_ir.c) against this library's C API, unchanged, into oracle/_ref/.

The programs are the reference's sources read where they lie under the
reference tree (default /root/reference, or $XAMG_REFERENCE_ROOT); nothing is
copied.  They are compiled for XAMG_NV = 1 and 4 with gcc, against
include/xamg_c_api.h, and linked to xamg-test_b200/libxamg_b200.so with a
relative run path, so the binaries run wherever the repository is unpacked.
The GPU tests run them (tests/test_gpu_examples.py); without the reference
tree this step does nothing and those tests skip."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
NAMES = ("example", "example_ir")
NVS = (1, 4)


def ref_examples_dir():
    return os.path.join(os.environ.get("XAMG_REFERENCE_ROOT", "/root/reference"), "examples", "c")


def binary(name, nv):
    return os.path.join(OUT, "%s_nv%d" % (name, nv))


def build():
    src_dir = ref_examples_dir()
    if not os.path.isdir(src_dir):
        return []
    os.makedirs(OUT, exist_ok=True)
    libdir = os.path.join(ROOT, "xamg-test_b200")
    rel = os.path.relpath(libdir, OUT)
    built = []
    for name in NAMES:
        src = os.path.join(src_dir, name + ".c")
        for nv in NVS:
            exe = binary(name, nv)
            obj = exe + ".o"
            subprocess.run(["gcc", "-O1", "-DXAMG_NV=%d" % nv, "-I", os.path.join(ROOT, "include"), "-c", src,
                            "-o", obj], check=True)
            subprocess.run(["gcc", obj, "-L", libdir, "-lxamg_b200", "-Wl,-rpath,$ORIGIN/" + rel, "-lm", "-o", exe],
                           check=True)
            os.remove(obj)
            built.append(exe)
    return built


if __name__ == "__main__":
    for b in build():
        sys.stdout.write(b + "\n")
