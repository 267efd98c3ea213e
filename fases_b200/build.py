"""Build recipe for libfz.so, the sm_100a stepper behind include/fz.h.

Compiles the CUDA kernels and the C++ host code in fases_b200/csrc/ with nvcc into
fases_b200/libfz.so (in-tree, so the library travels with the repository to the GPU host).
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfz.so")
# the same sources with -DFZ_BOUNDS_CHECK: every computed index of the stepping kernels is checked
CHECKED_LIB = os.path.join(HERE, "libfz_checked.so")
# the same sources with -DFZ_WAIT_TEST: bounded waits give up after about a millisecond, and a test
# hook (fz_test_skip_plane) makes the stage kernels skip one tile so that the wait for it runs out
WAIT_TEST_LIB = os.path.join(HERE, "libfz_waittest.so")
SOURCES = ["fz_kernels.cu", "fz_adjoint.cu", "fz_geometry.cu", "fz_api.cpp", "fz_project.cpp", "fz_group.cpp",
           "fz_adjoint.cpp", "fz_noalloc.cu", "fz_tune.cpp", "fz_legacy2d.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "fz.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, out: str = None, defines=()) -> str:
    out = out or LIB
    if not force and out == LIB and not _stale():
        return LIB
    cmd = ["nvcc", "-std=c++17", "-O3", *ARCH, "-lineinfo", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp", "-lgomp",
           "-I", os.path.join(HERE, "..", "include")]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += ["-D" + d for d in defines]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    cmd += ["-o", out]
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    import sys
    print(build(force=True, verbose="-v" in sys.argv))
