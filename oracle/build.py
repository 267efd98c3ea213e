"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/fz_oracle.cpp, the FP64 restatement of the reference 3D update loop, and
oracle/fz_legacy2d_oracle.cpp, the restatement of the reference 2D legacy solver, into
oracle/liboracle.so. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("fz_oracle.cpp", "fz_legacy2d_oracle.cpp")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(s) for s in srcs):
        return LIB
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-shared", "-fPIC", "-std=c++17",
           *srcs, "-o", LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
