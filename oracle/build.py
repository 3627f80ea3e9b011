"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/tg_oracle.cpp into oracle/libtg_oracle.so with IEEE arithmetic
(no fast-math, no fused multiply-add contraction) and OpenMP.  The reference's
own CUDA build cannot be produced on these machines (its sources include GLM
headers from an empty git submodule), so there is no oracle/_ref build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "tg_oracle.cpp")
OUT = os.path.join(HERE, "libtg_oracle.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    cmd = [
        "g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
        "-ffp-contract=off", "-fno-fast-math", "-fvisibility=hidden",
        SRC, "-o", OUT + ".tmp",
    ]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
