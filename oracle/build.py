"""Build the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

The oracle is the checker for the CUDA product: only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs load it.  Built with g++ -O3 and OpenMP; the ISA level is x86-64-v3 so
that the same .so runs on the host cores of the GPU machine.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "liboracle.so")
SRCS = [os.path.join(HERE, "oracle_capi.cpp")]
DEPS = SRCS + [os.path.join(HERE, "mdref.hpp")]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in DEPS)


def build(force=False, march="x86-64-v3"):
    if not force and not needs_build():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-O3", f"-march={march}", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
           "-o", OUT + ".tmp"] + SRCS
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
