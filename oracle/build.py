"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/ifgf_oracle.cpp into oracle/_build/libifgf_oracle.so with g++
and OpenMP.  The product library never links or loads this file's output.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ifgf_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libifgf_oracle.so")

# x86-64-v3 (AVX2 + FMA) so the prebuilt library also runs on other hosts.
FLAGS = ["-O3", "-march=x86-64-v3", "-std=c++17", "-fopenmp", "-fPIC", "-shared"]


def build_oracle(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["g++", *FLAGS, SRC, "-o", LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force=True))
