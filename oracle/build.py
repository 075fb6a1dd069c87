"""Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

Also builds oracle/_ref/libref_coeff.so from the reference's own coeff.cu when the
reference sources are present (see build_ref.sh). Neither library is product code.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "rbc_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "liboracle.so")


def build(force=False, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    if force or not os.path.exists(OUT) or os.path.getmtime(OUT) < os.path.getmtime(SRC):
        cmd = ["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-std=c++17",
               "-fPIC", "-shared", SRC, "-o", OUT]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    ref_script = os.path.join(HERE, "build_ref.sh")
    ref_out = os.path.join(HERE, "_ref", "libref_coeff.so")
    if os.path.exists(ref_script) and (force or not os.path.exists(ref_out)):
        subprocess.call(["sh", ref_script])
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
