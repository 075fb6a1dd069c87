"""Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

Also builds, when the reference sources are present, oracle/_ref/libref_coeff.so from the
reference's own coeff.cu (build_ref.sh) and oracle/_ref/ref_step, the reference's own FP64
step (build_ref_step.sh). None of these is product code.
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
    root = reference_root()
    if root:
        for script, out in (("build_ref.sh", "libref_coeff.so"), ("build_ref_step.sh", "ref_step")):
            if force or not os.path.exists(os.path.join(HERE, "_ref", out)):
                subprocess.call(["sh", os.path.join(HERE, script), root])
    return OUT


def reference_root():
    """The reference project's root for the checker builds in oracle/_ref: SDC_REFERENCE,
    else the reference's usual read-only mount when present (None where there is no copy
    of the reference: the prebuilt files are used there)."""
    for r in (os.environ.get("SDC_REFERENCE"), "/root/reference"):
        if r and os.path.isdir(os.path.join(r, "gpu_flow", "code")):
            return r
    return None


if __name__ == "__main__":
    print(build(force=True, verbose=True))
