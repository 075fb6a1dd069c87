"""Generates tests/golden/coeff_L{4,8,12}.npz from the reference's own Galerkin
coefficient code (gpu_flow/code/util/coeff.cu), compiled by oracle/build_ref.sh into
oracle/_ref/libref_coeff.so. Run in a container where the reference sources exist:
    python tests/golden/make_golden.py
The tables are the reference's outputs for the getters the RBC step uses, in the
getter index order (i + j*L [+ k*L*L]).
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
NAMES2 = ["Iac", "Ia1", "Ia2"]
NAMES3 = ["Ibbb", "Ibb1", "Ib11", "I111", "Iabc", "Iac1", "Iaab", "Iaa1", "Iab2", "Ia12"]


def main():
    so = os.path.join(ROOT, "oracle", "_ref", "libref_coeff.so")
    if not os.path.exists(so):
        subprocess.check_call(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")])
    lib = ctypes.CDLL(so)
    lib.ref_coeff_table.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    for L in (4, 8, 12):
        tabs = {}
        for name in NAMES2 + NAMES3 + ["lambda"]:
            out = np.zeros(L ** 3)
            m = lib.ref_coeff_table(L, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            assert m > 0, name
            tabs[name] = out[:m]
        path = os.path.join(HERE, f"coeff_L{L}.npz")
        np.savez_compressed(path, **tabs)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    sys.exit(main())
