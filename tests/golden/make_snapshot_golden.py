"""Generates tests/golden/snapshot_00030000.npz from the reference's own FP32 state
snapshots (gpu_flow/data/{theta,f,g,F,G}_00030000.bin, written by
matrix_folder_writer::write_binary_file, gpu_flow/code/output/matrix_folder_writer.cu:3-101).
Run where the reference exists:
    python tests/golden/make_snapshot_golden.py <reference root>
The fixture keeps, per file, the header words, the file size and its SHA-256, and for
theta the complete kx = 0 column of both vertical planes (raw FP32 pairs), which is
enough to rebuild a file of the same header and size and to check the Hermitian
symmetry that make_real leaves in a saved state.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["theta", "f", "g", "F", "G"]


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_snapshot_golden.py <reference root>")
    root = sys.argv[1]
    data = os.path.join(root, "gpu_flow", "data")
    out = {}
    for n in NAMES:
        raw = open(os.path.join(data, f"{n}_00030000.bin"), "rb").read()
        nmat, ndim = np.frombuffer(raw[:8], "<i4")
        dims = np.frombuffer(raw[8:8 + 4 * ndim], "<i4")
        out[f"{n}_header"] = np.frombuffer(raw[:8 + 4 * ndim], "<i4").copy()
        out[f"{n}_size"] = np.int64(len(raw))
        out[f"{n}_sha256"] = np.frombuffer(hashlib.sha256(raw).digest(), np.uint8).copy()
        if n == "theta":
            mox, ny, L = (int(d) for d in dims)
            vals = np.frombuffer(raw[8 + 4 * ndim:], "<f4").reshape(L, ny, mox, 2)
            out["theta_col0"] = vals[:, :, 0, :].copy()          # [L][Ny][re, im]
        if n == "F":
            out["F_values"] = np.frombuffer(raw[8 + 4 * ndim:], "<f4").copy()
    np.savez_compressed(os.path.join(HERE, "snapshot_00030000.npz"), **out)


if __name__ == "__main__":
    main()
