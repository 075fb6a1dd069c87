"""Golden step fixtures from the reference's OWN FP64 step (tests/golden/ref_step_*.npz).

The reference's step, nonlinear operator and operator constructors are compiled from its
sources by oracle/build_ref_step.sh into oracle/_ref/ref_step (a driver that calls
implicit_explicit_step::step_time + make_real_signal per iteration, as
gpu_flow/code/main.cu:612-616 does, or nonlinear_operator_rayleigh_noslip::
calculate_operator once). It needs a GPU. Usage, on a machine with one:

    python tests/golden/make_ref_step_golden.py run <workdir>      # inputs, runs, fixtures

`run` writes every case's input state (seeded generators only: the oracle's seeded
theta, and tests.helpers.splitmix_state), runs ref_step on it and writes
<workdir>/ref_step_<case>.npz; copy those into tests/golden/. The fixtures hold no
inputs: the tests rebuild them from the same seeds. Per output they keep F and G whole,
per (field, vertical mode) the plane's sum of |c|^2 over all wavenumbers, and the
values at NSAMPLE seeded kept-band positions per field, or every kept-band value where
`full` is set.
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.helpers import kept_mask, splitmix64, splitmix_state  # noqa: E402

NSAMPLE = 512
# (nx, ny, L, lx, ly, ra, pr, dt)
C1 = (64, 64, 4, 8.0, 8.0, 2000.0, 1.0, 1e-3)
C2 = (256, 256, 8, 32.0, 32.0, 5000.0, 0.9, 5e-4)
C3 = (512, 512, 12, 64.0, 64.0, 6000.0, 1.0, 2.5e-4)

# name: (params, input, mode, step marks, marks stored in full)
#   input ("seeded", seed, amp, kmax) = the seeded theta of the workload configs;
#         ("splitmix", seed, amp, decay) = tests.helpers.splitmix_state
CASES = {
    "c1_seeded": (C1, ("seeded", 1, 1e-3, 4.0), "steps", (1, 10, 100, 1000), (1000,)),
    "c1_random": (C1, ("splitmix", 5, 0.05, 0.15), "steps", (20, 100), (100,)),
    "op_64x64x4": (C1, ("splitmix", 11, 1.0, 0.15), "operator", (), ("op",)),
    "op_64x64x8": ((64, 64, 8, 8.0, 8.0, 5000.0, 0.9, 5e-4), ("splitmix", 12, 1.0, 0.15), "operator", (), ()),
    "op_48x32x3": ((48, 32, 3, 12.0, 8.0, 2500.0, 0.7, 1e-3), ("splitmix", 13, 1.0, 0.15), "operator", (), ()),
    "c2_seeded": (C2, ("seeded", 2, 1e-3, 8.0), "steps", (20,), ()),
    "c2_random": (C2, ("splitmix", 21, 0.05, 0.08), "steps", (20,), ()),
    "op_512x512x12": (C3, ("splitmix", 31, 1.0, 0.05), "operator", (), ()),
}


def case_input(name):
    """The input state of a case: [theta, f, g, F, G] in the reference layout."""
    prm, inp = CASES[name][0], CASES[name][1]
    nx, ny, L = prm[:3]
    if inp[0] == "seeded":
        import oracle
        o = oracle.Oracle(*prm, threads=1)
        o.init_theta(inp[1], inp[2], inp[3])
        return o.get_state()
    return splitmix_state(nx, ny, L, seed=inp[1], amp=inp[2], decay=inp[3])


def sample_index(nx, ny, L, seed):
    """NSAMPLE distinct flat indices into [L][ny][nx/2+1] inside the kept band."""
    m = np.broadcast_to(kept_mask(nx, ny)[None], (L, ny, nx // 2 + 1)).ravel()
    cand = np.flatnonzero(m)
    order = np.argsort(splitmix64(seed, cand.size), kind="stable")
    return np.sort(cand[order[:min(NSAMPLE, cand.size)]])


def summarize(state, nx, ny, L, tag, full, seed):
    out = {}
    idx = sample_index(nx, ny, L, seed)
    m = kept_mask(nx, ny)
    for nm, a in zip(("theta", "f", "g"), state[:3]):
        out[f"{tag}_{nm}_norm2"] = (np.abs(a) ** 2).sum(axis=(1, 2))
        if full:
            out[f"{tag}_{nm}_kept"] = a[:, m]
        else:
            out[f"{tag}_{nm}_sample"] = a.ravel()[idx]
    out[f"{tag}_F"] = state[3]
    out[f"{tag}_G"] = state[4]
    return out


def write_bin(path, state):
    with open(path, "wb") as fp:
        for a in state:
            fp.write(np.ascontiguousarray(a, dtype="<c16").tobytes())


def read_bin(path, nx, ny, L):
    raw = np.fromfile(path, dtype="<c16")
    n = L * ny * (nx // 2 + 1)
    assert raw.size == 3 * n + 2 * L, path
    planes = [raw[i * n:(i + 1) * n].reshape(L, ny, nx // 2 + 1) for i in range(3)]
    return planes + [raw[3 * n:3 * n + L], raw[3 * n + L:]]


def run(workdir):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_step")
    if not os.path.exists(exe):
        raise SystemExit("oracle/_ref/ref_step is not built (sh oracle/build_ref_step.sh <reference root>)")
    os.makedirs(workdir, exist_ok=True)
    for name, (prm, inp, mode, marks, full) in CASES.items():
        nx, ny, L, lx, ly, ra, pr, dt = prm
        src = os.path.join(workdir, name + "_in.bin")
        write_bin(src, case_input(name))
        prefix = os.path.join(workdir, name)
        args = [exe, str(nx), str(ny), str(L), repr(lx), repr(ly), repr(ra), repr(pr), repr(dt), src, prefix]
        args += ["operator"] if mode == "operator" else ["steps", ",".join(str(m) for m in marks)]
        subprocess.run(args, check=True, timeout=1800)
        fx = {"params": np.array(prm, dtype=np.float64), "nsample": np.int64(NSAMPLE)}
        tags = ["op"] if mode == "operator" else [str(m) for m in marks]
        for i, tag in enumerate(tags):
            path = prefix + ("_op.bin" if mode == "operator" else f"_{tag}.bin")
            st = read_bin(path, nx, ny, L)
            key = "op" if mode == "operator" else int(tag)
            fx.update(summarize(st, nx, ny, L, f"s{tag}", key in full, seed=1000 + i))
        np.savez_compressed(os.path.join(workdir, f"ref_step_{name}.npz"), **fx)
        print("wrote", name, flush=True)


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] != "run":
        raise SystemExit(__doc__)
    run(sys.argv[2])
