"""Generates the golden fixtures in this directory from the reference's own
kernels (src/cuda/algorithms/ptc_updater.cu push/deposit and
field_solver.cu e/b/divs), run on the host by oracle/ref_build.

Needs the reference tree (to build oracle/_ref/libapref.so). Run from the
repository root:  python tests/golden/make_golden.py
Each fixture holds seeded inputs (particles, E/B, backgrounds, J) and the
reference outputs: particles and J/Rho after push + deposit, and E/B/divE/
divB after one E update, one B update and compute_divs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from _cases import CHARGES, MASSES, mesh_1d, mesh_2d, random_fields, random_particles  # noqa: E402

CASES = [
    # name, kind, N, seed, particles, step, data_interval
    ("ref_1d_a", "1d", 512, 11, 600, 0, 1),
    ("ref_1d_b", "1d", 512, 12, 600, 4, 5),
    ("ref_2d_a", "2d", (32, 16), 21, 800, 0, 1),
    ("ref_2d_b", "2d", (64, 32), 22, 800, 3, 2),
    ("ref_2d_c", "2d", (32, 32), 23, 800, 1, 1),
]


def main():
    if oracle.load_ref(build=True) is None:
        raise SystemExit("reference pin library unavailable (needs the reference tree)")
    for name, kind, N, seed, n, step, di in CASES:
        rng = np.random.default_rng(seed)
        m = mesh_1d(N) if kind == "1d" else mesh_2d(*N)
        f = random_fields(m, rng)
        for c in range(3):
            f["J"][c][:] = rng.standard_normal(f["J"][c].shape).astype(np.float32)
        p = random_particles(m, n, rng)
        dt = np.float32(0.5 * m.delta[0])
        out = {}
        for k, v in oracle.mesh_dict(m).items():
            out["mesh_" + k] = np.asarray(v)
        out["dt"] = np.float32(dt)
        out["step"] = np.int64(step)
        out["data_interval"] = np.int64(di)
        for k in p:
            out["in_" + k] = p[k].copy()
        F = f["E"] + f["B"]
        for k in range(6):
            out[f"in_F{k}"] = F[k].copy()
        for k in range(3):
            out[f"in_Ebg{k}"] = f["Ebg"][k].copy()
            out[f"in_Bbg{k}"] = f["Bbg"][k].copy()
            out[f"in_J{k}"] = f["J"][k].copy()
        pr = oracle.copy_ptc(p)
        oracle.ref_push(m, pr, n, dt, F, CHARGES, MASSES)
        J = [np.zeros_like(F[0]) for _ in range(3)]
        R = [np.zeros_like(F[0]) for _ in range(2)]
        oracle.ref_deposit(m, pr, n, dt, step, di, J, R, CHARGES)
        for k in pr:
            out["out_" + k] = pr[k]
        for c in range(3):
            out[f"out_J{c}"] = J[c]
        for s in range(2):
            out[f"out_Rho{s}"] = R[s]
        fr = oracle.copy_fields(f)
        oracle.ref_update_e(m, fr, dt)
        oracle.ref_update_b(m, fr, dt)
        oracle.ref_compute_divs(m, fr)
        for k in range(3):
            out[f"fs_E{k}"] = fr["E"][k]
            out[f"fs_B{k}"] = fr["B"][k]
        out["fs_divE"] = fr["divE"]
        out["fs_divB"] = fr["divB"]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
