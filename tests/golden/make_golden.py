"""Generates the golden fixtures in this directory from the reference's own
kernels (src/cuda/algorithms/ptc_updater.cu push/deposit and
field_solver.cu e/b/divs; for logsph_*.npz the log-spherical
ptc_updater_logsph.cu / field_solver_logsph.cu kernels and
grid_log_sph.cpp coefficients), run on the host by oracle/ref_build.

Needs the reference tree (to build oracle/_ref/libapref.so). Run from the
repository root:  python tests/golden/make_golden.py [logsph | gap | gr | rad]
(gap_*.npz: the 1D gap lab's update_ptc_1dgap, ptc_updater_1dgap.cu;
gr_a.npz: the 1D GR lab's compute_coef and update_ptc_1dgr; rad_a.npz: the
pulsar lab's user radiative functions through emit_photons and
produce_pairs).
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
from oracle import logsph as ls  # noqa: E402
from _cases import (CHARGES, LS_CHARGES, LS_MASSES, MASSES, logsph_dt,  # noqa: E402
                    logsph_fields, logsph_particles, mesh_1d, mesh_2d, mesh_logsph,
                    random_fields, random_particles)

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

    main_logsph()


LS_CASES = [
    # name, N, seed, particles, params
    ("logsph_a", (64, 32), 31, 600, {}),
    ("logsph_b", (64, 32), 32, 600, {"gravity": 0.3, "rad_cooling_on": True,
                                     "rad_cooling_coef": 0.05, "compactness": 0.4}),
]


def main_logsph():
    """One push + deposit (step 0, data_interval 1) and one field update of
    the reference's log-spherical code on seeded dipole-field inputs."""
    if ls.load_ref(build=True) is None:
        raise SystemExit("reference pin library unavailable (needs the reference tree)")
    for name, N, seed, n, opts in LS_CASES:
        rng = np.random.default_rng(seed)
        m = mesh_logsph(*N)
        f = logsph_fields(m, rng)
        p = logsph_particles(m, n, rng, gamma_max=1e6)
        lp = ls.ls_params(**opts)
        dt = logsph_dt(m)
        out = {}
        for k, v in oracle.mesh_dict(m).items():
            out["mesh_" + k] = np.asarray(v)
        out["lp"] = np.array([lp.compactness, lp.omega, lp.gravity, lp.rad_cooling_coef,
                              lp.B0, lp.damping_coef, lp.rad_cooling_on, lp.damping_length],
                             np.float64)
        out["dt"] = np.float32(dt)
        c = ls.ref_coef(m)
        for k, cn in enumerate(ls.COEF_NAMES):
            out["coef_" + cn] = c[k]
        for k in p:
            out["in_p_" + k] = p[k].copy()
        for key in ("E", "B", "Ebg", "Bbg"):
            for k in range(3):
                out[f"in_{key}{k}"] = f[key][k].copy()
        ls.ref_push(m, lp, p, n, dt, f["E"] + f["B"], LS_CHARGES, LS_MASSES)
        J = [np.zeros_like(f["E"][0]) for _ in range(3)]
        R = [np.zeros_like(f["E"][0]) for _ in range(3)]
        ls.ref_deposit(m, lp, p, n, dt, 0, 1, J, R, c, LS_CHARGES)
        for k in p:
            out["out_p_" + k] = p[k]
        for k in range(3):
            out[f"out_J{k}"] = J[k]
            out[f"out_Rho{k}"] = R[k]
        f["J"] = J
        f["Rho"] = R
        ls.ref_update_fields(m, lp, f, c, dt)
        for key in ("E", "B"):
            for k in range(3):
                out[f"out_{key}{k}"] = f[key][k]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


def main_gap():
    """gap_*.npz: the 1D gap lab's update_ptc_1dgap (oracle/_ref/
    libapref_gap.so) on seeded particles and E3; outputs are the particles,
    J1 and Rho after one call."""
    from _cases import GAP_CHARGES, GAP_MASSES, gap_state, mesh_gap
    ref = oracle.load_ref_gap(build=True)
    if ref is None:
        raise SystemExit("gap pin library unavailable (needs the reference tree)")
    for name, N, lower, seed in [("gap_a", 256, 0.0, 31), ("gap_b", 300, -0.6, 32)]:
        rng = np.random.default_rng(seed)
        m = mesh_gap(N, lower)
        E3, p = gap_state(m, 500, rng)
        dt = np.float32(0.5 * m.delta[0])
        out = {}
        for k, v in oracle.mesh_dict(m).items():
            out["mesh_" + k] = np.asarray(v)
        out["dt"] = dt
        out["E3"] = E3.copy()
        for k in p:
            out["in_" + k] = p[k].copy()
        J = np.zeros(m.dims[0], np.float32)
        R = [np.zeros(m.dims[0], np.float32) for _ in range(2)]
        s_ = oracle.ptc_struct(p)
        ref.ref_gap_push_deposit(oracle.C.byref(m), oracle.C.byref(s_), len(p["x1"]), dt,
                                 oracle._p(E3), oracle._p(J), oracle._arr(R, 8), 2,
                                 oracle._fa(GAP_CHARGES), oracle._fa(GAP_MASSES))
        for k in p:
            out["out_" + k] = p[k]
        out["out_J1"] = J
        for sp in range(2):
            out[f"out_Rho{sp}"] = R[sp]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


def main_gr():
    """gr_a.npz: the 1D GR lab's Grid_1dGR::compute_coef and
    update_ptc_1dgr (oracle/_ref/libapref_gr.so) on a synthetic field-line
    table and seeded particles (tracked ones included, output step);
    outputs are the coefficients, the particles, J1 and Rho after one call."""
    from _cases import GR_A, GR_OMEGA, gr_dt, gr_mesh, gr_particles, gr_table
    ref = oracle.load_ref_gr(build=True)
    if ref is None:
        raise SystemExit("GR pin library unavailable (needs the reference tree)")
    N, B0, seed, step = 384, 2.0, 41, 8
    m = gr_mesh(N)
    tab = gr_table(n=200)
    cols = [np.ascontiguousarray(tab[k], np.float32) for k in oracle.GR_TABLE_KEYS]
    co = [np.zeros(m.dims[0], np.float32) for _ in range(oracle.GR_NCOEF)]
    ref.ref_gr_coef(oracle.C.byref(m), np.float32(GR_A), np.float32(GR_OMEGA), np.float32(B0),
                    *[oracle._p(c) for c in cols], len(cols[0]), oracle._arr(co, 15))
    rng = np.random.default_rng(seed)
    p = gr_particles(m, co, 700, rng)
    dt = np.float32(gr_dt(m, co, p))
    E3 = (0.05 * np.sin(0.013 * np.arange(m.dims[0]))).astype(np.float32)
    out = {"N": np.int64(N), "B0": np.float32(B0), "dt": dt, "step": np.int64(step),
           "E3": E3, "coef": np.stack(co)}
    for k in oracle.GR_TABLE_KEYS:
        out["tab_" + k] = tab[k]
    for k in p:
        out["in_" + k] = p[k].copy()
    charges, masses = [-1.2, 1.2] + [1.2] * 6, [1.2] * 8
    J = np.zeros(m.dims[0], np.float32)
    R = [np.zeros(m.dims[0], np.float32) for _ in range(2)]
    ref.ref_gr_push(oracle.C.byref(m), oracle.C.byref(oracle.ptc_struct(p)), len(p["x1"]), dt,
                    step, 4, np.float32(GR_A), np.float32(GR_OMEGA), oracle._p(E3),
                    oracle._arr(co, 15), oracle._p(J), oracle._arr(R, 8), 2,
                    oracle._fa(charges), oracle._fa(masses))
    for k in p:
        out["out_" + k] = p[k]
    out["J1"] = J
    out["Rho"] = np.stack(R)
    path = os.path.join(HERE, "gr_a.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


def main_rad():
    """rad_a.npz: the pulsar lab's check_emit_photon / emit_photon and
    check_produce_pair / produce_pair (oracle/_ref/libapref_rad.so, run by
    the pin driver with the build's draws) on a small seeded log-spherical
    state: inputs are the particles, photons and B / Rho fields; outputs the
    particles and photons after emit_photons, then after produce_pairs."""
    from oracle import rad
    from _cases import logsph_fields, logsph_particles, mesh_logsph, rad_photons, rad_rho
    if rad.load_ref(build=True) is None:
        raise SystemExit("radiation pin library unavailable (needs the reference tree)")
    seed, N, n, ph_n = 12, 40, 1000, 500
    m = mesh_logsph(N, N, rmax=8.0)
    rng = np.random.default_rng(seed)
    f = logsph_fields(m, rng, omega=0.1, noise=0.0, num_species=2)
    rad_rho(f, rng)
    p = logsph_particles(m, n, rng, gamma_max=3e4)
    ph = rad_photons(m, ph_n, 3 * ph_n, rng, E_range=(2.5, 500.0))
    rp = rad.rad_params(rad.RAD_PULSAR, delta_t=0.01, e_curv=2e-8, l_curv=2.0, BQ=0.05,
                        omega=0.1, r_cutoff=6.0, track_percent=0.3, seed=77)
    out = {"N": np.int64(N), "ph_num": np.int64(ph_n), "ph_cap": np.int64(ph["x1"].size),
           "B": np.stack(f["B"]), "Rho": np.stack(f["Rho"])}
    for k in p:
        out["in_ptc_" + k] = p[k].copy()
    for k in ph:
        out["in_ph_" + k] = ph[k][:ph_n].copy()
    no, _ = rad.ref_emit_photons(m, rp, p, n, ph, ph_n, ph["x1"].size, f, None, 4, 700)
    for k in ("p1", "p2", "p3", "E"):
        out["emit_ptc_" + k] = p[k].copy()
    for k in ph:
        out["emit_ph_" + k] = ph[k][:no].copy()
    cap = n + 2 * no + 60
    big = {k: np.concatenate([v, np.zeros(cap - n, v.dtype)]) for k, v in p.items()}
    big["cell"][n:] = oracle.MAX_CELL
    nb, _ = rad.ref_produce_pairs(m, rp, ph, no, big, n, cap, f, None, 4, 123_456)
    out["pairs_ph_cell"] = ph["cell"][:no].copy()
    for k in big:
        out["pairs_ptc_" + k] = big[k][n:nb].copy()
    path = os.path.join(HERE, "rad_a.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "logsph":
        main_logsph()
    elif len(sys.argv) > 1 and sys.argv[1] == "gap":
        main_gap()
    elif len(sys.argv) > 1 and sys.argv[1] == "gr":
        main_gr()
    elif len(sys.argv) > 1 and sys.argv[1] == "rad":
        main_rad()
    else:
        main()
