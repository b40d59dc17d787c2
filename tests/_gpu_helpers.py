"""Shared setup for the GPU parity tests: one simulation on the device
through the C ABI and the same state in the CPU oracle."""
import numpy as np

import oracle
from aperture3_b200 import SimData, SimEnvironment, SimParams, field_solver, ptc_updater

BITS = {np.dtype(np.float32): np.uint32, np.dtype(np.float64): np.uint64}


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        return np.array_equal(a.view(BITS[a.dtype]), b.view(BITS[b.dtype]))
    return np.array_equal(a, b)


def assert_bits(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if not bits_equal(a, b):
        if a.dtype.kind == "f":
            bad = np.flatnonzero(a.view(BITS[a.dtype]).ravel() != b.view(BITS[b.dtype]).ravel())
        else:
            bad = np.flatnonzero(a.ravel() != b.ravel())
        raise AssertionError(f"{what}: {bad.size} of {a.size} differ; first {bad[:4]}: "
                             f"{a.ravel()[bad[:4]]} vs {b.ravel()[bad[:4]]}")


def make_params(N, guard=2, periodic=(True, True), data_interval=1, tile=(0, 0), smoothing=0,
                capacity=100, size=None):
    N = list(N) + [1] * (3 - len(N))
    dim = 1 if N[1] == 1 else 2
    g = (guard, guard if dim > 1 else 0, 0)
    size = size or (1.0, 1.0 if dim > 1 else 1.0, 1.0)
    dt = float(np.float32(0.5 * np.float32(size[0]) / np.float32(N[0])))
    return SimParams(N=tuple(N), guard=g, size=tuple(size), delta_t=dt, q_e=1.0, num_species=2,
                     periodic_boundary=(periodic[0], periodic[1] if dim > 1 else False, False),
                     data_interval=data_interval, current_smoothing=smoothing,
                     max_ptc_number=capacity, tile_size=(tile[0], tile[1], 0))


class Pair:
    """The same simulation state on the GPU (env/data) and in the oracle."""

    def __init__(self, params: SimParams, fields, ptc, capacity=None, row_align=4):
        self.params = params
        self.env = SimEnvironment(params)
        self.data = SimData(self.env, capacity=capacity or max(len(ptc["x1"]), 1),
                            row_align=row_align)
        self.m = oracle.make_mesh(params.N, params.guard, params.lower, params.size)
        self.f = oracle.new_fields(self.m, params.num_species)
        for key in ("E", "B", "Ebg", "Bbg", "J"):
            if key in fields:
                for c in range(3):
                    self.f[key][c][:] = fields[key][c]
        self.data.set_fields(self.f)
        self.p = oracle.copy_ptc(ptc)
        self.data.set_particles(self.p)
        self.pusher = ptc_updater(self.env)
        self.solver = field_solver(self.env)
        self.dt = params.delta_t
        self.J64 = None

    @property
    def periodic(self):
        return self.env.periodic

    def oracle_update_particles(self):
        """ptc_updater::update_particles in the oracle, with FP64 J/Rho
        accumulation; returns (lost,) and leaves J64/R64 on self."""
        m, p, f = self.m, self.p, self.f
        n = len(p["x1"])
        dtf = np.float32(self.dt)
        F = f["E"] + f["B"]
        oracle.push(m, p, n, dtf, F, self.env.charges, self.env.masses)
        shape = f["J"][0].shape
        J64 = [np.zeros(shape) for _ in range(3)]
        R64 = [np.zeros(shape) for _ in range(self.params.num_species)]
        oracle.deposit(m, p, n, dtf, self.step, self.params.data_interval, J64, R64,
                       self.env.charges, f64=True)
        for a in J64 + R64:
            oracle.send_add_guard_cells(m, a, self.periodic)
        lost = oracle.wrap_particles(m, p, n, self.periodic)
        self.J64, self.R64 = J64, R64
        for c in range(3):
            f["J"][c][:] = J64[c].astype(np.float32)
        return lost

    step = 0

    def both_update_particles(self, step):
        self.step = step
        self.pusher.update_particles(self.data, self.dt, step)
        return self.oracle_update_particles()

    def both_update_fields(self, step):
        self.solver.update_fields(self.data, self.dt, step)
        oracle.update_fields(self.m, self.f, self.dt, step, self.periodic)

    def check_particles(self, keys=("p1", "p2", "p3", "E", "x1", "x2", "x3", "cell", "weight",
                                    "flag", "id")):
        got = self.data.particles_host()
        for k in keys:
            assert_bits(got[k], self.p[k], f"particles.{k}")
        return got

    def check_current(self, rel=1e-6, rho=False):
        g = self.data.fields_host()
        out = {}
        for c in range(3):
            ref = self.J64[c]
            scale = max(np.abs(ref).max(), 1e-30)
            err = np.abs(g["J"][c].astype(np.float64) - ref).max() / scale
            assert err <= rel, f"J{c + 1}: {err:.3g} of max|J|"
            out[f"J{c + 1}"] = err
        if rho:
            for s in range(self.params.num_species):
                ref = self.R64[s]
                scale = max(np.abs(ref).max(), 1e-30)
                err = np.abs(g["Rho"][s].astype(np.float64) - ref).max() / scale
                assert err <= rel, f"Rho{s}: {err:.3g} of max|rho|"
                out[f"Rho{s}"] = err
        return out
