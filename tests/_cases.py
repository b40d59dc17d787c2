"""Seeded random particle/field cases shared by the CPU and GPU tests."""
import numpy as np

import oracle

STAG = [(0, 1), (1, 0), (1, 1), (1, 0), (0, 1), (0, 0)]  # E1..E3, B1..B3 (x, y)


def empty_ptc(n):
    return {name: np.zeros(n, dt) for name, dt in oracle.PTC_FIELDS}


def random_particles(m, n, rng, gamma_max=20.0, edge_frac=0.2, species=(0, 1), ncells=None):
    """n particles in random bulk cells; a fraction sits exactly on or next to
    cell edges; momenta isotropic with gamma log-uniform in [1, gamma_max]."""
    p = empty_ptc(n)
    g0, g1 = m.guard[0], m.guard[1]
    c1 = rng.integers(g0, m.dims[0] - g0, n)
    if m.dimension > 1:
        c2 = rng.integers(g1, m.dims[1] - g1, n)
    else:
        c2 = np.zeros(n, np.int64)
    p["cell"][:] = (c1 + c2 * m.dims[0]).astype(np.uint32)
    for k in ("x1", "x2"):
        x = rng.random(n, dtype=np.float32)
        e = rng.random(n) < edge_frac
        choice = rng.integers(0, 4, n)
        edge_vals = np.array([0.0, np.nextafter(np.float32(1), np.float32(0)), 0.5,
                              np.float32(1e-7)], np.float32)
        x[e] = edge_vals[choice[e]]
        p[k][:] = x
    if m.dimension == 1:
        p["x2"][:] = rng.standard_normal(n).astype(np.float32)
    p["x3"][:] = rng.standard_normal(n).astype(np.float32)
    gamma = np.exp(rng.random(n) * np.log(gamma_max))
    pm = np.sqrt(np.maximum(gamma * gamma - 1.0, 0.0))
    ct = 2 * rng.random(n) - 1
    st = np.sqrt(1 - ct * ct)
    ph = 2 * np.pi * rng.random(n)
    p["p1"][:] = (pm * st * np.cos(ph)).astype(np.float32)
    p["p2"][:] = (pm * st * np.sin(ph)).astype(np.float32)
    p["p3"][:] = (pm * ct).astype(np.float32)
    p["E"][:] = np.sqrt(1 + p["p1"].astype(np.float64) ** 2 + p["p2"].astype(np.float64) ** 2
                        + p["p3"].astype(np.float64) ** 2).astype(np.float32)
    p["weight"][:] = (0.5 + rng.random(n)).astype(np.float32)
    sp = rng.choice(np.array(species), n)
    p["flag"][:] = (sp.astype(np.uint32) << np.uint32(29))
    p["id"][:] = np.arange(n, dtype=np.uint64)
    return p


def random_fields(m, rng, amp=0.5, num_species=2, bg=True):
    f = oracle.new_fields(m, num_species)
    for key in ("E", "B"):
        for c in range(3):
            f[key][c][:] = (amp * rng.standard_normal(f[key][c].shape)).astype(np.float32)
    if bg:
        for key in ("Ebg", "Bbg"):
            for c in range(3):
                f[key][c][:] = (0.1 * amp * rng.standard_normal(f[key][c].shape)).astype(np.float32)
    return f


def mesh_1d(N, guard=2, size=1.0):
    return oracle.make_mesh((N, 1, 1), (guard, 0, 0), size=(size, 1, 1))


def mesh_2d(N0, N1, guard=2, size=(1.0, 1.0)):
    return oracle.make_mesh((N0, N1, 1), (guard, guard, 0), size=(size[0], size[1], 1))


CHARGES = [-1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
MASSES = [1.0] * 8


# ---------------------------------------------------------------------------
# Log-spherical (ln r, theta) cases: r in [1, rmax], theta in [0, pi].

def mesh_logsph(N0, N1, guard=2, rmax=50.0):
    return oracle.make_mesh((N0, N1, 1), (guard, guard, 0),
                            size=(float(np.log(rmax)), float(np.pi), 1.0))


def _node_pos(m, dim, n, stagger):
    """Quadmesh::pos(dim, n, stagger) in float64 for the initial fields."""
    x = 1.0 if stagger else 0.5
    return m.lower[dim] + m.delta[dim] * (n - m.guard[dim] + x)


def logsph_fields(m, rng, omega=0.1, B0=1.0, noise=0.02, num_species=3):
    """Dipole background B_r = 2 B0 cos(theta) / r^3, B_theta = B0 sin(theta) / r^3
    and the corotation field E = -(Omega x r) x B of a rotating conductor,
    each sampled at its Yee stagger, plus seeded noise in E and B."""
    f = oracle.new_fields(m, num_species)
    i = np.arange(m.dims[0])[None, :]
    j = np.arange(m.dims[1])[:, None]
    for comp, (sx, sy) in enumerate(STAG[3:]):
        r = np.exp(_node_pos(m, 0, i, sx))
        th = _node_pos(m, 1, j, sy)
        br = 2 * B0 * np.cos(th) / r ** 3
        bt = B0 * np.sin(th) / r ** 3
        val = [br, bt, np.zeros_like(br)][comp]
        f["Bbg"][comp][:] = val.astype(np.float32)
    for comp, (sx, sy) in enumerate(STAG[:3]):
        r = np.exp(_node_pos(m, 0, i, sx))
        th = _node_pos(m, 1, j, sy)
        br = 2 * B0 * np.cos(th) / r ** 3
        bt = B0 * np.sin(th) / r ** 3
        v = omega * r * np.sin(th)
        val = [v * bt, -v * br, np.zeros_like(br)][comp]
        f["Ebg"][comp][:] = val.astype(np.float32)
    for c in range(3):
        f["E"][c][:] = f["Ebg"][c] + (noise * rng.standard_normal(f["E"][c].shape)).astype(np.float32)
        f["B"][c][:] = f["Bbg"][c] + (noise * rng.standard_normal(f["B"][c].shape)).astype(np.float32)
    return f


def logsph_particles(m, n, rng, gamma_max=1e3, species=(0, 1, 2)):
    p = random_particles(m, n, rng, gamma_max=gamma_max, species=species)
    p["x3"][:] = (np.pi * (2 * rng.random(n) - 1)).astype(np.float32)
    return p


def logsph_dt(m, frac=0.4):
    return np.float32(frac * min(m.delta[0], m.delta[1]))


LS_CHARGES = [-1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
LS_MASSES = [1.0, 1.0, 10.0, 1.0, 1.0, 1.0, 1.0, 1.0]


# ---------------------------------------------------------------------------
# 1D gap lab cases (ptc_updater_1dgap.cu): beta_phi(x) = x, so the grid's
# lower edge decides the sign of beta.

GAP_CHARGES = [-1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
GAP_MASSES = [1.0] * 8


def mesh_gap(N, lower=0.0, size=1.0, guard=2):
    return oracle.make_mesh((N, 1, 1), (guard, 0, 0), lower=(lower, 0.0, 0.0),
                            size=(size, 1.0, 1.0))


def gap_state(m, n, rng, pmax=50.0):
    """E1 / E3 / J fields and n particles in the bulk of a 1D gap grid:
    x1 uniform with a share on cell edges, p1 = +-pmax * u^3, E the gamma
    of p1 at the particle's beta, weights in [0.5, 1.5], e- / e+, a few
    with ignore_current."""
    nc = m.dims[0]
    x = np.arange(nc, dtype=np.float64)
    E1 = (0.8 * np.sin(2 * np.pi * x / nc) + 0.1 * rng.standard_normal(nc)).astype(np.float32)
    p = empty_ptc(n)
    g = m.guard[0]
    c = rng.integers(g, nc - g, n)
    p["cell"][:] = c.astype(np.uint32)
    x1 = rng.random(n, dtype=np.float32)
    e = rng.random(n) < 0.2
    edge = np.array([0.0, np.nextafter(np.float32(1), np.float32(0)), 0.5,
                     np.nextafter(np.float32(0.5), np.float32(0))], np.float32)
    x1[e] = edge[rng.integers(0, 4, n)[e]]
    p["x1"][:] = x1
    p["p1"][:] = (pmax * rng.uniform(-1, 1, n) ** 3).astype(np.float32)
    beta = (m.lower[0] + m.delta[0] * ((c - g).astype(np.float32) + x1)).astype(np.float32)
    p["E"][:] = np.sqrt(1.0 + p["p1"].astype(np.float64) ** 2 + beta.astype(np.float64) ** 2
                        ).astype(np.float32)
    p["weight"][:] = rng.uniform(0.5, 1.5, n).astype(np.float32)
    sp = rng.integers(0, 2, n).astype(np.uint32)
    p["flag"][:] = sp << 29
    ign = rng.random(n) < 0.05
    p["flag"][ign] |= np.uint32(1 << 3)
    p["id"][:] = np.arange(n, dtype=np.uint64)
    return E1, p


# ---------------------------------------------------------------------------
# 1D GR lab cases (labs/1dgr/config.toml grid: lower -6.273, size 6.138,
# guard 3; spin a = 0.99, field-line angular velocity 0.211765; q_e 1.2).

GR_A, GR_OMEGA = 0.99, 0.211765


def gr_table(n=600, rmin=1.15, rmax=14.0):
    """A synthetic field-line table (the reference reads one from coef.h5):
    B^3 / B^1 large enough near the horizon that u_0 is real in every cell."""
    a, om = GR_A, GR_OMEGA
    r = np.geomspace(rmin, rmax, n)
    theta = 0.3 + 0.2 / r
    Sigma = r * r + a * a * np.cos(theta) ** 2
    Delta = r * r - 2 * r + a * a
    A = (r * r + a * a) ** 2 - Delta * a * a * np.sin(theta) ** 2
    w = 2 * a * r / A
    g11, g33, al2 = Sigma / Delta, A * np.sin(theta) ** 2 / Sigma, Delta * Sigma / A
    b31 = 1.5 * np.sqrt(np.maximum(0.0, g11 * (g33 * (om - w) ** 2 - al2) / (g33 * al2))) + 0.1
    B1 = 1.0 / r ** 2
    tab = {"r": r, "B1": B1, "B3": b31 * B1, "jr": 0.5 / r ** 2, "rho": 0.2 / r ** 2,
           "theta": theta, "dpsidth": 0.5 * np.sin(theta)}
    return {k: v.astype(np.float32) for k, v in tab.items()}


def gr_mesh(N, guard=3):
    return oracle.make_mesh((N, 1, 1), (guard, 0, 0), lower=(-6.273, 0, 0), size=(6.138, 1, 1))


def gr_particles(m, co, n, rng, p_sigma=2.0, tracked_frac=0.1, ignore_frac=0.05):
    """n particles in bulk cells away from the ends, momenta N(0, p_sigma),
    u_0 = E consistent with p1 at each position (as the lab's initial
    condition sets it, ptc_updater_1dgr.cu:37-39)."""
    p = empty_ptc(n)
    g = m.guard[0]
    c = rng.integers(g + 2, m.dims[0] - g - 2, n)
    x1 = rng.random(n, dtype=np.float32)
    p["cell"][:] = c.astype(np.uint32)
    p["x1"][:] = x1
    p1 = (p_sigma * rng.standard_normal(n)).astype(np.float32)
    p["p1"][:] = p1
    nx = 1.0 - x1.astype(np.float64)
    it = lambda k: co[k][c] * x1 + co[k][c - 1] * nx  # noqa: E731
    D1, D2, D3, al = it(0), it(1), it(2), it(3)
    u0 = np.sqrt((D2 + p1.astype(np.float64) ** 2) / (D2 * (al * al - D3) + D1 * D1))
    p["E"][:] = u0.astype(np.float32)
    p["weight"][:] = (0.5 + rng.random(n)).astype(np.float32)
    sp = rng.integers(0, 2, n).astype(np.uint32)
    flag = sp << np.uint32(29)
    flag |= ((rng.random(n) < tracked_frac).astype(np.uint32) << np.uint32(1))  # tracked
    flag |= ((rng.random(n) < ignore_frac).astype(np.uint32) << np.uint32(3))  # ignore_current
    p["flag"][:] = flag
    p["id"][:] = np.arange(n, dtype=np.uint64)
    return p


def gr_dt(m, co, p):
    """A time step that moves the fastest particle half a cell."""
    c = p["cell"].astype(np.int64)
    D1, D2 = co[0][c], co[1][c]
    vr = np.abs((p["p1"] / p["E"] - D1) / D2).max()
    return float(np.float32(0.5 * m.delta[0] / max(vr, 1e-6)))


# ---------------------------------------------------------------------------
# Photons and pair production (radiative_transfer with the default and the
# pulsar lab's user functions).

def rad_photons(m, n, cap, rng, E_range=(2.5, 200.0), path_range=(-0.2, 1.0), holes=0.2,
                first_id=10_000_000):
    """cap photon slots, the first n in use: random bulk cells (a fifth of
    them holes), direction isotropic, energy log-uniform in E_range."""
    from oracle import rad
    ph = rad.new_photons(cap)
    g0, g1 = m.guard[0], m.guard[1]
    c1 = rng.integers(g0, m.dims[0] - g0, n)
    c2 = rng.integers(g1, m.dims[1] - g1, n) if m.dimension > 1 else np.zeros(n, np.int64)
    cell = (c1 + c2 * m.dims[0]).astype(np.uint32)
    cell[rng.random(n) < holes] = np.uint32(0xFFFFFFFF)
    ph["cell"][:n] = cell
    ph["x1"][:n] = rng.random(n, dtype=np.float32)
    ph["x2"][:n] = rng.random(n, dtype=np.float32)
    ph["x3"][:n] = (np.pi * (2 * rng.random(n) - 1)).astype(np.float32)
    E = np.exp(np.log(E_range[0]) + rng.random(n) * np.log(E_range[1] / E_range[0]))
    ct = 2 * rng.random(n) - 1
    st = np.sqrt(1 - ct * ct)
    phi = 2 * np.pi * rng.random(n)
    ph["p1"][:n] = (E * st * np.cos(phi)).astype(np.float32)
    ph["p2"][:n] = (E * st * np.sin(phi)).astype(np.float32)
    ph["p3"][:n] = (E * ct).astype(np.float32)
    ph["E"][:n] = E.astype(np.float32)
    ph["weight"][:n] = (0.5 + rng.random(n)).astype(np.float32)
    ph["path_left"][:n] = (path_range[0] + (path_range[1] - path_range[0]) * rng.random(n)
                           ).astype(np.float32)
    ph["id"][:n] = np.arange(first_id, first_id + n, dtype=np.uint64)
    return ph


def rad_rho(f, rng, frac_dense=0.3):
    """Charge densities with a multiplicity |rho0| + |rho1| over |rho0 + rho1|
    above 50 in about frac_dense of the cells."""
    shape = f["Rho"][0].shape
    a = rng.random(shape) + 0.1
    dense = rng.random(shape) < frac_dense
    f["Rho"][0][:] = (-a).astype(np.float32)
    f["Rho"][1][:] = np.where(dense, a * (1 + 1e-3), a * 3.0).astype(np.float32)


def gap_rad_case(ng, ne, n=6000, n_ph=6000, ic_path=0.004, seed=13):
    """The 1D gap lab's radiative transfer: a 512-cell gap grid with hot
    particles (gamma log-uniform in [2, 1e5]), photons of energy 10 .. 1e6,
    inverse-Compton tables of ng x ng entries and the oracle's parameters
    (model, tables, e_min 1e-3). Returns (mesh, params, tables holder,
    particles, photons, n, n_ph, capacity, photon capacity)."""
    from oracle import rad
    rng = np.random.default_rng(seed)
    m = oracle.make_mesh((512, 1, 1), (2, 0, 0), lower=(0.0, 0, 0), size=(1.0, 1, 1))
    cap, ph_cap = 4 * n + 1024, 3 * n_ph + 1024
    p = empty_ptc(cap)
    p["cell"][:n] = rng.integers(m.guard[0], m.dims[0] - m.guard[0], n).astype(np.uint32)
    p["cell"][n:] = oracle.MAX_CELL
    p["x1"][:n] = rng.random(n, dtype=np.float32)
    g = np.exp(np.log(2.0) + rng.random(n) * np.log(5e4))
    p["E"][:n] = g.astype(np.float32)
    p["p1"][:n] = (np.where(rng.random(n) < 0.5, -1, 1) * np.sqrt(g * g - 1)).astype(np.float32)
    p["weight"][:n] = (0.5 + rng.random(n)).astype(np.float32)
    p["flag"][:n] = (rng.integers(0, 2, n).astype(np.uint32) << np.uint32(29))
    p["id"][:n] = np.arange(n, dtype=np.uint64) + 31
    ph = rad.new_photons(ph_cap)
    ph["cell"][:n_ph] = rng.integers(m.guard[0], m.dims[0] - m.guard[0], n_ph).astype(np.uint32)
    ph["x1"][:n_ph] = rng.random(n_ph, dtype=np.float32)
    E = np.exp(np.log(10.0) + rng.random(n_ph) * np.log(1e5))
    ph["p1"][:n_ph] = (np.where(rng.random(n_ph) < 0.5, -1, 1) * E).astype(np.float32)
    ph["E"][:n_ph] = E.astype(np.float32)
    ph["weight"][:n_ph] = (0.5 + rng.random(n_ph)).astype(np.float32)
    ph["id"][:n_ph] = np.arange(n_ph, dtype=np.uint64) + 700_000
    tables = rad.IcTables(rad.gr1d_spectrum(1e-3), 1e-10, 0.1, 1.5e24 / ic_path, ng, ne)
    gap = rad.GapRad(tables)
    rp = rad.gap_rad_params(gap, 2e-3, e_min=1e-3, track_percent=0.3, seed=9)
    return m, rp, gap, p, ph, n, n_ph, cap, ph_cap
