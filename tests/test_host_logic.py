"""Host-side logic of the Python mirror that needs no device: the mesh
built as Grid::init does, charges and masses as setup_env does, the
parameter file reader, and the seeded initial conditions."""
import numpy as np

import oracle
from aperture3_b200 import ic
from aperture3_b200.sim import SimEnvironment, SimParams


def test_mesh_matches_grid_init():
    p = SimParams(N=(1024, 1024, 1), guard=(2, 2, 0), size=(10.0, 10.0, 10.0))
    m = SimEnvironment._make_mesh(p)
    o = oracle.make_mesh(p.N, p.guard, size=p.size)
    for k in ("dims", "guard", "delta", "inv_delta", "lower", "sizes"):
        assert list(getattr(m, k)) == list(getattr(o, k)), k
    assert m.dimension == 2
    assert m.delta[0] == np.float32(10.0) / np.float32(1024)


def test_params_from_toml(tmp_path):
    cfg = tmp_path / "config.toml"
    cfg.write_text('delta_t = 0.0025\nq_e = 1000.0\nnum_species = 2\n'
                   'periodic_boundary = [true, true]\n[Grid]\nN = [64, 32, 1]\n'
                   'guard = [2, 2, 0]\n[Simulation]\ndata_interval = 10\nsort_interval = 20\n')
    p = SimParams.from_toml(str(cfg))
    assert p.N == [64, 32, 1] and p.guard == [2, 2, 0]
    assert p.q_e == 1000.0 and p.data_interval == 10 and p.periodic_boundary == [True, True]


def test_box2d_initial_state():
    params, fields, ptc = ic.box2d(seed=3, N=32, ppc=8)
    assert ptc["x1"].numel() == 32 * 32 * 8
    cells = ptc["cell"].numpy()
    assert np.all(np.diff(cells) >= 0)  # filled cell by cell
    assert np.array_equal(ptc["x1"][0::2], ptc["x1"][1::2])  # pairs share positions
    sp = (ptc["flag"].numpy() >> 29)
    assert np.array_equal(sp[0::2], np.zeros(len(sp) // 2)) and np.all(sp[1::2] == 1)
    g = ptc["E"].double()
    assert float(g.min()) >= 1.0 and float(g.max()) <= 1000.0 * 1.0001
    assert abs(float(fields["B"][2].mean()) - 1.0) < 0.05


def test_box1d_initial_state():
    params, fields, ptc = ic.box1d(seed=0, N=256, num_particles=4096)
    assert ptc["x1"].numel() == 4096
    assert abs(float(ptc["p1"].std()) - 0.1) < 0.01
    assert float(fields["B"][0].min()) == 1.0
