"""Host-side mirror of the reference's lab-facing interface.

Same class and method names as the reference's algorithm classes and the
parts of sim_environment / sim_data they use (src/algorithms/ptc_updater.h,
field_solver.h, src/sim_environment.h, src/sim_data.h), without MPI: one
rank, one GPU, periodic exchange done by device kernels. Every operation
goes through libaperture_b200.so; device memory comes from torch.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import (AP_MAX_CELL, AP_MAX_SPECIES, ApArray, ApDiag, ApFields, ApLogsphParams,
                   ApMesh, ApParams, ApParticles, ApPhotons, ApRadCounts, ApRadParams,
                   ApStepStats, check)

PTC_FIELDS = (
    ("x1", torch.float32), ("x2", torch.float32), ("x3", torch.float32),
    ("p1", torch.float32), ("p2", torch.float32), ("p3", torch.float32),
    ("E", torch.float32), ("weight", torch.float32),
    ("cell", torch.int32), ("id", torch.int64), ("flag", torch.int32),
)
NP_DTYPES = {"cell": np.uint32, "id": np.uint64, "flag": np.uint32}
# photon_data (src/data/particle_data.h:68-80)
PH_FIELDS = (
    ("x1", torch.float32), ("x2", torch.float32), ("x3", torch.float32),
    ("p1", torch.float32), ("p2", torch.float32), ("p3", torch.float32),
    ("E", torch.float32), ("weight", torch.float32), ("path_left", torch.float32),
    ("cell", torch.int32), ("id", torch.int64), ("flag", torch.int32),
)

ELECTRON, POSITRON, ION = 0, 1, 2
FLAG_IGNORE_CURRENT = 1 << 3
FLAG_IGNORE_EM = 1 << 4


def species_flag(sp: int) -> int:
    """gen_ptc_type_flag (src/utils/util_functions.h:71-74)."""
    return (sp & 7) << 29


@dataclasses.dataclass
class SimParams:
    """The SimParams fields the particle update uses (src/sim_params.h:17-123),
    with the reference's key names."""
    N: Sequence[int] = (1, 1, 1)
    guard: Sequence[int] = (0, 0, 0)
    lower: Sequence[float] = (0.0, 0.0, 0.0)
    size: Sequence[float] = (1.0, 1.0, 1.0)
    delta_t: float = 0.01
    q_e: float = 1.0
    ion_mass: float = 1.0
    num_species: int = 2
    periodic_boundary: Sequence[bool] = (False, False, False)
    data_interval: int = 100
    current_smoothing: int = 0
    sort_interval: int = 20
    max_ptc_number: int = 100
    B0: float = 1.0
    max_steps: int = 0
    tile_size: Sequence[int] = (0, 0, 0)
    chunk: int = 0
    # log-spherical grids (coord_system "LogSpherical"; src/sim_params.h:31-48)
    coord_system: str = "Cartesian"
    compactness: float = 0.5
    omega: float = 0.2
    gravity: float = 0.0
    rad_cooling_on: bool = False
    rad_cooling_coef: float = 1.0
    damping_length: int = 30
    damping_coef: float = 0.002
    # 1D GR lab (coord_system "1DGR"): black hole spin (src/sim_params.h:63)
    a: float = 0.0
    # photons and pair production (src/sim_params.h:23, 50-88); rad_model
    # selects the user radiative functions: "default" (src/cuda/radiation/
    # user_radiative_functions.cu), "pulsar" (the pulsar lab's), "gr1d" (the
    # 1D GR lab's) or "gap1d" (the 1D gap lab's), the last two with the
    # inverse-Compton tables of e_min, ic_path, n_gamma, n_ep; rad_seed keys
    # the counter-based random stream that replaces cuRAND
    max_photon_number: int = 100
    create_pairs: bool = False
    gamma_thr: float = 20.0
    track_percent: float = 0.2
    BQ: float = 1.0
    photon_path: float = 1.0
    E_secondary: float = 4.0
    r_cutoff: float = 4.0
    l_curv: float = 6.0
    e_curv: float = 6.4e-9
    e_min: float = 1.0e-3
    ic_path: float = 1.0
    n_gamma: int = 600
    n_ep: int = 600
    rad_model: str = "default"
    rad_seed: int = 1

    @classmethod
    def from_toml(cls, path: str) -> "SimParams":
        """parse_config (src/sim_params.cpp:34-219) for the keys above."""
        import tomllib
        with open(path, "rb") as f:
            d = tomllib.load(f)
        p = cls()
        flat = dict(d)
        flat.update(d.get("Grid", {}))
        flat.update(d.get("Simulation", {}))
        for k in dataclasses.fields(cls):
            if k.name in flat:
                setattr(p, k.name, flat[k.name])
        return p


def _pad3(v, fill):
    v = list(v) + [fill] * (3 - len(v))
    return v[:3]


class SimEnvironment:
    """sim_environment (src/sim_environment.h) for one rank."""

    def __init__(self, params: SimParams, device: Optional[int] = None,
                 gr_table: Optional[Dict[str, np.ndarray]] = None):
        """gr_table (1D GR lab only): the tabulated field-line data the
        reference reads from coef.h5 -- arrays r, B1, B3, jr, rho, theta and
        dpsidth of equal length, r increasing."""
        self.params = params
        if device is not None:
            torch.cuda.set_device(device)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.mesh = self._make_mesh(params)
        # setup_env (sim_environment_impl.hpp:90-101)
        q = np.float32(params.q_e)
        self.charges = [float(q)] * AP_MAX_SPECIES
        self.masses = [float(q)] * AP_MAX_SPECIES
        self.charges[ELECTRON] = float(-q)
        self.masses[ION] = float(np.float32(q * np.float32(params.ion_mass)))
        self.periodic = [int(bool(x)) for x in _pad3(params.periodic_boundary, False)]
        ap = ApParams()
        ap.num_species = int(params.num_species)
        ap.data_interval = int(params.data_interval)
        ap.current_smoothing = int(params.current_smoothing)
        for i in range(3):
            ap.periodic[i] = self.periodic[i]
        for i in range(AP_MAX_SPECIES):
            ap.charges[i] = self.charges[i]
            ap.masses[i] = self.masses[i]
        ts = _pad3(params.tile_size, 0)
        ap.tile[0], ap.tile[1] = int(ts[0]), int(ts[1])
        ap.chunk = int(params.chunk)
        self.ap_params = ap
        self._lib = _lib.lib()
        ctx = C.c_void_p()
        self.logsph = str(params.coord_system).lower() in ("logspherical", "logsph", "log_sph")
        self.gap = str(params.coord_system).lower() in ("1dgap", "gap")
        self.gr = str(params.coord_system).lower() in ("1dgr", "gr")
        if self.gr:
            if gr_table is None:
                raise ValueError("a 1D GR environment needs gr_table")
            cols = [np.ascontiguousarray(gr_table[k], dtype=np.float32)
                    for k in _lib.GR_TABLE_KEYS]
            if len({len(c) for c in cols}) != 1:
                raise ValueError("gr_table arrays differ in length")
            self._gr_cols = cols  # kept alive for the call
            tab = _lib.ApGrTable(*[c.ctypes.data for c in cols], len(cols[0]))
            gp = _lib.ApGrParams(float(params.a), float(params.omega), float(params.B0))
            check(self._lib.ap_ctx_create_1dgr(C.byref(self.mesh), C.byref(ap), C.byref(gp),
                                               C.byref(tab), C.byref(ctx)), "ap_ctx_create_1dgr")
        elif self.gap:
            gp = _lib.ApGapParams(float(params.B0))
            check(self._lib.ap_ctx_create_1dgap(C.byref(self.mesh), C.byref(ap), C.byref(gp),
                                                C.byref(ctx)), "ap_ctx_create_1dgap")
        elif self.logsph:
            lp = ApLogsphParams(float(params.compactness), float(params.omega),
                                float(params.gravity), float(params.rad_cooling_coef),
                                float(params.B0), float(params.damping_coef),
                                int(bool(params.rad_cooling_on)), int(params.damping_length))
            self.ls_params = lp
            check(self._lib.ap_ctx_create_logsph(C.byref(self.mesh), C.byref(ap), C.byref(lp),
                                                 C.byref(ctx)), "ap_ctx_create_logsph")
        else:
            check(self._lib.ap_ctx_create(C.byref(self.mesh), C.byref(ap), C.byref(ctx)),
                  "ap_ctx_create")
        self.ctx = ctx

    @staticmethod
    def _make_mesh(p: SimParams) -> ApMesh:
        """Grid::init (src/core/grid.cpp:31-48)."""
        N = _pad3(p.N, 1)
        g = _pad3(p.guard, 0)
        lo = _pad3(p.lower, 0.0)
        sz = _pad3(p.size, 1.0)
        m = ApMesh()
        for i in range(3):
            m.guard[i] = int(g[i])
            m.dims[i] = int(N[i]) + 2 * int(g[i])
            m.lower[i] = float(np.float32(lo[i]))
            m.sizes[i] = float(np.float32(sz[i]))
            d = np.float32(np.float32(sz[i]) / np.float32(N[i]))
            m.delta[i] = float(d)
            m.inv_delta[i] = float(np.float32(1.0 / np.float64(d)))
        if m.dims[1] <= 1 and m.dims[2] <= 1:
            m.dimension = 1
        elif m.dims[2] <= 1:
            m.dimension = 2
        else:
            m.dimension = 3
        return m

    @property
    def dims(self):
        return [self.mesh.dims[i] for i in range(3)]

    def dim(self):
        return self.mesh.dimension

    def set_stream(self, stream: torch.cuda.Stream):
        check(self._lib.ap_set_stream(self.ctx, C.c_void_p(stream.cuda_stream)), "ap_set_stream")

    def set_sync(self, sync: bool):
        check(self._lib.ap_set_sync(self.ctx, int(sync)), "ap_set_sync")

    def sync(self):
        check(self._lib.ap_sync(self.ctx), "ap_sync")

    def send_guard_cells(self, field):
        """send_guard_cells for a scalar array or a list of components."""
        for a in (field if isinstance(field, (list, tuple)) else [field]):
            check(self._lib.ap_send_guard_cells(self.ctx, array_view(a)), "ap_send_guard_cells")

    def send_add_guard_cells(self, field):
        for a in (field if isinstance(field, (list, tuple)) else [field]):
            check(self._lib.ap_send_add_guard_cells(self.ctx, array_view(a)),
                  "ap_send_add_guard_cells")

    def set_pair_params(self, gamma_thr: float = 1e6, free_path: float = 0.05,
                        pair_energy: float = 50.0, seed: int = 0, first_id: int = 1 << 40,
                        enabled: bool = True):
        """Pair injection of this run (ap_pair_params)."""
        pp = _lib.ApPairParams(float(gamma_thr), float(free_path), float(pair_energy),
                               int(bool(enabled)), int(seed), int(first_id))
        check(self._lib.ap_set_pair_params(self.ctx, C.byref(pp)), "ap_set_pair_params")

    def set_compaction(self, interval: int):
        """Rewrite the 2D particle store in tile order every `interval`
        updates (0: never). Particles change slots, not values."""
        check(self._lib.ap_set_compaction(self.ctx, int(interval)), "ap_set_compaction")

    def set_tile_shape(self, tx: int, ty: int):
        """Tile shape of the 2D particle update (16x16, 32x16, 16x8, 8x8 or
        4x4); the tile order is rebuilt at the next update."""
        check(self._lib.ap_set_tile_shape(self.ctx, int(tx), int(ty)), "ap_set_tile_shape")

    def set_continuity_check(self, on: bool = True):
        """Record max |rho(t+1) - rho(t) + div J| (FP64, on the device) on
        every update with charge output that follows one; read it from
        SimData.diagnostics().continuity_residual (NaN when not recorded)."""
        check(self._lib.ap_set_continuity_check(self.ctx, int(bool(on))),
              "ap_set_continuity_check")

    def logsph_coef(self, which: int) -> np.ndarray:
        """Host copy of one Grid_LogSph coefficient array (grid_log_sph.h:45-47),
        shape (dims[1], dims[0])."""
        a = ApArray()
        check(self._lib.ap_logsph_coef(self.ctx, int(which), C.byref(a)), "ap_logsph_coef")
        d0, d1 = self.mesh.dims[0], self.mesh.dims[1]
        rows = device_to_host(a.ptr, a.pitch * d1).view(np.float32).reshape(d1, -1)
        return rows[:, :d0].copy()

    def gr_coef(self, which) -> np.ndarray:
        """Host copy of one Grid_1dGR coefficient array (grid_1dgr.h:16-20),
        by index or by its name in _lib.GR_COEF_NAMES."""
        k = _lib.GR_COEF_NAMES.index(which) if isinstance(which, str) else int(which)
        a = ApArray()
        check(self._lib.ap_gr_coef(self.ctx, k, C.byref(a)), "ap_gr_coef")
        return device_to_host(a.ptr, 4 * self.mesh.dims[0]).view(np.float32).copy()

    def launch_count(self) -> int:
        return int(self._lib.ap_launch_count(self.ctx))

    def close(self):
        if getattr(self, "ctx", None):
            self._lib.ap_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def array_view(t: torch.Tensor) -> ApArray:
    """ApArray of a pitched field tensor (rows x padded row)."""
    pitch = t.stride(0) * t.element_size()
    return ApArray(t.data_ptr(), pitch)


def _view_or_null(t: Optional[torch.Tensor]) -> ApArray:
    return array_view(t) if t is not None else ApArray(None, 0)


def _alloc_field(dims, device, row_align=4):
    rows = dims[1] * dims[2]
    padded = (dims[0] + row_align - 1) // row_align * row_align
    full = torch.zeros((rows, padded), dtype=torch.float32, device=device)
    return full[:, : dims[0]]


class SimData:
    """sim_data (src/sim_data.h:14-70): fields and the particle store."""

    def __init__(self, env: SimEnvironment, capacity: Optional[int] = None, row_align: int = 4,
                 photon_capacity: Optional[int] = None):
        """row_align: field rows are padded to a multiple of this many floats
        (4 gives the 16-byte row pitch the TMA field loads need; 1 packs the
        rows, which makes the kernels read the field tiles with plain loads
        when dims[0] is not a multiple of 4). photon_capacity: photon slots
        (default max_photon_number when create_pairs is set, else none)."""
        self.env = env
        dims = env.dims
        dev = env.device
        mk = lambda: _alloc_field(dims, dev, row_align)  # noqa: E731
        self.E = [mk() for _ in range(3)]
        self.B = [mk() for _ in range(3)]
        self.Ebg = [mk() for _ in range(3)]
        self.Bbg = [mk() for _ in range(3)]
        self.J = [mk() for _ in range(3)]
        self.Rho = [mk() for _ in range(env.params.num_species)]
        self.divE = mk()
        self.divB = mk()
        cap = int(capacity if capacity is not None else env.params.max_ptc_number)
        self.capacity = cap
        self.particles: Dict[str, torch.Tensor] = {
            name: torch.zeros(max(cap, 1), dtype=dt, device=dev) for name, dt in PTC_FIELDS}
        self.particles["cell"].fill_(-1)  # MAX_CELL
        self._number_stale = False
        self.number = 0
        # photons (sim_data.h: photons, photon_produced, pair_produced) when
        # the run creates pairs or a photon capacity is given
        if photon_capacity is None:
            photon_capacity = env.params.max_photon_number if env.params.create_pairs else 0
        self.photon_capacity = int(photon_capacity)
        self.photons: Optional[Dict[str, torch.Tensor]] = None
        self.photon_produced = self.pair_produced = None
        if self.photon_capacity > 0:
            self.photons = {name: torch.zeros(self.photon_capacity, dtype=dt, device=dev)
                            for name, dt in PH_FIELDS}
            self.photons["cell"].fill_(-1)
            self.photon_produced = mk()
            self.pair_produced = mk()
        self._bind()

    @property
    def number(self) -> int:
        """Particle count (slots [0, number) or the occupied slot range's
        end). After a batched step that may have changed it on the device it
        is read back on first use."""
        if self._number_stale:
            self.refresh_number()
        return self._number

    @number.setter
    def number(self, n: int):
        self._number = int(n)
        self._number_stale = False

    def mark_number_stale(self):
        """The device-side count may have changed (batched pair injection or
        sort); the next read of `number` fetches it."""
        self._number_stale = True

    def _bind(self):
        f = ApFields()
        for key in ("E", "B", "Ebg", "Bbg", "J"):
            arr = getattr(f, key)
            for c in range(3):
                arr[c] = array_view(getattr(self, key)[c])
        for s, r in enumerate(self.Rho):
            f.Rho[s] = array_view(r)
        f.divE = array_view(self.divE)
        f.divB = array_view(self.divB)
        lib = self.env._lib
        check(lib.ap_bind_fields(self.env.ctx, C.byref(f)), "ap_bind_fields")
        p = ApParticles()
        for name, _ in PTC_FIELDS:
            setattr(p, name, self.particles[name].data_ptr())
        check(lib.ap_bind_particles(self.env.ctx, C.byref(p), self.number, self.capacity),
              "ap_bind_particles")
        if self.photons is not None:
            self._bind_photons(0)

    def _bind_photons(self, number: int):
        ph = ApPhotons()
        for name, _ in PH_FIELDS:
            setattr(ph, name, self.photons[name].data_ptr())
        check(self.env._lib.ap_bind_photons(self.env.ctx, C.byref(ph), int(number),
                                            self.photon_capacity), "ap_bind_photons")

    # -- photons ---------------------------------------------------------
    @property
    def photon_number(self) -> int:
        n = C.c_size_t()
        check(self.env._lib.ap_get_photon_number(self.env.ctx, C.byref(n)),
              "ap_get_photon_number")
        return int(n.value)

    def photons_modified(self, number: int):
        """The photon count after the photon arrays were written on the
        device (slots [0, number) in use)."""
        if self.photons is None:
            raise _lib.ApError(1, "photons_modified: no photon storage")
        self._bind_photons(int(number))

    def set_photons(self, host: Dict[str, np.ndarray]):
        """Copies host photon arrays into slots [0, n)."""
        if self.photons is None:
            raise _lib.ApError(1, "set_photons: no photon storage")
        n = len(host["x1"])
        if n > self.photon_capacity:
            raise _lib.ApError(5, "set_photons")
        for name, dt in PH_FIELDS:
            a = np.ascontiguousarray(host[name])
            t = torch.from_numpy(a.view(np.int32) if dt == torch.int32 else
                                 (a.view(np.int64) if dt == torch.int64 else a))
            self.photons[name][:n].copy_(t)
        self._bind_photons(n)

    def photons_host(self) -> Dict[str, np.ndarray]:
        n = self.photon_number
        torch.cuda.synchronize()
        out = {}
        for name, _ in PH_FIELDS:
            a = self.photons[name][:n].cpu().numpy()
            out[name] = a.view(NP_DTYPES[name]) if name in NP_DTYPES else a
        return out

    # -- particles -------------------------------------------------------
    def set_particles(self, host: Dict[str, np.ndarray]):
        """Copies host SoA arrays into slots [0, n) and marks the tile order
        for rebuild."""
        n = len(host["x1"])
        if n > self.capacity:
            raise _lib.ApError(5, "set_particles")
        for name, dt in PTC_FIELDS:
            a = np.ascontiguousarray(host[name])
            t = torch.from_numpy(a.view(np.int32) if dt == torch.int32 else
                                 (a.view(np.int64) if dt == torch.int64 else a))
            self.particles[name][:n].copy_(t)
        self.number = n
        self.particles_modified()

    def set_particles_device(self, ptc: Dict[str, torch.Tensor]):
        """Copies device SoA tensors (any integer dtype for cell/id/flag) into
        slots [0, n) and marks the tile order for rebuild."""
        n = ptc["x1"].numel()
        if n > self.capacity:
            raise _lib.ApError(5, "set_particles_device")
        for name, dt in PTC_FIELDS:
            src = ptc[name]
            if dt == torch.int32 and src.dtype != torch.int32:
                src = (src.to(torch.int64) & 0xFFFFFFFF)
                src = torch.where(src >= 2 ** 31, src - 2 ** 32, src).to(torch.int32)
            self.particles[name][:n].copy_(src)
        self.number = n
        self.particles_modified()

    def set_fields_device(self, fields: Dict[str, List[torch.Tensor]]):
        for key in ("E", "B", "Ebg", "Bbg", "J"):
            if key in fields:
                for c in range(3):
                    getattr(self, key)[c].copy_(fields[key][c])

    def particles_modified(self, number: Optional[int] = None):
        if number is not None:
            self.number = int(number)
        check(self.env._lib.ap_particles_modified(self.env.ctx, self.number),
              "ap_particles_modified")

    def particles_host(self) -> Dict[str, np.ndarray]:
        self.refresh_number()
        torch.cuda.synchronize()
        out = {}
        for name, _ in PTC_FIELDS:
            a = self.particles[name][: self.number].cpu().numpy()
            out[name] = a.view(NP_DTYPES[name]) if name in NP_DTYPES else a
        return out

    def sort_particles(self):
        """sim_data::sort_particles (sim_data_impl.hpp:78-89)."""
        lib = self.env._lib
        check(lib.ap_sort_by_cell(self.env.ctx), "ap_sort_by_cell")
        self.refresh_number()

    def refresh_number(self):
        n = C.c_size_t()
        check(self.env._lib.ap_get_number(self.env.ctx, C.byref(n)), "ap_get_number")
        self.number = int(n.value)

    def slot_range(self):
        """(first, end): slots [first, end) hold every particle."""
        a, b = C.c_size_t(), C.c_size_t()
        check(self.env._lib.ap_get_slot_range(self.env.ctx, C.byref(a), C.byref(b)),
              "ap_get_slot_range")
        self.number = int(b.value)
        return int(a.value), int(b.value)

    def pair_stats(self):
        """(particle_steps, pairs created, pairs dropped) since pair injection
        was enabled."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(self.env._lib.ap_get_pair_stats(self.env.ctx, C.byref(a), C.byref(b), C.byref(c)),
              "ap_get_pair_stats")
        return int(a.value), int(b.value), int(c.value)

    def sort_particles_async(self):
        """sort_by_cell without reading the new count back (1D runs with pair
        injection keep it on the device; `number` fetches it on next use)."""
        check(self.env._lib.ap_sort_by_cell(self.env.ctx), "ap_sort_by_cell")
        self.mark_number_stale()

    def inject_pairs(self, dt: float, step: int):
        """Pair injection after the particle update of `step` (see
        SimEnvironment.set_pair_params); returns (emitted, dropped)."""
        em, dr = C.c_uint64(), C.c_uint64()
        check(self.env._lib.ap_inject_pairs(self.env.ctx, float(dt), int(step), C.byref(em),
                                            C.byref(dr)), "ap_inject_pairs")
        self.refresh_number()
        return int(em.value), int(dr.value)

    def tile_order(self):
        """(order, tile_start) of the per-step tile counting sort, as host arrays."""
        lib = self.env._lib
        o, ts = C.c_void_p(), C.c_void_p()
        nt, live = C.c_uint32(), C.c_size_t()
        check(lib.ap_get_tile_order(self.env.ctx, C.byref(o), C.byref(ts), C.byref(nt),
                                    C.byref(live)), "ap_get_tile_order")
        order = device_to_host(o.value, live.value * 4).view(np.uint32)
        start = device_to_host(ts.value, (nt.value + 1) * 4).view(np.uint32)
        return order, start

    def stats(self) -> ApStepStats:
        s = ApStepStats()
        check(self.env._lib.ap_get_stats(self.env.ctx, C.byref(s)), "ap_get_stats")
        return s

    def diagnostics(self) -> ApDiag:
        d = ApDiag()
        check(self.env._lib.ap_diagnostics(self.env.ctx, C.byref(d)), "ap_diagnostics")
        return d

    # -- fields ----------------------------------------------------------
    def fields_host(self):
        torch.cuda.synchronize()
        g = lambda t: t.contiguous().cpu().numpy()  # noqa: E731
        return {
            "E": [g(a) for a in self.E], "B": [g(a) for a in self.B],
            "Ebg": [g(a) for a in self.Ebg], "Bbg": [g(a) for a in self.Bbg],
            "J": [g(a) for a in self.J], "Rho": [g(a) for a in self.Rho],
            "divE": g(self.divE), "divB": g(self.divB),
        }

    def set_fields(self, host):
        for key in ("E", "B", "Ebg", "Bbg", "J"):
            if key in host:
                for c in range(3):
                    getattr(self, key)[c].copy_(torch.from_numpy(np.ascontiguousarray(host[key][c])))
        if "Rho" in host:
            for s, a in enumerate(host["Rho"]):
                self.Rho[s].copy_(torch.from_numpy(np.ascontiguousarray(a)))


def _wrap_device_ptr(ptr: int, n: int) -> torch.Tensor:
    """Non-owning uint8 tensor over device memory [ptr, ptr + n)."""
    class _Holder:
        __cuda_array_interface__ = {
            "shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Holder(), device="cuda")


def device_to_host(ptr: int, nbytes: int) -> np.ndarray:
    """Copy of nbytes of device memory at ptr, as a uint8 numpy array."""
    if nbytes == 0:
        return np.empty(0, np.uint8)
    torch.cuda.synchronize()
    return _wrap_device_ptr(ptr, nbytes).cpu().numpy().copy()


class ptc_updater:
    """ptc_updater (src/algorithms/ptc_updater.h:11-24)."""

    def __init__(self, env: SimEnvironment):
        self.env = env

    def update_particles(self, data: SimData, dt: float, step: int = 0):
        """ptc_updater::update_particles (ptc_updater.cu:748-841)."""
        check(self.env._lib.ap_update_particles(self.env.ctx, float(dt), int(step)),
              "ap_update_particles")

    def apply_boundary(self, data: SimData, dt: float, step: int = 0):
        """No-op, as in the reference (ptc_updater.cu:843-850)."""

    def smooth_current(self, data_or_array, step: int = 0):
        """smooth_current(sim_data&, step) or smooth_current(multi_array&)."""
        if isinstance(data_or_array, SimData):
            check(self.env._lib.ap_smooth_current(self.env.ctx, int(step)), "ap_smooth_current")
        else:
            check(self.env._lib.ap_smooth_array(self.env.ctx, array_view(data_or_array)),
                  "ap_smooth_array")


class field_solver:
    """field_solver (src/algorithms/field_solver.h:11-25)."""

    def __init__(self, env: SimEnvironment):
        self.env = env

    def update_fields(self, data: SimData, dt: float, step: int = 0):
        check(self.env._lib.ap_update_fields(self.env.ctx, float(dt), int(step)),
              "ap_update_fields")

    def apply_outflow_boundary(self, data: SimData, time: float = 0.0):
        """No-op, as in the reference (field_solver.cu:451-452)."""

    def compute_divs(self, data: SimData):
        check(self.env._lib.ap_compute_divs(self.env.ctx), "ap_compute_divs")

    def update_e_field(self, data: SimData, dt: float):
        check(self.env._lib.ap_update_e_field(self.env.ctx, float(dt)), "ap_update_e_field")

    def update_b_field(self, data: SimData, dt: float):
        check(self.env._lib.ap_update_b_field(self.env.ctx, float(dt)), "ap_update_b_field")


class Batch:
    """Batched mode (ap_batch_*): many independent 2D Cartesian runs, each a
    SimData of its own SimEnvironment, advanced with one persistent
    push / deposit launch per tile shape and no host synchronisation between
    steps. Each run's particles equal those of the same run advanced alone."""

    def __init__(self, runs: Sequence["SimData"] = ()):
        self.runs = list(runs)
        self._lib = _lib.lib()
        arr = (C.c_void_p * max(len(self.runs), 1))(*[d.env.ctx.value for d in self.runs])
        b = C.c_void_p()
        check(self._lib.ap_batch_create(arr, len(self.runs), C.byref(b)), "ap_batch_create")
        self.handle = b
        self._dt_arr = None  # each run's own delta_t as a ctypes array (membership cache)

    @property
    def dt(self):
        """Each run's own time step (SimParams.delta_t)."""
        return [float(d.env.params.delta_t) for d in self.runs]

    def add(self, data: "SimData"):
        check(self._lib.ap_batch_add(self.handle, data.env.ctx), "ap_batch_add")
        self.runs.append(data)
        self._dt_arr = None

    def remove(self, data: "SimData"):
        check(self._lib.ap_batch_remove(self.handle, data.env.ctx), "ap_batch_remove")
        self.runs.remove(data)
        self._dt_arr = None

    def _dts(self, dt):
        if dt is None:
            if self._dt_arr is None:
                self._dt_arr = (C.c_double * len(self.runs))(*self.dt)
            return self._dt_arr
        vals = [float(dt)] * len(self.runs) if np.isscalar(dt) else [float(x) for x in dt]
        return (C.c_double * len(self.runs))(*vals)

    def step_array(self, steps):
        """Per-run step numbers as the ctypes array the batched calls take;
        a loop that makes several calls per step can build it once."""
        if isinstance(steps, C.Array):
            return steps
        vals = [int(steps)] * len(self.runs) if np.isscalar(steps) else [int(x) for x in steps]
        return (C.c_uint32 * len(self.runs))(*vals)

    _steps = step_array

    def set_capture(self, on: bool):
        """Graph-capture mode (ap_batch_set_capture)."""
        check(self._lib.ap_batch_set_capture(self.handle, int(bool(on))), "ap_batch_set_capture")

    def set_stream(self, stream: torch.cuda.Stream):
        check(self._lib.ap_batch_set_stream(self.handle, C.c_void_p(stream.cuda_stream)),
              "ap_batch_set_stream")

    def update_particles(self, steps, dt=None):
        """One particle update of every run. steps: the step number of all
        runs or one per run; dt: None for each run's own delta_t, a scalar,
        or one value per run."""
        check(self._lib.ap_batch_update_particles(self.handle, self._dts(dt),
                                                  self._steps(steps)),
              "ap_batch_update_particles")

    def update_fields(self, steps, dt=None):
        check(self._lib.ap_batch_update_fields(self.handle, self._dts(dt), self._steps(steps)),
              "ap_batch_update_fields")

    def inject_pairs(self, steps, dt=None):
        """Pair injection of every run that has it enabled, without a host
        synchronisation; each run's particle number is read back when it is
        next used."""
        check(self._lib.ap_batch_inject_pairs(self.handle, self._dts(dt), self._steps(steps)),
              "ap_batch_inject_pairs")
        for d in self.runs:
            d.mark_number_stale()

    def sort_particles(self):
        check(self._lib.ap_batch_sort_by_cell(self.handle), "ap_batch_sort_by_cell")

    def advance(self, steps, nsteps: int, sort_interval: int = 0, inject: bool = False,
                dt=None):
        """`nsteps` lab-loop steps of every run in one call (ap_batch_advance):
        run r goes from step steps[r] to steps[r] + nsteps - 1; runs whose
        step is a positive multiple of sort_interval are sorted after it."""
        check(self._lib.ap_batch_advance(self.handle, self._dts(dt), self._steps(steps),
                                         int(nsteps), int(sort_interval), int(bool(inject))),
              "ap_batch_advance")
        for d in self.runs:
            d.mark_number_stale()

    def sync(self):
        bad = C.c_int(-1)
        st = self._lib.ap_batch_sync(self.handle, C.byref(bad))
        check(st, f"ap_batch_sync (run {bad.value})")

    def autotune(self, steps, dt=None) -> int:
        """Runs the tile-shape autotuner; returns the number of complete
        steps (particles, then fields) it advanced every run by."""
        used = C.c_int(0)
        check(self._lib.ap_batch_autotune(self.handle, self._dts(dt), self._steps(steps),
                                          C.byref(used)),
              "ap_batch_autotune")
        return int(used.value)

    def tile_shapes(self):
        out = []
        for d in self.runs:
            tx, ty = C.c_int(), C.c_int()
            check(self._lib.ap_get_tile_shape(d.env.ctx, C.byref(tx), C.byref(ty)),
                  "ap_get_tile_shape")
            out.append((tx.value, ty.value))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self._lib.ap_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ptc_updater_logsph:
    """ptc_updater_logsph (src/algorithms/ptc_updater_logsph.h:13-28)."""

    def __init__(self, env: SimEnvironment):
        if not env.logsph:
            raise ValueError("ptc_updater_logsph needs coord_system = 'LogSpherical'")
        self.env = env

    def update_particles(self, data: SimData, dt: float, step: int = 0):
        """update_particles then apply_boundary (ptc_updater_logsph.cu:681-836)."""
        check(self.env._lib.ap_update_particles(self.env.ctx, float(dt), int(step)),
              "ap_update_particles")

    def apply_boundary(self, data: SimData, dt: float, step: int = 0):
        """Run by update_particles already (axis current, outflow flags, and
        dropping particles that left the grid)."""

    def smooth_current(self, data: SimData, step: int = 0):
        """The smoothing passes of update_particles alone (filter_current_logsph
        weighted by face areas / cell volumes, then the axis current;
        ptc_updater_logsph.cu:616-666, 414-438) on the fields as they are."""
        check(self.env._lib.ap_smooth_current(self.env.ctx, int(step)), "ap_smooth_current")

    def inject_ptc(self, data: SimData, inj_per_cell: int, p1: float, p2: float, p3: float,
                   w: float, omega: float, seed: int = 0x5EED):
        """inject_ptc (ptc_updater_logsph.cu:849-870): pairs at the stellar
        surface where it is not yet dense (see ap_logsph_inject)."""
        check(self.env._lib.ap_logsph_inject(self.env.ctx, int(inj_per_cell), float(p1),
                                             float(p2), float(p3), float(w), float(omega),
                                             int(seed)), "ap_logsph_inject")
        data.refresh_number()


class field_solver_logsph:
    """field_solver_logsph (src/algorithms/field_solver_logsph.h:10-20)."""

    def __init__(self, env: SimEnvironment):
        if not env.logsph:
            raise ValueError("field_solver_logsph needs coord_system = 'LogSpherical'")
        self.env = env

    def update_fields(self, data: SimData, dt: float, time: float = 0.0):
        check(self.env._lib.ap_update_fields(self.env.ctx, float(dt), 0), "ap_update_fields")

    def apply_boundary(self, data: SimData, omega: float, time: float = 0.0):
        check(self.env._lib.ap_logsph_field_boundary(self.env.ctx, float(omega)),
              "ap_logsph_field_boundary")

    def compute_divs(self, data: SimData):
        check(self.env._lib.ap_compute_divs(self.env.ctx), "ap_compute_divs")


class ptc_updater_1dgap:
    """ptc_updater_1dgap (src/algorithms/ptc_updater_1dgap.h:11-27), for an
    environment with coord_system = '1dgap'."""

    def __init__(self, env: SimEnvironment):
        if not env.gap:
            raise ValueError("ptc_updater_1dgap needs coord_system = '1dgap'")
        self.env = env

    def update_particles(self, data: SimData, dt: float, step: int = 0):
        """ptc_updater_1dgap::update_particles (ptc_updater_1dgap.cu:219-272)."""
        check(self.env._lib.ap_update_particles(self.env.ctx, float(dt), int(step)),
              "ap_update_particles")


class field_solver_1dgap:
    """field_solver_1dgap (src/algorithms/field_solver_1dgap.h:9-20)."""

    def __init__(self, env: SimEnvironment):
        if not env.gap:
            raise ValueError("field_solver_1dgap needs coord_system = '1dgap'")
        self.env = env

    def update_fields(self, data: SimData, dt: float, time: float = 0.0):
        """E1 += (1.6 B0 - J1) dt (field_solver_1dgap.cu:28-40)."""
        check(self.env._lib.ap_update_fields(self.env.ctx, float(dt), 0), "ap_update_fields")


class ptc_updater_1dgr:
    """ptc_updater_1dgr (src/algorithms/ptc_updater_1dgr.h:11-30), for an
    environment with coord_system = '1DGR'."""

    def __init__(self, env: SimEnvironment):
        if not env.gr:
            raise ValueError("ptc_updater_1dgr needs coord_system = '1DGR'")
        self.env = env

    def update_particles(self, data: SimData, dt: float, step: int = 0):
        """ptc_updater_1dgr::update_particles (ptc_updater_1dgr.cu:418-473)."""
        check(self.env._lib.ap_update_particles(self.env.ctx, float(dt), int(step)),
              "ap_update_particles")


class field_solver_1dgr:
    """field_solver_1dgr (src/algorithms/field_solver_1dgr.h:11-22)."""

    def __init__(self, env: SimEnvironment):
        if not env.gr:
            raise ValueError("field_solver_1dgr needs coord_system = '1DGR'")
        self.env = env

    def update_fields(self, data: SimData, dt: float, time: float = 0.0):
        """E1 += (j0 - J1) dt (field_solver_1dgr.cu:14-44)."""
        check(self.env._lib.ap_update_fields(self.env.ctx, float(dt), 0), "ap_update_fields")


class radiative_transfer:
    """radiative_transfer (src/radiation/radiative_transfer.h:11-29): photon
    emission and pair production with the user radiative functions that
    SimParams.rad_model names ("default": src/cuda/radiation/
    user_radiative_functions.cu; "pulsar": the pulsar lab's; "gr1d" and
    "gap1d": the 1D GR and gap labs', whose inverse-Compton tables are built
    here as their user_rt_init builds them). The photon move itself is part of
    update_particles, as in the reference."""

    MODELS = {"default": _lib.RAD_DEFAULT, "pulsar": _lib.RAD_PULSAR, "gr1d": _lib.RAD_GR1D,
              "gap1d": _lib.RAD_GAP1D}

    def __init__(self, env: SimEnvironment, first_photon_id: int = 1 << 60,
                 first_particle_id: int = (1 << 60) + (1 << 59)):
        self.env = env
        pr = env.params
        rp = ApRadParams()
        rp.model = self.MODELS[pr.rad_model]
        rp.delta_t = pr.delta_t
        rp.gamma_thr = pr.gamma_thr
        rp.E_secondary = pr.E_secondary
        rp.photon_path = pr.photon_path
        rp.r_cutoff = pr.r_cutoff
        rp.track_percent = pr.track_percent
        rp.e_curv = pr.e_curv
        rp.l_curv = pr.l_curv
        rp.BQ = pr.BQ
        rp.omega = pr.omega
        rp.seed = int(pr.rad_seed)
        rp.first_photon_id = int(first_photon_id)
        rp.first_particle_id = int(first_particle_id)
        rp.e_min = pr.e_min
        rp.ic_path = pr.ic_path
        rp.n_gamma = int(pr.n_gamma)
        rp.n_ep = int(pr.n_ep)
        check(env._lib.ap_set_rad_params(env.ctx, C.byref(rp)), "ap_set_rad_params")
        self.last: Dict[str, int] = {}

    @staticmethod
    def _counts(c: ApRadCounts) -> Dict[str, int]:
        return {"marked": int(c.marked), "written": int(c.written), "dropped": int(c.dropped)}

    def emit_photons(self, data: SimData) -> Dict[str, int]:
        """radiative_transfer::emit_photons (radiative_transfer.cu:196-243);
        photon_produced accumulates the emitters' weights per cell."""
        cnt = ApRadCounts()
        check(self.env._lib.ap_emit_photons(self.env.ctx, _view_or_null(data.photon_produced),
                                             C.byref(cnt)), "ap_emit_photons")
        self.last = self._counts(cnt)
        return self.last

    def produce_pairs(self, data: SimData) -> Dict[str, int]:
        """radiative_transfer::produce_pairs (radiative_transfer.cu:245-301);
        pair_produced accumulates the converted photons' weights per cell."""
        cnt = ApRadCounts()
        check(self.env._lib.ap_produce_pairs(self.env.ctx, _view_or_null(data.pair_produced),
                                             C.byref(cnt)), "ap_produce_pairs")
        data.refresh_number()
        self.last = self._counts(cnt)
        return self.last


class inverse_compton:
    """inverse_compton (src/cuda/radiation/rt_ic.h, rt_ic.cu): the rate and
    photon-energy tables for a background spectrum, built on the device of
    an environment. `spectrum` is one of SPECTRA with its constructor's
    arguments, e.g. ("broken_power_law", 1.25, 1.1, 1e-3, 1e-10, 0.1)."""

    SPECTRA = {"power_law_hard": _lib.SPEC_POWER_LAW_HARD,
               "power_law_soft": _lib.SPEC_POWER_LAW_SOFT,
               "broken_power_law": _lib.SPEC_BROKEN_POWER_LAW,
               "black_body": _lib.SPEC_BLACK_BODY,
               "mono_energetic": _lib.SPEC_MONO_ENERGETIC}

    def __init__(self, env: SimEnvironment):
        self.env = env
        self.n_gamma = int(env.params.n_gamma)
        self.n_ep = int(env.params.n_ep)

    def init(self, spectrum, emin: float, emax: float, n0: float):
        sp = _lib.ApSpectrum()
        sp.kind = self.SPECTRA[spectrum[0]]
        for k, v in enumerate(spectrum[1:]):
            sp.p[k] = float(v)
        check(self.env._lib.ap_ic_init(self.env.ctx, C.byref(sp), float(emin), float(emax),
                                       float(n0), self.n_gamma, self.n_ep), "ap_ic_init")

    def tables(self) -> Dict[str, np.ndarray]:
        """ic_rate, gg_rate, gammas (n_gamma), dNde, dNde_thomson (n_gamma x
        n_ep) and the steps dep, dg, dlep."""
        ng, ne = self.n_gamma, self.n_ep
        out = {k: np.zeros(ng, np.float32) for k in ("ic_rate", "gg_rate", "gammas")}
        out.update({k: np.zeros((ng, ne), np.float32) for k in ("dNde", "dNde_thomson")})
        steps = np.zeros(3, np.float32)
        check(self.env._lib.ap_ic_tables(
            self.env.ctx, *[out[k].ctypes.data for k in ("ic_rate", "gg_rate", "gammas", "dNde",
                                                          "dNde_thomson")],
            steps.ctypes.data), "ap_ic_tables")
        out["dep"], out["dg"], out["dlep"] = (float(x) for x in steps)
        return out


# Python-style aliases
PtcUpdater = ptc_updater
FieldSolver = field_solver
PtcUpdaterLogsph = ptc_updater_logsph
FieldSolverLogsph = field_solver_logsph
PtcUpdater1dGap = ptc_updater_1dgap
FieldSolver1dGap = field_solver_1dgap
