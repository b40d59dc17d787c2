"""Seeded synthetic initial conditions for the benchmark configurations.

The reference labs build their initial state in main.cpp (fields from
closures, particles from sim_data::fill_multiplicity,
cuda/sim_data.cu:268-293: e-/e+ pairs at one position, then a sort). These
generators produce the same kind of state for the configurations this
package is measured on, as host or device tensors, from a seed:

* box1d: 1D periodic plain PIC, 4096 cells, dx = 1/4096, dt = dx/2,
  2^20 particles (e-/e+ pairs at one position, weight 1), positions uniform,
  momenta Gaussian (sigma 0.1 per component), E1 = 0.5 sin(2 pi x), B1 = 1.
* box2d: 2D periodic box, N x N Yee cells, dx = 1/N, dt = dx/2, ppc/2 pairs
  per cell at uniform positions, isotropic momenta with gamma log-uniform in
  [1, gamma_max], B3 = B0 plus random Fourier modes (integer |k| <= 8,
  amplitude 0.1, random phase) in every E and B component.

Particles come out sorted by cell (fill order). All values are computed in
float64 and rounded once to float32.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np
import torch

from .sim import POSITRON, ELECTRON, SimParams, species_flag


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def box1d_params(N: int = 4096, num_particles: int = 1 << 20, data_interval: int = 1) -> SimParams:
    dx = 1.0 / N
    return SimParams(N=(N, 1, 1), guard=(2, 0, 0), lower=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0),
                     delta_t=float(np.float32(0.5 * dx)), q_e=1.0, num_species=2,
                     periodic_boundary=(True, False, False), data_interval=data_interval,
                     max_ptc_number=num_particles, B0=1.0)


def box2d_params(N: int = 1024, ppc: int = 64, data_interval: int = 100, capacity=None,
                 tile=(0, 0)) -> SimParams:
    dx = 1.0 / N
    return SimParams(N=(N, N, 1), guard=(2, 2, 0), lower=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0),
                     delta_t=float(np.float32(0.5 * dx)), q_e=1.0, num_species=2,
                     periodic_boundary=(True, True, False), data_interval=data_interval,
                     max_ptc_number=int(capacity or N * N * ppc), B0=1.0,
                     tile_size=(tile[0], tile[1], 0))


def _stagger_pos(n_idx: torch.Tensor, guard: int, delta: float, stagger: int) -> torch.Tensor:
    """Quadmesh::pos(i, n, stagger) (src/core/quadmesh.h:132-150), lower = 0."""
    return delta * (n_idx.double() - guard + (1.0 if stagger else 0.5))


def _pairs(cells: torch.Tensor, g: torch.Generator, device, p_sampler) -> Dict[str, torch.Tensor]:
    """e-/e+ pairs at shared positions, one pair per entry of `cells`."""
    npair = cells.numel()
    n = 2 * npair
    rel1 = torch.rand(npair, generator=g, device=device, dtype=torch.float32)
    rel2 = torch.rand(npair, generator=g, device=device, dtype=torch.float32)
    p = p_sampler(n)  # (3, n) float64
    out = {
        "x1": rel1.repeat_interleave(2), "x2": rel2.repeat_interleave(2),
        "x3": torch.zeros(n, dtype=torch.float32, device=device),
        "p1": p[0].float(), "p2": p[1].float(), "p3": p[2].float(),
        "weight": torch.ones(n, dtype=torch.float32, device=device),
        "cell": cells.repeat_interleave(2).to(torch.int64),
        "id": torch.arange(n, dtype=torch.int64, device=device),
    }
    sp = torch.tensor([species_flag(ELECTRON), species_flag(POSITRON)], dtype=torch.int64,
                      device=device)
    out["flag"] = sp.repeat(npair)
    pp = out["p1"].double() ** 2 + out["p2"].double() ** 2 + out["p3"].double() ** 2
    out["E"] = torch.sqrt(1.0 + pp).float()
    return out


def box1d(seed: int = 0, N: int = 4096, num_particles: int = 1 << 20, device="cpu"):
    """Config: 1D periodic plain PIC. Returns (params, fields, particles)."""
    params = box1d_params(N, num_particles)
    g = _gen(seed, device)
    guard = 2
    npair = num_particles // 2
    cells = torch.sort(torch.randint(0, N, (npair,), generator=g, device=device)).values + guard

    def sampler(n):
        return 0.1 * torch.randn((3, n), generator=g, device=device, dtype=torch.float64)

    ptc = _pairs(cells, g, device, sampler)
    ptc["x2"].zero_()
    dims0 = N + 2 * guard
    dx = 1.0 / N
    n_idx = torch.arange(dims0, device=device)
    z = lambda: torch.zeros((1, dims0), dtype=torch.float32, device=device)  # noqa: E731
    E = [z(), z(), z()]
    B = [z(), z(), z()]
    E[0][0] = (0.5 * torch.sin(2 * math.pi * _stagger_pos(n_idx, guard, dx, 0))).float()
    B[0][0] = 1.0
    fields = {"E": E, "B": B}
    return params, fields, ptc


def box2d(seed: int = 0, N: int = 1024, ppc: int = 64, gamma_max: float = 1e3,
          modes: int = 8, amp: float = 0.1, kmax: int = 8, device="cpu", tile=(0, 0),
          data_interval: int = 100):
    """Config: 2D periodic box. Returns (params, fields, particles)."""
    params = box2d_params(N, ppc, data_interval=data_interval, tile=tile)
    g = _gen(seed, device)
    guard = 2
    dims0 = N + 2 * guard
    cx = torch.arange(N, device=device) + guard
    cells = (cx[None, :] + cx[:, None] * dims0).reshape(-1)
    cells = cells.repeat_interleave(ppc // 2)

    def sampler(n):
        u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
        gamma = torch.exp(u * math.log(gamma_max))
        pm = torch.sqrt(torch.clamp(gamma * gamma - 1.0, min=0.0))
        ct = 2.0 * torch.rand(n, generator=g, device=device, dtype=torch.float64) - 1.0
        st = torch.sqrt(torch.clamp(1.0 - ct * ct, min=0.0))
        ph = 2.0 * math.pi * torch.rand(n, generator=g, device=device, dtype=torch.float64)
        return torch.stack([pm * st * torch.cos(ph), pm * st * torch.sin(ph), pm * ct])

    ptc = _pairs(cells, g, device, sampler)
    # fields: random Fourier modes per component, on each component's stagger
    dx = 1.0 / N
    n_idx = torch.arange(dims0, device=device)
    stag = [(0, 1), (1, 0), (1, 1), (1, 0), (0, 1), (0, 0)]  # E1..E3, B1..B3 (x, y)
    rng = np.random.default_rng(seed + 7919)
    comps = []
    for k in range(6):
        X = _stagger_pos(n_idx, guard, dx, stag[k][0])[None, :]
        Y = _stagger_pos(n_idx, guard, dx, stag[k][1])[:, None]
        f = torch.zeros((dims0, dims0), dtype=torch.float64, device=device)
        for _ in range(modes):
            while True:
                kx, ky = rng.integers(-kmax, kmax + 1, size=2)
                if kx or ky:
                    break
            ph = rng.uniform(0.0, 2.0 * math.pi)
            f += amp * torch.sin(2.0 * math.pi * (kx * X + ky * Y) + ph)
        if k == 5:
            f += params.B0
        comps.append(f.float())
    fields = {"E": comps[:3], "B": comps[3:]}
    return params, fields, ptc


def logsph(seed: int = 0, N: int = 1024, ppc: int = 32, rmax: float = 50.0,
           scale_height: float = 0.5, gamma_max: float = 1e6, omega: float = 0.1,
           B0: float = 1.0, device="cpu"):
    """Config: 2D log-spherical grid, x1 = ln r in [0, ln rmax], x2 = theta in
    [0, pi], N x N cells, guard 2. Dipole background B_r = 2 B0 cos(theta) /
    r^3, B_theta = B0 sin(theta) / r^3 (labs/pulsar/src/main.cpp:49-58) and
    the corotation field E = -(Omega x r) x B, each on its Yee stagger; B and
    E start equal to their backgrounds. Pairs per cell drawn from a Poisson
    law of mean ppc / 2 * exp(-(r - 1) / scale_height) at the cell centre;
    momenta along the local B direction (random sign) with gamma
    log-uniform in [1, gamma_max]; dt = 0.4 * min(delta). Returns (params,
    fields, particles); params.coord_system is "LogSpherical"."""
    from .sim import SimParams
    guard = 2
    d0 = float(np.float32(np.float32(math.log(rmax)) / np.float32(N)))
    d1 = float(np.float32(np.float32(math.pi) / np.float32(N)))
    params = SimParams(N=(N, N, 1), guard=(guard, guard, 0), lower=(0.0, 0.0, 0.0),
                       size=(float(np.float32(math.log(rmax))), float(np.float32(math.pi)), 1.0),
                       delta_t=float(np.float32(0.4 * min(d0, d1))), q_e=1.0, num_species=2,
                       periodic_boundary=(False, False, False), data_interval=100, B0=B0,
                       coord_system="LogSpherical", compactness=0.0, omega=omega,
                       damping_length=32)
    g = _gen(seed, device)
    dims = N + 2 * guard
    n_idx = torch.arange(dims, device=device)
    stag = [(0, 1), (1, 0), (1, 1), (1, 0), (0, 1), (0, 0)]  # E1..E3, B1..B3 (x, y)

    def pos(d, n, s, delta):
        return delta * (n.double() - guard + (1.0 if s else 0.5))
    comps = []
    for k in range(6):
        r = torch.exp(pos(0, n_idx, stag[k][0], d0))[None, :]
        th = pos(1, n_idx, stag[k][1], d1)[:, None]
        br = 2.0 * B0 * torch.cos(th) / r ** 3
        bt = B0 * torch.sin(th) / r ** 3
        if k >= 3:
            val = [br, bt, torch.zeros_like(br)][k - 3]
        else:
            v = omega * r * torch.sin(th)
            val = [v * bt, -v * br, torch.zeros_like(br)][k]
        comps.append(val.float().contiguous())
    # particles
    rc = torch.exp(pos(0, n_idx[guard:guard + N], 0, d0))
    lam = (ppc / 2.0) * torch.exp(-(rc - 1.0) / scale_height)
    lam2 = lam[None, :].expand(N, N).contiguous()
    npc = torch.poisson(lam2.double(), generator=g).long().reshape(-1)
    cx = torch.arange(N, device=device) + guard
    cells = (cx[None, :] + cx[:, None] * dims).reshape(-1).repeat_interleave(npc)
    c1 = cells % dims
    c2 = cells // dims
    th = pos(1, c2, 0, d1)
    rr = torch.exp(pos(0, c1, 0, d0))
    br = 2.0 * torch.cos(th) / rr ** 3
    bt = torch.sin(th) / rr ** 3
    bn = torch.sqrt(br * br + bt * bt)

    def sampler(n):
        u = torch.rand(n // 2, generator=g, device=device, dtype=torch.float64)
        gam = torch.exp(u * math.log(gamma_max))
        pm = torch.sqrt(torch.clamp(gam * gam - 1.0, min=0.0))
        sgn = torch.where(torch.rand(n // 2, generator=g, device=device) < 0.5, -1.0, 1.0)
        pm = (pm * sgn).repeat_interleave(2)
        return torch.stack([pm * br.repeat_interleave(2) / bn.repeat_interleave(2),
                            pm * bt.repeat_interleave(2) / bn.repeat_interleave(2),
                            torch.zeros_like(pm)])
    ptc = _pairs(cells, g, device, sampler)
    params.max_ptc_number = int(ptc["x1"].numel())
    fields = {"E": comps[:3], "B": comps[3:], "Ebg": [c.clone() for c in comps[:3]],
              "Bbg": [c.clone() for c in comps[3:]]}
    return params, fields, ptc


def to_numpy_ptc(ptc: Dict[str, torch.Tensor]) -> Dict[str, np.ndarray]:
    out = {}
    for k, v in ptc.items():
        a = v.cpu().numpy()
        if k in ("cell", "flag"):
            a = a.astype(np.uint32)
        elif k == "id":
            a = a.astype(np.uint64)
        out[k] = np.ascontiguousarray(a)
    return out
