"""Named workloads (synthetic lattices; no dataset is involved).

  duct     16x32x32 square duct, walls in y and z, tau=0.8, fx=1e-6, 20000 steps
  slit     128x64x64 slit channel (walls in y), neutral squirmer a=6, B1=1.5e-3,
           tau=1.0, centre at mid-height, 15 deg toward the wall, 50000 steps
  bulk_*   256x128x128 fully periodic box, squirmer a=8, B1=1e-3, tau=0.9,
           beta in {-3, 0, 3}, random unit orientation from seed 12345+beta
           (numpy default_rng, normalised Gaussian), 10000 steps
  ensemble 256 slit-channel squirmers of uneven sizes (see ensemble_members)
"""
from __future__ import annotations

import numpy as np

from .params import Params

SLIT_DECK = dict(  # the reference's inputs/channel_neutral.in keys
    walls_y=1, walls_z=0, squirmer=1, planar=1, eps=0.2, hc=2.0, hmin=0.5,
    print_every=2000, traj_every=50)


def bulk_orientation(beta: float) -> tuple:
    g = np.random.default_rng(12345 + int(beta)).standard_normal(3)
    g = g / np.linalg.norm(g)
    return tuple(float(v) for v in g)


def workload_params(name: str, precision: str = "fp64") -> Params:
    p = Params()
    if name == "duct":
        p.update(nx=16, ny=32, nz=32, tau=0.8, fx=1e-6, walls_y=1, walls_z=1, squirmer=0,
                 steps=20000, tol=0.0, print_every=1000)
    elif name == "slit":
        p.update(**SLIT_DECK)
        p.update(nx=128, ny=64, nz=64, radius=6, beta=0, b1=1.5e-3, tau=1.0, angle=15, steps=50000)
    elif name.startswith("bulk_"):
        beta = {"m3": -3.0, "0": 0.0, "p3": 3.0}[name[5:]]
        p.update(nx=256, ny=128, nz=128, walls_y=0, walls_z=0, squirmer=1, radius=8, b1=1e-3,
                 tau=0.9, beta=beta, planar=0, steps=10000, traj_every=50, print_every=1000)
        ex, ey, ez = bulk_orientation(beta)
        p.update(ex=ex, ey=ey, ez=ez)
    else:
        raise KeyError(f"unknown workload '{name}'")
    p.update(precision=precision)
    p.validate()
    return p


def ensemble_members(n: int = 256, seed: int = 2024) -> list[Params]:
    """Slit-channel squirmers: Nx ~ U[64,160], Ny, Nz ~ U[48,96] (integers),
    a ~ U[4,8], beta ~ U[-5,5], angle ~ U[-30,30] deg, y0 = 0.5 + U[1.5a, H-1.5a]
    with H = Ny - 2. Walls in y only; B1 = 0.015 and tau = 1.0 (the reference
    defaults, params.hpp:20, :44); FP32-shifted storage."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.integers(64, 161))
        ny = int(rng.integers(48, 97))
        nz = int(rng.integers(48, 97))
        a = float(rng.uniform(4.0, 8.0))
        beta = float(rng.uniform(-5.0, 5.0))
        angle = float(rng.uniform(-30.0, 30.0))
        H = ny - 2
        y0 = 0.5 + float(rng.uniform(1.5 * a, H - 1.5 * a))
        p = Params()
        p.update(**SLIT_DECK)
        p.update(nx=nx, ny=ny, nz=nz, radius=a, beta=beta, angle=angle, y0=y0, b1=0.015, tau=1.0,
                 steps=30000, precision="fp32")
        p.validate()
        out.append(p)
    return out
