"""Readers of the drop-in's result files (the reference's formats, written by
src/utils/io.cpp and src/main.cpp in the reference) and the analytic flows the
reference's acceptance tests compare against. Test helpers only."""
from __future__ import annotations

from pathlib import Path

import numpy as np


def read_vtk(path) -> dict:
    """Legacy binary STRUCTURED_POINTS file as written by writeVTK (io.cpp:44-67):
    the header lines, flag (u8), density (big-endian f64) and velocity (3 x
    big-endian f64). Arrays are indexed [z, y, x]."""
    raw = Path(path).read_bytes()
    pos = 0
    header = []

    def line():
        nonlocal pos
        end = raw.index(b"\n", pos)
        s = raw[pos:end].decode()
        pos = end + 1
        return s

    while True:
        s = line()
        header.append(s)
        if s.startswith("POINT_DATA"):
            break
    dims = [int(v) for v in next(h for h in header if h.startswith("DIMENSIONS")).split()[1:]]
    n = dims[0] * dims[1] * dims[2]
    shape = (dims[2], dims[1], dims[0])
    out = {"header": header, "dims": dims}
    assert line() == "SCALARS flag unsigned_char 1" and line() == "LOOKUP_TABLE default"
    out["flag"] = np.frombuffer(raw, np.uint8, n, pos).reshape(shape)
    pos += n + 1
    assert line() == "SCALARS density double 1" and line() == "LOOKUP_TABLE default"
    out["density"] = np.frombuffer(raw, ">f8", n, pos).astype(float).reshape(shape)
    pos += 8 * n + 1
    assert line() == "VECTORS velocity double"
    out["velocity"] = np.frombuffer(raw, ">f8", 3 * n, pos).astype(float).reshape(shape + (3,))
    pos += 24 * n + 1
    assert pos == len(raw)
    return out


def read_keyvalue(path) -> dict:
    """`key v1 [v2 ...]` lines (_summary.txt, _squirmer.dat)."""
    out = {}
    for s in Path(path).read_text().splitlines():
        tok = s.split()
        if tok:
            out[tok[0]] = np.array([float(v) for v in tok[1:]])
    return out


TRAJ_COLS = ("t", "X", "Y", "Z", "ex", "ey", "ez", "Ux", "Uy", "Uz", "Wx", "Wy", "Wz", "Fwall_y", "Fwall_z")


def read_traj(path) -> dict:
    """The trajectory file (io.cpp:72-83) by column name, plus the in-plane
    angle of e in degrees."""
    a = np.loadtxt(path, ndmin=2)
    tr = {k: a[:, j] for j, k in enumerate(TRAJ_COLS)}
    tr["angle"] = np.degrees(np.arctan2(tr["ey"], tr["ex"]))
    return tr


def blake_velocity(x, y, z, R, B1, beta, e=(1.0, 0.0, 0.0)):
    """Lab-frame Stokes flow around a two-mode squirmer of radius R centred at
    the origin and swimming along e (Blake, J. Fluid Mech. 46, 1971): the
    source dipole B1 (R/r)^3 (cos th r^ - e/3) plus the B2 = beta B1 stresslet
    and its companion terms. Shape (3, ...); NaN inside the sphere."""
    x, y, z = np.broadcast_arrays(*(np.asarray(v, float) for v in (x, y, z)))
    e = np.asarray(e, float)
    r = np.maximum(np.sqrt(x * x + y * y + z * z), 1e-12)
    rh = np.stack([x / r, y / r, z / r])
    ct = np.tensordot(e, rh, axes=1)
    E = e.reshape((3,) + (1,) * x.ndim)
    q = R / r
    B2 = beta * B1
    u = (B1 * q ** 3 * (ct * rh - E / 3.0)
         + B2 * (q ** 4 - q ** 2) * (1.5 * ct * ct - 0.5) * rh
         + B2 * q ** 4 * ct * (ct * rh - E))
    u[:, r < R] = np.nan
    return u


def near_field_error(vtk: dict, X, R, B1, beta) -> float:
    """Relative L2 difference of (u_x, u_y) between the simulated flow and the
    Blake flow over the lattice plane z nearest below the centre, at distances
    1.25 R < r < 3 R from it (minimum image in a periodic box), fluid nodes
    only -- the near-field figure of the reference's acceptance test."""
    nx, ny, nz = vtk["dims"]
    zp = int(np.floor(X[2] % nz))
    dz = zp - X[2] % nz
    dx = np.arange(nx) - X[0] % nx
    dx -= nx * np.round(dx / nx)
    dy = np.arange(ny) - X[1]
    dy -= ny * np.round(dy / ny)
    PX, PY = np.meshgrid(dx, dy)
    v = vtk["velocity"][zp]
    fl = vtk["flag"][zp]
    ub = blake_velocity(PX, PY, np.full_like(PX, dz), R, B1, beta)
    rr = np.sqrt(PX ** 2 + PY ** 2 + dz ** 2)
    m = (rr > 1.25 * R) & (rr < 3 * R) & (fl == 0)
    num = np.sum((v[..., 0][m] - ub[0][m]) ** 2 + (v[..., 1][m] - ub[1][m]) ** 2)
    den = np.sum(ub[0][m] ** 2 + ub[1][m] ** 2)
    return float(np.sqrt(num / den))
