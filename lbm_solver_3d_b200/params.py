"""Simulation parameters: the reference's ``key = value`` system in Python.

Mirrors ``lbm::Params`` (src/utils/params.hpp:14-63, src/utils/params.cpp:37-157):
the same keys and aliases, the same boolean spellings, the same file syntax
(``#`` comments, one ``key = value`` per line, later command-line
``key=value`` overrides), the same validation rules and messages. The keys
this library adds are listed in ``EXTRA_KEYS``; everything else unknown is an
error, as in the reference.
"""
from __future__ import annotations

import ctypes
import math
import dataclasses
from dataclasses import dataclass, field, fields
from pathlib import Path

__all__ = ["Params", "ParamError", "PRECISIONS", "EXTRA_KEYS"]

PRECISIONS = {"fp64": 0, "fp32": 1, "fp16": 2}

# Keys beyond the reference's set: storage precision and a 3-D initial
# orientation (the reference only takes an in-plane angle, squirmer.cpp:26-27).
EXTRA_KEYS = ("precision", "ex", "ey", "ez", "device", "checkpoint_every", "restart")


class ParamError(RuntimeError):
    """Raised where the reference throws std::runtime_error."""


def _to_bool(v: str) -> bool:
    # params.cpp:25-30
    s = v.strip().lower()
    if s in ("1", "true", "yes", "on"):
        return True
    if s in ("0", "false", "no", "off"):
        return False
    raise ParamError(f"cannot interpret '{v}' as a boolean")


def _stoi(v: str) -> int:
    # std::stoi semantics: leading whitespace, optional sign, digits; trailing
    # characters are ignored ("12abc" -> 12), no digits -> invalid_argument.
    s = v.strip()
    k = 0
    if k < len(s) and s[k] in "+-":
        k += 1
    j = k
    while j < len(s) and s[j].isdigit():
        j += 1
    if j == k:
        raise ValueError(v)
    return int(s[:j])


def _stod(v: str) -> float:
    # std::stod semantics: the longest valid floating-point prefix.
    s = v.strip()
    for end in range(len(s), 0, -1):
        try:
            return float(s[:end])
        except ValueError:
            continue
    raise ValueError(v)


@dataclass
class Params:
    """Same fields and defaults as lbm::Params (params.hpp:16-56)."""

    NX: int = 64
    NY: int = 34
    NZ: int = 32
    tau: float = 1.0
    Lambda: float = 3.0 / 16.0
    Fx: float = 0.0
    Fy: float = 0.0
    Fz: float = 0.0
    wallsY: bool = True
    wallsZ: bool = False
    steps: int = 10000
    printEvery: int = 1000
    vtkEvery: int = 0
    trajEvery: int = 50
    tol: float = 0.0
    massCorrectionEvery: int = 10
    outputDir: str = "outputs"
    prefix: str = "run"
    squirmer: bool = False
    R: float = 4.0
    B1: float = 0.015
    beta: float = 0.0
    rhoP: float = 1.0
    x0: float = -1.0
    y0: float = -1.0
    z0: float = -1.0
    angle: float = 30.0
    planar: bool = True
    eps: float = 0.2
    hc: float = 2.0
    hmin: float = 0.5
    # additions
    precision: str = "fp64"
    orientation: tuple | None = None
    device: int = 0
    checkpoint_every: int = 0   # the driver writes <prefix>_checkpoint.bin every this many steps
    restart: str = ""           # the driver continues from this checkpoint file

    # ---- key = value (params.cpp:37-75) ----
    def set(self, key: str, v: str) -> None:
        k = key.strip().lower()
        v = str(v)
        try:
            if k == "nx": self.NX = _stoi(v)
            elif k == "ny": self.NY = _stoi(v)
            elif k == "nz": self.NZ = _stoi(v)
            elif k == "tau": self.tau = _stod(v)
            elif k == "lambda": self.Lambda = _stod(v)
            elif k == "fx": self.Fx = _stod(v)
            elif k == "fy": self.Fy = _stod(v)
            elif k == "fz": self.Fz = _stod(v)
            elif k in ("walls_y", "wallsy"): self.wallsY = _to_bool(v)
            elif k in ("walls_z", "wallsz"): self.wallsZ = _to_bool(v)
            elif k == "steps": self.steps = _stoi(v)
            elif k in ("print_every", "print"): self.printEvery = _stoi(v)
            elif k in ("vtk_every", "vtk"): self.vtkEvery = _stoi(v)
            elif k in ("traj_every", "traj"): self.trajEvery = _stoi(v)
            elif k == "tol": self.tol = _stod(v)
            elif k == "mass_correction_every": self.massCorrectionEvery = _stoi(v)
            elif k == "output_dir": self.outputDir = v
            elif k == "prefix": self.prefix = v
            elif k in ("squirmer", "sq"): self.squirmer = _to_bool(v)
            elif k in ("radius", "r"): self.R = _stod(v)
            elif k == "b1": self.B1 = _stod(v)
            elif k == "beta": self.beta = _stod(v)
            elif k in ("rho_p", "rhop"): self.rhoP = _stod(v)
            elif k == "x0": self.x0 = _stod(v)
            elif k == "y0": self.y0 = _stod(v)
            elif k == "z0": self.z0 = _stod(v)
            elif k == "angle": self.angle = _stod(v)
            elif k == "planar": self.planar = _to_bool(v)
            elif k == "eps": self.eps = _stod(v)
            elif k == "hc": self.hc = _stod(v)
            elif k == "hmin": self.hmin = _stod(v)
            elif k == "precision":
                s = v.strip().lower()
                if s not in PRECISIONS:
                    raise ParamError(f"precision must be one of {', '.join(PRECISIONS)}")
                self.precision = s
            elif k in ("ex", "ey", "ez"):
                o = list(self.orientation or (0.0, 0.0, 0.0))
                o["xyz".index(k[1])] = _stod(v)
                self.orientation = tuple(o)
            elif k == "device": self.device = _stoi(v)
            elif k == "checkpoint_every": self.checkpoint_every = _stoi(v)
            elif k == "restart": self.restart = v.strip()
            else:
                raise ParamError(f"unknown parameter '{k}'")
        except ValueError:
            raise ParamError(f"invalid value '{v}' for parameter '{k}'") from None

    def copy(self) -> "Params":
        return dataclasses.replace(self)

    def update(self, **kv) -> "Params":
        for k, v in kv.items():
            self.set(k, v if isinstance(v, str) else _fmt(v))
        return self

    # ---- input file (params.cpp:81-101) ----
    def load_file(self, path) -> None:
        path = str(path)
        try:
            text = Path(path).read_text()
        except OSError:
            raise ParamError(f"cannot open input file '{path}'") from None
        for line_no, line in enumerate(text.splitlines(), 1):
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            if "=" not in line:
                raise ParamError(f"{path}:{line_no}: expected 'key = value'")
            key, val = line.split("=", 1)
            try:
                self.set(key, val.strip())
            except ParamError as e:
                raise ParamError(f"{path}:{line_no}: {e}") from None

    # ---- command line (params.cpp:107-114) ----
    def parse_command_line(self, args) -> None:
        for a in args:
            if "=" not in a:
                self.load_file(a)
            else:
                k, v = a.split("=", 1)
                self.set(k, v)

    @classmethod
    def from_args(cls, *args, **overrides) -> "Params":
        p = cls()
        p.parse_command_line([str(a) for a in args])
        p.update(**overrides)
        return p

    # ---- validation (params.cpp:120-140) ----
    def validate(self) -> None:
        def fail(m):
            raise ParamError(m)

        if self.NX < 1 or self.NY < 1 or self.NZ < 1: fail("grid dimensions must be positive")
        if self.wallsY and self.NY < 4: fail("ny must be >= 4 with walls in y")
        if self.wallsZ and self.NZ < 4: fail("nz must be >= 4 with walls in z")
        if self.tau <= 0.5: fail("tau must be > 0.5")
        if self.Lambda <= 0.0: fail("lambda must be > 0")
        if self.steps < 0: fail("steps must be >= 0")
        if self.printEvery < 1 or self.trajEvery < 1: fail("print_every and traj_every must be >= 1")
        if self.orientation is not None and math.sqrt(sum(c * c for c in self.orientation)) == 0.0:
            fail("orientation (ex, ey, ez) must be non-zero")
        if not self.squirmer:
            return
        if self.R <= 1.0: fail("squirmer radius must be > 1 lattice unit")
        if abs(self.angle) >= 45.0: fail("initial angle must satisfy |angle| < 45 deg from the x-axis")
        if self.rhoP <= 0.0: fail("rho_p must be > 0")
        if self.eps < 0.0 or self.hc <= 0.0 or self.hmin < 0.0: fail("eps >= 0, hc > 0, hmin >= 0 required")
        y = self.y0 if self.y0 >= 0 else 0.5 * (self.NY - 1)
        if self.wallsY and (y - self.R - 0.5 < self.hmin or (self.NY - 1.5) - y - self.R < self.hmin):
            fail("squirmer initially overlaps (or is too close to) a y-wall")
        if (2.0 * self.R + 2.0 > self.NX or (not self.wallsY and 2.0 * self.R + 2.0 > self.NY)
                or 2.0 * self.R + 2.0 > self.NZ):
            fail("domain too small for the squirmer")
        if 2.0 * self.B1 / 3.0 > 0.05:
            fail("swimming speed U0 = 2 B1 / 3 too large (Mach number); keep U0 < 0.05")

    @property
    def ncells(self) -> int:
        return self.NX * self.NY * self.NZ

    @property
    def nu(self) -> float:
        return (self.tau - 0.5) / 3.0

    def to_c(self):
        """The C-ABI parameter block (include/lbmgpu.h: lbmgpu_params)."""
        from ._lib import LbmgpuParams
        c = LbmgpuParams()
        c.nx, c.ny, c.nz = self.NX, self.NY, self.NZ
        c.tau, c.lambda_, c.fx, c.fy, c.fz = self.tau, self.Lambda, self.Fx, self.Fy, self.Fz
        c.walls_y, c.walls_z = int(self.wallsY), int(self.wallsZ)
        c.traj_every, c.mass_correction_every = self.trajEvery, self.massCorrectionEvery
        c.squirmer = int(self.squirmer)
        c.radius, c.b1, c.beta, c.rho_p = self.R, self.B1, self.beta, self.rhoP
        c.x0, c.y0, c.z0, c.angle = self.x0, self.y0, self.z0, self.angle
        c.planar = int(self.planar)
        c.eps, c.hc, c.hmin = self.eps, self.hc, self.hmin
        if self.orientation is not None:
            c.use_orientation = 1
            c.ex, c.ey, c.ez = self.orientation
        c.precision = PRECISIONS[self.precision]
        c.device = self.device
        return c

    def to_kv(self, reference_only: bool = False) -> list[str]:
        """key=value strings the reference's Params::set accepts."""
        kv = [f"nx={self.NX}", f"ny={self.NY}", f"nz={self.NZ}", f"tau={_fmt(self.tau)}",
              f"lambda={_fmt(self.Lambda)}", f"fx={_fmt(self.Fx)}", f"fy={_fmt(self.Fy)}",
              f"fz={_fmt(self.Fz)}", f"walls_y={int(self.wallsY)}", f"walls_z={int(self.wallsZ)}",
              f"steps={self.steps}", f"print_every={self.printEvery}", f"vtk_every={self.vtkEvery}",
              f"traj_every={self.trajEvery}", f"tol={_fmt(self.tol)}",
              f"mass_correction_every={self.massCorrectionEvery}", f"output_dir={self.outputDir}",
              f"prefix={self.prefix}", f"squirmer={int(self.squirmer)}", f"radius={_fmt(self.R)}",
              f"b1={_fmt(self.B1)}", f"beta={_fmt(self.beta)}", f"rho_p={_fmt(self.rhoP)}",
              f"x0={_fmt(self.x0)}", f"y0={_fmt(self.y0)}", f"z0={_fmt(self.z0)}",
              f"angle={_fmt(self.angle)}", f"planar={int(self.planar)}", f"eps={_fmt(self.eps)}",
              f"hc={_fmt(self.hc)}", f"hmin={_fmt(self.hmin)}"]
        if not reference_only:
            kv.append(f"precision={self.precision}")
            if self.orientation is not None:
                kv += [f"ex={_fmt(self.orientation[0])}", f"ey={_fmt(self.orientation[1])}",
                       f"ez={_fmt(self.orientation[2])}"]
            if self.checkpoint_every:
                kv.append(f"checkpoint_every={self.checkpoint_every}")
            if self.restart:
                kv.append(f"restart={self.restart}")
        return kv


def _fmt(v) -> str:
    if isinstance(v, bool):
        return str(int(v))
    if isinstance(v, float):
        return repr(v)  # round-trips exactly through strtod
    return str(v)
