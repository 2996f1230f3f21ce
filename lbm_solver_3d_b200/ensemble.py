"""Ensembles of independent lattices advanced together (lbmgpu_batch_* of
include/lbmgpu.h).

The reference runs one lattice per process (src/main.cpp); a parameter study
there is one process per case (postprocessing/lbm_post.py:39-56). ``Ensemble``
holds many cases on one GPU and advances all of them with one persistent bulk
launch, one zone launch and one squirmer launch per time step, captured in
CUDA graphs. Each member computes exactly what ``Solver(params).run(n)``
computes for it alone; ``member(i)`` returns a read-only ``Solver`` view for
its squirmer state, trajectory rows, fields and diagnostics.
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import LbmgpuParams, check_batch
from .params import Params
from .solver import Solver


def shard_members(members: list[Params], rank: int, world: int) -> list[int]:
    """Indices of the members that rank `rank` of `world` runs: the members are
    independent, so a multi-GPU ensemble splits them across ranks with no
    exchange. Largest first, each to the rank with the fewest nodes so far
    (ties to the lower rank): every rank computes the same assignment."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(members)), key=lambda i: (-members[i].ncells, i))
    load = [0] * world
    owner = {}
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += members[i].ncells
    return sorted(i for i in range(len(members)) if owner[i] == rank)


class Ensemble:
    def __init__(self, members: list[Params], autotune: bool = False, tune_reps: int = 5):
        if not members:
            raise ValueError("an ensemble needs at least one member")
        for p in members:
            p.validate()
        self.params = list(members)
        self.lib = _lib.load()
        arr = (LbmgpuParams * len(members))(*[p.to_c() for p in members])
        b = ctypes.c_void_p()
        check_batch(self.lib.lbmgpu_batch_create(arr, len(members), ctypes.byref(b)), None)
        self.b = b
        self._views: dict[int, Solver] = {}
        self.tiling = None
        if autotune:
            self.autotune(tune_reps)

    def __len__(self) -> int:
        return len(self.params)

    @property
    def cells(self) -> int:
        n = ctypes.c_int()
        c = ctypes.c_longlong()
        check_batch(self.lib.lbmgpu_batch_size(self.b, ctypes.byref(n), ctypes.byref(c)), self.b)
        return c.value

    def run(self, nsteps: int) -> None:
        check_batch(self.lib.lbmgpu_batch_run(self.b, int(nsteps)), self.b)

    def member(self, i: int) -> Solver:
        if i not in self._views:
            h = ctypes.c_void_p()
            check_batch(self.lib.lbmgpu_batch_member(self.b, int(i), ctypes.byref(h)), self.b)
            self._views[i] = Solver._member(self.params[i], h, self)
        return self._views[i]

    STAGED2, STAGED3 = -2, -3

    def set_tiling(self, tile: int, ctas_per_sm: int) -> None:
        """tile 32/64/128: threads per row of the row kernel; 1: one CTA per
        row; 2 / 3: 32-node chunks (3: persistent warps); 4: staged row runs;
        -3 / -4: the staged kernel with 3 / 4 shared-memory stages
        (include/lbmgpu.h, LBMGPU_TILE_*)."""
        check_batch(self.lib.lbmgpu_batch_set_tiling(self.b, int(tile), int(ctas_per_sm)), self.b)
        self.tiling = (tile, ctas_per_sm)

    def autotune(self, reps: int = 5) -> dict:
        """Chooses the bulk launch's tiling by timing every candidate; the
        members' populations are restored afterwards."""
        tx, bps = ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_double()
        check_batch(self.lib.lbmgpu_batch_autotune(self.b, int(reps), ctypes.byref(tx), ctypes.byref(bps),
                                                   ctypes.byref(ms)), self.b)
        self.tiling = (tx.value, bps.value)
        return dict(tile=tx.value, ctas_per_sm=bps.value, ms=ms.value)

    def time_bulk(self, reps: int = 10) -> float:
        ms = ctypes.c_double()
        check_batch(self.lib.lbmgpu_batch_time_bulk(self.b, int(reps), ctypes.byref(ms)), self.b)
        return ms.value

    def set_stream(self, stream_handle: int | None) -> None:
        check_batch(self.lib.lbmgpu_batch_set_stream(self.b, ctypes.c_void_p(stream_handle or 0)), self.b)

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        check_batch(self.lib.lbmgpu_batch_launch_count(self.b, ctypes.byref(v)), self.b)
        return v.value

    def close(self) -> None:
        if getattr(self, "b", None):
            for v in self._views.values():
                v.h = None
            self._views.clear()
            self.lib.lbmgpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def main(argv=None) -> None:
    """Run the first --members members of ensemble_members(256) for --steps
    steps with a given bulk tiling (used for profiling):
        python -m lbm_solver_3d_b200.ensemble --members 64 --steps 61 --tile 2"""
    import argparse
    from .workloads import ensemble_members
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--steps", type=int, default=61)
    ap.add_argument("--tile", type=int, default=2)
    ap.add_argument("--ctas-per-sm", type=int, default=1)
    ap.add_argument("--precision", default="fp32")
    args = ap.parse_args(argv)
    ps = ensemble_members(256)[: args.members]
    for p in ps:
        p.update(precision=args.precision)
    with Ensemble(ps) as ens:
        ens.set_tiling(args.tile, args.ctas_per_sm)
        ens.run(args.steps)
        print(f"{len(ps)} members, {ens.cells} nodes, {args.steps} steps, tile {args.tile}: ok")


if __name__ == "__main__":
    main()
