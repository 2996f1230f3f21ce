"""Collect the reference's shipped result files into tests/golden/shipped.npz.

    python tests/golden/extract_shipped.py REFERENCE_ROOT

Reads (from the reference checkout given as the argument):
  outputs/duct_summary.txt, outputs/duct_profile_{y,z}.dat
  outputs/channel_{neutral,puller,pusher}_{summary.txt,squirmer.dat}
  outputs/channel_puller_traj.dat
  examples/reference_data/channel_{neutral,puller,pusher}_traj.dat
and stores their numbers (not the files) as arrays. The tests compare the
oracle and the CUDA path against them; nothing reads the reference at test time.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def keyvalue(path: Path) -> dict:
    out = {}
    for line in path.read_text().splitlines():
        tok = line.split()
        if tok:
            out[tok[0]] = np.array([float(v) for v in tok[1:]])
    return out


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_shipped.py REFERENCE_ROOT")
    ref = Path(sys.argv[1])
    arrays = {}
    for name in ("duct", "channel_neutral", "channel_puller", "channel_pusher"):
        for k, v in keyvalue(ref / "outputs" / f"{name}_summary.txt").items():
            arrays[f"{name}_summary_{k}"] = v
        if name != "duct":
            for k, v in keyvalue(ref / "outputs" / f"{name}_squirmer.dat").items():
                arrays[f"{name}_squirmer_{k}"] = v
    for ax in ("y", "z"):
        arrays[f"duct_profile_{ax}"] = np.loadtxt(ref / "outputs" / f"duct_profile_{ax}.dat")
    arrays["outputs_channel_puller_traj"] = np.loadtxt(ref / "outputs" / "channel_puller_traj.dat")
    for name in ("neutral", "puller", "pusher"):
        arrays[f"example_{name}_traj"] = np.loadtxt(ref / "examples" / "reference_data" / f"channel_{name}_traj.dat")
    np.savez_compressed(HERE / "shipped.npz", **arrays)
    print(f"wrote {HERE / 'shipped.npz'} ({len(arrays)} arrays)")


if __name__ == "__main__":
    main()
