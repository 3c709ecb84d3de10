"""Generates tests/golden/ref_ibb.npz from the reference's own geometry kernels.

Runs oracle/_ref/libkofm_ref.so (updateIBBOnly and bcFindIntersectionLS of the
reference's source/Kernels/lsKernels.cl, updateWallD of kOmegaKernels.cl,
compiled for the CPU by oracle/Makefile) on two walls given as polylines
through one point per column: the interpolated bounce-back list (population
index, wall fraction) in the builder's order, duplicates included, and the
wall distance of every node.

    make -C oracle && python tests/golden/make_golden_ibb.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from komegafoulingmodel_b200 import geometry as G  # noqa: E402
from oracle.orc import RefKernels, make_cfg  # noqa: E402

NX, NY = 256, 66


def walls(name):
    x = np.arange(NX)
    if name == "wavy":    # flat at the seam, amplitude 8, wavelength 100
        h = 8.0 * 0.5 * (1 - np.cos(2 * np.pi * x / 100))
        return 0.5 + h, NY - 1.5 - h
    if name == "sine":    # a sine not aligned with the rows
        h = 4.0 * np.sin(2 * np.pi * x / 64) + 5.3
        return h, NY - 1 - h
    raise KeyError(name)


def main():
    rk = RefKernels()
    out = {}
    for name in ("wavy", "sine"):
        yb, yt = walls(name)
        ch = G.channel_from_walls(NX, NY, yb, yt, ibb_all=True)
        idx, dist = rk.ibb_list(make_cfg(NX, NY, 1.0, 0.0, 0.1), ch.ntype, yb, yt)
        out[f"{name}_yb"], out[f"{name}_yt"] = yb, yt
        out[f"{name}_ntype"] = ch.ntype
        out[f"{name}_idx"], out[f"{name}_dist"] = idx, dist
        out[f"{name}_walld"] = rk.wall_distance(make_cfg(NX, NY, 1.0, 0.0, 0.1), ch.ntype, yb, yt)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_ibb.npz")
    np.savez_compressed(path, nx=NX, ny=NY, **out)
    print("wrote", path, {k: v.shape for k, v in out.items() if k.endswith("_idx")})


if __name__ == "__main__":
    main()
