"""Generates tests/golden/ref_shear.npz from the reference's own shear kernels.

Runs oracle/_ref/libkofm_ref.so (source/Kernels/trKernelsShear.cl of the
reference compiled for the CPU by oracle/Makefile) on a small wavy channel:
TR_Find_Shear_Coeffs1 on the shear-node list, then TR_shear_1 on a seeded
near-equilibrium state with and without an eddy viscosity.  Only the values at
the shear nodes are stored (the kernels read nothing else).

    make -C oracle && python tests/golden/make_golden_shear.py
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from komegafoulingmodel_b200 import geometry as G  # noqa: E402
from komegafoulingmodel_b200 import shear  # noqa: E402
from oracle.orc import RefKernels, make_cfg  # noqa: E402
from tests.cases import komega_state, perturbed_state  # noqa: E402

NX, NY, AMP, WAVELEN = 64, 24, 4.0, 32
TAU, FTERM, MU = 1.9, 1e-5, 0.01


def state(ch):
    F = perturbed_state(ch, seed=21, u_mean=0.02)
    _, _, nut, _ = komega_state(ch, seed=22)
    rng = np.random.default_rng(23)
    fl = ch.fluid_mask().ravel()
    rho = np.where(fl, 1.0 + 1e-3 * rng.standard_normal(ch.n), 0.0)
    ux = np.where(fl, 0.02 + 1e-2 * rng.standard_normal(ch.n), 0.0)
    uy = np.where(fl, 5e-3 * rng.standard_normal(ch.n), 0.0)
    return F, rho, ux, uy, nut


def main():
    ch = G.wavy_channel(NX, NY, AMP, WAVELEN)
    cfg = make_cfg(NX, NY, TAU, FTERM, MU)
    nodes, _ = shear.shear_nodes(ch)
    n = len(nodes)
    R = RefKernels()
    cfss = np.zeros(16 * n)
    R.L.ref_shear_coeffs1(C.byref(cfg), nodes, ch.ntype, cfss, n, shear.CUTOFF_RADIUS)
    F, rho, ux, uy, nut = state(ch)
    out = dict(nx=NX, ny=NY, amp=AMP, wavelength=WAVELEN, tau=TAU, fterm=FTERM, mu=MU,
               nodes=nodes, cfss=cfss.reshape(n, 16),
               F=F.reshape(9, -1)[:, nodes].T.copy(), rho=rho[nodes], ux=ux[nodes],
               uy=uy[nodes], nut=nut[nodes])
    for tag, nu in (("lam", np.zeros(ch.n)), ("turb", nut)):
        tau = np.zeros(n)
        R.L.ref_wall_shear_nodes(C.byref(cfg), rho, ux, uy, cfss, F.copy(), tau, nodes, nu, n)
        out[f"tau_{tag}"] = tau
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_shear.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
