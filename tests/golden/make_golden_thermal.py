"""Generates tests/golden/ref_thermal.npz from the reference's own kernel.

Runs Update_T_Coeffs_Implicit (source/Kernels/tfdKernels.cl:122-279 of the
reference, compiled for the CPU by oracle/Makefile into oracle/_ref) on a small
seeded wavy channel with a k-omega eddy viscosity, and stores its inputs and
the CSR values and right-hand side it writes.

    make -C oracle && python tests/golden/make_golden_thermal.py
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from komegafoulingmodel_b200 import geometry as G  # noqa: E402
from oracle.orc import Oracle, RefKernels, make_cfg  # noqa: E402
from tests.cases import komega_state  # noqa: E402

NX, NY, AMP, WAVELEN = 40, 20, 3.0, 20
RATE, FTERM, MU = 1.3, 1e-5, 0.02
TH = (MU / 0.708, 0.004, 1 / 0.9, 2.0)   # alpha_fluid, alpha_foul, 1/Pr_t, T_in
DT = 0.7


def inputs(ch):
    rng = np.random.default_rng(31)
    n = ch.n
    fl = ch.fluid_mask().ravel()
    T = np.where(fl, 0.5 + 0.8 * rng.random(n), 0.0)
    T[fl & (rng.random(n) < 0.05)] = 2.5          # above the inlet clamp
    ux = np.where(fl, 0.03 + 0.01 * rng.standard_normal(n), 0.0)
    uy = np.where(fl, 0.005 * rng.standard_normal(n), 0.0)
    _, _, nut, _ = komega_state(ch, seed=32)
    return T, ux, uy, nut


def main():
    ch = G.wavy_channel(NX, NY, AMP, WAVELEN)
    cfg = make_cfg(NX, NY, RATE, FTERM, MU)
    IA, JA, ind = Oracle().csr_thermal(cfg, ch.ntype)
    T, ux, uy, nut = inputs(ch)
    A = np.zeros(len(JA))
    Oracle().L.orc_csr_fill_solid_boundary_thermal(C.byref(cfg), ch.ntype, ind, A)
    b = np.zeros(ch.n)
    RefKernels().L.ref_thermal_coeffs(C.byref(cfg), np.array(TH), ind, ch.ntype, ch.dX.copy(),
                                      A, b, T.copy(), ux.copy(), uy.copy(), nut.copy(), DT)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_thermal.npz")
    np.savez_compressed(path, nx=NX, ny=NY, amp=AMP, wavelength=WAVELEN, rate=RATE, fterm=FTERM,
                        mu=MU, th=np.array(TH), dt=DT, T=T, ux=ux, uy=uy, nut=nut, IA=IA, JA=JA,
                        A=A, b=b)
    print("wrote", path, "nnz", len(JA))


if __name__ == "__main__":
    main()
