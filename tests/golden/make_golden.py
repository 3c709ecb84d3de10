"""Generates tests/golden/ref_kernels.npz from the reference's own kernels.

Runs oracle/_ref/libkofm_ref.so (source/Kernels/*.cl of the reference compiled
for the CPU by oracle/Makefile) on a small seeded straight channel and stores
inputs and outputs of LB_collision_SRT_Fluid, LB_collision_SRT_Fluid_w_kOmega,
Update_kOmega_Diffusivities and Update_kOmega_Coeffs_Implicit.

    make -C oracle && python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from komegafoulingmodel_b200 import geometry as G  # noqa: E402
from oracle.orc import Oracle, RefKernels, make_cfg  # noqa: E402
from tests.cases import komega_state, perturbed_state  # noqa: E402


def main():
    nx, ny = 32, 12
    tau, fterm, mu = 1.9, 1e-5, 0.01
    cfg = make_cfg(nx, ny, tau, fterm, mu)
    ch = G.straight_channel(nx, ny)
    n = ch.n
    F = perturbed_state(ch, seed=11)
    K, O, nut, S = komega_state(ch, seed=12)
    R = RefKernels()
    out = dict(nx=nx, ny=ny, tau=tau, fterm=fterm, mu=mu, F=F, K=K, O=O, S=S)
    for komega in (0, 1):
        FB = np.zeros(9 * n)
        rho, ux, uy, nt = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        k, o, s = K.copy(), O.copy(), S.copy()
        if komega:
            R.L.ref_collide_komega(C.byref(cfg), rho, ux, uy, F.copy(), FB, ch.ntype,
                                   ch.wallD, nt, k, o, s, 2)
        else:
            R.L.ref_collide_laminar(C.byref(cfg), rho, ux, uy, F.copy(), FB, ch.ntype, 2)
        for key, v in dict(FB=FB, rho=rho, ux=ux, uy=uy, nut=nt, K=k, O=o, S=s).items():
            out[f"{key}_{komega}"] = v
    # k-omega assembly on the k-omega collide outputs
    IA, JA, ind = Oracle().csr(cfg, ch.ntype)
    nnz = len(JA)
    Dk, Do, F1, dk = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(2 * n)
    kA, oA, kb, ob = np.zeros(nnz), np.zeros(nnz), np.zeros(n), np.zeros(n)
    dbg = np.zeros(40 * n)
    k1, o1 = out["K_1"].copy(), out["O_1"].copy()
    R.L.ref_komega_diffusivities(C.byref(cfg), ch.ntype, k1, o1, out["nut_1"], ch.wallD,
                                 Dk, Do, F1, dk, out["rho_1"], ch.dX, dbg)
    R.L.ref_komega_coeffs(C.byref(cfg), ind, k1, o1, out["nut_1"], Dk, Do, F1, dk,
                          out["S_1"], out["rho_1"], out["ux_1"], out["uy_1"], kA, oA,
                          kb, ob, ch.dX, ch.wallD, ch.ntype, 1.0, dbg)
    out.update(Dk=Dk, Do=Do, F1=F1, dkdo=dk, kA=kA, oA=oA, kb=kb, ob=ob)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_kernels.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
