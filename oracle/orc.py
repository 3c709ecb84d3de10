"""ctypes bindings for the checker libraries (test infrastructure only).

* ``Oracle``  -- oracle/liboracle.so, the FP64 C restatement of the
  reference's LB + k-omega time step (oracle/kofm_oracle.c).
* ``RefKernels`` -- oracle/_ref/libkofm_ref.so, the reference's OWN kernel
  sources (source/Kernels/*.cl) compiled for the CPU by oracle/Makefile.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Arrays use the reference layout: node (i, j) at i + nxf*j,
population q at node + q*nxf*ny.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libkofm_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i16 = np.ctypeslib.ndpointer(dtype=np.int16, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

OPTION_SAVE_MACRO_FIELDS = 0x2
M_SOLID = 0x0001
M_FLUID = 0x0002
SOLID_BOUNDARY = 0x0010
NESW_BOUNDARY = 0x0F00


def build(force: bool = False) -> None:
    """Build liboracle.so and (when the reference tree is mounted) _ref."""
    if force or not os.path.exists(LIB_ORACLE) or (
        os.path.exists(os.path.join(HERE, "..", "..", "reference"))
    ):
        pass
    subprocess.run(["make", "-s", "-C", HERE, "CXX=g++", "CC=gcc"], check=True)


class _Cfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("nxf", C.c_int), ("ny", C.c_int),
        ("tau0", C.c_double), ("fterm", C.c_double), ("mu", C.c_double),
        ("max_turb_visc", C.c_double),
    ]


class GmresStats(C.Structure):
    _fields_ = [
        ("iters", C.c_int), ("restarts", C.c_int), ("nan", C.c_int),
        ("rho0", C.c_double), ("norm_rhs", C.c_double), ("prev_err", C.c_double),
    ]


class KOmegaState(C.Structure):
    _fields_ = [
        ("steps_per_lb", C.c_int), ("time_since_change", C.c_int),
        ("dt", C.c_double), ("max_iters", C.c_int),
        ("rel_tol", C.c_double), ("abs_tol", C.c_double),
        ("last_k", GmresStats), ("last_o", GmresStats),
    ]


def make_cfg(nx, ny, tau0, fterm, mu, max_turb_visc=10.0, nxf=None) -> _Cfg:
    return _Cfg(nx, nxf or nx, ny, tau0, fterm, mu, max_turb_visc)


class Oracle:
    def __init__(self, path: str = LIB_ORACLE):
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self.L = L
        cp = C.POINTER(_Cfg)
        L.orc_feq.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        L.orc_collide_push.argtypes = [cp, _dp, _dp, _i16, _dp, _dp, _dp, _dp,
                                       _dp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.orc_ibb.argtypes = [cp, _i32, _dp, _dp, C.c_int]
        L.orc_macro.argtypes = [cp, _dp, _i16, _dp, _dp, _dp]
        L.orc_komega_diffusivities.argtypes = [cp, _i16, _dp, _dp, _dp, _dp,
                                               _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_komega_coeffs.argtypes = [cp, _i32, _dp, _dp, _dp, _dp, _dp, _dp,
                                        _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                        _dp, _dp, _dp, _i16, C.c_double]
        L.orc_csr_build.argtypes = [cp, _i16, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_csr_build.restype = C.c_int
        L.orc_csr_fill_solid_boundary.argtypes = [cp, _i16, _i32, _dp]
        L.orc_gmres_solve.argtypes = [C.c_int, _i32, _i32, _dp, _dp, _dp, C.c_int,
                                      C.c_int, C.c_double, C.c_double,
                                      C.POINTER(GmresStats)]
        L.orc_komega_solve.argtypes = [cp, C.POINTER(KOmegaState), _i16, _i32,
                                       _i32, _i32, _dp, _dp, _dp, _dp, _dp, _dp,
                                       _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                       _dp, _dp, _dp]
        L.orc_geom_straight.argtypes = [cp, _i16, _dp, _dp]
        L.orc_sum.argtypes = [_dp, C.c_int64]
        L.orc_sum.restype = C.c_double
        L.orc_min.argtypes = [_dp, C.c_int64]
        L.orc_min.restype = C.c_double

    # thin wrappers -------------------------------------------------------
    def feq(self, rho, ux, uy):
        out = np.zeros(9)
        self.L.orc_feq(rho, ux, uy, out)
        return out

    def geom_straight(self, cfg):
        n = cfg.nxf * cfg.ny
        m = np.zeros(n, np.int16)
        dX = np.zeros(4 * n)
        wd = np.zeros(n)
        self.L.orc_geom_straight(C.byref(cfg), m, dX, wd)
        return m, dX, wd

    def csr(self, cfg, m):
        n = cfg.nxf * cfg.ny
        nnz = self.L.orc_csr_build(C.byref(cfg), m, None, None, None)
        IA = np.zeros(n + 1, np.int32)
        JA = np.zeros(nnz, np.int32)
        ind = np.zeros(5 * n, np.int32)
        self.L.orc_csr_build(C.byref(cfg), m, IA.ctypes.data, JA.ctypes.data,
                             ind.ctypes.data)
        return IA, JA, ind


class RefKernels:
    """The reference's kernels compiled for the CPU (oracle/_ref)."""

    def __init__(self, path: str = LIB_REF):
        L = C.CDLL(path)
        self.L = L
        cp = C.POINTER(_Cfg)
        L.ref_collide_komega.argtypes = [cp, _dp, _dp, _dp, _dp, _dp, _i16, _dp,
                                         _dp, _dp, _dp, _dp, C.c_int]
        L.ref_collide_laminar.argtypes = [cp, _dp, _dp, _dp, _dp, _dp, _i16, C.c_int]
        L.ref_ibb.argtypes = [cp, _i32, _dp, _dp, C.c_int]
        L.ref_calc_ro_j.argtypes = [cp, _dp, _dp, _dp, _dp, _i16]
        L.ref_komega_diffusivities.argtypes = [cp, _i16, _dp, _dp, _dp, _dp, _dp,
                                               _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_komega_coeffs.argtypes = [cp, _i32, _dp, _dp, _dp, _dp, _dp, _dp,
                                        _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                        _dp, _dp, _dp, _i16, C.c_double, _dp]

    @staticmethod
    def available(path: str = LIB_REF) -> bool:
        return os.path.exists(path)
