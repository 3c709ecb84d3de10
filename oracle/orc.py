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


def build() -> None:
    """Builds liboracle.so and, when the reference tree is mounted, _ref."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


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
        ("fail_solves", C.c_int), ("fail_mask", C.c_int),
    ]


class ThermalCfg(C.Structure):
    _fields_ = [("alpha_fluid", C.c_double), ("alpha_foul", C.c_double),
                ("pr_turb_inv", C.c_double), ("t_in", C.c_double)]


class BicgStats(C.Structure):
    _fields_ = [("iters", C.c_int), ("checks", C.c_int), ("conv", C.c_int), ("reset", C.c_int),
                ("residual", C.c_double), ("initial_residual", C.c_double)]


class ThermalState(C.Structure):
    _fields_ = [("steps_per_lb", C.c_int), ("time_since_change", C.c_int),
                ("dt", C.c_double), ("max_iters", C.c_int),
                ("rel_tol", C.c_double), ("abs_tol", C.c_double),
                ("solves", C.c_int), ("resets", C.c_int), ("last", BicgStats)]


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
        L.orc_wall_shear_nodes.argtypes = [cp, _dp, _dp, _dp, _dp, C.c_void_p, _i32, C.c_int,
                                           _dp, _dp]
        L.orc_wall_shear_links.argtypes = [_dp, _i32, _dp, C.c_int, _dp]
        L.orc_csr_build_thermal.argtypes = [cp, _i16, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_csr_build_thermal.restype = C.c_int
        L.orc_csr_fill_solid_boundary_thermal.argtypes = [cp, _i16, _i32, _dp]
        tp = C.POINTER(ThermalCfg)
        L.orc_thermal_coeffs.argtypes = [cp, tp, _i32, _i16, _dp, _dp, _dp, _dp, _dp, _dp,
                                         C.c_void_p, C.c_double]
        L.orc_bicgstab_solve.argtypes = [C.c_int, _i32, _i32, _dp, _dp, _dp, C.c_int, C.c_double,
                                         C.c_double, C.c_int, C.POINTER(BicgStats)]
        L.orc_thermal_solve.argtypes = [cp, tp, C.POINTER(ThermalState), _i16, _i32, _i32, _i32,
                                        _dp, _dp, _dp, _dp, _dp, C.c_void_p, _dp, _dp]
        L.orc_adj_collide.argtypes = [cp, _i16, _dp, _dp]
        L.orc_adj_stream.argtypes = [cp, _i16, _i32, _dp, C.c_int, _dp, _dp]
        L.orc_adj_stream_T.argtypes = [cp, _i16, _i32, _dp, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_adj_j.argtypes = [cp, _i16, _dp, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.orc_adj_j.restype = C.c_double
        L.orc_adj_run.argtypes = [cp, _i16, _i32, _dp, C.c_int, _dp, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_adj_run.restype = C.c_double
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

    def csr_thermal(self, cfg, m):
        """CSR_Inds (non-periodic) with the thermal flags."""
        n = cfg.nxf * cfg.ny
        nnz = self.L.orc_csr_build_thermal(C.byref(cfg), m, None, None, None)
        IA = np.zeros(n + 1, np.int32)
        JA = np.zeros(nnz, np.int32)
        ind = np.zeros(5 * n, np.int32)
        self.L.orc_csr_build_thermal(C.byref(cfg), m, IA.ctypes.data, JA.ctypes.data,
                                     ind.ctypes.data)
        return IA, JA, ind


def adj_run(orc, cfg, ch, FA0, T, q=None, shear_setup=None, want_dF0=False):
    """orc_adj_run: (J, dJ/dq per IBB entry, dJ/dFA0 or None)."""
    q = np.ascontiguousarray(ch.ibb_q if q is None else q, np.float64)
    ibb = np.ascontiguousarray(ch.ibb_idx, np.int32)
    dq = np.zeros(len(ibb))
    dF0 = np.zeros_like(FA0) if want_dF0 else None
    if shear_setup is not None:
        sn = np.ascontiguousarray(shear_setup.nodes, np.int32)
        cf = np.ascontiguousarray(shear_setup.cfss.ravel(), np.float64)
        sp, cpp, ns = sn.ctypes.data, cf.ctypes.data, len(sn)
    else:
        sn = cf = None
        sp = cpp = None
        ns = 0
    J = orc.L.orc_adj_run(C.byref(cfg), np.ascontiguousarray(ch.ntype, np.int16), ibb, q, len(ibb),
                          np.ascontiguousarray(FA0, np.float64), T, sp, cpp, ns,
                          dq.ctypes.data if len(dq) else None,
                          dF0.ctypes.data if dF0 is not None else None)
    del sn, cf
    return J, dq, dF0


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
        if hasattr(L, "ref_thermal_coeffs"):
            L.ref_thermal_coeffs.argtypes = [cp, _dp, _i32, _i16, _dp, _dp, _dp, _dp, _dp, _dp,
                                             _dp, C.c_double]
        if hasattr(L, "ref_wall_shear_nodes"):
            L.ref_wall_shear_nodes.argtypes = [cp, _dp, _dp, _dp, _dp, _dp, _dp, _i32, _dp, C.c_int]
            L.ref_shear_coeffs1.argtypes = [cp, _i32, _i16, _dp, C.c_int, C.c_double]
        if hasattr(L, "ref_update_node_boundary_info"):
            L.ref_update_node_boundary_info.argtypes = [cp, _i16]
        if hasattr(L, "ref_ini_dx"):
            L.ref_ini_dx.argtypes = [_dp, C.c_int, _i32, C.c_int, _i16, C.c_int, C.c_int, C.c_int,
                                     C.c_double, _dp, _dp]
        if hasattr(L, "ref_ini_lsmap"):
            L.ref_ini_lsmap.argtypes = [_dp, _i32, C.c_int, C.c_int, C.c_int,
                                        np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")]
        if hasattr(L, "ref_update_walld"):
            L.ref_update_walld.argtypes = [cp, _dp, C.c_int,
                                           np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS"),
                                           _i16, _dp, C.c_int]
        if hasattr(L, "ref_update_ibb_only"):
            L.ref_update_ibb_only.argtypes = [cp, _dp, C.c_int, _i16, _i32, _dp, C.c_int,
                                              C.POINTER(C.c_int)]

    @staticmethod
    def wall_points(nx, y_bot, y_top):
        """The reference's polyline layout for walls through (x, y_w[x]),
        x = -1 .. nx (periodic heights): bottom wall left to right, then top
        wall right to left."""
        xs = np.arange(-1, nx + 1)
        bot = np.column_stack([xs, np.asarray(y_bot)[xs % nx]])
        top = np.column_stack([xs[::-1], np.asarray(y_top)[xs[::-1] % nx]])
        return np.ascontiguousarray(np.vstack([bot, top]), np.float64)

    def wall_distance(self, cfg, ntype, y_bot, y_top, radius=50):
        """The reference's updateWallD on walls laid out as wall_points, each
        column mapped to the segment that starts at it."""
        nx, nxf = cfg.nx, cfg.nxf
        pts = self.wall_points(nx, y_bot, y_top)
        n2 = len(pts) // 2
        lsmap = np.zeros((2, nxf), np.uint16)
        lsmap[0, :nx] = np.arange(nx) + 1                 # bottom segment from x = i
        lsmap[1, :nx] = n2 + (nx - 1 - np.arange(nx))     # top segment from x = i + 1 to x = i
        return self.wall_distance_pts(cfg, ntype, pts, lsmap, radius)

    def wall_distance_pts(self, cfg, ntype, pts, lsmap, radius=50):
        """updateWallD on the polyline pts (the reference's point order) with
        the column map lsmap [2][nx] (entries as the kernel uses them)."""
        nx, nxf, ny = cfg.nx, cfg.nxf, cfg.ny
        lm = np.zeros((2, nxf), np.uint16)
        lm[:, :nx] = np.asarray(lsmap)[:, :nx]
        wd = np.zeros(nxf * ny)
        self.L.ref_update_walld(C.byref(cfg), np.ascontiguousarray(pts, np.float64).ravel(), len(pts), lm.ravel(),
                                np.ascontiguousarray(ntype, np.int16), wd, radius)
        return wd

    def ls_map(self, pts, segs, nx, nxf):
        """clVariablesLS::iniLSMap on points pts and segments segs (the
        lsc0 / lsbl tables): [2][nxf] segment index per column and wall."""
        m = np.zeros((2, nxf), np.uint16)
        self.L.ref_ini_lsmap(np.ascontiguousarray(pts, np.float64).ravel(),
                             np.ascontiguousarray(segs, np.int32).ravel(), len(segs), nx, nxf, m)
        return m

    def link_fractions(self, cfg, ntype, pts, segs, min_dx=0.001):
        """The reference's host set-up of dXArr and dXArr0 (bcFindNodes over
        every segment) for points pts and segments segs: two [4][nxf*ny]."""
        n = cfg.nxf * cfg.ny
        dx, dx0 = np.zeros(4 * n), np.zeros(4 * n)
        self.L.ref_ini_dx(np.ascontiguousarray(pts, np.float64).ravel(), len(pts),
                          np.ascontiguousarray(segs, np.int32).ravel(), len(segs),
                          np.ascontiguousarray(ntype, np.int16), cfg.nx, cfg.nxf, cfg.ny, min_dx, dx, dx0)
        return dx, dx0

    def ibb_list_pts(self, cfg, ntype, pts, cap=1 << 20):
        """updateIBBOnly on the polyline pts (the reference's point order)."""
        pts = np.ascontiguousarray(pts, np.float64)
        ibb = np.zeros(cap, np.int32)
        dist = np.zeros(cap)
        n = C.c_int()
        self.L.ref_update_ibb_only(C.byref(cfg), pts.ravel(), len(pts),
                                   np.ascontiguousarray(ntype, np.int16), ibb, dist, cap, C.byref(n))
        if n.value > cap:
            raise RuntimeError("reference link list larger than cap")
        return ibb[:n.value], dist[:n.value]

    def ibb_list(self, cfg, ntype, y_bot, y_top, cap=1 << 20):
        """The reference's interpolated-link list (updateIBBOnly) for walls
        through (x, y_w[x]), x = -1 .. nx (periodic heights): (population
        index, wall fraction) in the builder's order, duplicates kept."""
        return self.ibb_list_pts(cfg, ntype, self.wall_points(cfg.nx, y_bot, y_top), cap)

    @staticmethod
    def available(path: str = LIB_REF) -> bool:
        return os.path.exists(path)


class OracleSim:
    """FP64 CPU run of the reference step loop (Solve_no_TR, LBLS.cpp:185-205):
    collide + push (LB_collision_SRT_Fluid[_w_kOmega]), lbIBB, then
    kOmega::Solve (diffusivities, coefficients, GMRES for omega then k).

    State arrays use the reference layout; ``f`` is the FA buffer."""

    def __init__(self, orc: Oracle, cfg, ntype, dX, wallD, f, k=None, omega=None,
                 nut=None, sxy=None, komega=False, ibb_idx=None, ibb_q=None,
                 max_iters=1000, rel_tol=1e-4, abs_tol=1e-7, dt=1.0, thermal=None):
        self.o, self.cfg, self.komega = orc, cfg, komega
        n = cfg.nxf * cfg.ny
        self.n = n
        self.m = np.ascontiguousarray(ntype, np.int16)
        self.dX = np.ascontiguousarray(dX, np.float64)
        self.wallD = np.ascontiguousarray(wallD, np.float64)
        self.FA = np.ascontiguousarray(f, np.float64).copy()
        self.FB = np.zeros_like(self.FA)
        self.rho, self.ux, self.uy = np.zeros(n), np.zeros(n), np.zeros(n)
        z = np.zeros(n)
        self.K = z.copy() if k is None else np.array(k, np.float64)
        self.O = z.copy() if omega is None else np.array(omega, np.float64)
        self.nut = z.copy() if nut is None else np.array(nut, np.float64)
        self.S = np.zeros(3 * n) if sxy is None else np.array(sxy, np.float64)
        self.ibb_idx = np.zeros(0, np.int32) if ibb_idx is None else np.ascontiguousarray(ibb_idx, np.int32)
        self.ibb_q = np.zeros(0) if ibb_q is None else np.ascontiguousarray(ibb_q, np.float64)
        if komega:
            self.IA, self.JA, self.ind = orc.csr(cfg, self.m)
            nnz = len(self.JA)
            self.kA, self.oA = np.zeros(nnz), np.zeros(nnz)
            orc.L.orc_csr_fill_solid_boundary(C.byref(cfg), self.m, self.ind, self.kA)
            orc.L.orc_csr_fill_solid_boundary(C.byref(cfg), self.m, self.ind, self.oA)
            self.kb, self.ob = np.zeros(n), np.zeros(n)
            self.Dk = np.where((self.m & M_FLUID) != 0, cfg.mu, 0.0)
            self.Do = self.Dk.copy()
            self.F1 = np.zeros(n)
            self.dkdo = np.zeros(2 * n)
            self.kst = KOmegaState(1, 0, dt, max_iters, rel_tol, abs_tol)
        # thermal: dict(T=..., cfg=ThermalCfg, dX0=..., max_iters, rel_tol, abs_tol, dt,
        # every=LB steps per thermal solve)
        self.thermal = thermal
        if thermal is not None:
            self.T = np.array(thermal["T"], np.float64)
            self.Tprev = np.zeros(n)
            self.tcfg = thermal["cfg"]
            self.dX0 = np.ascontiguousarray(thermal.get("dX0", self.dX), np.float64)
            self.tIA, self.tJA, self.tind = orc.csr_thermal(cfg, self.m)
            self.tA = np.zeros(len(self.tJA))
            orc.L.orc_csr_fill_solid_boundary_thermal(C.byref(cfg), self.m, self.tind, self.tA)
            self.tb = np.zeros(n)
            self.tst = ThermalState(1, 0, thermal.get("dt", 1.0), thermal.get("max_iters", 1000),
                                    thermal.get("rel_tol", 1e-4), thermal.get("abs_tol", 1e-7))
            self.t_every = thermal.get("every", 1)
            self.time_n = 0

    def step(self, nsteps=1, options=OPTION_SAVE_MACRO_FIELDS):
        L, cp = self.o.L, C.byref(self.cfg)
        opt = options | (OPTION_SAVE_MACRO_FIELDS if self.komega or self.thermal is not None else 0)
        for _ in range(nsteps):
            L.orc_collide_push(cp, self.FA, self.FB, self.m, self.rho, self.ux, self.uy,
                               self.K, self.O, self.wallD, self.nut, self.S, opt,
                               1 if self.komega else 0)
            if len(self.ibb_idx):
                L.orc_ibb(cp, self.ibb_idx, self.ibb_q, self.FB, len(self.ibb_idx))
            self.FA, self.FB = self.FB, self.FA
            if self.komega:
                self.komega_solve()
            if self.thermal is not None:
                if self.time_n % self.t_every == 0:
                    self.thermal_solve()
                self.time_n += 1

    def komega_solve(self):
        L, cp = self.o.L, C.byref(self.cfg)
        L.orc_komega_solve(cp, C.byref(self.kst), self.m, self.IA, self.JA, self.ind,
                           self.K, self.O, self.nut, self.wallD, self.rho, self.ux,
                           self.uy, self.S, self.dX, self.Dk, self.Do, self.F1,
                           self.dkdo, self.kA, self.oA, self.kb, self.ob)

    def thermal_solve(self):
        L, cp = self.o.L, C.byref(self.cfg)
        L.orc_thermal_solve(cp, C.byref(self.tcfg), C.byref(self.tst), self.m, self.tIA,
                            self.tJA, self.tind, self.dX0, self.T, self.Tprev, self.ux, self.uy,
                            self.nut.ctypes.data if self.komega else None, self.tA, self.tb)
