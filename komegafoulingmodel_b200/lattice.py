"""Python handle on one kofm context (one lattice on one GPU).

A thin wrapper over the C ABI (include/kofm.h): numpy arrays in the
reference's padded FP64 layout go in and out; the state lives on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import KofmDesc, KofmStats, check

_dp = C.POINTER(C.c_double)


def _ptr(a, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def desc_default() -> KofmDesc:
    lib = _abi.load()
    d = KofmDesc()
    check("kofm_desc_default", lib.kofm_desc_default(C.byref(d)))
    return d


class Lattice:
    """Device-resident D2Q9 (+ k-omega) lattice driven through the C ABI."""

    def __init__(self, desc: KofmDesc):
        self.lib = _abi.load()
        self.desc = desc
        self._ctx = C.c_void_p()
        check("kofm_create", self.lib.kofm_create(C.byref(desc), C.byref(self._ctx)))
        self.nxf, self.ny = desc.nx_full, desc.ny
        self.n = self.nxf * self.ny

    # -- lifecycle ------------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.kofm_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- geometry / state ---------------------------------------------------------
    def set_geometry(self, ntype, wallD=None, dX=None, ibb_idx=None, ibb_q=None):
        ntype = np.ascontiguousarray(ntype, np.int16)
        wallD = None if wallD is None else np.ascontiguousarray(wallD, np.float64)
        dX = None if dX is None else np.ascontiguousarray(dX, np.float64)
        n_ibb = 0 if ibb_idx is None else len(ibb_idx)
        ii = None if ibb_idx is None else np.ascontiguousarray(ibb_idx, np.int32)
        qq = None if ibb_q is None else np.ascontiguousarray(ibb_q, np.float64)
        check("kofm_set_geometry", self.lib.kofm_set_geometry(
            self._ctx, _ptr(ntype, C.c_int16), _ptr(wallD), _ptr(dX),
            _ptr(ii, C.c_int32), _ptr(qq), n_ibb))
        self._n_ibb = n_ibb

    def set_walls(self, y_bot, y_top, y_bot0=None, y_top0=None, ibb_all=False, seam_ibb=False,
                  min_dx=0.001, wall_radius=50):
        """Geometry built on the device from the wall heights at every column
        (kofm_set_walls): what geometry.channel_from_walls builds on the host,
        plus, with the thermal update, the unfouled-wall fractions."""
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64)
                for a in (y_bot, y_top, y_bot0, y_top0)]
        for a in arrs:
            if a is not None and a.shape != (self.desc.nx,):
                raise ValueError("wall heights need one value per column")
        check("kofm_set_walls", self.lib.kofm_set_walls(
            self._ctx, *[_ptr(a) for a in arrs], float(min_dx), int(wall_radius),
            (_abi.WALLS_IBB_ALL if ibb_all else 0) | (_abi.WALLS_SEAM_IBB if seam_ibb else 0)))
        n = C.c_int32()
        check("kofm_get_geometry", self.lib.kofm_get_geometry(
            self._ctx, None, None, None, None, None, None, 0, C.byref(n)))
        self._n_ibb = n.value

    def get_geometry(self):
        """The context's geometry in the host layout: dict with ntype, dX,
        ibb_idx, ibb_q, and wallD (k-omega) / dX0 (thermal) (kofm_get_geometry)."""
        d = self.desc
        n = C.c_int32()
        check("kofm_get_geometry", self.lib.kofm_get_geometry(
            self._ctx, None, None, None, None, None, None, 0, C.byref(n)))
        out = dict(ntype=np.empty(self.n, np.int16), dX=np.empty(4 * self.n),
                   ibb_idx=np.empty(max(n.value, 1), np.int32), ibb_q=np.empty(max(n.value, 1)))
        out["wallD"] = np.empty(self.n) if d.use_komega else None
        out["dX0"] = np.empty(4 * self.n) if d.use_thermal else None
        check("kofm_get_geometry", self.lib.kofm_get_geometry(
            self._ctx, _ptr(out["ntype"], C.c_int16), _ptr(out["wallD"]), _ptr(out["dX"]),
            _ptr(out["dX0"]), _ptr(out["ibb_idx"], C.c_int32), _ptr(out["ibb_q"]),
            len(out["ibb_idx"]), C.byref(n)))
        out["ibb_idx"], out["ibb_q"] = out["ibb_idx"][:n.value], out["ibb_q"][:n.value]
        return out

    def set_state(self, f, k=None, omega=None, nut=None, sxy=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64)
                for a in (f, k, omega, nut, sxy)]
        check("kofm_set_state", self.lib.kofm_set_state(self._ctx, *[_ptr(a) for a in arrs]))

    def get_state(self):
        f = np.empty(9 * self.n)
        if self.desc.use_komega:
            k, o, nut, s = np.empty(self.n), np.empty(self.n), np.empty(self.n), np.empty(3 * self.n)
        else:
            k = o = nut = s = None
        check("kofm_get_state", self.lib.kofm_get_state(
            self._ctx, _ptr(f), _ptr(k), _ptr(o), _ptr(nut), _ptr(s)))
        return f, k, o, nut, s

    def set_temperature(self, T):
        """tempArray in (host layout, FP64; kofm_set_temperature)."""
        T = np.ascontiguousarray(T, np.float64)
        check("kofm_set_temperature", self.lib.kofm_set_temperature(self._ctx, _ptr(T)))

    def get_temperature(self):
        T = np.empty(self.n)
        check("kofm_get_temperature", self.lib.kofm_get_temperature(self._ctx, _ptr(T)))
        return T

    def set_thermal_geometry(self, dX0):
        """Link fractions of the unfouled walls (dXArr0) for the thermal rows."""
        dX0 = np.ascontiguousarray(dX0, np.float64)
        check("kofm_set_thermal_geometry", self.lib.kofm_set_thermal_geometry(self._ctx, _ptr(dX0)))

    def thermal_update(self):
        """One clVariablesFD::Solve (kofm_thermal_update)."""
        check("kofm_thermal_update", self.lib.kofm_thermal_update(self._ctx))

    def adjoint(self, nsteps, n_ibb=None):
        """(J, dJ/dq) over nsteps from the current state (kofm_adjoint); dJ/dq
        in the order of the IBB links given to set_geometry."""
        n = self._n_ibb if n_ibb is None else n_ibb
        J = C.c_double()
        dq = np.zeros(max(n, 1))
        check("kofm_adjoint", self.lib.kofm_adjoint(self._ctx, nsteps, C.byref(J), _ptr(dq)))
        return J.value, dq[:n]

    def set_adjoint_memory(self, nbytes):
        """Cap on the device memory adjoint() keeps states in (< 0: half the
        free memory; 0: sqrt(T) checkpoints only) (kofm_set_adjoint_memory)."""
        check("kofm_set_adjoint_memory", self.lib.kofm_set_adjoint_memory(self._ctx, int(nbytes)))

    def set_shear(self, sh):
        """Uploads a shear.ShearSetup (kofm_set_shear)."""
        nodes = np.ascontiguousarray(sh.nodes, np.int32)
        cf = np.ascontiguousarray(sh.cfss, np.float64)
        bn = np.ascontiguousarray(sh.bl_nodes, np.int32)
        bw = np.ascontiguousarray(sh.bl_weights, np.float64)
        self._shear_sizes = (len(nodes), len(bn))
        check("kofm_set_shear", self.lib.kofm_set_shear(
            self._ctx, _ptr(nodes, C.c_int32), len(nodes), _ptr(cf), _ptr(bn, C.c_int32), _ptr(bw),
            len(bn)))

    def wall_shear(self):
        """(tau at the shear nodes, tau at the boundary links) of the current state."""
        n, nb = self._shear_sizes
        t, b = np.empty(n), np.empty(nb)
        check("kofm_wall_shear", self.lib.kofm_wall_shear(self._ctx, _ptr(t), _ptr(b) if nb else None))
        return t, b

    def get_macro(self):
        rho, ux, uy = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        check("kofm_get_macro", self.lib.kofm_get_macro(self._ctx, _ptr(rho), _ptr(ux), _ptr(uy)))
        return rho, ux, uy

    # -- stepping -------------------------------------------------------------------
    def lb_step(self, options=_abi.OPTION_SAVE_MACRO_FIELDS):
        check("kofm_lb_step", self.lib.kofm_lb_step(self._ctx, options))

    def komega_assemble(self, dt=1.0):
        check("kofm_komega_assemble", self.lib.kofm_komega_assemble(self._ctx, dt))

    def komega_solve(self, raise_on_error=True):
        it = (C.c_int32 * 2)()
        rr = (C.c_double * 2)()
        st = self.lib.kofm_komega_solve(self._ctx, it, rr)
        if raise_on_error:
            check("kofm_komega_solve", st)
        return st, (it[0], it[1]), (rr[0], rr[1])

    def komega_update(self):
        check("kofm_komega_update", self.lib.kofm_komega_update(self._ctx))

    def step(self, nsteps=1, options=_abi.OPTION_SAVE_MACRO_FIELDS):
        check("kofm_step", self.lib.kofm_step(self._ctx, nsteps, options))

    def sync(self):
        check("kofm_sync", self.lib.kofm_sync(self._ctx))

    def reduce(self, field, op=_abi.OP_SUM) -> float:
        out = C.c_double()
        check("kofm_reduce", self.lib.kofm_reduce(self._ctx, field, op, C.byref(out)))
        return out.value

    def stats(self) -> KofmStats:
        s = KofmStats()
        check("kofm_get_stats", self.lib.kofm_get_stats(self._ctx, C.byref(s)))
        return s

    def debug_barrier_timeout(self, spin_limit: int) -> int:
        return self.lib.kofm_debug_barrier_timeout(self._ctx, spin_limit)

    def debug_fail_solves(self, n: int, mask: int = 1):
        """The next n k-omega solves report a NaN residual for the systems in
        mask (1: omega, 2: k), host-made (kofm_debug_fail_solves)."""
        check("kofm_debug_fail_solves", self.lib.kofm_debug_fail_solves(self._ctx, n, mask))

    def solver_trace(self):
        """Device times (ns from the launch's start) at which the last
        k-omega solve's grid barriers released (kofm_debug_solver_trace)."""
        buf = (C.c_int64 * 32)()
        n = C.c_int32()
        check("kofm_debug_solver_trace", self.lib.kofm_debug_solver_trace(self._ctx, buf, 32, C.byref(n)))
        return [buf[i] for i in range(min(n.value, 32))]

    def komega_rows(self, system: int):
        """(coef [4, ny * nx_full] E/W/N/S off-diagonals normalised by the
        diagonal, rhs [ny * nx_full] = b - A x0) of one k-omega system (0:
        omega, 1: k) as the last assembly left them (kofm_debug_komega_rows)."""
        n = self.nxf * self.ny
        coef = np.zeros((4, n))
        rhs = np.zeros(n)
        check("kofm_debug_komega_rows",
              self.lib.kofm_debug_komega_rows(self._ctx, system, coef.ctypes.data_as(_abi._dp),
                                              rhs.ctypes.data_as(_abi._dp)))
        return coef, rhs

    def komega_update_status(self) -> int:
        """kofm_komega_update's status without raising."""
        return self.lib.kofm_komega_update(self._ctx)

    @property
    def stream(self) -> int:
        return self.lib.kofm_stream(self._ctx) or 0
