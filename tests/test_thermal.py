"""Thermal implicit finite differences (clVariablesFD::Solve): the oracle's
coefficient rows pinned to the reference's Update_T_Coeffs_Implicit, its
BiCGStab restatement checked against the reference's step list and a direct
solve, and the device update (kofm_thermal_update / kofm_step) against the
oracle."""
import ctypes as C
import os

import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from oracle.orc import BicgStats, OracleSim, ThermalCfg, ThermalState, make_cfg
from tests.cases import fp32_state, komega_state, rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_thermal.npz")


def _coeffs(orc, cfg, ch, th, T, ux, uy, nut, dt):
    IA, JA, ind = orc.csr_thermal(cfg, ch.ntype)
    A = np.zeros(len(JA))
    orc.L.orc_csr_fill_solid_boundary_thermal(C.byref(cfg), ch.ntype, ind, A)
    b = np.zeros(ch.n)
    orc.L.orc_thermal_coeffs(C.byref(cfg), C.byref(th), ind, ch.ntype, ch.dX, A, b, T, ux, uy,
                             None if nut is None else np.ascontiguousarray(nut).ctypes.data, dt)
    return IA, JA, ind, A, b


# ---- CPU: pattern, coefficients, solver ------------------------------------------

def test_thermal_csr_pattern(oracle):
    """CSR_Inds (non-periodic, M0 flags): wall-boundary rows hold only the
    diagonal, inner wall rows are empty, domain rows hold S, W, C, E, N in
    that column order, and x = 0 / nx-1 have no W / E entry (no wrap)."""
    ch = G.wavy_channel(64, 24, 4.0, 32)
    cfg = make_cfg(ch.nx, ch.ny, 1.2, 0.0, 0.05)
    IA, JA, ind = oracle.csr_thermal(cfg, ch.ntype)
    t = ch.ntype.astype(np.int32) & 0xFFFF
    nxf = ch.nx_full
    for g in range(ch.n):
        row = JA[IA[g]:IA[g + 1]]
        x = g % nxf
        if t[g] & G.M0_SOLID:
            assert list(row) == ([g] if t[g] & G.SOLID_BOUNDARY0 else [])
            continue
        want = [g - nxf] + ([g - 1] if x > 0 else []) + [g] + ([g + 1] if x < ch.nx - 1 else []) + [g + nxf]
        assert list(row) == want, (g, row, want)


def test_thermal_coeffs_match_reference_golden(oracle):
    """Update_T_Coeffs_Implicit (tfdKernels.cl:122-279) outputs of the
    reference, bit for bit: CSR values and right-hand side."""
    z = np.load(GOLDEN)
    ch = G.wavy_channel(int(z["nx"]), int(z["ny"]), float(z["amp"]), int(z["wavelength"]))
    cfg = make_cfg(ch.nx, ch.ny, float(z["rate"]), float(z["fterm"]), float(z["mu"]))
    th = ThermalCfg(*[float(v) for v in z["th"]])
    IA, JA, ind, A, b = _coeffs(oracle, cfg, ch, th, z["T"], z["ux"], z["uy"], z["nut"], float(z["dt"]))
    assert np.array_equal(IA, z["IA"]) and np.array_equal(JA, z["JA"])
    assert np.array_equal(A, z["A"])
    assert np.array_equal(b, z["b"])


def test_thermal_coeffs_match_reference_live(oracle, refk):
    ch = G.wavy_channel(120, 36, 6.0, 60)
    cfg = make_cfg(ch.nx, ch.ny, 1.4, 1e-5, 0.01)
    th = ThermalCfg(0.01 / 0.708, 0.002, 1 / 0.9, 2.0)
    rng = np.random.default_rng(41)
    fl = ch.fluid_mask().ravel()
    T = np.where(fl, 2.2 * rng.random(ch.n), 0.0)
    ux = np.where(fl, 0.04 * rng.random(ch.n), 0.0)
    uy = np.where(fl, 0.004 * rng.standard_normal(ch.n), 0.0)
    _, _, nut, _ = komega_state(ch, seed=42)
    for dt in (1.0, 0.25):
        IA, JA, ind, A, b = _coeffs(oracle, cfg, ch, th, T, ux, uy, nut, dt)
        A2 = np.zeros(len(JA))
        oracle.L.orc_csr_fill_solid_boundary_thermal(C.byref(cfg), ch.ntype, ind, A2)
        b2 = np.zeros(ch.n)
        refk.L.ref_thermal_coeffs(C.byref(cfg), np.array([th.alpha_fluid, th.alpha_foul,
                                                          th.pr_turb_inv, th.t_in]),
                                  ind, ch.ntype, ch.dX.copy(), A2, b2, T.copy(), ux.copy(),
                                  uy.copy(), nut.copy(), dt)
        assert np.array_equal(A, A2) and np.array_equal(b, b2)


def _bicgstab_steps(IA, JA, A, b, x, max_iters, rel_tol, abs_tol, reset_flag=True):
    """The step list of BiCGStabSolver::solve (BiCGStabSolver.cpp:628-723)
    with the kernels it enqueues and reduceAndCheckConvergence (509-545),
    written out in numpy for a small system: scalars filled with 1, omega
    never reduced, L1-norm checks.  Returns (x, iterCount, checks, reset)."""
    import scipy.sparse as sp
    n = len(b)
    M = sp.csr_matrix((A, JA, IA), shape=(n, n))
    b = b.copy()
    x = x.copy()
    rho = alpha = omega = 1.0
    normb = np.abs(b).sum()
    b = b - M @ x
    r0 = b.copy()
    p = b.copy()
    rho = (b * b).sum()
    it, checks, state = 0, 0, {"first": True, "init": 0.0, "avg": 0.0}
    v = np.zeros(n)

    def check(r):
        res = np.abs(r).sum() / normb
        if state["first"]:
            state["init"] = res
        state["first"] = False
        if reset_flag and (np.isnan(res) or (it > 1 and res > 10.0 * state["avg"])):
            return "reset"
        if res <= rel_tol or res <= abs_tol * state["init"]:
            return "conv"
        state["avg"] = res
        return None

    while it < max_iters:
        if it > 0:
            rho_new = (b * r0).sum()
            beta = (rho_new / rho) * (alpha / omega)
            rho = rho_new
            p = b + beta * (p - omega * v)
        v = M @ p
        alpha = rho / (v * r0).sum()
        x = x + alpha * p
        b = b - alpha * v
        checks += 1
        out = check(b)
        if out:
            return x, it, checks, out == "reset"
        t = M @ b
        x = x + omega * b
        b = b - omega * t
        checks += 1
        out = check(b)
        if out:
            return x, it, checks, out == "reset"
        it += 1
    return x, it, checks, False


def test_bicgstab_restates_reference_steps(oracle):
    ch = G.wavy_channel(48, 24, 3.0, 24)
    cfg = make_cfg(ch.nx, ch.ny, 1.2, 0.0, 0.05)
    th = ThermalCfg(0.05 / 0.708, 0.0, 1 / 0.9, 2.0)
    rng = np.random.default_rng(5)
    fl = ch.fluid_mask().ravel()
    T = np.where(fl, 0.5 + rng.random(ch.n), 0.0)
    ux = np.where(fl, 0.05 * rng.random(ch.n), 0.0)
    uy = np.where(fl, 0.01 * rng.standard_normal(ch.n), 0.0)
    for dt, tol in ((1.0, 1e-4), (4.0, 1e-10)):
        IA, JA, ind, A, b = _coeffs(oracle, cfg, ch, th, T, ux, uy, None, dt)
        want, it, checks, reset = _bicgstab_steps(IA, JA, A, b, T, 1000, tol, 1e-7)
        x, bb, st = T.copy(), b.copy(), BicgStats()
        oracle.L.orc_bicgstab_solve(ch.n, IA, JA, A, bb, x, 1000, tol, 1e-7, 1, C.byref(st))
        assert not reset and st.conv == 1 and st.reset == 0
        assert (st.iters, st.checks) == (it, checks)
        assert np.abs(x - want).max() <= 1e-12 * np.abs(want).max()


def _rough_case(oracle):
    """Random T and velocities on a wavy channel with an eddy viscosity: the
    omega = 1 iteration's residual jumps tenfold at its fifth check."""
    ch = G.wavy_channel(96, 40, 5.0, 48)
    cfg = make_cfg(ch.nx, ch.ny, 1.3, 0.0, 0.02)
    th = ThermalCfg(0.02 / 0.708, 0.0, 1 / 0.9, 2.0)
    rng = np.random.default_rng(6)
    fl = ch.fluid_mask().ravel()
    T = np.where(fl, 0.5 + rng.random(ch.n), 0.0)
    ux = np.where(fl, 0.03 + 0.01 * rng.standard_normal(ch.n), 0.0)
    uy = np.where(fl, 0.005 * rng.standard_normal(ch.n), 0.0)
    _, _, nut, _ = komega_state(ch, seed=7)
    return ch, cfg, th, T, ux, uy, nut


def test_bicgstab_growth_triggers_reset(oracle):
    """reduceAndCheckConvergence's resetTimeFunc path: a residual ten times
    the previous check's (after the second iteration) ends the solve."""
    ch, cfg, th, T, ux, uy, nut = _rough_case(oracle)
    IA, JA, ind, A, b = _coeffs(oracle, cfg, ch, th, T, ux, uy, nut, 1.0)
    _, it, checks, reset = _bicgstab_steps(IA, JA, A, b, T, 1000, 1e-4, 1e-7)
    x, bb, st = T.copy(), b.copy(), BicgStats()
    oracle.L.orc_bicgstab_solve(ch.n, IA, JA, A, bb, x, 1000, 1e-4, 1e-7, 1, C.byref(st))
    assert reset and st.reset == 1 and st.conv == 0
    assert (st.iters, st.checks) == (it, checks) == (2, 5)


def test_bicgstab_matches_direct_solve(oracle):
    """Without the growth test the same system converges; the solution
    matches a direct solve."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sl
    ch, cfg, th, T, ux, uy, nut = _rough_case(oracle)
    IA, JA, ind, A, b = _coeffs(oracle, cfg, ch, th, T, ux, uy, nut, 1.0)
    x, bb, st = T.copy(), b.copy(), BicgStats()
    oracle.L.orc_bicgstab_solve(ch.n, IA, JA, A, bb, x, 1000, 1e-12, 1e-30, 0, C.byref(st))
    assert st.conv == 1
    rows = np.diff(IA) > 0
    M = sp.csr_matrix((A, JA, IA), shape=(ch.n, ch.n))[rows][:, rows]
    ref = sl.spsolve(M.tocsc(), b[rows])
    assert np.abs(x[rows] - ref).max() <= 1e-9 * np.abs(ref).max()


# ---- GPU ---------------------------------------------------------------------------

def _thermal_lattice(ch, rate, g, mu, komega, **desc):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = rate, g, mu
    d.use_komega = 1 if komega else 0
    d.use_thermal = 1
    for key, v in desc.items():
        setattr(d, key, v)
    L = Lattice(d)
    L.set_geometry(ch.ntype, ch.wallD if komega else None, ch.dX, ch.ibb_idx, ch.ibb_q)
    return L, d


def _wavy_case():
    ch = G.wavy_channel(256, 66, 8.0, 128)
    nu, u_max = 5e-4, 0.05
    R = ch.pipe_radius
    y = np.arange(ch.ny)[:, None] - 0.5
    ux = np.clip(u_max * (1 - ((y - R) / R) ** 2), 0, None) * np.ones((1, ch.nx))
    f = G.equilibrium_state(ch, ux=ux)
    g = G.force_from_re((2.0 / 3.0) * u_max * R / nu, nu, R)
    k0 = 1.5 * (0.05 * u_max) ** 2
    o0 = np.sqrt(k0) / (0.09 ** 0.25 * 0.07 * 2 * R)
    k, o, nut = G.komega_fields(ch, k0, o0)
    f, k, o, nut = fp32_state(f, k, o, nut)
    return ch, f, k, o, nut, 1.0 / (3 * nu + 0.5), g, nu


TIGHT_KO = dict(komega_rel_tol=1e-10, komega_abs_tol=1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("tol,dt,npre", [(1e-4, 1.0, 5), (1e-12, 1.0, 5), (1e-12, 64.0, 0)])
def test_gpu_thermal_update_of_device_state(kofm_lib, oracle, tol, dt, npre):
    """kofm_thermal_update against orc_thermal_solve on the state the device
    holds (T, the step's u and nu_t, the sub-step count and dt): one
    clVariablesFD::Solve after npre full steps and one LB + k-omega step.  At
    dt = 64 the residual growth test halves the time step twice (the
    resetTimeFunc path: T restored, sub-steps doubled) in both."""
    ch, f, k, o, nut, rate, g, nu = _wavy_case()
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    L, d = _thermal_lattice(ch, rate, g, nu, True, thermal_rel_tol=tol, thermal_dt=dt, **TIGHT_KO)
    with L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.set_temperature(G.temperature_field(ch))
        L.step(npre)
        L.lb_step()
        L.komega_update()
        T5 = L.get_temperature()
        _, ux, uy = L.get_macro()
        nut5 = L.get_state()[3]
        st5 = L.stats()
        L.thermal_update()
        T6 = L.get_temperature()
        st6 = L.stats()
    th = ThermalCfg(nu / d.pr_number, d.alpha_foul, 1.0 / d.pr_turb_number, d.t_in)
    ts = ThermalState(st5.thermal_steps_per_lb, st5.thermal_time_since_change, st5.thermal_dt,
                      d.thermal_max_iters, tol, d.thermal_abs_tol)
    IA, JA, ind = oracle.csr_thermal(cfg, ch.ntype)
    A = np.zeros(len(JA))
    oracle.L.orc_csr_fill_solid_boundary_thermal(C.byref(cfg), ch.ntype, ind, A)
    T, Tprev, b = T5.copy(), np.zeros(ch.n), np.zeros(ch.n)
    oracle.L.orc_thermal_solve(C.byref(cfg), C.byref(th), C.byref(ts), ch.ntype, IA, JA, ind, ch.dX,
                               T, Tprev, ux, uy, np.ascontiguousarray(nut5).ctypes.data, A, b)
    fl = ch.fluid_mask().ravel()
    err = rel_l2(T6, T, fl)
    dT = rel_l2(T6, T5, fl)
    print(dict(err=err, change=dT, gpu_iters=st6.thermal_iters, oracle_iters=ts.last.iters,
               gpu_res=st6.thermal_residual, oracle_res=ts.last.residual))
    print(dict(solves=(st6.thermal_solves, ts.solves), resets=(st6.thermal_resets, ts.resets),
               dt=(st6.thermal_dt, ts.dt), steps5=(st5.thermal_steps_per_lb, st5.thermal_dt)))
    assert (st6.thermal_solves, st6.thermal_resets) == (ts.solves, ts.resets)
    assert (ts.resets > 0) == (dt > 32)
    assert (st6.thermal_steps_per_lb, st6.thermal_dt) == (ts.steps_per_lb, ts.dt)
    assert abs(st6.thermal_iters - ts.last.iters) <= (0 if tol < 1e-8 else 1)
    # both solves meet the tolerance; at 1e-4 they may stop an iteration apart
    assert err < (1e-10 if tol < 1e-8 else 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("komega", [False, True])
def test_gpu_thermal_run_matches_oracle(kofm_lib, oracle, komega):
    """T after LB (+ k-omega) + thermal steps on the GPU against the FP64
    oracle run from the same start (solves to 1e-12 / 1e-10 so that only the
    FP32 storage of the flow separates them)."""
    if komega:
        ch, f, k, o, nut, rate, g, nu = _wavy_case()
        nsteps = 10
    else:
        ch = G.wavy_channel(192, 40, 5.0, 96)
        rate, g, nu = 1.25, 2e-6, 0.1
        (f,) = fp32_state(G.equilibrium_state(ch, ux=0.01))
        k = o = nut = None
        nsteps = 60
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    L, d = _thermal_lattice(ch, rate, g, nu, komega, thermal_rel_tol=1e-12, **TIGHT_KO)
    T0 = G.temperature_field(ch)
    th = ThermalCfg(nu / d.pr_number, d.alpha_foul, 1.0 / d.pr_turb_number, d.t_in)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, None, komega=komega,
                    ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q, rel_tol=1e-10, abs_tol=1e-30,
                    thermal=dict(T=T0, cfg=th, rel_tol=1e-12, abs_tol=d.thermal_abs_tol))
    sim.step(nsteps)
    with L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n) if komega else None)
        L.set_temperature(T0)
        L.step(nsteps)
        T = L.get_temperature()
        tsum = L.reduce(_abi.FIELD_TEMP)
        tmin = L.reduce(_abi.FIELD_TEMP, _abi.OP_MIN)
    fl = ch.fluid_mask().ravel()
    err = rel_l2(T, sim.T, fl)
    change = rel_l2(sim.T, T0, fl)
    print(dict(err=err, change=change))
    assert change > 1e-3            # the inlet front has moved in
    assert err < 1e-6 * max(change, 1.0)
    assert abs(tsum - T.sum()) <= 1e-12 * abs(T.sum()) and tmin == T.min()


# ---- fouling layer: conjugate heat transfer ----------------------------------------

def _fouled_channel(nx=160, ny=40):
    """Straight unfouled walls at 0.5 and ny - 1.5 with a deposit 3-6 cells
    thick on both: the nodes between are the fouling layer (M0_FLUID |
    M_SOLID), where T diffuses with LB_ALPHA_FOUL.  The deposit is flat and
    half-way between rows at x = 0, so no link at the periodic seam has
    2q > 1 (where the reference's lbIBB reads an unwrapped neighbour)."""
    x = np.arange(nx)
    d = 3.0 + 1.5 * (1.0 - np.cos(2 * np.pi * x / 80.0))
    return G.channel_from_walls(nx, ny, 0.5 + d, ny - 1.5 - d,
                                y_bot0=np.full(nx, 0.5), y_top0=np.full(nx, ny - 1.5))


def test_fouled_channel_flags():
    ch = _fouled_channel()
    t = (ch.ntype.astype(np.int32) & 0xFFFF)
    foul = (t & G.M0_FLUID != 0) & (t & G.M_SOLID != 0)
    assert foul.sum() > 2 * ch.nx * 2
    clean = G.straight_channel(ch.nx, ch.ny)
    ct = clean.ntype.astype(np.int32) & 0xFFFF
    m0 = G.M0_SOLID | G.M0_FLUID | G.SOLID_BOUNDARY0 | G.NESW_BOUNDARY0 | G.BOUNDARY0
    # the unfouled flags and link fractions are those of the clean channel
    assert np.array_equal(t & m0, ct & m0)
    assert np.array_equal(ch.dX0, clean.dX)
    # the flow sees the deposit: its surface nodes are solid boundaries of the
    # flow, fluid nodes next to it carry wall bits, and its links are cut
    fl = ((t & G.M_FLUID) != 0).reshape(ch.ny, ch.nx_full)
    tt = t.reshape(ch.ny, ch.nx_full)
    assert np.any(foul & ((t & G.SOLID_BOUNDARY) != 0))
    below_solid = fl[1:, :] & ~fl[:-1, :]
    assert np.all((tt[1:, :][below_solid] & G.BOUND[4]) != 0)
    assert len(ch.ibb_idx) > 0 and not np.array_equal(ch.dX, ch.dX0)


def test_thermal_coeffs_fouling_layer_match_reference(oracle, refk):
    ch = _fouled_channel()
    cfg = make_cfg(ch.nx, ch.ny, 1.4, 1e-5, 0.02)
    th = ThermalCfg(0.02 / 0.708, 0.003, 1 / 0.9, 2.0)
    rng = np.random.default_rng(51)
    fl = ch.fluid_mask().ravel()
    T = 2.2 * rng.random(ch.n)
    ux = np.where(fl, 0.04 * rng.random(ch.n), 0.0)
    uy = np.where(fl, 0.004 * rng.standard_normal(ch.n), 0.0)
    _, _, nut, _ = komega_state(ch, seed=52)
    IA, JA, ind = oracle.csr_thermal(cfg, ch.ntype)
    A, A2 = np.zeros(len(JA)), np.zeros(len(JA))
    oracle.L.orc_csr_fill_solid_boundary_thermal(C.byref(cfg), ch.ntype, ind, A)
    A2[:] = A
    b, b2 = np.zeros(ch.n), np.zeros(ch.n)
    oracle.L.orc_thermal_coeffs(C.byref(cfg), C.byref(th), ind, ch.ntype, ch.dX0, A, b, T, ux, uy,
                                nut.ctypes.data, 1.0)
    refk.L.ref_thermal_coeffs(C.byref(cfg), np.array([th.alpha_fluid, th.alpha_foul, th.pr_turb_inv,
                                                      th.t_in]),
                              ind, ch.ntype, ch.dX0.copy(), A2, b2, T.copy(), ux.copy(), uy.copy(),
                              nut.copy(), 1.0)
    assert np.array_equal(A, A2) and np.array_equal(b, b2)


@pytest.mark.gpu
def test_gpu_thermal_fouling_layer_matches_oracle(kofm_lib, oracle):
    """Laminar flow over the deposit, heat conducted through it: the device
    update with the unfouled link fractions (kofm_set_thermal_geometry) and
    the fouling-layer diffusivity against the oracle run."""
    ch = _fouled_channel()
    rate, g, nu = 1.25, 2e-6, 0.1
    (f,) = fp32_state(G.equilibrium_state(ch, ux=0.01))
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    L, d = _thermal_lattice(ch, rate, g, nu, False, thermal_rel_tol=1e-12, alpha_foul=0.02)
    T0 = G.temperature_field(ch)
    th = ThermalCfg(nu / d.pr_number, d.alpha_foul, 1.0 / d.pr_turb_number, d.t_in)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q,
                    thermal=dict(T=T0, cfg=th, dX0=ch.dX0, rel_tol=1e-12, abs_tol=d.thermal_abs_tol))
    sim.step(40)
    with L:
        L.set_thermal_geometry(ch.dX0)
        L.set_state(f)
        L.set_temperature(T0)
        L.step(40)
        T = L.get_temperature()
    t = ch.ntype.astype(np.int32) & 0xFFFF
    dom = (t & G.M0_FLUID) != 0
    err = rel_l2(T, sim.T, dom)
    print(dict(err=err, change=rel_l2(sim.T, T0, dom)))
    assert err < 1e-8
