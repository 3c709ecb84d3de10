"""GPU parity of the LB collide-stream kernel against the FP64 oracle.

The oracle (oracle/kofm_oracle.c) is pinned to the reference's own kernels by
tests/test_oracle_pin.py.  The GPU stores populations as FP32 deviations
f - w with FP64 collide arithmetic; tolerances are stated per test.
"""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from oracle.orc import OracleSim, make_cfg
from tests.cases import fp32_state, komega_state, perturbed_state, rel_l2

pytestmark = pytest.mark.gpu


def lattice(nx, ny, tau, fterm, mu, komega=False, storage=_abi.STORE_FP32):
    d = desc_default()
    d.nx, d.nx_full, d.ny = nx, nx, ny
    d.tau, d.fterm, d.mu = tau, fterm, mu
    d.use_komega = 1 if komega else 0
    d.storage = storage
    return Lattice(d)


def fluid_pops(ch, f):
    return f.reshape(9, -1)[:, ch.fluid_mask().ravel()]


def assert_pops_close(gpu, ref):
    """FP32-stored deviations d = f - w: each stored value carries half an
    ulp of its own magnitude, and the collision mixes the 9 populations of a
    node, so the error of one population is bounded by the FP32 resolution of
    the largest deviation of its node (plus FP64 round-off)."""
    dev = np.abs(ref - G.W[:, None])
    scale = dev.max(axis=0, keepdims=True)
    err = np.abs(gpu - ref)
    assert np.all(err <= 4e-7 * scale + 1e-14), float((err / (scale + 1e-300)).max())
    assert np.linalg.norm(err) <= 1e-7 * np.linalg.norm(dev)


def test_state_round_trip_phase0(kofm_lib):
    ch = G.straight_channel(128, 16)
    f = perturbed_state(ch, seed=1)
    with lattice(128, 16, 1.25, 0.0, 0.1) as L:
        L.set_geometry(ch.ntype)
        L.set_state(f)
        g, *_ = L.get_state()
    a, b = fluid_pops(ch, g), fluid_pops(ch, f)
    # FP32 rounding of the deviation f - w
    dev = np.abs(b - G.W[:, None])
    assert np.all(np.abs(a - b) <= 6e-8 * dev + 1e-15)


@pytest.mark.parametrize("nsteps", [1, 2, 5])
def test_laminar_steps_match_oracle(kofm_lib, oracle, nsteps):
    nx, ny = 128, 20
    ch = G.straight_channel(nx, ny)
    (f,) = fp32_state(perturbed_state(ch, seed=2))
    cfg = make_cfg(nx, ny, 1.25, 1e-5, 0.1)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f)
    sim.step(nsteps)
    with lattice(nx, ny, 1.25, 1e-5, 0.1) as L:
        L.set_geometry(ch.ntype)
        L.set_state(f)
        for _ in range(nsteps):
            L.lb_step()
        g, *_ = L.get_state()
        rho, ux, uy = L.get_macro()
    fl = ch.fluid_mask().ravel()
    assert_pops_close(fluid_pops(ch, g), fluid_pops(ch, sim.FA))
    # moments of the last step are FP32 copies of FP64 values
    assert np.max(np.abs(rho[fl] - sim.rho[fl])) < 2e-7
    assert np.max(np.abs(ux[fl] - sim.ux[fl])) < 1e-8
    assert np.max(np.abs(uy[fl] - sim.uy[fl])) < 1e-8


def test_komega_collide_matches_oracle(kofm_lib, oracle):
    nx, ny = 128, 20
    ch = G.straight_channel(nx, ny)
    f = perturbed_state(ch, seed=3)
    k, o, nut, s = komega_state(ch, seed=4)
    fl = ch.fluid_mask().ravel()
    idx = np.nonzero(fl)[0]
    k[idx[:4]] *= -1.0
    o[idx[10:13]] *= -1.0
    f, k, o, nut, s = fp32_state(f, k, o, nut, s)
    cfg = make_cfg(nx, ny, 1.9, 1e-6, 0.01)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, s, komega=True)
    import ctypes as C
    oracle.L.orc_collide_push(C.byref(cfg), sim.FA, sim.FB, sim.m, sim.rho, sim.ux, sim.uy,
                              sim.K, sim.O, sim.wallD, sim.nut, sim.S, 2, 1)
    with lattice(nx, ny, 1.9, 1e-6, 0.01, komega=True) as L:
        L.set_geometry(ch.ntype, ch.wallD, ch.dX)
        L.set_state(f, k, o, nut, s)
        L.lb_step()
        g, k2, o2, nut2, s2 = L.get_state()
    assert_pops_close(fluid_pops(ch, g), fluid_pops(ch, sim.FB))
    assert np.allclose(k2[fl], sim.K[fl], rtol=1e-7, atol=0)     # clamp k<0 -> 1e-16
    assert np.allclose(o2[fl], sim.O[fl], rtol=1e-7, atol=0)     # clamp omega<0 -> |omega|
    assert np.allclose(nut2[fl], sim.nut[fl], rtol=1e-6, atol=1e-20)
    for c in range(3):
        a = s2[c * ch.n:(c + 1) * ch.n][fl]
        b = sim.S[c * ch.n:(c + 1) * ch.n][fl]
        assert np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(b)) + 1e-12


def test_poiseuille_c1_1000_steps_parity(kofm_lib, oracle):
    """Config 1 (256 x 64, tau = 0.8, nu = 0.1, g = 1e-6, start from rest):
    rho and u within rel-L2 1e-5 of the FP64 oracle after 1000 steps."""
    nx, ny, rate, g = 256, 64, 1.0 / 0.8, 1e-6
    mu = (0.8 - 0.5) / 3.0
    ch = G.straight_channel(nx, ny)
    f = G.equilibrium_state(ch)
    cfg = make_cfg(nx, ny, rate, g, mu)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f)
    sim.step(1000)
    with lattice(nx, ny, rate, g, mu) as L:
        L.set_geometry(ch.ntype)
        L.set_state(f)
        L.step(1000)
        rho, ux, uy = L.get_macro()
        sums = [L.reduce(_abi.FIELD_RHO), L.reduce(_abi.FIELD_UX)]
    fl = ch.fluid_mask().ravel()
    assert rel_l2(rho, sim.rho, fl) < 1e-5
    assert rel_l2(ux, sim.ux, fl) < 1e-5
    assert np.max(np.abs(uy[fl])) < 1e-9
    # FP64 reductions over the padded array (Reducer<double>::reduceSingle)
    assert abs(sums[0] - np.sum(rho)) < 1e-6
    assert abs(sums[1] - np.sum(ux)) <= 1e-9 * abs(np.sum(ux)) + 1e-12


def _startup_poiseuille(y, t, g, nu, H, nterms=200):
    """Start-up flow between plates (fluid from y'=0 to H), series solution."""
    yp = y
    u = g / (2 * nu) * yp * (H - yp)
    for n in range(1, 2 * nterms, 2):
        u -= 4 * g * H * H / (nu * n ** 3 * np.pi ** 3) * np.sin(n * np.pi * yp / H) * np.exp(-nu * n * n * np.pi ** 2 * t / H ** 2)
    return u


def test_poiseuille_c1_10000_steps_analytic(kofm_lib):
    """Config 1 over its full 10,000 steps against the analytic start-up
    profile (walls half-way at y = 0.5 and 62.5)."""
    nx, ny, rate, g = 256, 64, 1.0 / 0.8, 1e-6
    mu = (0.8 - 0.5) / 3.0
    ch = G.straight_channel(nx, ny)
    with lattice(nx, ny, rate, g, mu) as L:
        L.set_geometry(ch.ntype)
        L.set_state(G.equilibrium_state(ch))
        L.step(10000)
        rho, ux, uy = L.get_macro()
    prof = ux.reshape(ny, nx)[1:-1, :].mean(axis=1)
    y = np.arange(1, ny - 1) - 0.5
    ua = _startup_poiseuille(y, 10000.0, g, mu, ny - 2.0)
    assert np.linalg.norm(prof - ua) / np.linalg.norm(ua) < 2e-3


@pytest.mark.parametrize("storage", [_abi.STORE_FP16_DEV, _abi.STORE_BF16_DEV, _abi.STORE_FP16_NEQ,
                                     _abi.STORE_FP16_ROW])
def test_half_storage_forms_run_and_conserve_mass(kofm_lib, oracle, storage):
    nx, ny = 256, 64
    ch = G.straight_channel(nx, ny)
    f = G.equilibrium_state(ch, ux=0.02)
    cfg = make_cfg(nx, ny, 1.25, 1e-6, 0.1)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f)
    sim.step(200)
    with lattice(nx, ny, 1.25, 1e-6, 0.1, storage=storage) as L:
        L.set_geometry(ch.ntype)
        L.set_state(f)
        L.step(200)
        rho, ux, uy = L.get_macro()
    fl = ch.fluid_mask().ravel()
    # 16-bit deviations round to 2^-11 (FP16) / 2^-8 (BF16) of their size
    # every step; the non-equilibrium forms round only f - feq (of the node's
    # own moments, or of its row's at the upload)
    bound = {_abi.STORE_FP16_DEV: 2e-2, _abi.STORE_BF16_DEV: 5e-2, _abi.STORE_FP16_NEQ: 1e-3,
             _abi.STORE_FP16_ROW: 1e-3}[storage]
    assert rel_l2(ux, sim.ux, fl) < bound
    assert abs(rho[fl].mean() - 1.0) < 1e-2


def test_fp16_neq_round_trip_and_first_step(kofm_lib, oracle):
    """The non-equilibrium form stores f - feq(rho, u) of each node: a state
    upload and download reproduces f to FP16 precision of that difference, and
    one step matches the oracle at that level."""
    nx, ny = 128, 20
    ch = G.straight_channel(nx, ny)
    (f,) = fp32_state(perturbed_state(ch, seed=5))
    with lattice(nx, ny, 1.25, 1e-5, 0.1, storage=_abi.STORE_FP16_NEQ) as L:
        L.set_geometry(ch.ntype)
        L.set_state(f)
        g, *_ = L.get_state()
        L.lb_step()
        g1, *_ = L.get_state()
    a, b = fluid_pops(ch, g), fluid_pops(ch, f)
    # e = f - feq(rho, u) of each node, rounded to FP16 (half an ulp: 2^-11 of |e|)
    fr = f.reshape(9, -1)
    rho = fr.sum(0)
    ux = (G.CX[:, None] * fr).sum(0) / np.where(rho == 0, 1, rho)
    uy = (G.CY[:, None] * fr).sum(0) / np.where(rho == 0, 1, rho)
    e = fluid_pops(ch, fr - G.feq(rho, ux, uy))
    assert np.all(np.abs(a - b) <= 2.0 ** -11 * np.abs(e) + 2e-8)
    cfg = make_cfg(nx, ny, 1.25, 1e-5, 0.1)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f)
    sim.step(1)
    err = np.abs(fluid_pops(ch, g1) - fluid_pops(ch, sim.FA))
    # input rounding carried through one collision plus the new rounding
    assert err.max() < 2.0 ** -9 * np.abs(e).max(), (err.max(), np.abs(e).max())


def test_fp16_row_round_trip_and_first_step(kofm_lib, oracle):
    """The row-reference form stores f - feq(rho_R, u_R) with one reference
    per row, the mean density and velocity of the row's fluid nodes at the
    upload: a state upload and download reproduces f to FP16 precision of
    that difference, and one step matches the oracle at that level."""
    nx, ny = 128, 20
    ch = G.straight_channel(nx, ny)
    (f,) = fp32_state(perturbed_state(ch, seed=5, u_mean=0.02))
    with lattice(nx, ny, 1.25, 1e-5, 0.1, storage=_abi.STORE_FP16_ROW) as L:
        L.set_geometry(ch.ntype)
        L.set_state(f)
        g, *_ = L.get_state()
        L.lb_step()
        g1, *_ = L.get_state()
    a, b = fluid_pops(ch, g), fluid_pops(ch, f)
    fr = f.reshape(9, ny, ch.nx_full)
    fl = ch.fluid_mask()
    rho = fr.sum(0)
    jx = (G.CX[:, None, None] * fr).sum(0)
    jy = (G.CY[:, None, None] * fr).sum(0)
    cnt = np.maximum(fl.sum(1), 1)
    srho = np.where(fl, rho, 0).sum(1)
    rr = np.where(srho > 0, srho / cnt, 1.0)
    ru = np.where(srho > 0, np.where(fl, jx, 0).sum(1) / np.where(srho > 0, srho, 1), 0.0)
    rv = np.where(srho > 0, np.where(fl, jy, 0).sum(1) / np.where(srho > 0, srho, 1), 0.0)
    R = lambda a: np.repeat(a[:, None], ch.nx_full, 1).ravel()  # noqa: E731
    e = fluid_pops(ch, f.reshape(9, -1) - G.feq(R(rr), R(ru), R(rv)))
    # e rounded to FP16 (half an ulp: 2^-11 of |e|), plus the FP32 equilibrium
    assert np.all(np.abs(a - b) <= 2.0 ** -11 * np.abs(e) + 2e-8)
    cfg = make_cfg(nx, ny, 1.25, 1e-5, 0.1)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f)
    sim.step(1)
    err = np.abs(fluid_pops(ch, g1) - fluid_pops(ch, sim.FA))
    assert err.max() < 2.0 ** -9 * np.abs(e).max() + 1e-7, (err.max(), np.abs(e).max())
