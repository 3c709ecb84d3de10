"""Wall shear: the set-up (shear nodes, coefficient rows, boundary-link
weights), the oracle's TR_shear_1 / TR_shear_2 pinned to the reference's own
kernels, and the GPU's kofm_wall_shear against the oracle."""
import ctypes as C
import os

import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from komegafoulingmodel_b200 import shear
from oracle.orc import OracleSim, make_cfg
from tests.cases import fp32_state, komega_state, perturbed_state, rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_shear.npz")


def _golden_case():
    z = np.load(GOLDEN)
    ch = G.wavy_channel(int(z["nx"]), int(z["ny"]), float(z["amp"]), int(z["wavelength"]))
    cfg = make_cfg(int(z["nx"]), int(z["ny"]), float(z["tau"]), float(z["fterm"]), float(z["mu"]))
    return z, ch, cfg


def _scatter(n, nodes, v):
    a = np.zeros(n)
    a[nodes] = v
    return a


def oracle_tau(orc, cfg, sh, FA, rho, ux, uy, nut=None):
    """TR_shear_1 then TR_shear_2 in the oracle on a full state (host layout)."""
    n = len(sh.nodes)
    t = np.zeros(n)
    orc.L.orc_wall_shear_nodes(C.byref(cfg), np.ascontiguousarray(FA), rho, ux, uy,
                               None if nut is None else np.ascontiguousarray(nut).ctypes.data,
                               np.ascontiguousarray(sh.nodes, np.int32), n,
                               np.ascontiguousarray(sh.cfss.ravel()), t)
    b = np.zeros(len(sh.bl_nodes))
    orc.L.orc_wall_shear_links(t, np.ascontiguousarray(sh.bl_nodes.ravel(), np.int32),
                               np.ascontiguousarray(sh.bl_weights.ravel()), len(b), b)
    return t, b


# ---- set-up ---------------------------------------------------------------

def test_straight_channel_shear_nodes_and_normals():
    nx, ny = 40, 12
    ch = G.straight_channel(nx, ny)
    nodes, col_start = shear.shear_nodes(ch)
    # one node next to each wall per column, column by column
    assert np.array_equal(col_start, 2 * np.arange(nx + 1))
    assert np.array_equal(nodes[0::2], np.arange(nx) + nx * 1)
    assert np.array_equal(nodes[1::2], np.arange(nx) + nx * (ny - 2))
    cf = shear.shear_coeffs(ch, nodes)
    # wall normal (0, -1) at the bottom, (0, 1) at the top: s_k = -/+ c_ky,
    # x row 3 s_k c_kx, y row 3 s_k (c_ky - n_y s_k) = 0
    cx, cy = G.CX[1:].astype(float), G.CY[1:].astype(float)
    for row, ny_ in ((cf[0], -1.0), (cf[1], 1.0)):
        s = cy * ny_
        assert np.allclose(row[:8], 3 * s * cx) and np.allclose(row[8:], 0.0)


def test_shear_window():
    ch = G.wavy_channel(96, 30, 5.0, 48)
    full = shear.setup(ch)
    win = shear.setup(ch, 20, 60)
    x = win.nodes % ch.nx_full
    assert x.min() >= 20 and x.max() <= 60
    sel = ((full.nodes % ch.nx_full) >= 20) & ((full.nodes % ch.nx_full) <= 60)
    assert np.array_equal(win.nodes, full.nodes[sel])
    assert len(win.bl_nodes) == 2 * 41
    assert np.all(win.col_start[20:62] - win.col_start[20] == full.col_start[20:62] - full.col_start[20])


def test_shear_coeffs_match_reference_golden():
    """TR_Find_Shear_Coeffs1 (trKernelsShear.cl:333-375) outputs of the
    reference on a wavy channel, bit for bit."""
    z, ch, _ = _golden_case()
    nodes, _ = shear.shear_nodes(ch)
    assert np.array_equal(nodes, z["nodes"])
    assert np.array_equal(shear.shear_coeffs(ch, nodes), z["cfss"])


def test_shear_coeffs_match_reference_live(refk):
    ch = G.wavy_channel(160, 44, 7.0, 80)
    cfg = make_cfg(ch.nx, ch.ny, 1.5, 1e-5, 0.05)
    nodes, _ = shear.shear_nodes(ch)
    ref = np.zeros(16 * len(nodes))
    refk.L.ref_shear_coeffs1(C.byref(cfg), nodes, ch.ntype, ref, len(nodes), shear.CUTOFF_RADIUS)
    assert np.array_equal(shear.shear_coeffs(ch, nodes).ravel(), ref)


def test_bl_weights_are_the_four_nearest():
    """TR_Find_Shear_Coeffs2 (trKernelsShear.cl:414-505): the four nearest
    shear nodes within the cut-off among the columns within the search radius,
    ascending list indices, Gaussian weights that sum to one."""
    ch = G.wavy_channel(128, 36, 6.0, 64)
    sh = shear.setup(ch)
    mids = shear.wall_midpoints(ch)
    x = (sh.nodes % ch.nx_full).astype(float)
    y = (sh.nodes // ch.nx_full).astype(float)
    assert len(sh.bl_nodes) == 2 * ch.nx
    for b in range(len(mids)):
        idx, w = sh.bl_nodes[b], sh.bl_weights[b]
        assert np.all(np.diff(idx) >= 0)
        assert abs(w.sum() - 1.0) < 1e-14
        d = np.hypot(mids[b, 0] - x, mids[b, 1] - y)
        ival = int(mids[b, 0])
        lo = sh.col_start[max(0, ival - shear.INDEX_RADIUS_SEARCH)]
        hi = sh.col_start[min(ch.nx - 1, ival + shear.INDEX_RADIUS_SEARCH + 1)]
        cand = np.arange(lo, hi)
        cand = cand[d[cand] < shear.CUTOFF_RADIUS]
        want = cand[np.argsort(d[cand], kind="stable")][:4]
        got = idx[idx >= 0]
        assert set(got) == set(want), (b, got, want)
        # weights follow the distances: exp(-(d/R)^2/2), normalised
        ww = np.exp(-0.5 * (d[got] / shear.CUTOFF_RADIUS) ** 2)
        assert np.allclose(w[idx >= 0] * ww.sum() / (w[idx >= 0].sum()), ww, rtol=1e-12)


# ---- TR_shear_1 / TR_shear_2 in the oracle ----------------------------------

def test_oracle_wall_shear_matches_reference_golden(oracle):
    z, ch, cfg = _golden_case()
    nodes = z["nodes"]
    n = ch.n
    FA = np.zeros(9 * n)
    FA.reshape(9, -1)[:, nodes] = z["F"].T
    rho, ux, uy, nut = (_scatter(n, nodes, z[k]) for k in ("rho", "ux", "uy", "nut"))
    for tag, nu in (("lam", None), ("turb", nut)):
        t = np.zeros(len(nodes))
        oracle.L.orc_wall_shear_nodes(C.byref(cfg), FA, rho, ux, uy,
                                      None if nu is None else nu.ctypes.data,
                                      np.ascontiguousarray(nodes, np.int32), len(nodes),
                                      np.ascontiguousarray(z["cfss"].ravel()), t)
        ref = z[f"tau_{tag}"]
        assert np.all(np.sign(t) == np.sign(ref))
        assert np.abs(t - ref).max() <= 1e-12 * np.abs(ref).max(), tag


def test_oracle_wall_shear_matches_reference_live(oracle, refk):
    ch = G.wavy_channel(96, 32, 5.0, 48)
    cfg = make_cfg(ch.nx, ch.ny, 1.2, 1e-5, 0.03)
    sh = shear.setup(ch)
    FA = perturbed_state(ch, seed=5, u_mean=0.03)
    _, _, nut, _ = komega_state(ch, seed=6)
    rng = np.random.default_rng(7)
    rho = 1.0 + 1e-3 * rng.standard_normal(ch.n)
    ux = 0.03 + 1e-2 * rng.standard_normal(ch.n)
    uy = 5e-3 * rng.standard_normal(ch.n)
    n = len(sh.nodes)
    ref = np.zeros(n)
    refk.L.ref_wall_shear_nodes(C.byref(cfg), rho, ux, uy, sh.cfss.ravel().copy(), FA.copy(), ref,
                                sh.nodes, nut, n)
    t, b = oracle_tau(oracle, cfg, sh, FA, rho, ux, uy, nut)
    assert np.abs(t - ref).max() <= 1e-12 * np.abs(ref).max()
    # TR_shear_2: dot(weights, tau of the four nodes)
    want = np.array([sum(w * t[j] for j, w in zip(jj, ww) if j >= 0)
                     for jj, ww in zip(sh.bl_nodes, sh.bl_weights)])
    assert np.allclose(b, want, rtol=1e-14, atol=0)


# ---- GPU ------------------------------------------------------------------

def _lattice(ch, rate, g, mu, komega, storage=_abi.STORE_FP32, **desc):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = rate, g, mu
    d.use_komega = 1 if komega else 0
    d.storage = storage
    for key, v in desc.items():
        setattr(d, key, v)
    L = Lattice(d)
    L.set_geometry(ch.ntype, ch.wallD if komega else None, ch.dX if komega else None,
                   ch.ibb_idx, ch.ibb_q)
    return L


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [_abi.STORE_FP32, _abi.STORE_FP16_NEQ])
@pytest.mark.parametrize("komega", [False, True])
def test_gpu_wall_shear_of_device_state(kofm_lib, oracle, storage, komega):
    """kofm_wall_shear against TR_shear_1/2 of the oracle applied to the
    state the device holds (downloaded populations, moments, nu_t)."""
    ch = G.wavy_channel(192, 48, 6.0, 96)
    rate, g, mu = 1.3, 2e-6, 0.05
    cfg = make_cfg(ch.nx, ch.ny, rate, g, mu)
    sh = shear.setup(ch)
    f = G.equilibrium_state(ch, ux=0.02)
    with _lattice(ch, rate, g, mu, komega, storage) as L:
        if komega:
            k, o, nut, s = komega_state(ch, seed=3)
            L.set_state(f, k, o, nut, s)
        else:
            L.set_state(f)
        L.set_shear(sh)
        L.step(40)
        t_gpu, b_gpu = L.wall_shear()
        st = L.get_state()
        FA = st[0]
        nu = st[3] if komega else None
        rho, ux, uy = L.get_macro()
    t, b = oracle_tau(oracle, cfg, sh, FA, rho, ux, uy, nu)
    scale = np.abs(t).max()
    assert scale > 0
    assert np.abs(t_gpu - t).max() <= 1e-9 * scale
    assert np.abs(b_gpu - b).max() <= 1e-9 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("komega,nsteps,tol", [(False, 300, 1e-5), (True, 10, 1e-5)])
def test_gpu_wall_shear_matches_oracle_run(kofm_lib, oracle, komega, nsteps, tol):
    """Shear after a run on the GPU against the shear of the FP64 oracle run
    from the same start (wavy walls: interpolated bounce-back at the shear
    nodes)."""
    ch = G.wavy_channel(192, 48, 6.0, 96)
    rate, g, mu = 1.3, 2e-6, 0.05
    cfg = make_cfg(ch.nx, ch.ny, rate, g, mu)
    sh = shear.setup(ch)
    if komega:
        k, o, nut, s = komega_state(ch, seed=3)
        f, k, o, nut, s = fp32_state(G.equilibrium_state(ch, ux=0.02), k, o, nut, s)
    else:
        (f,) = fp32_state(G.equilibrium_state(ch, ux=0.02))
        k = o = nut = s = None
    # k-omega: GMRES to 1e-10 in both, so that no solve's result depends on
    # where its cycle is cut (tests/test_wavy_gpu.py explains the tie)
    tight = dict(rel_tol=1e-10, abs_tol=1e-30, max_iters=1000)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, s, komega=komega,
                    ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q, **tight)
    sim.step(nsteps)
    t, b = oracle_tau(oracle, cfg, sh, sim.FA, sim.rho, sim.ux, sim.uy,
                      sim.nut if komega else None)
    with _lattice(ch, rate, g, mu, komega, komega_rel_tol=tight["rel_tol"],
                  komega_abs_tol=tight["abs_tol"], komega_max_iters=tight["max_iters"]) as L:
        L.set_state(f, k, o, nut, s)
        L.set_shear(sh)
        L.step(nsteps)
        t_gpu, b_gpu = L.wall_shear()
    et, eb = rel_l2(t_gpu, t), rel_l2(b_gpu, b)
    print(dict(nodes=et, links=eb))
    assert et < tol and eb < tol


@pytest.mark.gpu
def test_gpu_set_shear_rejects_bad_input(kofm_lib):
    ch = G.straight_channel(64, 16)
    sh = shear.setup(ch)
    with _lattice(ch, 1.0, 1e-6, 0.1, False) as L:
        lib, ctx = L.lib, L._ctx
        bad = sh.nodes.astype(np.int32).copy()
        bad[0] = ch.n
        cf = np.ascontiguousarray(sh.cfss)
        i32 = C.POINTER(C.c_int32)
        dp = C.POINTER(C.c_double)
        rc = lib.kofm_set_shear(ctx, bad.ctypes.data_as(i32), len(bad), cf.ctypes.data_as(dp),
                                None, None, 0)
        assert rc == _abi.ERR_INVALID_ARG
        bl = sh.bl_nodes.astype(np.int32).copy()
        bl[0, 0] = len(sh.nodes)
        nodes = sh.nodes.astype(np.int32)
        w = np.ascontiguousarray(sh.bl_weights)
        rc = lib.kofm_set_shear(ctx, nodes.ctypes.data_as(i32), len(nodes), cf.ctypes.data_as(dp),
                                bl.ctypes.data_as(i32), w.ctypes.data_as(dp), len(bl))
        assert rc == _abi.ERR_INVALID_ARG
        # no state yet: the shear needs one
        L.set_shear(sh)
        rc = lib.kofm_wall_shear(ctx, None, None)
        assert rc == _abi.ERR_STATE
