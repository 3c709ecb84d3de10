"""The reference's padded host layout: rows of XsizeFull = nX rounded up to a
multiple of 128 (clProblem.cpp:469), the columns nX..XsizeFull-1 unused.  The
device keeps its own pitch; every host array (populations, fields, IBB link
indices, temperature) is read and written in the padded layout.  A channel of
nx = 200 (XsizeFull 256) against the oracle on the same padded arrays."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from oracle.orc import OracleSim, ThermalCfg, make_cfg
from tests.cases import fp32_state, rel_l2

NX, NY = 200, 40
NXF = G.xsize_full(NX)


def test_padded_geometry():
    assert NXF == 256
    ch = G.wavy_channel(NX, NY, 5.0, 100, nx_full=NXF)
    t = (ch.ntype.astype(np.int32) & 0xFFFF).reshape(NY, NXF)
    assert np.all((t[:, NX:] & G.M_SOLID) != 0)
    node = ch.ibb_idx % ch.n
    assert np.all(node % NXF < NX)
    assert np.all(ch.dX.reshape(4, NY, NXF)[:, :, NX:] == 0)


def _lattice(ch, rate, g, mu, komega=False, thermal=False, **desc):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = rate, g, mu
    d.use_komega = 1 if komega else 0
    d.use_thermal = 1 if thermal else 0
    for key, v in desc.items():
        setattr(d, key, v)
    L = Lattice(d)
    L.set_geometry(ch.ntype, ch.wallD if komega else None, ch.dX if (komega or thermal) else None,
                   ch.ibb_idx, ch.ibb_q)
    return L, d


@pytest.mark.gpu
def test_padded_laminar_thermal_matches_oracle(kofm_lib, oracle):
    ch = G.wavy_channel(NX, NY, 5.0, 100, nx_full=NXF)
    rate, g, mu = 1.25, 2e-6, 0.1
    (f,) = fp32_state(G.equilibrium_state(ch, ux=0.01))
    cfg = make_cfg(NX, NY, rate, g, mu, nxf=NXF)
    L, d = _lattice(ch, rate, g, mu, thermal=True, thermal_rel_tol=1e-12)
    T0 = G.temperature_field(ch)
    th = ThermalCfg(mu / d.pr_number, d.alpha_foul, 1.0 / d.pr_turb_number, d.t_in)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q,
                    thermal=dict(T=T0, cfg=th, rel_tol=1e-12, abs_tol=d.thermal_abs_tol))
    sim.step(50)
    with L:
        L.set_state(f)
        L.set_temperature(T0)
        L.step(50)
        rho, ux, uy = L.get_macro()
        f2 = L.get_state()[0]
        T = L.get_temperature()
    fl = ch.fluid_mask().ravel()
    assert rel_l2(ux, sim.ux, fl) < 1e-5 and rel_l2(rho, sim.rho, fl) < 1e-6
    dom = ((ch.ntype.astype(np.int32) & 0xFFFF) & G.M0_FLUID) != 0
    assert rel_l2(T, sim.T, dom) < 1e-8
    # padding columns come back as zeros
    pad = np.zeros((NY, NXF), bool)
    pad[:, NX:] = True
    assert np.all(f2.reshape(9, -1)[:, pad.ravel()] == 0) and np.all(T[pad.ravel()] == 0)


@pytest.mark.gpu
def test_padded_komega_matches_oracle(kofm_lib, oracle):
    from tests.test_komega_gpu import channel_case
    ch0, f0, k0, o0, nut0, rate, g, nu = channel_case(nx=NX, ny=34)
    ch = G.straight_channel(NX, 34, nx_full=NXF)

    def pad(a, planes=1):
        a = np.asarray(a).reshape(planes, 34, NX)
        out = np.zeros((planes, 34, NXF))
        out[:, :, :NX] = a
        return out.ravel()

    f, k, o, nut = pad(f0, 9), pad(k0), pad(o0), pad(nut0)
    cfg = make_cfg(NX, 34, rate, g, nu, nxf=NXF)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, komega=True)
    sim.step(20)
    L, _ = _lattice(ch, rate, g, nu, komega=True)
    with L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.step(20)
        _, k2, o2, _, _ = L.get_state()
        ux = L.get_macro()[1]
    fl = ch.fluid_mask().ravel()
    for name, a, b in (("ux", ux, sim.ux), ("k", k2, sim.K), ("omega", o2, sim.O)):
        assert rel_l2(a, b, fl) < 1e-5, name
