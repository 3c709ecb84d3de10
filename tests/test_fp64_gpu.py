"""The FP64 storage form (KOFM_STORE_FP64): populations, node fields and all
arithmetic in FP64 -- the reference's own precision (Kernels/Heading.cl:7,
FTYPE double) -- against the FP64 oracle.  With the GMRES solves run to a
tight tolerance the device and the oracle compute the same step in different
summation orders only, so the fields agree to ~1e-12 after 100 steps."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from oracle.orc import OracleSim, make_cfg
from tests.cases import rel_l2
from tests.test_komega_gpu import channel_case

pytestmark = pytest.mark.gpu

TIGHT = dict(rel_tol=1e-12, abs_tol=1e-30, max_iters=1000)


def _fp64_lattice(ch, rate, g, nu, komega, **desc):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = rate, g, nu
    d.use_komega = 1 if komega else 0
    d.storage = _abi.STORE_FP64
    for key, v in desc.items():
        setattr(d, key, v)
    L = Lattice(d)
    L.set_geometry(ch.ntype, ch.wallD if komega else None, ch.dX if komega else None,
                   ch.ibb_idx if len(ch.ibb_idx) else None, ch.ibb_q if len(ch.ibb_q) else None)
    return L


@pytest.mark.parametrize("classic", [0, 1])
def test_komega_channel_100_steps_at_1e10(kofm_lib, oracle, classic):
    """rho, u, k, omega within rel-L2 1e-10 of the oracle after 100 steps of
    the k-omega channel (both solve forms), from the same FP64 state."""
    ch, f, k, o, nut, rate, g, nu = channel_case()
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, komega=True, **TIGHT)
    sim.step(100)
    with _fp64_lattice(ch, rate, g, nu, True, komega_rel_tol=TIGHT["rel_tol"],
                       komega_abs_tol=TIGHT["abs_tol"], komega_classic=classic) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.step(100)
        rho, ux, uy = L.get_macro()
        _, k2, o2, nut2, _ = L.get_state()
    fl = ch.fluid_mask().ravel()
    errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl), k=rel_l2(k2, sim.K, fl),
                omega=rel_l2(o2, sim.O, fl), nut=rel_l2(nut2, sim.nut, fl))
    print(errs)
    for key, e in errs.items():
        assert e < 1e-10, errs


def test_komega_channel_reference_tolerance(kofm_lib, oracle):
    """At the reference's GMRES tolerances the cycles end where rounding puts
    the xi-test tie, so the solves agree to the size of the correction's
    residual: fields within 1e-6 after 100 steps, and the same restart counts
    in the last step."""
    ch, f, k, o, nut, rate, g, nu = channel_case()
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, komega=True)
    sim.step(100)
    with _fp64_lattice(ch, rate, g, nu, True) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.step(100)
        st = L.stats()
        rho, ux, _ = L.get_macro()
        _, k2, o2, _, _ = L.get_state()
    fl = ch.fluid_mask().ravel()
    errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl), k=rel_l2(k2, sim.K, fl),
                omega=rel_l2(o2, sim.O, fl))
    print(errs, (st.omega_restarts, st.k_restarts))
    assert (st.omega_restarts, st.k_restarts) == (sim.kst.last_o.restarts, sim.kst.last_k.restarts)
    for key, e in errs.items():
        assert e < 1e-6, errs


def test_laminar_wavy_1000_steps(kofm_lib, oracle):
    """Laminar wavy channel with interpolated bounce-back: FP64 device vs FP64
    oracle after 1000 steps within 1e-12."""
    nx, ny = 256, 40
    ch = G.wavy_channel(nx, ny, 6.0, 128)
    rate, g, mu = 1.25, 2e-6, 0.1
    f = G.equilibrium_state(ch, ux=0.01)
    sim = OracleSim(oracle, make_cfg(nx, ny, rate, g, mu), ch.ntype, ch.dX, ch.wallD, f,
                    ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q)
    sim.step(1000)
    with _fp64_lattice(ch, rate, g, mu, False) as L:
        L.set_state(f)
        L.step(1000)
        rho, ux, uy = L.get_macro()
        f2, *_ = L.get_state()
    fl = ch.fluid_mask().ravel()
    errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl),
                uy=float(np.linalg.norm((uy - sim.uy)[fl]) / np.linalg.norm(sim.ux[fl])),
                f=rel_l2(f2, sim.FA))
    print(errs)
    for key, e in errs.items():
        assert e < 1e-12, errs


def test_fp64_form_reductions_and_refusals(kofm_lib):
    """Reductions read the FP64 fields; the thermal update and the device
    geometry builder are not offered with this form."""
    ch, f, k, o, nut, rate, g, nu = channel_case(nx=128, ny=34)
    with _fp64_lattice(ch, rate, g, nu, True) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.step(3)
        _, k2, _, _, _ = L.get_state()
        assert L.reduce(_abi.FIELD_K) == pytest.approx(float(np.sum(k2)), rel=1e-13)
        assert L.reduce(_abi.FIELD_K, _abi.OP_MAX) == float(np.max(k2))
        y = np.full(ch.nx, 0.5)
        assert L.lib.kofm_set_walls(L._ctx, y.ctypes.data_as(_abi.C.POINTER(_abi.C.c_double)),
                                    (y + ch.ny - 2).ctypes.data_as(_abi.C.POINTER(_abi.C.c_double)),
                                    None, None, 0.001, 50, 0) == _abi.ERR_STATE
    d = desc_default()
    d.storage = _abi.STORE_FP64
    d.use_thermal = 1
    ctx = _abi.C.c_void_p()
    assert kofm_lib.kofm_create(_abi.C.byref(d), _abi.C.byref(ctx)) == -110
