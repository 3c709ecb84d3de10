"""The k-omega sub-stepping on the GPU: kOmega::Solve's dt halving on a NaN
residual and its doubling after 20 calm steps (kOmega.cpp:31-73, 387-414;
GMRESSolver::checkConvergence, GMRESSolver.cpp:1535-1546), what the fields
hold after a NaN solve, and the solver's non-convergence status.

Failures are made on the host: either a solve is told to report a NaN
residual (kofm_debug_fail_solves, and the same hook in the oracle's
kOmega::Solve), or NaN values are uploaded through kofm_set_state.  Nothing
faults on the device."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from oracle.orc import OracleSim, make_cfg
from tests.cases import fp32_state, rel_l2
from tests.test_komega_gpu import channel_case, make_lattice

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mask", [1, 2, 3])
def test_halving_and_doubling_follow_the_oracle(kofm_lib, oracle, mask):
    """A NaN residual in the omega solve (mask 1), the k solve (2) or both (3)
    of step 4: dt halves once per failed system, the failed field keeps its
    value, the sub-steps of the halved dt run, and dt doubles back after 20
    calm steps -- step by step as the FP64 oracle's kOmega::Solve given the
    same failure; fields within 1e-5 after 30 steps."""
    ch, f, k, o, nut, rate, g, nu = channel_case(nx=128, ny=34)
    f, k, o, nut = fp32_state(f, k, o, nut)
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, komega=True)
    seen = []
    with make_lattice(ch, rate, g, nu) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        for step in range(30):
            if step == 3:
                L.debug_fail_solves(1, mask)
                sim.kst.fail_solves, sim.kst.fail_mask = 1, mask
            L.step(1)
            sim.step(1)
            st = L.stats()
            seen.append((st.steps_per_lb, st.dt, st.time_since_change))
            assert (st.steps_per_lb, st.dt, st.time_since_change) == (
                sim.kst.steps_per_lb, sim.kst.dt, sim.kst.time_since_change), step
        rho, ux, _ = L.get_macro()
        _, k2, o2, _, _ = L.get_state()
    halved = 2 if mask == 3 else 1
    assert seen[3][0] == 2 ** halved and seen[3][1] == 0.5 ** halved
    assert seen[2][0] == 1 and seen[-1][0] < seen[3][0]   # doubled back after calm steps
    fl = ch.fluid_mask().ravel()
    errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl),
                k=rel_l2(k2, sim.K, fl), omega=rel_l2(o2, sim.O, fl))
    print(seen[:6], errs)
    for key, e in errs.items():
        assert e < 1e-5, errs


def _nan_state(nodes=(0.3, 0.5, 0.7)):
    ch, f, k, o, nut, rate, g, nu = channel_case(nx=128, ny=34)
    fl = np.flatnonzero(ch.fluid_mask().ravel())
    bad = fl[(np.array(nodes) * len(fl)).astype(int)]
    k, o = k.copy(), o.copy()
    k[bad] = np.nan
    o[bad] = np.nan
    return ch, f, k, o, nut, rate, g, nu, bad


def test_nan_fields_halve_until_the_cap_and_keep_their_values(kofm_lib):
    """NaN in k and omega at three fluid nodes: every solve of the update
    meets a NaN residual, so dt halves until more than 2^20 sub-steps would
    be needed and the update returns KOFM_ERR_NAN (the reference would halve
    for ever).  k and omega are then exactly the fields from before the
    update (the NaN stays at its three nodes and spreads nowhere), and a
    repaired state steps again from dt = 1."""
    ch, f, k, o, nut, rate, g, nu, bad = _nan_state()
    with make_lattice(ch, rate, g, nu) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.lb_step()
        _, k_pre, o_pre, _, _ = L.get_state()
        assert np.isnan(k_pre[bad]).all() and np.isnan(o_pre[bad]).all()
        assert L.komega_update_status() == _abi.ERR_NAN
        st = L.stats()
        assert st.steps_per_lb > 2 ** 20 and st.dt == 1.0 / st.steps_per_lb
        assert st.omega_nan == 1 and st.k_nan == 1
        _, k_post, o_post, _, _ = L.get_state()
        assert np.array_equal(k_post, k_pre, equal_nan=True)
        assert np.array_equal(o_post, o_pre, equal_nan=True)
        # a repaired state starts the sub-stepping again
        ch2, f2, k2, o2, nut2, *_ = channel_case(nx=128, ny=34)
        L.set_state(f2, k2, o2, nut2, np.zeros(3 * ch.n))
        L.step(3)
        st = L.stats()
        assert st.steps_per_lb == 1 and st.dt == 1.0 and st.omega_nan == 0 and st.k_nan == 0
        _, k3, o3, _, _ = L.get_state()
        assert np.isfinite(k3).all() and np.isfinite(o3).all()


def test_solve_reports_nan_and_leaves_the_fields(kofm_lib):
    """kofm_komega_solve on NaN systems returns KOFM_ERR_NAN and leaves k and
    omega as they were."""
    ch, f, k, o, nut, rate, g, nu, bad = _nan_state()
    with make_lattice(ch, rate, g, nu) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        L.lb_step()
        L.komega_assemble(1.0)
        _, k_pre, o_pre, _, _ = L.get_state()
        st, iters, rel = L.komega_solve(raise_on_error=False)
        assert st == _abi.ERR_NAN
        _, k_post, o_post, _, _ = L.get_state()
        assert np.array_equal(k_post, k_pre, equal_nan=True)
        assert np.array_equal(o_post, o_pre, equal_nan=True)


def test_iteration_cap_reports_not_converged(kofm_lib):
    """komega_max_iters = 10 with Krylov dimension 10 leaves one restart
    (maxRestarts = max_iters / krylov, GMRESSolver.cpp:1412): one cycle runs
    and no convergence check follows, so the solve returns
    KOFM_ERR_NOT_CONVERGED; with the default cap the same systems converge."""
    ch, f, k, o, nut, rate, g, nu = channel_case(nx=128, ny=34)
    for cap, want in ((10, _abi.ERR_NOT_CONVERGED), (1000, 0)):
        d = desc_default()
        d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
        d.tau, d.fterm, d.mu = rate, g, nu
        d.use_komega = 1
        d.komega_max_iters = cap
        with Lattice(d) as L:
            L.set_geometry(ch.ntype, ch.wallD, ch.dX)
            L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
            L.lb_step()
            L.komega_assemble(1.0)
            st, iters, rel = L.komega_solve(raise_on_error=False)
            assert st == want, (cap, st, iters, rel)
            s = L.stats()
            if cap == 10:
                assert s.omega_restarts == 1 and s.k_restarts == 1
