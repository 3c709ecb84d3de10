"""The oracle's GMRES restatement (GMRESSolver::solve) against direct solves."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from komegafoulingmodel_b200 import geometry as G
from oracle.orc import GmresStats, OracleSim, make_cfg
from tests.cases import komega_state, perturbed_state


def _assembled(oracle, nx=64, ny=20, seed=3, dt=1.0):
    cfg = make_cfg(nx, ny, 1.9, 1e-6, 0.01)
    ch = G.straight_channel(nx, ny)
    F = perturbed_state(ch, seed=seed)
    k, o, nut, s = komega_state(ch, seed=seed + 1)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, F, k, o, nut, s, komega=True)
    L, cp = oracle.L, C.byref(cfg)
    L.orc_collide_push(cp, sim.FA, sim.FB, sim.m, sim.rho, sim.ux, sim.uy, sim.K, sim.O,
                       sim.wallD, sim.nut, sim.S, 2, 1)
    L.orc_komega_diffusivities(cp, sim.m, sim.K, sim.O, sim.nut, sim.wallD, sim.Dk, sim.Do,
                               sim.F1, sim.dkdo, sim.rho, sim.dX)
    L.orc_komega_coeffs(cp, sim.ind, sim.K, sim.O, sim.nut, sim.Dk, sim.Do, sim.F1,
                        sim.dkdo, sim.S, sim.rho, sim.ux, sim.uy, sim.kA, sim.oA, sim.kb,
                        sim.ob, sim.dX, sim.wallD, sim.m, dt)
    return sim


def _direct(IA, JA, A, b, n):
    M = sp.csr_matrix((A, JA, IA), shape=(n, n))
    rows = np.diff(IA) > 0
    x = np.zeros(n)
    x[rows] = sla.spsolve(M[rows][:, rows].tocsc(), b[rows])
    return x


@pytest.mark.parametrize("which", ["omega", "k"])
def test_gmres_reaches_reference_tolerance_and_tight_solution(oracle, which):
    sim = _assembled(oracle)
    A, b, x0 = (sim.oA, sim.ob, sim.O) if which == "omega" else (sim.kA, sim.kb, sim.K)
    n = sim.n
    sol = _direct(sim.IA, sim.JA, A, b, n)
    for tol, bound in ((1e-4, 1e-3), (1e-13, 1e-11)):
        x, bb, st = x0.copy(), b.copy(), GmresStats()
        oracle.L.orc_gmres_solve(n, sim.IA, sim.JA, A, bb, x, 10, 1000, tol, 1e-30, C.byref(st))
        assert st.nan == 0
        # the correction solved for is sol - x0; its error is bounded by the tolerance
        err = np.linalg.norm(x - sol) / np.linalg.norm(sol - x0)
        assert err < bound, (tol, err, st.iters, st.restarts)
        # the estimate the solver stops on matches the true residual of A d = b - A x0
        M = sp.csr_matrix((A, sim.JA, sim.IA), shape=(n, n))
        true_rel = np.linalg.norm(b - M @ x) / np.linalg.norm(b - M @ x0)
        assert true_rel <= max(tol, 1e-13) * 1.01


def test_gmres_zero_rhs_takes_the_nan_path(oracle):
    """rho0 / norm_rhs = 0/0 is NaN: the reference calls resetTimeFunc
    (GMRESSolver.cpp:1537-1546), i.e. halves the k-omega time step."""
    sim = _assembled(oracle)
    n = sim.n
    M = sp.csr_matrix((sim.oA, sim.JA, sim.IA), shape=(n, n))
    x0 = sim.O.copy()
    b = M @ x0  # exact solution already: b - A x0 == 0
    st = GmresStats()
    oracle.L.orc_gmres_solve(n, sim.IA, sim.JA, sim.oA, b, x0, 10, 1000, 1e-4, 1e-7, C.byref(st))
    assert st.nan == 1 and st.iters == 0


def test_komega_solve_halves_dt_on_nan(oracle):
    """kOmega::Solve: a NaN residual doubles stepsPerLB and halves dt."""
    nx, ny = 32, 12
    cfg = make_cfg(nx, ny, 1.9, 0.0, 0.01)
    ch = G.straight_channel(nx, ny)
    F = G.equilibrium_state(ch)
    k, o, nut = G.komega_fields(ch, 1e-4, 1e-2)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, F, k, o, nut, komega=True)
    sim.O[:] = np.nan  # poison omega -> NaN residual on every sub-step
    sim.step(1)
    # dt halves on every NaN until the runaway bound of 2^20 sub-steps
    assert sim.kst.last_o.nan == 1
    assert sim.kst.steps_per_lb > (1 << 20) and sim.kst.dt < 1e-6
