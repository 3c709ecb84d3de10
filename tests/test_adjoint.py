"""Discrete adjoint of the laminar step (kofm_adjoint; no counterpart in the
reference): the FP64 oracle adjoint (oracle/kofm_adjoint.c) against central
finite differences, its forward against the oracle step, and the device
adjoint against the oracle adjoint."""
import ctypes as C

import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, desc_default
from komegafoulingmodel_b200 import geometry as G
from komegafoulingmodel_b200 import shear
from oracle.orc import adj_run, make_cfg
from tests.cases import fp32_state, perturbed_state, rel_l2

RATE, FTERM = 1.3, 1e-5
MU = (1.0 / RATE - 0.5) / 3.0


def _case(nx=48, ny=20, amp=3.0, lam=24, ibb_all=True):
    ch = G.wavy_channel(nx, ny, amp, lam, ibb_all=ibb_all)
    cfg = make_cfg(nx, ny, RATE, FTERM, MU)
    return ch, cfg, shear.setup(ch)


def test_adjoint_forward_is_the_oracle_step(oracle):
    ch, cfg, _ = _case()
    F = perturbed_state(ch, seed=2, u_mean=0.02)
    n = ch.n
    fs, FA = np.zeros(9 * n), np.zeros(9 * n)
    oracle.L.orc_adj_collide(C.byref(cfg), ch.ntype, F, fs)
    oracle.L.orc_adj_stream(C.byref(cfg), ch.ntype, ch.ibb_idx, ch.ibb_q, len(ch.ibb_idx), fs, FA)
    FB = np.zeros(9 * n)
    z = np.zeros(n)
    oracle.L.orc_collide_push(C.byref(cfg), F, FB, ch.ntype, z.copy(), z.copy(), z.copy(), z.copy(),
                              z.copy(), z.copy(), z.copy(), np.zeros(3 * n), 0, 0)
    oracle.L.orc_ibb(C.byref(cfg), ch.ibb_idx, ch.ibb_q, FB, len(ch.ibb_idx))
    assert np.array_equal(FA, FB)


def test_oracle_adjoint_matches_finite_differences(oracle):
    """Links with q = 1/2 are left out here: the Bouzidi interpolation changes
    formula there (2q <= 1 / 2q > 1), so J has a kink in q at 1/2 and the
    adjoint gives the 2q <= 1 side's derivative."""
    ch, cfg, sh = _case(ibb_all=False)
    F0 = perturbed_state(ch, seed=3, u_mean=0.02)
    T = 12
    J, dq, dF0 = adj_run(oracle, cfg, ch, F0, T, shear_setup=sh, want_dF0=True)
    rng = np.random.default_rng(1)
    for _ in range(3):   # wall fractions
        d = rng.standard_normal(len(dq))
        h = 1e-6
        Jp, _, _ = adj_run(oracle, cfg, ch, F0, T, q=ch.ibb_q + h * d, shear_setup=sh)
        Jm, _, _ = adj_run(oracle, cfg, ch, F0, T, q=ch.ibb_q - h * d, shear_setup=sh)
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - dq @ d) <= 1e-6 * max(abs(fd), np.abs(dq).sum() * 1e-3), (fd, dq @ d)
    fl = np.tile(ch.fluid_mask().ravel(), 9)
    for _ in range(2):   # initial populations
        d = rng.standard_normal(F0.shape) * fl
        h = 1e-7
        Jp, _, _ = adj_run(oracle, cfg, ch, F0 + h * d, T, shear_setup=sh)
        Jm, _, _ = adj_run(oracle, cfg, ch, F0 - h * d, T, shear_setup=sh)
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - dF0 @ d) <= 1e-7 * abs(fd)


def _gpu_adjoint(ch, sh, F0, T, q=None):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = RATE, FTERM, MU
    with Lattice(d) as L:
        L.set_geometry(ch.ntype, None, None, ch.ibb_idx, ch.ibb_q if q is None else q)
        if sh is not None:
            L.set_shear(sh)
        L.set_state(F0)
        L.step(1)   # g^0 = collide(FA^0)
        return L.adjoint(T)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [1, 7, 16])
def test_gpu_adjoint_matches_oracle(kofm_lib, oracle, T):
    """sqrt(T) checkpoints: T = 7 recomputes segments of 3, 3, 1 states; the
    device forward stores FP32 populations, so J and dJ/dq differ from the
    FP64 oracle by that rounding only."""
    ch, cfg, sh = _case(96, 40, 5.0, 48)
    (F0,) = fp32_state(perturbed_state(ch, seed=4, u_mean=0.02))
    J, dq, _ = adj_run(oracle, cfg, ch, F0, T, shear_setup=sh)
    Jg, dqg = _gpu_adjoint(ch, sh, F0, T)
    print(dict(T=T, J=(J, Jg), dq_err=rel_l2(dqg, dq)))
    assert abs(Jg - J) <= 1e-6 * abs(J)
    assert rel_l2(dqg, dq) < 1e-4


@pytest.mark.gpu
def test_gpu_adjoint_pressure_term_only(kofm_lib, oracle):
    ch, cfg, _ = _case(96, 40, 5.0, 48)
    (F0,) = fp32_state(perturbed_state(ch, seed=5, u_mean=0.02))
    J, dq, _ = adj_run(oracle, cfg, ch, F0, 9)
    Jg, dqg = _gpu_adjoint(ch, None, F0, 9)
    assert abs(Jg - J) <= 1e-6 * abs(J) + 1e-12 and rel_l2(dqg, dq) < 1e-4
