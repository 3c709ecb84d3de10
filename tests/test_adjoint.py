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


def _gpu_adjoint(ch, sh, F0, T, q=None, mem=None):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = RATE, FTERM, MU
    with Lattice(d) as L:
        L.set_geometry(ch.ntype, None, None, ch.ibb_idx, ch.ibb_q if q is None else q)
        if sh is not None:
            L.set_shear(sh)
        if mem is not None:
            L.set_adjoint_memory(mem)
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
def test_gpu_adjoint_memory_cap_does_not_change_results(kofm_lib, oracle):
    """Every state stored (default cap), sqrt(T) checkpoints only (cap 0) and a
    cap between (segments of 6 states + 2 checkpoints for T = 17): the same
    kernels on the same states, so J and dJ/dq agree bit for bit."""
    ch, cfg, sh = _case(96, 40, 5.0, 48)
    (F0,) = fp32_state(perturbed_state(ch, seed=6, u_mean=0.02))
    T = 17
    state = 4 * 9 * (-(-ch.nx_full // 128) * 128) * ch.ny   # FP32 state at the device row pitch
    runs = [_gpu_adjoint(ch, sh, F0, T, mem=m) for m in (None, 0, 7 * state + 6 * 9 * 8 * len(sh.nodes))]
    for J, dq in runs[1:]:
        assert J == runs[0][0] and np.array_equal(dq, runs[0][1])
    J, dq, _ = adj_run(oracle, cfg, ch, F0, T, shear_setup=sh)
    assert abs(runs[0][0] - J) <= 1e-6 * abs(J) and rel_l2(runs[0][1], dq) < 1e-4


@pytest.mark.gpu
def test_gpu_adjoint_pressure_term_only(kofm_lib, oracle):
    ch, cfg, _ = _case(96, 40, 5.0, 48)
    (F0,) = fp32_state(perturbed_state(ch, seed=5, u_mean=0.02))
    J, dq, _ = adj_run(oracle, cfg, ch, F0, 9)
    Jg, dqg = _gpu_adjoint(ch, None, F0, 9)
    assert abs(Jg - J) <= 1e-6 * abs(J) + 1e-12 and rel_l2(dqg, dq) < 1e-4


def test_shape_gradient_matches_finite_differences(oracle):
    """dJ/d(wall heights) = (dq/dy)^T dJ/dq against central differences of J
    over rebuilt geometries (walls 0.3 cell off the half-way positions and a
    perturbation small enough that no node changes type)."""
    nx, ny = 48, 20
    x = np.arange(nx)
    h = 2.0 * 0.5 * (1 - np.cos(2 * np.pi * x / 24))
    yb, yt = 0.8 + h, ny - 1.8 - h
    ch = G.channel_from_walls(nx, ny, yb, yt, ibb_all=True)
    cfg = make_cfg(nx, ny, RATE, FTERM, MU)
    sh = shear.setup(ch)
    F0 = perturbed_state(ch, seed=6, u_mean=0.02)
    T = 8
    J, dq, _ = adj_run(oracle, cfg, ch, F0, T, shear_setup=sh)
    gb, gt = G.shape_gradient(ch, dq)
    rng = np.random.default_rng(2)
    db, dt_ = rng.standard_normal(nx), rng.standard_normal(nx)
    eps = 1e-6
    Js = []
    for sgn in (1, -1):
        c2 = G.channel_from_walls(nx, ny, yb + sgn * eps * db, yt + sgn * eps * dt_, ibb_all=True)
        assert np.array_equal(c2.ntype, ch.ntype) and np.array_equal(c2.ibb_idx, ch.ibb_idx)
        Js.append(adj_run(oracle, cfg, c2, F0, T, shear_setup=sh)[0])
    fd = (Js[0] - Js[1]) / (2 * eps)
    want = gb @ db + gt @ dt_
    assert abs(fd - want) <= 1e-6 * abs(fd), (fd, want)


class WallShapeObjective:
    """Thin torch.autograd.Function over kofm_adjoint: J(y_bot, y_top) of a
    laminar wavy channel run from F0, with the gradient the device adjoint
    gives through dq/dy (test wrapper)."""

    @staticmethod
    def apply(y_bot, y_top, F0, T, nx, ny):
        import torch

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, yb, yt):
                ch = G.channel_from_walls(nx, ny, yb.detach().numpy(), yt.detach().numpy(),
                                          ibb_all=True)
                J, dq = _gpu_adjoint(ch, shear.setup(ch), F0, T)
                gb, gt = G.shape_gradient(ch, dq)
                ctx.save_for_backward(torch.from_numpy(gb), torch.from_numpy(gt))
                return torch.tensor(J, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gJ):
                gb, gt = ctx.saved_tensors
                return gJ * gb, gJ * gt

        return _Fn.apply(y_bot, y_top)


@pytest.mark.gpu
def test_torch_wrapper_gradient(kofm_lib, oracle):
    """autograd through the wrapper gives the device shape gradient; it agrees
    with the FP64 oracle's, and a small step against it lowers J."""
    import torch
    nx, ny, T = 96, 40, 10
    x = np.arange(nx)
    h = 3.0 * 0.5 * (1 - np.cos(2 * np.pi * x / 48))
    yb = torch.tensor(0.8 + h, dtype=torch.float64, requires_grad=True)
    yt = torch.tensor(ny - 1.8 - h, dtype=torch.float64, requires_grad=True)
    ch = G.channel_from_walls(nx, ny, yb.detach().numpy(), yt.detach().numpy(), ibb_all=True)
    (F0,) = fp32_state(perturbed_state(ch, seed=7, u_mean=0.02))
    J = WallShapeObjective.apply(yb, yt, F0, T, nx, ny)
    J.backward()
    cfg = make_cfg(nx, ny, RATE, FTERM, MU)
    Jo, dqo, _ = adj_run(oracle, cfg, ch, F0, T, shear_setup=shear.setup(ch))
    gbo, gto = G.shape_gradient(ch, dqo)
    g = np.concatenate([yb.grad.numpy(), yt.grad.numpy()])
    go = np.concatenate([gbo, gto])
    assert abs(J.item() - Jo) <= 1e-6 * abs(Jo) and rel_l2(g, go) < 1e-4
    # descent: the step moves the walls by < 1e-3 cell (no node changes type)
    step = 5e-4 / np.abs(g).max()
    with torch.no_grad():
        yb2, yt2 = yb - step * yb.grad, yt - step * yt.grad
    c2 = G.channel_from_walls(nx, ny, yb2.numpy(), yt2.numpy(), ibb_all=True)
    assert np.array_equal(c2.ntype, ch.ntype)
    J2 = WallShapeObjective.apply(yb2, yt2, F0, T, nx, ny)
    assert J2.item() < J.item()


@pytest.mark.gpu
def test_gpu_adjoint_c4_against_fp64_adjoint(kofm_lib, oracle):
    """The adjoint case's lattice (1024 x 256, wall h(x) = sum_{m<=64} a_m
    cos(2 pi m x / nx), a_m ~ N(0, (4/m)^2), seed 0) over 20 steps: device J
    and dJ/dq against the FP64 oracle adjoint of the same run."""
    from komegafoulingmodel_b200.adjoint import Case
    case = Case(1024, 256)
    ch = case.channel()
    # the oracle follows the reference's lbIBB where it reads outside the
    # fluid (the unwrapped seam neighbour, the wall node of a one-node notch);
    # the case's walls have neither
    assert case.seam_ok(ch) and case.notches(ch) == 0
    (F0,) = fp32_state(case.start(ch))
    sh = shear.setup(ch)
    T = 20
    cfg = make_cfg(ch.nx, ch.ny, case.rate, case.fterm, case.nu)
    J, dq, _ = adj_run(oracle, cfg, ch, F0, T, shear_setup=sh)
    with case.lattice(ch) as L:
        L.set_state(F0)
        L.step(1)
        Jg, dqg = L.adjoint(T)
    print(dict(J=(J, Jg), dq_err=rel_l2(dqg, dq)))
    assert abs(Jg - J) <= 1e-6 * abs(J) and rel_l2(dqg, dq) < 1e-4
