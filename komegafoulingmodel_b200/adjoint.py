"""The adjoint/gradient case: d(objective)/d(wall-shape coefficients) of a
laminar channel whose wall height is h(x) = sum_{m=1..64} a_m cos(2 pi m x / nx),
a_m ~ N(0, (4/m)^2) from one seed, through kofm_adjoint (every state stored;
also timed with sqrt(T) checkpoints),
checked against central finite differences of the device forward along seeded
random directions, with the adjoint's cost against the forward's.

    python -m komegafoulingmodel_b200.adjoint [--nx 1024 --ny 256 --steps 2000]

Prints one JSON line.  The k-omega adjoint is not built: the flow is laminar
(nu = 0.01, Re ~ 1.3e3 on the height), the objective that of kofm_adjoint
(mean-density drop between the first and last columns / 3 plus the TR_shear_1
wall shear at the shear nodes, summed over the steps).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import geometry as G
from . import shear


def coefficients(n_modes: int = 64, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    m = np.arange(1, n_modes + 1)
    return rng.standard_normal(n_modes) * (4.0 / m)


def walls(a: np.ndarray, nx: int, ny: int, with_source: bool = False):
    """Bottom wall y = b + h(x) - h(0), top wall mirrored (ny - 1 - y).

    The offset b puts the wall at x = 0 (where every cosine is flat) 0.6
    above a row, so the first fluid row there is 0.4 away and no link across
    the periodic seam has 2q > 1 even when the seam columns are given
    interpolated links (seam_ibb; such links read an unwrapped upstream
    neighbour in the reference's lbIBB); b is the smallest such value that
    keeps the wall at least 0.8 above row 0 (piecewise constant in a).

    A column that dips below both neighbours across a lattice row would leave
    a one-node notch whose fluid node has wall links on both sides; there the
    reference's lbIBB reads populations of a solid node (2q > 1 needs the
    upstream neighbour, which is wall).  Such columns are lifted to their
    lower neighbour's height; with_source also returns, per column, the
    column whose height it carries."""
    x = np.arange(nx)
    m = np.arange(1, len(a) + 1)
    h = (a[:, None] * np.cos(2 * np.pi * m[:, None] * x[None, :] / nx)).sum(0)
    h = h - h[0]
    b = np.ceil(0.8 - h.min() - 0.6) + 0.6
    yb = b + h
    src = np.arange(nx)
    for i in range(nx):
        lo = min(yb[(i - 1) % nx], yb[(i + 1) % nx])
        if yb[i] < lo and np.floor(lo) > np.floor(yb[i]) and np.floor(lo) != lo:
            j = (i - 1) % nx if yb[(i - 1) % nx] <= yb[(i + 1) % nx] else (i + 1) % nx
            yb[i] = yb[j]
            src[i] = j
    if with_source:
        return yb, (ny - 1) - yb, src
    return yb, (ny - 1) - yb


def modes(nx: int, n_modes: int) -> np.ndarray:
    x = np.arange(nx)
    m = np.arange(1, n_modes + 1)
    return np.cos(2 * np.pi * m[:, None] * x[None, :] / nx)


class Case:
    def __init__(self, nx, ny, nu=0.01, u_mean=0.05, seed=0):
        from .lattice import desc_default
        self.nx, self.ny = nx, ny
        self.a = coefficients(seed=seed)
        self.rate = 1.0 / (3.0 * nu + 0.5)
        self.nu = nu
        R = 0.5 * (ny - 2)
        self.fterm = G.force_from_re((2.0 / 3.0) * 1.5 * u_mean * R / nu, nu, R)
        self.u_mean = u_mean
        self.desc_default = desc_default

    def channel(self, a=None):
        yb, yt = walls(self.a if a is None else a, self.nx, self.ny)
        return G.channel_from_walls(self.nx, self.ny, yb, yt, ibb_all=True, wall_distance=False)

    @staticmethod
    def notches(ch) -> int:
        """Fluid nodes with wall links in two opposite directions."""
        t = ch.ntype.astype(np.int32) & 0xFFFF
        fl = (t & G.M_SOLID) == 0
        n = 0
        for q in (1, 3, 5, 7):
            n += int(np.sum(fl & ((t & G.BOUND[q]) != 0) & ((t & G.BOUND[G.REV[q]]) != 0)))
        return n

    def seam_ok(self, ch) -> bool:
        """No interpolated link across the periodic seam has 2q > 1."""
        D = ch.n
        d = ch.ibb_idx // D
        x = (ch.ibb_idx % D) % ch.nx_full
        cx = G.CX[d]
        seam = ((x == 0) & (cx == 1)) | ((x == ch.nx - 1) & (cx == -1))
        return not np.any(seam & (ch.ibb_q > 0.5))

    def start(self, ch):
        y = np.arange(self.ny)[:, None]
        yb, yt = ch.y_bot[None, :], ch.y_top[None, :]
        prof = np.clip(6.0 * self.u_mean * (y - yb) * (yt - y) / (yt - yb) ** 2, 0.0, None)
        return G.equilibrium_state(ch, ux=prof)

    def lattice(self, ch):
        from .lattice import Lattice
        d = self.desc_default()
        d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
        d.tau, d.fterm, d.mu = self.rate, self.fterm, self.nu
        L = Lattice(d)
        L.set_geometry(ch.ntype, None, None, ch.ibb_idx, ch.ibb_q)
        L.set_shear(shear.setup(ch))
        return L


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--directions", type=int, default=8)
    ap.add_argument("--h", type=float, default=1e-3)
    ap.add_argument("--nu", type=float, default=0.01,
                    help="viscosity (0.01: Re ~ 1.3e3 on the height at 1024x256; 1.27e-3: ~1e4)")
    args = ap.parse_args(argv)
    case = Case(args.nx, args.ny, nu=args.nu)
    ch = case.channel()
    F0 = case.start(ch)
    T = args.steps

    def run_adjoint(c, Fs):
        with case.lattice(c) as L:
            L.set_state(Fs)
            L.step(1)
            return L.adjoint(T)

    # cost: forward T steps against the adjoint (forward + recomputation + backward)
    with case.lattice(ch) as L:
        L.set_state(F0)
        L.step(1)
        stream = torch.cuda.ExternalStream(L.stream)
        L.step(3)
        L.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.step(T)
        e1.record(stream)
        L.sync()
        torch.cuda.synchronize()
        fwd_ms = e0.elapsed_time(e1)
    # the first call allocates the work buffers (every state stored at this
    # size); the cost is the best of three later calls (host wall clock, all
    # three reported), then the same with the memory cap at 0 (states
    # recomputed from sqrt(T) checkpoints; its first call re-allocates)
    def timed(L, n):
        out = []
        for _ in range(n):
            L.sync()
            t0 = time.perf_counter()
            L.adjoint(T)
            out.append((time.perf_counter() - t0) * 1e3)
        return out

    with case.lattice(ch) as L:
        L.set_state(F0)
        L.step(1)
        L.sync()
        t0 = time.perf_counter()
        J, dq = L.adjoint(T)
        cold_ms = (time.perf_counter() - t0) * 1e3
        adj_runs = timed(L, 3)
        L.set_adjoint_memory(0)
        ckpt_runs = timed(L, 4)[1:]
    adj_ms, ckpt_ms = min(adj_runs), min(ckpt_runs)
    gb, gt = G.shape_gradient(ch, dq)
    M = modes(args.nx, len(case.a))
    # y_bot = b + h(x) - h(0): d y_bot / d a_m = cos(2 pi m x / nx) - 1 (a
    # lifted column follows the column it copies), y_top = ny - 1 - y_bot
    src = walls(case.a, args.nx, args.ny, with_source=True)[2]
    dyb = (M - 1.0)[:, src]
    dJda = dyb @ gb - dyb @ gt
    rng = np.random.default_rng(1)
    checks = []
    for k in range(args.directions):
        d = rng.standard_normal(len(case.a))
        d /= np.linalg.norm(d)
        h = args.h
        b0 = walls(case.a, args.nx, args.ny)[0][0]
        while True:
            cp, cm = case.channel(case.a + h * d), case.channel(case.a - h * d)
            same_b = (walls(case.a + h * d, args.nx, args.ny)[0][0] == b0
                      and walls(case.a - h * d, args.nx, args.ny)[0][0] == b0)
            if (same_b and np.array_equal(cp.ntype, ch.ntype) and np.array_equal(cm.ntype, ch.ntype)
                    and np.array_equal(cp.ibb_idx, ch.ibb_idx) and np.array_equal(cm.ibb_idx, ch.ibb_idx)):
                break
            h *= 0.25
            if h < 1e-9:
                break
        Jp, _ = run_adjoint(cp, F0)
        Jm, _ = run_adjoint(cm, F0)
        fd = (Jp - Jm) / (2 * h)
        ad = float(dJda @ d)
        checks.append({"h": h, "fd": fd, "adjoint": ad, "rel": abs(fd - ad) / max(abs(fd), 1e-300)})
    line = {"case": f"laminar wall-shape gradient {args.nx}x{args.ny}, T={T}, nu={args.nu}",
            "re_height": case.u_mean * (args.ny - 2) / args.nu,
            "J": J, "n_links": len(dq), "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
            "adjoint_over_forward": adj_ms / fwd_ms, "adjoint_runs_ms": adj_runs,
            "adjoint_first_call_ms": cold_ms, "adjoint_sqrt_checkpoints_ms": ckpt_ms,
            "sqrt_checkpoints_runs_ms": ckpt_runs, "sqrt_checkpoints_over_forward": ckpt_ms / fwd_ms,
            "checkpoint_interval": int(np.ceil(np.sqrt(T))),
            "fd_checks": checks, "max_rel": max((c["rel"] for c in checks), default=None)}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
