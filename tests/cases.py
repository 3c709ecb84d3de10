"""Seeded test inputs shared by the CPU and GPU tests (no device code here)."""
from __future__ import annotations

import numpy as np

from komegafoulingmodel_b200 import geometry as G


def perturbed_state(ch, seed=0, rho_amp=1e-3, u_amp=1e-2, neq_amp=1e-3, u_mean=0.0):
    """Near-equilibrium FA with seeded perturbations on fluid nodes."""
    rng = np.random.default_rng(seed)
    shape = (ch.ny, ch.nx_full)
    rho = 1.0 + rho_amp * rng.standard_normal(shape)
    ux = u_mean + u_amp * rng.standard_normal(shape)
    uy = 0.5 * u_amp * rng.standard_normal(shape)
    f = G.feq(rho, ux, uy) * (1.0 + neq_amp * rng.standard_normal((9,) + shape))
    f[:, ~ch.fluid_mask()] = 0.0
    return f.reshape(9, -1).ravel()


def komega_state(ch, seed=1, k0=1e-4, o0=1e-2, s_amp=1e-4):
    rng = np.random.default_rng(seed)
    fl = ch.fluid_mask().ravel()
    n = ch.n
    k = np.where(fl, k0 * (1 + 0.3 * rng.random(n)), 0.0)
    o = np.where(fl, o0 * (1 + 0.3 * rng.random(n)), 0.0)
    nut = np.where(fl, k / np.where(fl, o, 1.0), 0.0)
    s = np.concatenate([np.where(fl, s_amp * rng.standard_normal(n), 0.0) for _ in range(3)])
    return k, o, nut, s


def rel_l2(a, b, mask=None):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    if mask is not None:
        a, b = a[mask], b[mask]
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def fp32_state(f, *fields):
    """The state as the FP32 device form holds it: populations rounded as
    deviations f - w, scalar fields rounded to FP32 (so the oracle starts
    from exactly the GPU's stored state)."""
    from komegafoulingmodel_b200 import geometry as G
    n = len(f) // 9
    w = np.repeat(G.W, n)
    out = [(f - w).astype(np.float32).astype(np.float64) + w]
    for a in fields:
        out.append(None if a is None else np.asarray(a).astype(np.float32).astype(np.float64))
    return out
