"""Seeded synthetic channels of the benchmark shapes.

No dataset is involved: every workload is a channel geometry plus an initial
state built on the host.  Names and sizes:

  poiseuille_256x64       laminar Poiseuille start-up, tau = 0.8 (nu = 0.1),
                          g = 1e-6, from rest (config 1)
  komega_straight_16384x1024  straight k-omega channel, 16.7M nodes, nu = 5e-4,
                          Re on the channel height about 5e4 (config 3)
  komega_straight_2048x256    the config-2 size as a straight, periodic,
                          body-forced channel (the variant with a reference)
  komega_wavy_2048x256    the config-2 shape: walls 0.5 + 16 (1 - cos(2 pi x /
                          512)) and mirrored (interpolated bounce-back), k-omega,
                          nu = 5e-4, periodic and body-forced
  komega_straight_<nx>x<ny>   other sizes of the straight k-omega channel
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import geometry as G


@dataclass
class Workload:
    name: str
    channel: G.Channel
    tau: float        # relaxation rate
    fterm: float
    mu: float
    komega: bool
    f: np.ndarray
    k: np.ndarray | None = None
    omega: np.ndarray | None = None
    nut: np.ndarray | None = None
    sxy: np.ndarray | None = None
    steps: int = 1000
    device_geometry: bool = False  # geometry from the walls on the device (kofm_set_walls)

    @property
    def nodes(self) -> int:
        return self.channel.nx * self.channel.ny


def poiseuille(nx=256, ny=64, tau=0.8, g=1e-6, steps=10000) -> Workload:
    ch = G.straight_channel(nx, ny)
    mu = (tau - 0.5) / 3.0
    return Workload(f"poiseuille_{nx}x{ny}", ch, 1.0 / tau, g, mu, False,
                    G.equilibrium_state(ch), steps=steps)


def komega_channel(nx, ny, re_height=5.0e4, nu=5.0e-4, steps=1000, intensity=0.05) -> Workload:
    """Straight channel, parabolic start whose mean velocity gives Re on the
    channel height, body force from the reference's Re -> Fval relation on the
    half-height (clVariablesLB.cpp:584-600); k = 1.5 (I u)^2 with I = 5% of the
    peak velocity and omega = k^0.5 / (0.09^0.25 * 0.07 H)."""
    ch = G.straight_channel(nx, ny)
    R = ch.pipe_radius
    H = 2.0 * R
    u_mean = re_height * nu / H
    u_max = 1.5 * u_mean
    y = np.arange(ny)[:, None] - 0.5
    ux = np.clip(u_max * (1.0 - ((y - R) / R) ** 2), 0.0, None) * np.ones((1, ch.nx_full))
    f = G.equilibrium_state(ch, ux=ux)
    g = G.force_from_re(u_mean * R / nu, nu, R)
    k0 = 1.5 * (intensity * u_max) ** 2
    o0 = np.sqrt(k0) / (0.09 ** 0.25 * 0.07 * H)
    k, o, nut = G.komega_fields(ch, k0, o0)
    return Workload(f"komega_straight_{nx}x{ny}", ch, 1.0 / (3.0 * nu + 0.5), g, nu, True,
                    f, k, o, nut, np.zeros(3 * ch.n), steps=steps)


def komega_wavy(nx=2048, ny=256, amplitude=32.0, wavelength=512, nu=5.0e-4, u_max=0.05,
                intensity=0.05, steps=1000) -> Workload:
    """Wavy k-omega channel: walls displaced by A (1 - cos(2 pi x / L)) / 2
    (mirrored, the seam at a crest), parabolic start of peak u_max between the
    mean walls, body force from the reference's Re -> Fval relation on the
    half-height, k and omega from the turbulence intensity as komega_channel."""
    ch = G.wavy_channel(nx, ny, amplitude, wavelength)
    R = ch.pipe_radius
    y = np.arange(ny)[:, None] - 0.5
    ux = np.clip(u_max * (1.0 - ((y - R) / R) ** 2), 0.0, None) * np.ones((1, ch.nx_full))
    f = G.equilibrium_state(ch, ux=ux)
    g = G.force_from_re((2.0 / 3.0) * u_max * R / nu, nu, R)
    k0 = 1.5 * (intensity * u_max) ** 2
    o0 = np.sqrt(k0) / (0.09 ** 0.25 * 0.07 * 2 * R)
    k, o, nut = G.komega_fields(ch, k0, o0)
    return Workload(f"komega_wavy_{nx}x{ny}", ch, 1.0 / (3.0 * nu + 0.5), g, nu, True,
                    f, k, o, nut, np.zeros(3 * ch.n), steps=steps)


def by_name(name: str) -> Workload:
    if name.startswith("poiseuille"):
        return poiseuille()
    if name == "komega_straight_16384x1024":
        return komega_channel(16384, 1024, steps=20000)
    if name == "komega_wavy_2048x256":
        return komega_wavy(steps=50000)
    if name == "komega_straight_2048x256":
        return komega_channel(2048, 256, re_height=2.5e4, steps=50000)
    if name.startswith("komega_straight_"):
        # other sizes of the same straight channel (profiling cases)
        nx, ny = (int(v) for v in name[len("komega_straight_"):].split("x"))
        return komega_channel(nx, ny)
    raise KeyError(name)


def apply(lattice, w: Workload) -> None:
    """Uploads geometry and state of a workload into a Lattice."""
    ch = w.channel
    if w.device_geometry:
        lattice.set_walls(ch.y_bot, ch.y_top)
    else:
        lattice.set_geometry(ch.ntype, ch.wallD, ch.dX, ch.ibb_idx if len(ch.ibb_idx) else None,
                             ch.ibb_q if len(ch.ibb_q) else None)
    lattice.set_state(w.f, w.k, w.omega, w.nut, w.sxy)


def descriptor(w: Workload, storage: int = 0, krylov: int = 10):
    from .lattice import desc_default
    d = desc_default()
    d.nx, d.nx_full, d.ny = w.channel.nx, w.channel.nx_full, w.channel.ny
    d.tau, d.fterm, d.mu = w.tau, w.fterm, w.mu
    d.use_komega = 1 if w.komega else 0
    d.storage = storage
    d.krylov_dim = krylov
    return d
