"""Host-side set-up of a channel: geometry flags and initial fields.

Covers what the reference computes on the host before its time loop, for the
straight channel (two straight wall polylines):
  * nType bits with fluid / solid / boundary flags and the per-direction wall
    flags (clVariablesLS::iniFillMap0 / iniFillMap / iniNodeBoundaryInfo0 /
    iniNodeBoundaryInfo, clVariablesLS.cpp:686-1000);
  * dXArr, the fraction of each E/W/N/S link that lies in the fluid
    (clVariablesLS::inidXArrays, clVariablesLS.cpp:650-684);
  * WallD, the distance to the nearest wall (kOmega::iniWallD,
    kOmega.cpp:330-349);
  * the equilibrium populations of a velocity field (calcFeqVals /
    iniDists, clVariablesLB.cpp:77-117, 407-428) and the k-omega initial
    values (kOmega::setInitialValues, kOmega.cpp:530-570).
Arrays use the reference's padded layout: node (i, j) at i + nx_full*j.
"""
from __future__ import annotations

import numpy as np

# nType bits (Kernels/Heading.cl:223-251)
M_SOLID, M_FLUID, M0_SOLID, M0_FLUID = 0x1, 0x2, 0x4, 0x8
SOLID_BOUNDARY, SOLID_BOUNDARY0, NESW_BOUNDARY0, BOUNDARY0 = 0x10, 0x20, 0x40, 0x80
BOUND = [0, 0x100, 0x200, 0x400, 0x800, 0x1000, 0x2000, 0x4000, 0x8000]
NESW_BOUNDARY = 0x0F00

CX = np.array([0, 1, -1, 0, 0, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 1, -1, 1, -1, -1, 1])
W = np.array([4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36])


def xsize_full(nx: int) -> int:
    """XsizeFull: nX rounded up to a multiple of 128 (clProblem.cpp:469)."""
    return ((nx + 127) // 128) * 128


class Channel:
    """Geometry arrays of one channel (reference padded layout)."""

    def __init__(self, nx, ny, nx_full, ntype, dX, wallD, ibb_idx=None, ibb_q=None,
                 y_bot=None, y_top=None):
        self.nx, self.ny, self.nx_full = nx, ny, nx_full
        self.ntype, self.dX, self.wallD = ntype, dX, wallD
        self.ibb_idx = np.zeros(0, np.int32) if ibb_idx is None else ibb_idx
        self.ibb_q = np.zeros(0) if ibb_q is None else ibb_q
        self.y_bot, self.y_top = y_bot, y_top

    @property
    def n(self):
        return self.nx_full * self.ny

    def fluid_mask(self) -> np.ndarray:
        m = (self.ntype.astype(np.int32) & 0xFFFF).reshape(self.ny, self.nx_full)
        out = (m & M_SOLID) == 0
        out[:, self.nx:] = False
        return out

    @property
    def pipe_radius(self) -> float:
        """Half-height between the walls (the reference's "Pipe Radius")."""
        return 0.5 * (float(np.mean(self.y_top)) - float(np.mean(self.y_bot)))


def straight_channel(nx: int, ny: int, nx_full: int | None = None) -> Channel:
    """Rows 0 and ny-1 solid; half-way walls at y = 0.5 and y = ny - 1.5."""
    nxf = nx if nx_full is None else nx_full
    yb, yt = 0.5, ny - 1.5
    j = np.arange(ny)
    solid_row = (j == 0) | (j == ny - 1)
    t = np.where(solid_row[:, None], M0_SOLID | M_SOLID, M0_FLUID | M_FLUID)
    t = np.broadcast_to(t, (ny, nxf)).astype(np.int32).copy()
    solid = (t & M_SOLID) != 0
    solid[:, nx:] = False
    fluid = ~solid
    fluid[:, nx:] = False
    for q in range(1, 9):
        # neighbour of (i, j) in direction q, periodic in x over nx
        nb_solid = np.zeros_like(solid)
        jj = j + CY[q]
        valid = (jj >= 0) & (jj < ny)
        src = np.roll(solid[:, :nx], -CX[q], axis=1)
        rows = np.where(valid)[0]
        nb_solid[rows, :nx] = src[jj[rows], :]
        hit = fluid & nb_solid
        t[hit] |= BOUND[q] | BOUNDARY0
        if q < 5:
            t[hit] |= NESW_BOUNDARY0
            # mark the solid neighbours of NESW links
            ii, jv = np.nonzero(hit.T)
            t[jv + CY[q], (ii + CX[q]) % nx] |= SOLID_BOUNDARY | SOLID_BOUNDARY0
    dX = np.zeros((4, ny, nxf))
    dX[:, fluid] = 1.0
    dX[2, ny - 2, :nx] = yt - (ny - 2)   # north link of the top fluid row
    dX[3, 1, :nx] = 1 - yb               # south link of the bottom fluid row
    wallD = np.where(fluid, np.minimum(j[:, None] - yb, yt - j[:, None]), 0.0)
    return Channel(nx, ny, nxf, t.astype(np.uint16).view(np.int16).ravel(),
                   dX.ravel(), wallD.ravel(), y_bot=np.full(nx, yb), y_top=np.full(nx, yt))


# ---------------------------------------------------------------------------
def feq(rho, ux, uy):
    """Product-form D2Q9 equilibrium (clVariablesLB.cpp:77-117): 9 x shape."""
    rho, ux, uy = np.broadcast_arrays(np.asarray(rho, float), np.asarray(ux, float),
                                      np.asarray(uy, float))

    def phi(c, u):
        return 2.0 / 3.0 - u * u if c == 0 else 0.5 * (1.0 / 3.0 + c * u + u * u)

    return np.stack([rho * phi(CX[q], ux) * phi(CY[q], uy) for q in range(9)])


def equilibrium_state(ch: Channel, rho=1.0, ux=0.0, uy=0.0) -> np.ndarray:
    """FA filled with feq(rho, u) on fluid nodes, 0 elsewhere (iniDists)."""
    shape = (ch.ny, ch.nx_full)
    f = feq(np.broadcast_to(rho, shape), np.broadcast_to(ux, shape), np.broadcast_to(uy, shape))
    f[:, ~ch.fluid_mask()] = 0.0
    return f.reshape(9, -1).ravel()


def komega_fields(ch: Channel, k0: float, omega0: float):
    """k, omega, nu_t = k/omega on fluid nodes (fillByNodeType, kOmega.cpp:567-569)."""
    fl = ch.fluid_mask().ravel()
    k = np.where(fl, k0, 0.0)
    o = np.where(fl, omega0, 0.0)
    nut = np.where(fl, k0 / omega0, 0.0)
    return k, o, nut


def komega_reference_initial(re: float, mu: float, pipe_radius: float, umean: float = 0.0,
                             geom_penalty: float = 1.0):
    """kOmega::setInitialValues (kOmega.cpp:538-553): turbulence intensity
    0.16 Re^(-1/8) and length scale 0.036 R."""
    if umean == 0.0:
        umean = re * mu / pipe_radius / 4.0 * geom_penalty
    re_ini = pipe_radius * 4.0 * umean / mu
    ti = 0.16 * re_ini ** (-1.0 / 8.0)
    k0 = 1.5 * (ti * umean) ** 2
    omega0 = np.sqrt(k0) / 0.5477225575 / (0.036 * pipe_radius)
    return k0, omega0


def force_from_re(re: float, mu: float, pipe_radius: float) -> float:
    """Fval = Re * 3 mu^2 / R^3 (clVariablesLB.cpp:584-600)."""
    return re * 3.0 * mu * mu / pipe_radius ** 3
