"""Wall shear set-up: shear nodes, their coefficient rows and the boundary-link
weights.

Restates what the reference computes once before its time loop (and after
every wall update) for its wall-shear output:
  * the shear-node list ssArr -- every fluid node with a solid E, W, N or S
    neighbour, ordered column by column (clVariablesLS::fillShearArray,
    clVariablesLS.cpp:288-320) -- with the index of each column's first node
    (ssArrInds);
  * per shear node the two coefficient rows CFSS (TR_Find_Shear_Coeffs1,
    Kernels/trKernelsShear.cl:333-375): a wall normal from the wall-link
    flags of the shear nodes within the cut-off radius among the 50 list
    neighbours on either side, then 3 s_k (c_k - n s_k) per direction, with
    s_k = c_k . n;
  * per boundary link (wall segment) the four nearest shear nodes to its
    midpoint within the cut-off radius, among the columns within
    INDEX_RADIUS_SEARCH of it, and normalised Gaussian weights
    (TR_Find_Shear_Coeffs2, trKernelsShear.cl:414-505).
Boundary links are the segments of the wall polylines between neighbouring
columns: bottom wall first, then the top wall.  The reference tracks shear
only over a window of columns [minSSArrNodeX, maxSSArrNodeX] around its
tracer release/stop positions (clVariablesLS.cpp:572-573); x_min/x_max give
that window (default: the whole channel), and the links kept are those whose
left column lies in it (NUM_BL_BOT / BL_BOT_START, Kernels/Heading.cl:427).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import geometry as G

CUTOFF_RADIUS = 5.0        # CUTOFF_RADIUS (ConstDef.h)
INDEX_RADIUS_SEARCH = 30   # INDEX_RADIUS_SEARCH (ConstDef.h)


@dataclass
class ShearSetup:
    nodes: np.ndarray      # int32 [n] node indices i + nx_full j
    col_start: np.ndarray  # int32 [nx + 1] first list index of every column
    cfss: np.ndarray       # float64 [n, 16] x row (8) then y row (8), directions 1..8
    bl_nodes: np.ndarray   # int32 [n_bl, 4] list indices of the nearest nodes (-1: none)
    bl_weights: np.ndarray  # float64 [n_bl, 4]
    x_min: int = 0
    x_max: int = -1


def shear_nodes(ch: G.Channel, x_min: int = 0, x_max: int | None = None):
    nx, ny, nxf = ch.nx, ch.ny, ch.nx_full
    x_max = nx - 1 if x_max is None else x_max
    solid = ~ch.fluid_mask()
    nodes, col_start = [], np.zeros(nx + 1, np.int32)
    for i in range(nx):
        col_start[i] = len(nodes)
        if i < x_min or i > x_max:
            continue
        for j in range(ny):
            if solid[j, i]:
                continue
            for k in range(1, 5):
                ii, jj = (i + G.CX[k]) % nx, j + G.CY[k]
                if 0 <= jj < ny and solid[jj, ii]:
                    nodes.append(i + nxf * j)
                    break
    col_start[nx] = len(nodes)
    return np.asarray(nodes, np.int32), col_start


def shear_coeffs(ch: G.Channel, nodes: np.ndarray, cutoff: float = CUTOFF_RADIUS) -> np.ndarray:
    nxf = ch.nx_full
    t = ch.ntype.astype(np.int32) & 0xFFFF
    x = (nodes % nxf).astype(float)
    y = (nodes // nxf).astype(float)
    n = len(nodes)
    cf = np.zeros((n, 16))
    cx = G.CX[1:].astype(float)
    cy = G.CY[1:].astype(float)
    for ii in range(n):
        lo, hi = max(ii - 50, 0), min(ii + 50, n)
        dx = x[ii] - x[lo:hi]
        dy = y[ii] - y[lo:hi]
        near = np.hypot(dx, dy) <= cutoff
        tn = t[nodes[lo:hi][near]]
        nv = np.array([np.sum((tn & G.BOUND[1]) != 0) - np.sum((tn & G.BOUND[2]) != 0),
                       np.sum((tn & G.BOUND[3]) != 0) - np.sum((tn & G.BOUND[4]) != 0)], float)
        nv /= np.hypot(nv[0], nv[1])
        s = cx * nv[0] + cy * nv[1]
        cf[ii, :8] = 3.0 * s * (cx - nv[0] * s)
        cf[ii, 8:] = 3.0 * s * (cy - nv[1] * s)
    return cf


def wall_midpoints(ch: G.Channel, x_min: int = 0, x_max: int | None = None) -> np.ndarray:
    """Midpoints of the wall segments from column x to x + 1 for x in
    [x_min, x_max]: bottom wall, then top wall (the segment's first point
    plus half its length along the tangent, trKernelsShear.cl:430-433)."""
    x_max = ch.nx - 1 if x_max is None else x_max
    x = np.arange(x_min, x_max + 1)
    out = []
    for y_w in (ch.y_bot, ch.y_top):
        y0 = np.asarray(y_w, float)
        y1 = np.roll(y0, -1)
        out.append(np.column_stack([x + 0.5, 0.5 * (y0[x] + y1[x])]))
    return np.vstack(out)


def bl_weights(ch: G.Channel, nodes, col_start, mids, cutoff: float = CUTOFF_RADIUS,
               radius: int = INDEX_RADIUS_SEARCH, x_min: int = 0, x_max: int | None = None):
    nxf = ch.nx_full
    x_max = ch.nx - 1 if x_max is None else x_max
    x = (nodes % nxf).astype(float)
    y = (nodes // nxf).astype(float)
    nb = len(mids)
    sind = np.full((nb, 4), -1, np.int32)
    wts = np.zeros((nb, 4))
    for b in range(nb):
        mx, my = mids[b]
        ival = int(mx)
        start = col_start[max(x_min, ival - radius)]
        stop = col_start[min(x_max, ival + radius + 1)]
        # the four nearest within the cut-off (slots kept largest-first, as
        # the reference's insertion does)
        d4 = [100.0] * 4
        i4 = [-1] * 4
        for j in range(start, stop):
            dist = float(np.hypot(mx - x[j], my - y[j]))
            if dist < d4[0] and dist < cutoff:
                d4[0], i4[0] = dist, j
                for a in range(3):
                    if d4[a] >= d4[a + 1]:
                        break
                    d4[a], d4[a + 1] = d4[a + 1], d4[a]
                    i4[a], i4[a + 1] = i4[a + 1], i4[a]
        w4 = [np.exp(-0.5 * (d / cutoff) ** 2) / np.sqrt(2.0 * np.pi) for d in d4]
        order = sorted(range(4), key=lambda a: i4[a])
        tot = sum(w4)
        sind[b] = [i4[a] for a in order]
        wts[b] = [w4[a] / tot for a in order]
    return sind, wts


def setup(ch: G.Channel, x_min: int = 0, x_max: int | None = None) -> ShearSetup:
    """The reference's shear set-up (clVariablesLS::fillShearArray, then
    TR_Find_Shear_Coeffs1 and TR_Find_Shear_Coeffs2) for channel ch."""
    x_max = ch.nx - 1 if x_max is None else x_max
    nodes, col_start = shear_nodes(ch, x_min, x_max)
    cf = shear_coeffs(ch, nodes)
    sind, wts = bl_weights(ch, nodes, col_start, wall_midpoints(ch, x_min, x_max),
                           x_min=x_min, x_max=x_max)
    return ShearSetup(nodes, col_start, cf, sind, wts, x_min, x_max)
