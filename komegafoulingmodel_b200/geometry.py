"""Host-side set-up of a channel: geometry flags and initial fields.

Covers what the reference computes on the host before its time loop, for a
channel between two wall polylines given by their height at every column:
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
REV = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7])


def xsize_full(nx: int) -> int:
    """XsizeFull: nX rounded up to a multiple of 128 (clProblem.cpp:469)."""
    return ((nx + 127) // 128) * 128


class Channel:
    """Geometry arrays of one channel (reference padded layout)."""

    def __init__(self, nx, ny, nx_full, ntype, dX, wallD, ibb_idx=None, ibb_q=None,
                 y_bot=None, y_top=None, dX0=None):
        self.nx, self.ny, self.nx_full = nx, ny, nx_full
        self.ntype, self.dX, self.wallD = ntype, dX, wallD
        self.ibb_idx = np.zeros(0, np.int32) if ibb_idx is None else ibb_idx
        self.ibb_q = np.zeros(0) if ibb_q is None else ibb_q
        self.y_bot, self.y_top = y_bot, y_top
        # link fractions of the unfouled walls (dXArr0); the same as dX when
        # the channel has no fouling layer
        self.dX0 = dX if dX0 is None else dX0

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


def _link_fractions(ii, jj, q, nx, y_bot, y_top):
    """Fraction t in (0, 1] of the links from nodes (ii, jj) in direction q at
    which they meet a wall; walls are linear between columns (periodic in x)."""
    cx, cy = int(CX[q]), int(CY[q])
    best = np.full(ii.shape, np.inf)
    for y_w in (y_bot, y_top):
        y0 = y_w[ii]
        d = (y_w[(ii + cx) % nx] - y0) if cx != 0 else np.zeros_like(y0)
        den = cy - d
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.where(den != 0.0, (y0 - jj) / np.where(den != 0.0, den, 1.0), np.inf)
        ok = (t > 0.0) & (t <= 1.0 + 1e-12)
        best = np.where(ok, np.minimum(best, np.minimum(t, 1.0)), best)
    return np.where(np.isfinite(best), best, 0.5)


def wall_fraction_jacobian(ch: Channel):
    """d q / d (wall heights) of every interpolated bounce-back link of ch, in
    the order of ch.ibb_idx: arrays (wall, col0, dq_dy0, col1, dq_dy1) with
    wall 0 = bottom, 1 = top, q = (y0 - j) / (c_y - (y1 - y0)) the crossing
    of the link from node (i, j) with the wall segment from (i, y0) to
    (i + c_x, y1) (y1 = y0 for the vertical links).  Links whose fraction was
    clamped to 1 get zero derivatives."""
    D = ch.n
    d = ch.ibb_idx // D
    node = ch.ibb_idx % D
    ii = node % ch.nx_full
    jj = node // ch.nx_full
    nx = ch.nx
    n = len(d)
    wall = np.zeros(n, np.int32)
    col0 = ii.astype(np.int64)
    col1 = np.zeros(n, np.int64)
    g0 = np.zeros(n)
    g1 = np.zeros(n)
    for k in range(n):
        q = int(d[k])
        cx, cy = int(CX[q]), int(CY[q])
        best, pick = np.inf, None
        for w, y_w in enumerate((ch.y_bot, ch.y_top)):
            y0 = y_w[ii[k]]
            y1 = y_w[(ii[k] + cx) % nx] if cx != 0 else y0
            den = cy - (y1 - y0)
            if den == 0.0:
                continue
            t = (y0 - jj[k]) / den
            if 0.0 < t <= 1.0 + 1e-12 and t < best:
                best, pick = t, (w, y0, y1, den)
        if pick is None:
            continue
        w, y0, y1, den = pick
        wall[k] = w
        col1[k] = (ii[k] + cx) % nx
        if best > 1.0:
            continue
        N = y0 - jj[k]
        if cx == 0:
            g0[k] = 1.0 / den
        else:
            g0[k] = (den - N) / den ** 2
            g1[k] = N / den ** 2
    return wall, col0, g0, col1, g1


def shape_gradient(ch: Channel, dJdq):
    """dJ/d(wall heights) from dJ/dq (kofm_adjoint): (dJ/dy_bot, dJ/dy_top),
    one value per column."""
    wall, c0, g0, c1, g1 = wall_fraction_jacobian(ch)
    out = np.zeros((2, ch.nx))
    np.add.at(out, (wall, c0), np.asarray(dJdq) * g0)
    np.add.at(out, (wall, c1), np.asarray(dJdq) * g1)
    return out[0], out[1]


def _wall_distance(nx, ny, nxf, fluid, y_bot, y_top, radius=50):
    """Distance of every fluid node to the walls as the reference computes it
    (kOmega::iniWallD / findMinDist, kOmega.cpp:136-193, 330-349, and the
    updateWallD kernel, kOmegaKernels.cl:751-840), for walls given as
    polylines through (x, y_w[x]) for x = -1 .. nx (periodic heights; the
    bottom wall left to right, the top wall right to left):
      * only the segments within `radius` of the segment that starts at the
        node's column ("Wall D Search Rad", WALLD_SEARCH_RADIUS = 50): bottom
        segments starting at x - radius .. x + radius - 1, top segments at
        x - radius + 1 .. x + radius, none outside -1 .. nx - 1;
      * per segment the distance to its line, |cross| / |P1 - P0|, replaced by
        the distance to P0 or P1 when the foot of the perpendicular, taken on
        the side the segment's normal points to, falls beyond that end in x;
      * the minimum over both walls (starting from 1000).
    The same floating-point operations in the same order as the reference,
    so the values agree bit for bit; where the node lies behind a segment's
    line the "foot" is the mirror image and the line distance can be shorter
    than the segment's true distance -- kept, as the reference."""
    wall = np.zeros((ny, nxf))
    jj, ii = np.nonzero(fluid)
    if len(jj) == 0:
        return wall
    px = ii.astype(float)
    py = jj.astype(float)
    dmin = np.full(len(jj), 1000.0)
    for top, y_w in ((False, y_bot), (True, y_top)):
        lo, hi = (-radius + 1, radius) if top else (-radius, radius - 1)
        for o in range(lo, hi + 1):
            xa = ii + o
            m = (xa >= -1) & (xa <= nx - 1)
            if not m.any():
                continue
            xa = xa[m]
            x, y = px[m], py[m]
            ax = xa.astype(float)
            ay = y_w[xa % nx]
            bx = ax + 1.0
            by = y_w[(xa + 1) % nx]
            P0x, P0y, P1x, P1y = (bx, by, ax, ay) if top else (ax, ay, bx, by)
            vTx = P1x - P0x
            vTy = P1y - P0y
            vTmag = np.sqrt(vTx * vTx + vTy * vTy)
            d = np.abs(vTy * x - vTx * y + P1x * P0y - P1y * P0x) / vTmag
            pcx = x - d * (-(vTy / vTmag))
            if top:
                c0 = pcx > P0x
                c1 = ~c0 & (pcx < P1x)
            else:
                c0 = pcx < P0x
                c1 = ~c0 & (pcx > P1x)
            e0x, e0y = x - P0x, y - P0y
            e1x, e1y = x - P1x, y - P1y
            d = np.where(c0, np.sqrt(e0x * e0x + e0y * e0y), d)
            d = np.where(c1, np.sqrt(e1x * e1x + e1y * e1y), d)
            cur = dmin[m]
            dmin[m] = np.where(d < cur, d, cur)
    wall[jj, ii] = dmin
    return wall


def _fluid(nx, ny, nxf, y_bot, y_top):
    j = np.arange(ny)
    fluid = np.zeros((ny, nxf), bool)
    fluid[:, :nx] = (j[:, None] > y_bot[None, :]) & (j[:, None] < y_top[None, :])
    fluid[0, :] = False
    fluid[ny - 1, :] = False
    return fluid


def _wall_links(nx, ny, nxf, fluid, q):
    """Fluid nodes whose link in direction q ends in a solid node."""
    solid = ~fluid
    solid[:, nx:] = False
    j = np.arange(ny)
    nb_solid = np.zeros((ny, nxf), bool)
    jn = j + CY[q]
    valid = (jn >= 0) & (jn < ny)
    src = np.roll(solid[:, :nx], -CX[q], axis=1)
    rows = np.where(valid)[0]
    nb_solid[rows, :nx] = src[jn[rows], :]
    return fluid & nb_solid


def channel_from_walls(nx: int, ny: int, y_bot, y_top, nx_full: int | None = None,
                       wall_radius: int = 50, y_bot0=None, y_top0=None,
                       ibb_all: bool = False, seam_ibb: bool = False,
                       min_dx: float = 0.001, wall_distance: bool = True) -> Channel:
    """Channel between two walls given by their heights at every column (the
    wall polylines of clVariablesLS).  Node (i, j) is fluid iff
    y_bot[i] < j < y_top[i].  Builds the nType flags (per-direction wall bits
    of the links whose upstream node is solid), the E/W/N/S link fractions
    dXArr, the interpolated bounce-back list (link from a fluid node into the
    wall, as node + D * dir, with its wall fraction q; links with q = 1/2 need
    no correction and are left out) and the wall distance.

    y_bot0 / y_top0 give unfouled walls outside the fouled ones: the nodes
    between them are the fouling layer (M0_FLUID | M_SOLID), the *0 flags and
    dX0 (dXArr0) follow the unfouled walls (iniFillMap0 /
    iniNodeBoundaryInfo0, clVariablesLS.cpp:920-951), everything the flow
    uses follows the fouled ones (iniNodeBoundaryInfo, 953-998).

    ibb_all keeps the links with q = 1/2 in the interpolated bounce-back list
    too (they give the half-way value exactly), so that every wall link has a
    wall fraction to differentiate (kofm_adjoint).

    As the reference's list builder (updateIBBOnly, lsKernels.cl:455-466),
    the nodes of columns 0 and nx-1 get no interpolated links: their wall
    links bounce back half-way.  seam_ibb = True lists them too.

    min_dx is the smallest link fraction dXArr / dXArr0 take ("Min dX Dist",
    MINIMUM_DX_DIST = 0.001: bcSetdXArr, clVariablesLS.cpp:248-286); the
    interpolated list keeps the unclamped fraction, as updateIBBOnly.

    The wall distance follows the reference's search (_wall_distance, over
    the segments within wall_radius columns); wall_distance = False leaves it
    0 (a laminar run does not read it)."""
    nxf = nx if nx_full is None else nx_full
    y_bot = np.asarray(y_bot, float)
    y_top = np.asarray(y_top, float)
    fouled = y_bot0 is not None or y_top0 is not None
    y_bot0 = y_bot if y_bot0 is None else np.asarray(y_bot0, float)
    y_top0 = y_top if y_top0 is None else np.asarray(y_top0, float)
    if np.any(y_bot0 > y_bot) or np.any(y_top0 < y_top):
        raise ValueError("the unfouled walls must lie outside the fouled ones")
    j = np.arange(ny)
    fluid = _fluid(nx, ny, nxf, y_bot, y_top)
    fluid0 = _fluid(nx, ny, nxf, y_bot0, y_top0)
    t = np.where(fluid0, M0_FLUID, M0_SOLID) | np.where(fluid, M_FLUID, M_SOLID)
    t = t.astype(np.int32)
    t[:, nx:] = M0_SOLID | M_SOLID
    dX = np.zeros((4, ny, nxf))
    dX[:, fluid] = 1.0
    dX0 = np.zeros((4, ny, nxf))
    dX0[:, fluid0] = 1.0
    D = nxf * ny
    ibb_idx, ibb_q = [], []
    for q in range(1, 9):
        # unfouled domain
        hit0 = _wall_links(nx, ny, nxf, fluid0, q)
        t[hit0] |= BOUNDARY0
        if q < 5:
            t[hit0] |= NESW_BOUNDARY0
            ii, jv = np.nonzero(hit0.T)
            t[jv + CY[q], (ii + CX[q]) % nx] |= SOLID_BOUNDARY0
            jv, ii = np.nonzero(hit0)
            dX0[q - 1, jv, ii] = np.maximum(_link_fractions(ii, jv, q, nx, y_bot0, y_top0), min_dx)
        # fouled domain (the flow)
        hit = _wall_links(nx, ny, nxf, fluid, q)
        t[hit] |= BOUND[q]
        if q < 5:
            ii, jv = np.nonzero(hit.T)
            t[jv + CY[q], (ii + CX[q]) % nx] |= SOLID_BOUNDARY
        jv, ii = np.nonzero(hit)
        frac = _link_fractions(ii, jv, q, nx, y_bot, y_top)
        if q < 5:
            dX[q - 1, jv, ii] = np.maximum(frac, min_dx)
        keep = np.abs(frac - 0.5) > 1e-12 if not ibb_all else np.ones(frac.shape, bool)
        if not seam_ibb:
            keep &= (ii != 0) & (ii != nx - 1)
        ibb_idx.extend((q * D + jv * nxf + ii)[keep].tolist())
        ibb_q.extend(frac[keep].tolist())
    if not wall_distance:
        wall = np.zeros((ny, nxf))
    elif np.all(y_bot == y_bot[0]) and np.all(y_top == y_top[0]):
        # straight walls: the vertical distance (the reference's line distance
        # equals it up to the rounding of (x + 1) y_w - x y_w, exactly for
        # half-way walls)
        wall = np.where(fluid, np.minimum(j[:, None] - y_bot[0], y_top[0] - j[:, None]), 0.0)
    else:
        wall = _wall_distance(nx, ny, nxf, fluid, y_bot, y_top, wall_radius)
    order = np.argsort(ibb_idx, kind="stable")
    return Channel(nx, ny, nxf, t.astype(np.uint16).view(np.int16).ravel(), dX.ravel(),
                   wall.ravel(), np.asarray(ibb_idx, np.int32)[order],
                   np.asarray(ibb_q, float)[order], y_bot=y_bot, y_top=y_top,
                   dX0=dX0.ravel() if fouled else None)


def read_reference_walls(directory: str):
    """The wall polylines of a reference run directory: lbsize.txt ("nX nY"),
    lsc0.txt (one "x y" point per line) and lsbl.txt (one "i j" segment per
    line, 0-based point indices) -- the files clVariablesLS::allocateArrays
    loads (clVariablesLS.cpp:45-50) and MakeChannel_Test.m writes.  Returns
    (nx, ny, y_bot, y_top): the two walls' heights at every column, where
    each column crosses exactly two segments (the lower wall and the upper)."""
    import os
    size = np.loadtxt(os.path.join(directory, "lbsize.txt")).ravel()
    nx, ny = int(size[0]), int(size[1])
    pts = np.loadtxt(os.path.join(directory, "lsc0.txt"), ndmin=2)
    segs = np.loadtxt(os.path.join(directory, "lsbl.txt"), ndmin=2).astype(np.int64)
    xa, ya = pts[segs[:, 0], 0], pts[segs[:, 0], 1]
    xb, yb = pts[segs[:, 1], 0], pts[segs[:, 1], 1]
    lo, hi = np.minimum(xa, xb), np.maximum(xa, xb)
    y_bot = np.full(nx, np.inf)
    y_top = np.full(nx, -np.inf)
    for x in range(nx):
        on = (lo <= x) & (x <= hi) & (hi > lo)
        if not np.any(on):
            raise ValueError(f"column {x} crosses no wall segment")
        t = (x - xa[on]) / (xb[on] - xa[on])
        y = ya[on] + t * (yb[on] - ya[on])
        y_bot[x], y_top[x] = y.min(), y.max()
        if not y_top[x] > y_bot[x]:
            raise ValueError(f"column {x} crosses only one wall")
    return nx, ny, y_bot, y_top


_CXY = ((1.0, 0.0), (-1.0, 0.0), (0.0, 1.0), (0.0, -1.0), (1.0, 1.0), (-1.0, -1.0), (1.0, -1.0), (-1.0, 1.0))
_REV8 = (1, 0, 3, 2, 5, 4, 7, 6)


def _ls_links(pts, nx, ny, nxf, ntype, xlo, xhi):
    """The reference's list builder updateIBBOnly (lsKernels.cl:428-492, with
    bcFindIntersectionLS, 172-228) on the polyline pts (bottom wall left to
    right, then top wall right to left; segment i joins points i and i + 1,
    except the one from the last bottom point to the first top point), in
    its order and floating-point operations: (population index, fraction)
    pairs, a link listed once per segment that finds it.  Columns xlo .. xhi
    are searched (the reference: 1 .. nx - 2)."""
    import math
    n_pts = len(pts)
    skip = n_pts // 2 - 1
    D = nxf * ny
    t = ntype.astype(np.int32) & 0xFFFF
    out = []
    for i in range(n_pts - 1):
        if i == skip:
            continue
        c0x, c0y = float(pts[i, 0]), float(pts[i, 1])
        c1x, c1y = float(pts[i + 1, 0]), float(pts[i + 1, 1])
        tx, ty = c1x - c0x, c1y - c0y
        bl = math.sqrt(tx * tx + ty * ty)
        tx, ty = tx / bl, ty / bl
        nvx, nvy = -ty, tx
        xmin, ymin = int(min(c0x, c1x)), int(min(c0y, c1y))           # convert_int2: toward zero
        xmax, ymax = int(math.ceil(max(c0x, c1x))), int(math.ceil(max(c0y, c1y)))
        if xmin < xlo:
            xmin = xlo
        if xmin > xhi or xmax < 0:
            continue
        if xmax > xhi:
            xmax = xhi
        if ymin < 0:
            ymin = 0
        if ymin >= ny or ymax < 0:
            continue
        if ymax >= ny:
            ymax = ny - 1
        for ii in range(xmin, xmax + 1):
            for jj in range(ymin, ymax + 1):
                gid = ii + nxf * jj
                if t.flat[gid] & M_SOLID:
                    continue
                lx, ly = float(ii), float(jj)
                for k in range(4):
                    d = 2 * k
                    cx, cy = _CXY[d]
                    den = nvx * cx + nvy * cy
                    if den == 0.0:
                        continue
                    if den > 0.0:
                        d = _REV8[d]
                        cx, cy = cx * -1.0, cy * -1.0
                        den *= -1.0
                    dist = (nvx * (c0x - lx) + nvy * (c0y - ly)) / den
                    if dist < 0.0 or dist > 1.0:
                        continue
                    ccx, ccy = lx + cx * dist, ly + cy * dist
                    a0x, a0y = ccx - c0x, ccy - c0y
                    a1x, a1y = ccx - c1x, ccy - c1y
                    if abs(bl - math.sqrt(a0x * a0x + a0y * a0y) - math.sqrt(a1x * a1x + a1y * a1y)) >= 1.0e-5:
                        continue
                    out.append((gid + D * (d + 1), dist))
    return out


def _ls_dx(pts, segs, nx, ny, nxf, ntype, min_dx=0.001, eps=1.0e-5):
    """dXArr as the reference's host set-up computes it (iniFillMap's 1 on
    fluid nodes, then bcFindNodes over every segment with bcFindDirection,
    bcFindIntersection, bcFindIntersectionLinePlane, testInside and bcSetdXArr,
    clVariablesLS.cpp:92-290, 330-356, 1195-1208) in its floating-point
    operations: [4][nxf*ny] (planes E, W, N, S).  A wall link whose crossing
    no segment reaches keeps 1, as there."""
    import math
    t = ntype.astype(np.int32).reshape(ny, nxf) & 0xFFFF
    dX = np.zeros((4, ny, nxf))
    dX[:, (t & M_FLUID) != 0] = 1.0
    dX[:, :, nx:] = 0.0
    cxy = ((0.0, 0.0), (1.0, 0.0), (-1.0, 0.0), (0.0, 1.0), (0.0, -1.0))
    rev = (0, 2, 1, 4, 3)

    def intersect(lx, ly, dx_, dy_, c0, c1):
        p10x, p10y = c1[0] - c0[0], c1[1] - c0[1]
        nvx, nvy = -p10y, p10x
        den = nvx * dx_ + nvy * dy_
        if den == 0.0:
            return None
        plx, ply = c0[0] - lx, c0[1] - ly
        distf = (nvx * plx + nvy * ply) / den
        cx_, cy_ = lx + dx_ * distf, ly + dy_ * distf
        d0x, d0y = cx_ - c0[0], cy_ - c0[1]
        d1x, d1y = cx_ - c1[0], cy_ - c1[1]
        if not abs(math.sqrt(p10x * p10x + p10y * p10y) - math.sqrt(d0x * d0x + d0y * d0y)
                   - math.sqrt(d1x * d1x + d1y * d1y)) < eps:
            return None
        n_cut = int(math.ceil(distf))
        dist = 1.0 - (n_cut - distf)
        c1x, c1y = int(lx + dx_ * n_cut), int(ly + dy_ * n_cut)
        c0x, c0y = c1x - int(dx_), c1y - int(dy_)
        if c0x % nx != c0x or c0y % ny != c0y:
            return None
        if t[c0y, c0x] & M_SOLID:
            if dist < eps:
                dist = 1.0
                n_cut -= 1
                c1x, c1y = int(lx + dx_ * n_cut), int(ly + dy_ * n_cut)
                c0x, c0y = c1x - int(dx_), c1y - int(dy_)
                if c0x % nx != c0x or c0y % ny != c0y:
                    return None
            else:
                return None
        return c0x, c0y, c1x, c1y, dist

    for a, b in segs:
        if a < 0:
            continue
        c0, c1 = (float(pts[a, 0]), float(pts[a, 1])), (float(pts[b, 0]), float(pts[b, 1]))
        cnx, cny = c0[1] - c1[1], c1[0] - c0[0]
        xmin, ymin = math.floor(min(c0[0], c1[0])), math.floor(min(c0[1], c1[1]))
        xmax, ymax = math.ceil(max(c0[0], c1[0])), math.ceil(max(c0[1], c1[1]))
        xmin = max(xmin, 0)
        if xmin > nx - 1 or xmax < 0:
            continue
        xmax = min(xmax, nx - 1)
        ymin = max(ymin, 0)
        if ymin > ny - 1 or ymax < 0:
            continue
        ymax = min(ymax, ny - 1)
        for d in (1, 3):
            dx_, dy_ = cxy[d]
            cn = cnx * dx_ + cny * dy_
            if cn == 0.0:
                continue
            if cn > 0.0:
                d = rev[d]
                dx_, dy_ = cxy[d]
            starts = []
            if dx_ != 0.0:
                i = xmin if dx_ == 1.0 else xmax
                starts += [(i, j) for j in range(ymin, ymax + 1)]
            if dy_ != 0.0:
                j = ymin if dy_ == 1.0 else ymax
                starts += [(i, j) for i in range(xmin, xmax + 1)]
            for i, j in starts:
                r = intersect(float(i), float(j), dx_, dy_, c0, c1)
                if r is None:
                    continue
                x0, y0, x1, y1, dist = r
                if not (0 <= x0 < nx and 0 <= y0 < ny):
                    continue
                x1 %= nx
                if not (0 <= y1 < ny):
                    continue
                if t[y0, x0] & M_SOLID or not (t[y1, x1] & M_SOLID):
                    continue
                v = dX[d - 1, y0, x0]
                v = dist if dist < v else v
                dX[d - 1, y0, x0] = v if v > min_dx else min_dx
    return dX.reshape(4, -1)


def _ls_map(pts, nx):
    """The segment each column starts its wall-distance search from
    (iniLSMap, clVariablesLS.cpp:895-918): per wall, the segment whose left
    end rounds up to the column, as an index among the wall segments (top
    segments counted after the bottom ones)."""
    import math
    n_pts = len(pts)
    nb = n_pts // 2 - 1                      # segments per wall
    lsmap = np.zeros((2, nx), np.int64)
    for ib in range(nb):
        cx1, cx2 = pts[ib, 0], pts[ib + 1, 0]
        if not (cx2 < 0.0 or cx1 >= nx - 1.0):
            loc = int(math.ceil(cx1))
            if 0 <= loc < nx:
                lsmap[0, loc] = ib
        it = n_pts // 2 + ib                 # top segment: points it, it + 1 (right to left)
        cx2, cx1 = pts[it, 0], pts[it + 1, 0]
        if not (cx2 < 0.0 or cx1 >= nx - 1.0):
            loc = int(math.ceil(cx1))
            if 0 <= loc < nx:
                lsmap[1, loc] = ib + nb
    return lsmap


def _ls_wall_distance(pts, lsmap, nx, ny, nxf, fluid, radius=50):
    """updateWallD / findMinDist (kOmegaKernels.cl:751-840) on the polyline
    pts with the column map lsmap, in the reference's operations: the window
    of radius segments around lsmap's entry, used as point indices into pts
    as the kernel does (bottom: [max(m - r, 0), min(m + r, n/2 - 1)), top:
    [max(m - r, n/2), min(m + r, n - 1)))."""
    wall = np.zeros((ny, nxf))
    jj, ii = np.nonzero(fluid)
    if len(jj) == 0:
        return wall
    n_pts = len(pts)
    px, py = ii.astype(float), jj.astype(float)
    dmin = np.full(len(jj), 1000.0)
    Cx, Cy = pts[:, 0].astype(float), pts[:, 1].astype(float)
    for top in (False, True):
        m = lsmap[1 if top else 0][ii]
        lo = np.maximum(m - radius, n_pts // 2 if top else 0)
        hi = np.minimum(m + radius, n_pts - 1 if top else n_pts // 2 - 1)
        for o in range(-radius, radius):
            k = m + o
            sel = (k >= lo) & (k < hi)
            if not sel.any():
                continue
            k = k[sel]
            x, y = px[sel], py[sel]
            P0x, P0y, P1x, P1y = Cx[k], Cy[k], Cx[k + 1], Cy[k + 1]
            vTx = P1x - P0x
            vTy = P1y - P0y
            vTmag = np.sqrt(vTx * vTx + vTy * vTy)
            d = np.abs(vTy * x - vTx * y + P1x * P0y - P1y * P0x) / vTmag
            pcx = x - d * (-(vTy / vTmag))
            if top:
                c0 = pcx > P0x
                c1 = ~c0 & (pcx < P1x)
            else:
                c0 = pcx < P0x
                c1 = ~c0 & (pcx > P1x)
            e0x, e0y = x - P0x, y - P0y
            e1x, e1y = x - P1x, y - P1y
            d = np.where(c0, np.sqrt(e0x * e0x + e0y * e0y), d)
            d = np.where(c1, np.sqrt(e1x * e1x + e1y * e1y), d)
            cur = dmin[sel]
            dmin[sel] = np.where(d < cur, d, cur)
    wall[jj, ii] = dmin
    return wall


def read_reference_polyline(directory: str):
    """lsc0.txt points in the order the reference's kernels walk them
    (bottom wall left to right, then top wall right to left) and lbsize."""
    import os
    size = np.loadtxt(os.path.join(directory, "lbsize.txt")).ravel()
    pts = np.loadtxt(os.path.join(directory, "lsc0.txt"), ndmin=2)
    return int(size[0]), int(size[1]), pts


def read_reference_segments(directory: str):
    """lsbl.txt: the wall segments as point-index pairs."""
    import os
    return np.loadtxt(os.path.join(directory, "lsbl.txt"), ndmin=2).astype(np.int64)


def channel_from_reference_files(directory: str, nx_full: int | None = None, ibb_all: bool = False,
                                 min_dx: float = 0.001, wall_radius: int = 50) -> Channel:
    """The geometry of a reference run directory on its own polylines: node
    types from the walls' heights at the columns (read_reference_walls, the
    fill of clVariablesLS), the interpolated links and their fractions from
    the reference's list builder on the actual segments (_ls_links; columns
    1 .. nx-2, a link found by two segments kept once, links with q = 1/2
    left out unless ibb_all), the E/W/N/S link fractions of the reference's
    host set-up on the same segments (_ls_dx: clamped at min_dx, 1 where no
    segment reaches the crossing, as at the ends of the polylines), and the
    wall distance of updateWallD on the actual segments (_ls_wall_distance)."""
    nx, ny, y_bot, y_top = read_reference_walls(directory)
    _, _, pts = read_reference_polyline(directory)
    ch = channel_from_walls(nx, ny, y_bot, y_top, nx_full, wall_distance=False, min_dx=min_dx)
    nxf, D = ch.nx_full, ch.n
    fl = ch.fluid_mask()
    first = {}
    for idx, dist in _ls_links(pts, nx, ny, nxf, ch.ntype, 1, nx - 2):
        first.setdefault(idx, dist)
    keep = sorted(k for k, v in first.items() if ibb_all or abs(v - 0.5) > 1e-12)
    ch.ibb_idx = np.asarray(keep, np.int32)
    ch.ibb_q = np.asarray([first[k] for k in keep], float)
    segs = read_reference_segments(directory)
    ch.dX = _ls_dx(pts, segs, nx, ny, nxf, ch.ntype, min_dx).ravel()
    ch.wallD = _ls_wall_distance(pts, _ls_map(pts, nx), nx, ny, nxf, fl, wall_radius).ravel()
    return ch


def wavy_channel(nx: int, ny: int, amplitude: float, wavelength: int,
                 nx_full: int | None = None, ibb_all: bool = False,
                 seam_ibb: bool = False, wall_distance: bool = True) -> Channel:
    """Walls displaced by h(x) = A (1 - cos(2 pi x / L)) / 2 from the half-way
    positions 0.5 and ny - 1.5, mirrored top and bottom.  h and its slope
    vanish at x = 0, so the links at the periodic seam keep q <= 1/2."""
    x = np.arange(nx)
    h = amplitude * 0.5 * (1.0 - np.cos(2.0 * np.pi * x / wavelength))
    return channel_from_walls(nx, ny, 0.5 + h, ny - 1.5 - h, nx_full, ibb_all=ibb_all, seam_ibb=seam_ibb,
                              wall_distance=wall_distance)


def straight_channel(nx: int, ny: int, nx_full: int | None = None) -> Channel:
    """Rows 0 and ny-1 solid; half-way walls at y = 0.5 and y = ny - 1.5."""
    return channel_from_walls(nx, ny, np.full(nx, 0.5), np.full(nx, ny - 1.5), nx_full)


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


def temperature_field(ch: Channel, t0: float = 0.5) -> np.ndarray:
    """tempArray at the start of a run that loads no temperature file:
    Tinitial (TFD_INI_TEMP, 0.5) on every node -- clVariablesFD::testRestartRun
    fills the whole array (clVariablesFD.cpp:813-823) and ini's
    fillByNodeType(ROE0, nType, M0_FLUID_NODE) (236-239) leaves the wall nodes
    as they are.  The wall-boundary rows of the thermal system (x = 0) pull
    those values to 0 over the first solves."""
    return np.full(ch.n, float(t0))


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


def main(argv=None):
    """Times the geometry set-up of a wavy k-omega channel: the device builder
    (kofm_set_walls, median of 5 calls on a live context after one warm-up)
    and, with --host, this module's host builder plus kofm_set_geometry.

        python -m komegafoulingmodel_b200.geometry [--nx 16384 --ny 1024 --host]
    """
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=16384)
    ap.add_argument("--ny", type=int, default=1024)
    ap.add_argument("--amplitude", type=float, default=32.0)
    ap.add_argument("--wavelength", type=int, default=512)
    ap.add_argument("--host", action="store_true")
    args = ap.parse_args(argv)
    from .lattice import Lattice, desc_default
    nx, ny = args.nx, args.ny
    h = args.amplitude * 0.5 * (1.0 - np.cos(2.0 * np.pi * np.arange(nx) / args.wavelength))
    yb, yt = 0.5 + h, ny - 1.5 - h
    d = desc_default()
    d.nx, d.nx_full, d.ny = nx, nx, ny
    d.use_komega = 1
    out = {"case": f"wavy k-omega channel {nx}x{ny}, amplitude {args.amplitude}, "
                   f"wavelength {args.wavelength}"}
    with Lattice(d) as L:
        L.set_walls(yb, yt)
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            L.set_walls(yb, yt)
            ts.append((time.perf_counter() - t0) * 1e3)
        out["device_ms"] = sorted(ts)[2]
        out["device_runs_ms"] = ts
        out["n_ibb"] = L._n_ibb
        if args.host:
            t0 = time.perf_counter()
            ch = wavy_channel(nx, ny, args.amplitude, args.wavelength)
            t1 = time.perf_counter()
            L.set_geometry(ch.ntype, ch.wallD, ch.dX, ch.ibb_idx, ch.ibb_q)
            t2 = time.perf_counter()
            out["host_builder_ms"] = (t1 - t0) * 1e3
            out["set_geometry_ms"] = (t2 - t1) * 1e3
            out["host_over_device"] = (t2 - t0) * 1e3 / out["device_ms"]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
