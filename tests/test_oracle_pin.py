"""Pins the oracle (FP64 C restatement) to the reference's own kernels.

oracle/_ref is the reference's source/Kernels/{Heading,lbKernels,
kOmegaKernels}.cl compiled for the CPU (oracle/Makefile).  Where it is
absent (the reference tree is not mounted) the committed fixtures in
tests/golden/ (made from it by tests/golden/make_golden.py) pin the oracle.
"""
import ctypes as C
import os

import numpy as np
import pytest

from komegafoulingmodel_b200 import geometry as G
from oracle.orc import make_cfg
from tests.cases import komega_state, perturbed_state

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_kernels.npz")


def _collide(lib_fn, cfg, F, m, wd, k, o, s, komega, oracle_call):
    n = cfg.nxf * cfg.ny
    FB = np.zeros(9 * n)
    rho, ux, uy, nut = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    K, O, S = k.copy(), o.copy(), s.copy()
    if oracle_call:
        lib_fn(C.byref(cfg), F, FB, m, rho, ux, uy, K, O, wd, nut, S, 2, komega)
    elif komega:
        lib_fn(C.byref(cfg), rho, ux, uy, F.copy(), FB, m, wd, nut, K, O, S, 2)
    else:
        lib_fn(C.byref(cfg), rho, ux, uy, F.copy(), FB, m, 2)
    return dict(FB=FB, rho=rho, ux=ux, uy=uy, nut=nut, K=K, O=O, S=S)


@pytest.mark.parametrize("komega", [0, 1])
@pytest.mark.parametrize("nx,ny", [(64, 20), (128, 33)])
def test_collide_matches_reference_kernel(oracle, refk, komega, nx, ny):
    cfg = make_cfg(nx, ny, 1.25 if not komega else 1.9, 1e-5, 0.01 if komega else 0.1)
    ch = G.straight_channel(nx, ny)
    F = perturbed_state(ch, seed=nx + ny)
    k, o, nut, s = komega_state(ch, seed=3)
    # a few negative k / omega exercise the in-place clamps (lbKernels.cl:400-410)
    k[ch.fluid_mask().ravel().nonzero()[0][:3]] *= -1
    o[ch.fluid_mask().ravel().nonzero()[0][5:7]] *= -1
    a = _collide(oracle.L.orc_collide_push, cfg, F, ch.ntype, ch.wallD, k, o, s, komega, True)
    fn = refk.L.ref_collide_komega if komega else refk.L.ref_collide_laminar
    b = _collide(fn, cfg, F, ch.ntype, ch.wallD, k, o, s, komega, False)
    fl = ch.fluid_mask().ravel()
    for key in a:
        if not komega and key in ("K", "O", "S", "nut"):
            continue
        x, y = a[key], b[key]
        if key == "FB":
            # slots of fluid nodes (solid slots are never written)
            x = x.reshape(9, -1)[:, fl]
            y = y.reshape(9, -1)[:, fl]
        scale = np.max(np.abs(y)) + 1e-300
        tol = 1e-11 if key == "S" else 1e-14
        assert np.max(np.abs(x - y)) <= tol * scale, key


def test_ibb_matches_reference_kernel(oracle, refk):
    nx, ny = 64, 20
    cfg = make_cfg(nx, ny, 1.25, 0.0, 0.1)
    ch = G.straight_channel(nx, ny)
    n = ch.n
    rng = np.random.default_rng(5)
    FB = rng.random(9 * n)
    # links from the bottom / top fluid rows into the walls, q both sides of 0.5
    idx, q = [], []
    for i in range(nx):
        for d, j in ((4, 1), (3, ny - 2), (6, 1), (5, ny - 2)):
            if d in (6,) and i == 0:
                continue
            idx.append(d * n + i + nx * j)
            q.append(rng.uniform(0.05, 0.95))
    idx = np.array(idx, np.int32)
    q = np.array(q)
    a = FB.copy()
    b = FB.copy()
    oracle.L.orc_ibb(C.byref(cfg), idx, q, a, len(idx))
    refk.L.ref_ibb(C.byref(cfg), idx, q, b, len(idx))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("nx,ny", [(64, 20), (96, 40)])
def test_komega_assembly_matches_reference_kernels(oracle, refk, nx, ny):
    cfg = make_cfg(nx, ny, 1.9, 1e-6, 0.01)
    ch = G.straight_channel(nx, ny)
    n = ch.n
    F = perturbed_state(ch, seed=7)
    k, o, nut, s = komega_state(ch, seed=8)
    a = _collide(oracle.L.orc_collide_push, cfg, F, ch.ntype, ch.wallD, k, o, s, 1, True)
    IA, JA, ind = oracle.csr(cfg, ch.ntype)
    nnz = len(JA)

    def assemble(lib, is_oracle):
        Dk, Do, F1, dk = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(2 * n)
        kA, oA, kb, ob = np.zeros(nnz), np.zeros(nnz), np.zeros(n), np.zeros(n)
        K, O = a["K"].copy(), a["O"].copy()
        if is_oracle:
            lib.orc_komega_diffusivities(C.byref(cfg), ch.ntype, K, O, a["nut"], ch.wallD,
                                         Dk, Do, F1, dk, a["rho"], ch.dX)
            lib.orc_komega_coeffs(C.byref(cfg), ind, K, O, a["nut"], Dk, Do, F1, dk, a["S"],
                                  a["rho"], a["ux"], a["uy"], kA, oA, kb, ob, ch.dX,
                                  ch.wallD, ch.ntype, 1.0)
        else:
            dbg = np.zeros(40 * n)
            lib.ref_komega_diffusivities(C.byref(cfg), ch.ntype, K, O, a["nut"], ch.wallD,
                                         Dk, Do, F1, dk, a["rho"], ch.dX, dbg)
            lib.ref_komega_coeffs(C.byref(cfg), ind, K, O, a["nut"], Dk, Do, F1, dk, a["S"],
                                  a["rho"], a["ux"], a["uy"], kA, oA, kb, ob, ch.dX,
                                  ch.wallD, ch.ntype, 1.0, dbg)
        return dict(Dk=Dk, Do=Do, F1=F1, dk=dk, kA=kA, oA=oA, kb=kb, ob=ob)

    x = assemble(oracle.L, True)
    y = assemble(refk.L, False)
    for key in x:
        assert np.array_equal(x[key], y[key]), key


def test_oracle_against_golden_fixtures(oracle):
    """Same comparisons against fixtures generated from oracle/_ref."""
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixtures not generated")
    g = np.load(GOLDEN)
    nx, ny = int(g["nx"]), int(g["ny"])
    cfg = make_cfg(nx, ny, float(g["tau"]), float(g["fterm"]), float(g["mu"]))
    ch = G.straight_channel(nx, ny)
    for komega in (0, 1):
        a = _collide(oracle.L.orc_collide_push, cfg, g["F"], ch.ntype, ch.wallD, g["K"],
                     g["O"], g["S"], komega, True)
        fl = ch.fluid_mask().ravel()
        for key in ("FB", "rho", "ux", "uy") + (("nut", "K", "O", "S") if komega else ()):
            ref = g[f"{key}_{komega}"]
            x = a[key]
            if key == "FB":
                x = x.reshape(9, -1)[:, fl].ravel()
                ref = ref.reshape(9, -1)[:, fl].ravel()
            tol = 1e-11 if key == "S" else 1e-14
            assert np.max(np.abs(x - ref)) <= tol * (np.max(np.abs(ref)) + 1e-300), (komega, key)


def test_oracle_assembly_against_golden_fixtures(oracle):
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixtures not generated")
    g = np.load(GOLDEN)
    nx, ny = int(g["nx"]), int(g["ny"])
    cfg = make_cfg(nx, ny, float(g["tau"]), float(g["fterm"]), float(g["mu"]))
    ch = G.straight_channel(nx, ny)
    n = ch.n
    IA, JA, ind = oracle.csr(cfg, ch.ntype)
    nnz = len(JA)
    Dk, Do, F1, dk = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(2 * n)
    kA, oA, kb, ob = np.zeros(nnz), np.zeros(nnz), np.zeros(n), np.zeros(n)
    K, O = g["K_1"].copy(), g["O_1"].copy()
    oracle.L.orc_komega_diffusivities(C.byref(cfg), ch.ntype, K, O, g["nut_1"], ch.wallD,
                                      Dk, Do, F1, dk, g["rho_1"], ch.dX)
    oracle.L.orc_komega_coeffs(C.byref(cfg), ind, K, O, g["nut_1"], Dk, Do, F1, dk, g["S_1"],
                               g["rho_1"], g["ux_1"], g["uy_1"], kA, oA, kb, ob, ch.dX,
                               ch.wallD, ch.ntype, 1.0)
    for key, v in dict(Dk=Dk, Do=Do, F1=F1, dkdo=dk, kA=kA, oA=oA, kb=kb, ob=ob).items():
        assert np.array_equal(v, g[key]), key


# ---- interpolated bounce-back list of the geometry builders ------------------------

def _same_list(idx, dist, ch):
    """The reference's list (duplicates included) against a builder's: every
    link once, the same wall fractions.  The reference lists a link twice
    where it meets the wall at a polyline point (both segments' tests accept
    it, lsKernels.cl:199-206): the two entries carry the same fraction."""
    uniq, first, inv = np.unique(idx, return_index=True, return_inverse=True)
    spread = np.zeros(len(uniq))
    np.maximum.at(spread, inv, np.abs(dist - dist[first][inv]))
    assert spread.max() <= 1e-15
    assert np.array_equal(uniq, ch.ibb_idx)   # the builder's list is sorted
    assert np.abs(dist[first] - ch.ibb_q).max() <= 1e-15
    return len(idx) - len(uniq)


@pytest.mark.parametrize("name", ["wavy", "sine", "random"])
def test_ibb_list_matches_reference_builder(refk, name):
    """channel_from_walls (and, through the GPU tests, kofm_set_walls) against
    the reference's updateIBBOnly on the same walls: the same links from the
    same nodes (none on columns 0 and nx-1) with the same wall fractions."""
    from komegafoulingmodel_b200 import adjoint as A
    if name == "random":
        nx, ny = 1024, 256
        yb, yt = A.walls(A.coefficients(), nx, ny)
    else:
        import tests.golden.make_golden_ibb as mk
        nx, ny = mk.NX, mk.NY
        yb, yt = mk.walls(name)
    ch = G.channel_from_walls(nx, ny, yb, yt, ibb_all=True)
    idx, dist = refk.ibb_list(make_cfg(nx, ny, 1.0, 0.0, 0.1), ch.ntype, yb, yt)
    dups = _same_list(idx, dist, ch)
    print(name, len(ch.ibb_idx), "links;", dups, "listed twice by the reference")


def test_geometry_against_golden_fixture():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_ibb.npz"))
    nx, ny = int(z["nx"]), int(z["ny"])
    for name in ("wavy", "sine"):
        ch = G.channel_from_walls(nx, ny, z[f"{name}_yb"], z[f"{name}_yt"], ibb_all=True)
        assert np.array_equal(ch.ntype, z[f"{name}_ntype"])
        _same_list(z[f"{name}_idx"], z[f"{name}_dist"], ch)
        assert np.array_equal(ch.wallD, z[f"{name}_walld"])


@pytest.mark.parametrize("name", ["wavy", "sine", "random", "fouled"])
def test_boundary_flags_match_reference_kernel(refk, name):
    """The builders' nType against the reference's updateNodeBoundaryInfo
    (lsKernels.cl:511-583): cleared to the bits it keeps and recomputed by it,
    the fouled-wall flags come back unchanged; run on the unfouled map, it
    gives the *0 flags the builders set (BOUNDARY_NODE0 for any wall link,
    NESW_BOUNDARY_NODE0 for an E/W/N/S one, SOLID_BOUNDARY_NODE0 from its
    SOLID_BOUNDARY_NODE, as iniNodeBoundaryInfo0, clVariablesLS.cpp:920-951)."""
    from komegafoulingmodel_b200 import adjoint as A
    import tests.golden.make_golden_ibb as mk
    yb0 = yt0 = None
    if name == "random":
        nx, ny = 1024, 256
        yb, yt = A.walls(A.coefficients(), nx, ny)
    elif name == "fouled":
        nx, ny = 160, 40
        dep = 3.0 + 1.5 * (1.0 - np.cos(2 * np.pi * np.arange(nx) / 80.0))
        yb, yt = 0.5 + dep, ny - 1.5 - dep
        yb0, yt0 = np.full(nx, 0.5), np.full(nx, ny - 1.5)
    else:
        nx, ny = mk.NX, mk.NY
        yb, yt = mk.walls(name)
    ch = G.channel_from_walls(nx, ny, yb, yt, y_bot0=yb0, y_top0=yt0)
    cfg = make_cfg(nx, ny, 1.0, 0.0, 0.1)
    t = ch.ntype.astype(np.int32) & 0xFFFF
    m = (t & 0x00EF).astype(np.uint16).view(np.int16)
    refk.L.ref_update_node_boundary_info(C.byref(cfg), m)
    assert np.array_equal(m, ch.ntype)
    # the unfouled map: M0 bits in the places of the M bits
    m0 = np.where(t & G.M0_SOLID, G.M_SOLID, G.M_FLUID).astype(np.uint16).view(np.int16)
    refk.L.ref_update_node_boundary_info(C.byref(cfg), m0)
    r = m0.astype(np.int32) & 0xFFFF
    fl0 = (t & G.M0_SOLID) == 0
    want = np.zeros_like(t)
    want |= np.where(fl0 & ((r & 0xFF00) != 0), G.BOUNDARY0, 0)
    want |= np.where(fl0 & ((r & G.NESW_BOUNDARY) != 0), G.NESW_BOUNDARY0, 0)
    want |= np.where(~fl0 & ((r & G.SOLID_BOUNDARY) != 0), G.SOLID_BOUNDARY0, 0)
    got = t & (G.BOUNDARY0 | G.NESW_BOUNDARY0 | G.SOLID_BOUNDARY0)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", ["wavy", "sine", "random"])
def test_wall_distance_matches_reference_kernel(refk, name):
    """channel_from_walls' wall distance against the reference's updateWallD
    (kOmegaKernels.cl:751-840) on the same polylines: bit for bit, including
    the nodes where the reference's line distance undercuts the segment's."""
    from komegafoulingmodel_b200 import adjoint as A
    import tests.golden.make_golden_ibb as mk
    if name == "random":
        nx, ny = 1024, 256
        yb, yt = A.walls(A.coefficients(), nx, ny)
    else:
        nx, ny = mk.NX, mk.NY
        yb, yt = mk.walls(name)
    ch = G.channel_from_walls(nx, ny, yb, yt)
    wd = refk.wall_distance(make_cfg(nx, ny, 1.0, 0.0, 0.1), ch.ntype, yb, yt)
    assert np.array_equal(ch.wallD, wd)


@pytest.mark.parametrize("name", ["wavy", "sine", "random"])
def test_link_fractions_match_reference_host_setup(refk, name):
    """channel_from_walls' dXArr against the reference's host set-up
    (bcFindNodes .. bcSetdXArr, clVariablesLS.cpp:92-290, compiled as C++) on
    the same walls through the columns: the same links, the same fractions
    up to the rounding of its 1 - (ceil(d) - d)."""
    from komegafoulingmodel_b200 import adjoint as A
    import tests.golden.make_golden_ibb as mk
    if name == "random":
        nx, ny = 1024, 256
        yb, yt = A.walls(A.coefficients(), nx, ny)
    else:
        nx, ny = mk.NX, mk.NY
        yb, yt = mk.walls(name)
    ch = G.channel_from_walls(nx, ny, yb, yt, wall_distance=False)
    pts = refk.wall_points(nx, yb, yt)
    n = len(pts) // 2
    segs = np.array([(i, i + 1) for i in range(n - 1)] + [(n + i, n + i + 1) for i in range(n - 1)])
    dx, _ = refk.link_fractions(make_cfg(nx, ny, 1.0, 0.0, 0.1), ch.ntype, pts, segs)
    assert np.array_equal(dx == 1.0, ch.dX == 1.0) and np.array_equal(dx == 0.0, ch.dX == 0.0)
    assert np.abs(dx - ch.dX).max() <= 1e-15
