"""Curved walls: the wall-polyline geometry builder on CPU, and the GPU step
on a wavy channel (interpolated bounce-back with wall fractions q != 1/2,
non-uniform FD weights from the link fractions, curved wall distance) against
the FP64 oracle."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from oracle.orc import OracleSim, make_cfg
from tests.cases import fp32_state, rel_l2


def test_straight_walls_need_no_interpolated_records():
    ch = G.straight_channel(128, 20)
    assert len(ch.ibb_idx) == 0
    fl = ch.fluid_mask()
    assert fl[1:-1, :].all() and not fl[0].any() and not fl[-1].any()


def test_no_interpolated_links_on_the_seam_columns():
    """As the reference's updateIBBOnly (lsKernels.cl:455-466): no interpolated
    links from the nodes of columns 0 and nx-1 unless asked for."""
    for ibb_all in (False, True):
        ch = G.wavy_channel(256, 66, 8.0, 100, ibb_all=ibb_all)
        x = (ch.ibb_idx % ch.n) % ch.nx_full
        assert len(x) > 0 and not np.any((x == 0) | (x == ch.nx - 1))
        cs = G.wavy_channel(256, 66, 8.0, 100, ibb_all=ibb_all, seam_ibb=True)
        xs = (cs.ibb_idx % cs.n) % cs.nx_full
        assert np.any(xs == ch.nx - 1)
        inner = (xs != 0) & (xs != ch.nx - 1)
        assert np.array_equal(cs.ibb_idx[inner], ch.ibb_idx) and np.array_equal(cs.ibb_q[inner], ch.ibb_q)
        assert np.array_equal(cs.ntype, ch.ntype) and np.array_equal(cs.dX, ch.dX)


def test_link_fractions_clamped_for_the_fd_weights_only():
    """dXArr takes at least "Min dX Dist" (bcSetdXArr, clVariablesLS.cpp:
    248-286); the interpolated list keeps the fraction itself."""
    nx, ny = 64, 20
    ch = G.channel_from_walls(nx, ny, np.full(nx, 0.9995), np.full(nx, ny - 1.9995))
    dX = ch.dX.reshape(4, ny, nx)
    assert np.allclose(dX[3, 1, :], 0.001) and np.allclose(dX[2, ny - 2, :], 0.001)
    assert len(ch.ibb_q) > 0 and np.allclose(ch.ibb_q, 0.0005)
    c0 = G.channel_from_walls(nx, ny, np.full(nx, 0.9995), np.full(nx, ny - 1.9995), min_dx=0.0)
    assert np.allclose(c0.dX.reshape(4, ny, nx)[3, 1, :], 0.0005)


def test_wavy_geometry_invariants():
    ch = G.wavy_channel(256, 66, 8.0, 128)
    n = ch.n
    fl = ch.fluid_mask().ravel()
    t = ch.ntype.astype(np.int32) & 0xFFFF
    q = ch.ibb_q
    assert len(q) > 0 and np.all((q > 0) & (q <= 1))
    d = ch.ibb_idx // n
    node = ch.ibb_idx % n
    # every record is a fluid node whose link in direction d ends in a solid node
    assert np.all(fl[node])
    bound = np.array(G.BOUND)[d]
    assert np.all((t[node] & bound) != 0)
    # link fractions of the E/W/N/S planes: 1 away from walls, (0, 1] at walls
    dX = ch.dX.reshape(4, -1)
    assert np.all(dX[:, fl] > 0) and np.all(dX[:, fl] <= 1) and np.all(dX[:, ~fl] == 0)
    # wall distance is positive in the fluid and at most half the opening
    assert np.all(ch.wallD[fl] > 0) and ch.wallD.max() < 33
    # the seam columns have no link with 2q > 1 (those read the upstream node)
    x = node % ch.nx_full
    cx = G.CX[d]
    seam = ((x == 0) & (cx == 1)) | ((x == ch.nx - 1) & (cx == -1))
    assert not np.any(seam & (q > 0.5))


def _lattice(ch, rate, g, mu, komega, storage=_abi.STORE_FP32, **desc):
    d = desc_default()
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = rate, g, mu
    d.use_komega = 1 if komega else 0
    d.storage = storage
    for key, v in desc.items():
        setattr(d, key, v)
    L = Lattice(d)
    L.set_geometry(ch.ntype, ch.wallD if komega else None, ch.dX if komega else None,
                   ch.ibb_idx, ch.ibb_q)
    return L


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [(_abi.STORE_FP32, 1e-5), (_abi.STORE_FP16_NEQ, 1e-4),
                                         (_abi.STORE_FP16_NEQ32, 1e-4), (_abi.STORE_FP16_ROW, 1e-4)])
def test_wavy_laminar_matches_oracle(kofm_lib, oracle, storage, tol):
    """Interpolated bounce-back with q from 0.03 to 0.97; the FP16 f - feq
    form decodes every gathered, bounced and interpolated population with the
    reference moments of the node it was read from."""
    nx, ny = 256, 40
    ch = G.wavy_channel(nx, ny, 6.0, 128)
    rate, g, mu = 1.25, 2e-6, 0.1
    (f,) = fp32_state(G.equilibrium_state(ch, ux=0.01))
    cfg = make_cfg(nx, ny, rate, g, mu)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q)
    sim.step(300)
    with _lattice(ch, rate, g, mu, False, storage) as L:
        L.set_state(f)
        L.step(300)
        rho, ux, uy = L.get_macro()
    fl = ch.fluid_mask().ravel()
    errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl))
    uy_rel = np.linalg.norm((uy - sim.uy)[fl]) / np.linalg.norm(sim.ux[fl])
    print(errs, uy_rel)
    assert errs["rho"] < tol / 10 and errs["ux"] < tol and uy_rel < tol, (errs, uy_rel)


def _wavy_komega_case(nx=256, ny=66, amp=8.0, lam=128):
    ch = G.wavy_channel(nx, ny, amp, lam)
    nu, u_max = 5e-4, 0.05
    R = ch.pipe_radius
    y = np.arange(ny)[:, None] - 0.5
    ux = np.clip(u_max * (1 - ((y - R) / R) ** 2), 0, None) * np.ones((1, nx))
    f = G.equilibrium_state(ch, ux=ux)
    g = G.force_from_re((2.0 / 3.0) * u_max * R / nu, nu, R)
    k0 = 1.5 * (0.05 * u_max) ** 2
    o0 = np.sqrt(k0) / (0.09 ** 0.25 * 0.07 * 2 * R)
    k, o, nut = G.komega_fields(ch, k0, o0)
    f, k, o, nut = fp32_state(f, k, o, nut)
    return ch, f, k, o, nut, 1.0 / (3 * nu + 0.5), g, nu


def _fields(L):
    rho, ux, _ = L.get_macro()
    _, k, o, _, _ = L.get_state()
    return rho, ux, k, o


# GMRES tolerances of the wavy k-omega comparison: tight, so that each solve's
# result does not depend on where a cycle is cut (see the test's docstring)
TIGHT = dict(rel_tol=1e-10, abs_tol=1e-30, max_iters=1000)


@pytest.mark.gpu
def test_wavy_komega_matches_oracle(kofm_lib, oracle):
    """k-omega on the wavy channel, with the GMRES solves run to 1e-10.

    At the reference tolerance (1e-4) some solves on this channel end a cycle
    on a tie: the xi-test |xi_k| >= rho compares two numbers that agree to
    ~1e-9 while each carries the rounding of a sum over all nodes, so whether
    the cycle stops at k or goes on depends on the summation order (the device
    and the oracle both meet the tolerance either way, ~2e-7 apart in omega).
    This flow then amplifies such differences: the oracle started from k
    perturbed by 1e-7 differs by 2e-5 after 20 steps and ~1e-2 in k after 50
    (near-wall limiter and clamp switches).  With 1e-10 solves the GPU is held
    to 1e-5 after 10 steps, and after 100 steps to a few times the oracle's own
    spread under that perturbation."""
    ch, f, k, o, nut, rate, g, nu = _wavy_komega_case()
    nx, ny = ch.nx, ch.ny
    cfg = make_cfg(nx, ny, rate, g, nu)
    mk = lambda kk: OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, kk, o, nut,  # noqa: E731
                              komega=True, ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q, **TIGHT)
    sim, pert = mk(k), mk(k * (1 + 1e-7))
    fl = ch.fluid_mask().ravel()
    with _lattice(ch, rate, g, nu, True, komega_rel_tol=TIGHT["rel_tol"],
                  komega_abs_tol=TIGHT["abs_tol"], komega_max_iters=TIGHT["max_iters"]) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        sim.step(10)
        L.step(10)
        rho, ux, k2, o2 = _fields(L)
        errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl),
                    k=rel_l2(k2, sim.K, fl), omega=rel_l2(o2, sim.O, fl))
        print("10 steps", errs)
        for key in ("rho", "ux", "k", "omega"):
            assert errs[key] < 1e-5, errs
        sim.step(90)
        pert.step(100)
        L.step(90)
        rho, ux, k2, o2 = _fields(L)
    for name, gpu, ref, alt in (("ux", ux, sim.ux, pert.ux), ("k", k2, sim.K, pert.K),
                                ("omega", o2, sim.O, pert.O)):
        spread = rel_l2(alt, ref, fl)
        err = rel_l2(gpu, ref, fl)
        print("100 steps", name, err, spread)
        assert err < 5 * spread + 1e-6, (name, err, spread)


@pytest.mark.gpu
def test_wavy_komega_2048x256_matches_oracle(kofm_lib, oracle):
    """The 2048 x 256 wavy k-omega channel (walls 0.5 + 16 (1 - cos(2 pi x /
    512)) and mirrored: a +-16 sine of wavelength 512 phased so that the
    periodic seam sits at a crest, where no interpolated link has 2q > 1),
    body-forced and periodic, nu = 5e-4, GMRES solves run to 1e-10: 10 steps
    within 1e-5 of the FP64 oracle, 40 within a few times the oracle's own
    spread under a 1e-7 perturbation of k."""
    ch, f, k, o, nut, rate, g, nu = _wavy_komega_case(2048, 256, 32.0, 512)
    from komegafoulingmodel_b200.adjoint import Case
    assert Case.notches(ch) == 0
    x = (ch.ibb_idx % ch.n) % ch.nx_full
    cx = G.CX[ch.ibb_idx // ch.n]
    assert not np.any((((x == 0) & (cx == 1)) | ((x == ch.nx - 1) & (cx == -1))) & (ch.ibb_q > 0.5))
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    mk = lambda kk: OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, kk, o, nut,  # noqa: E731
                              komega=True, ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q, **TIGHT)
    sim, pert = mk(k), mk(k * (1 + 1e-7))
    fl = ch.fluid_mask().ravel()
    with _lattice(ch, rate, g, nu, True, komega_rel_tol=TIGHT["rel_tol"],
                  komega_abs_tol=TIGHT["abs_tol"], komega_max_iters=TIGHT["max_iters"]) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        sim.step(10)
        L.step(10)
        rho, ux, k2, o2 = _fields(L)
        errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl),
                    k=rel_l2(k2, sim.K, fl), omega=rel_l2(o2, sim.O, fl))
        print("10 steps", errs)
        for key in ("rho", "ux", "k", "omega"):
            assert errs[key] < 1e-5, errs
        sim.step(30)
        pert.step(40)
        L.step(30)
        rho, ux, k2, o2 = _fields(L)
    for name, gpu, ref, alt in (("ux", ux, sim.ux, pert.ux), ("k", k2, sim.K, pert.K),
                                ("omega", o2, sim.O, pert.O)):
        spread = rel_l2(alt, ref, fl)
        err = rel_l2(gpu, ref, fl)
        print("40 steps", name, err, spread)
        assert err < 5 * spread + 1e-6, (name, err, spread)


@pytest.mark.gpu
def test_wavy_komega_2048x256_at_the_reference_tolerance(kofm_lib, oracle):
    """The same 2048 x 256 wavy channel with the reference's GMRES tolerances
    (relTol 1e-4, absTol 1e-7).  Measured against the FP64 oracle: rho, u, k,
    omega stay below 1e-5 for the first 6 steps (3.1e-6 at step 6); at step 7
    one discrete switch moves omega by 3.7e-5, and from there the difference
    grows as the flow's own sensitivity does -- the oracle started from
    k (1 + 1e-7) spreads from itself by 1e-4 in k by step 18 and 4e-3 by step
    60, where the GPU stands at 1.3x that spread in u and 1.5x in k.  Held
    here: 1e-5 after 6 steps, and u, k within 3x the oracle's spread after
    60."""
    ch, f, k, o, nut, rate, g, nu = _wavy_komega_case(2048, 256, 32.0, 512)
    cfg = make_cfg(ch.nx, ch.ny, rate, g, nu)
    mk = lambda kk: OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, kk, o, nut,  # noqa: E731
                              komega=True, ibb_idx=ch.ibb_idx, ibb_q=ch.ibb_q)
    sim, pert = mk(k), mk(k * (1 + 1e-7))
    fl = ch.fluid_mask().ravel()
    with _lattice(ch, rate, g, nu, True) as L:
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        sim.step(6)
        L.step(6)
        rho, ux, k2, o2 = _fields(L)
        errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl),
                    k=rel_l2(k2, sim.K, fl), omega=rel_l2(o2, sim.O, fl))
        print("6 steps", errs)
        for key in ("rho", "ux", "k", "omega"):
            assert errs[key] < 1e-5, errs
        sim.step(54)
        pert.step(60)
        L.step(54)
        rho, ux, k2, o2 = _fields(L)
    for name, gpu, ref, alt in (("ux", ux, sim.ux, pert.ux), ("k", k2, sim.K, pert.K)):
        spread = rel_l2(alt, ref, fl)
        err = rel_l2(gpu, ref, fl)
        print("60 steps", name, err, spread)
        assert err < 3 * spread + 1e-6, (name, err, spread)


def _write_reference_walls(d, nx, ny, bottom, top, dx=1.0):
    """Wall files in the layout of a reference run directory: points every dx
    from x = -0.75 along the lower wall to past nx - 0.5, then back along the
    upper wall; segments join consecutive points of each wall."""
    import os
    xs = [-0.75]
    while xs[-1] <= nx - 0.5:
        xs.append(xs[-1] + dx)
    xs = np.array(xs)
    pts = [(x, bottom(x)) for x in xs] + [(x, top(x)) for x in xs[::-1]]
    n = len(xs)
    segs = [(i, i + 1) for i in range(n - 1)] + [(n + i, n + i + 1) for i in range(n - 1)]
    os.makedirs(d, exist_ok=True)
    np.savetxt(os.path.join(d, "lsc0.txt"), np.array(pts))
    np.savetxt(os.path.join(d, "lsbl.txt"), np.array(segs), fmt="%d")
    np.savetxt(os.path.join(d, "lbsize.txt"), np.array([[nx, ny]]), fmt="%d")


def test_reference_wall_files(tmp_path):
    """lsc0 / lsbl / lbsize files (straight walls of the reference's channel
    script: y = nY/2 - 1 + 0.5 -/+ H) and a wavy pair give the channel that
    channel_from_walls builds from the same heights."""
    nx, H = 96, 20
    ny = 2 * H + 4
    yini = ny / 2 - 1 + 0.5
    _write_reference_walls(str(tmp_path / "s"), nx, ny, lambda x: yini - H, lambda x: yini + H)
    ch = G.channel_from_reference_files(str(tmp_path / "s"))
    ref = G.channel_from_walls(nx, ny, np.full(nx, yini - H), np.full(nx, yini + H))
    assert np.array_equal(ch.ntype, ref.ntype) and np.array_equal(ch.dX, ref.dX)
    assert np.array_equal(ch.ibb_idx, ref.ibb_idx) and np.allclose(ch.wallD, ref.wallD)
    # wavy walls with vertices at the columns (dx = 1 from x = -0.75 misses
    # them; dx = 0.25 from -0.75 hits every column)
    amp, lam = 4.0, 48
    h = lambda x: amp * 0.5 * (1 - np.cos(2 * np.pi * x / lam))  # noqa: E731
    _write_reference_walls(str(tmp_path / "w"), nx, ny, lambda x: 0.5 + h(x),
                           lambda x: ny - 1.5 - h(x), dx=0.25)
    ch = G.channel_from_reference_files(str(tmp_path / "w"))
    x = np.arange(nx)
    ref = G.channel_from_walls(nx, ny, 0.5 + h(x), ny - 1.5 - h(x))
    # the same nodes and links; the fractions follow the file's own segments
    # (points every quarter column) instead of chords between the columns
    assert np.array_equal(ch.ntype, ref.ntype) and np.array_equal(ch.ibb_idx, ref.ibb_idx)
    assert np.allclose(ch.ibb_q, ref.ibb_q, atol=2e-2) and not np.allclose(ch.ibb_q, ref.ibb_q, atol=1e-6)


@pytest.mark.parametrize("dx", [1.0, 0.25])
def test_reference_wall_files_match_reference_kernels(tmp_path, refk, dx):
    """channel_from_reference_files on a reference-style run directory
    (points from x = -0.75 every dx) against the reference's own
    updateIBBOnly, updateWallD, iniLSMap and dXArr set-up on the same points:
    the same links, fractions, link fractions and wall distances bit for
    bit."""
    from oracle.orc import make_cfg
    nx, ny = 128, 40
    h = lambda x: 3.0 * 0.5 * (1 - np.cos(2 * np.pi * x / 64))  # noqa: E731
    _write_reference_walls(str(tmp_path), nx, ny, lambda x: 0.5 + h(x), lambda x: ny - 1.5 - h(x), dx=dx)
    ch = G.channel_from_reference_files(str(tmp_path), ibb_all=True)
    _, _, pts = G.read_reference_polyline(str(tmp_path))
    cfg = make_cfg(nx, ny, 1.0, 0.0, 0.1)
    idx, dist = refk.ibb_list_pts(cfg, ch.ntype, pts)
    u, first = np.unique(idx, return_index=True)
    assert np.array_equal(u, ch.ibb_idx) and np.array_equal(dist[first], ch.ibb_q)
    lsmap = G._ls_map(pts, nx)
    segs = np.loadtxt(str(tmp_path / "lsbl.txt"), ndmin=2).astype(np.int32)
    assert np.array_equal(lsmap, refk.ls_map(pts, segs, nx, nx).astype(np.int64))   # iniLSMap
    wd = refk.wall_distance_pts(cfg, ch.ntype, pts, lsmap)
    assert np.array_equal(wd, ch.wallD)
    dx, _ = refk.link_fractions(cfg, ch.ntype, pts, segs)   # bcFindNodes .. bcSetdXArr (host code)
    assert np.array_equal(dx, ch.dX)
