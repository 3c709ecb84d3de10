"""The device geometry builder (kofm_set_walls) against the host builder
(geometry.channel_from_walls): the same nType flags, link fractions and
interpolated links bit for bit, the wall distance to FP32 rounding, and the
same time steps whichever built the geometry -- also when the walls move on a
live context."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, desc_default
from komegafoulingmodel_b200 import adjoint as A
from komegafoulingmodel_b200 import geometry as G
from tests.cases import fp32_state, komega_state, perturbed_state


def _desc(nx, ny, komega=False, thermal=False):
    d = desc_default()
    d.nx, d.nx_full, d.ny = nx, nx, ny
    d.tau, d.fterm, d.mu = 1.25, 1e-6, 0.1
    d.use_komega = 1 if komega else 0
    d.use_thermal = 1 if thermal else 0
    return d


def _walls(name):
    """(nx, ny, y_bot, y_top, y_bot0, y_top0, ibb_all) of the test geometries."""
    if name == "straight":
        nx, ny = 128, 20
        return nx, ny, np.full(nx, 0.5), np.full(nx, ny - 1.5), None, None, False
    if name in ("wavy", "wavy_all"):
        nx, ny = 256, 66
        h = 8.0 * 0.5 * (1 - np.cos(2 * np.pi * np.arange(nx) / 128))
        return nx, ny, 0.5 + h, ny - 1.5 - h, None, None, name == "wavy_all"
    if name == "random":   # the 64-mode random wall of the adjoint case
        nx, ny = 1024, 256
        yb, yt = A.walls(A.coefficients(), nx, ny)
        return nx, ny, yb, yt, None, None, True
    if name == "fouled":   # deposit inside straight unfouled walls
        nx, ny = 160, 40
        dep = 3.0 + 1.5 * (1.0 - np.cos(2 * np.pi * np.arange(nx) / 80.0))
        return nx, ny, 0.5 + dep, ny - 1.5 - dep, np.full(nx, 0.5), np.full(nx, ny - 1.5), False
    if name == "near":     # walls 5e-4 below / above a row: fractions under min_dx
        nx, ny = 64, 20
        return nx, ny, np.full(nx, 0.9995), np.full(nx, ny - 1.9995), None, None, False
    if name == "c2":
        nx, ny = 2048, 256
        h = 32.0 * 0.5 * (1 - np.cos(2 * np.pi * np.arange(nx) / 512))
        return nx, ny, 0.5 + h, ny - 1.5 - h, None, None, False
    raise KeyError(name)


@pytest.mark.gpu
@pytest.mark.parametrize("name,seam", [("straight", False), ("wavy", False), ("wavy", True),
                                       ("wavy_all", False), ("random", False), ("random", True),
                                       ("fouled", False), ("near", False), ("c2", False)])
def test_device_builder_matches_host_builder(kofm_lib, name, seam):
    nx, ny, yb, yt, yb0, yt0, ibb_all = _walls(name)
    thermal = yb0 is not None
    ch = G.channel_from_walls(nx, ny, yb, yt, y_bot0=yb0, y_top0=yt0, ibb_all=ibb_all, seam_ibb=seam)
    with Lattice(_desc(nx, ny, komega=True, thermal=thermal)) as L:
        L.set_walls(yb, yt, yb0, yt0, ibb_all=ibb_all, seam_ibb=seam)
        geo = L.get_geometry()
    assert np.array_equal(geo["ntype"], ch.ntype)
    assert np.array_equal(geo["ibb_idx"], ch.ibb_idx)
    assert np.array_equal(geo["ibb_q"], ch.ibb_q)
    assert np.array_equal(geo["dX"], ch.dX)
    if thermal:
        assert np.array_equal(geo["dX0"], ch.dX0)
    # the device stores the wall distance in FP32; it searches every segment,
    # the host the three around the nearest of its samples
    fl = ch.fluid_mask().ravel()
    host = ch.wallD.astype(np.float32).astype(np.float64)
    err = np.abs(geo["wallD"] - host)[fl] / host[fl]
    print(name, len(ch.ibb_idx), "wallD max rel", err.max(), "differing", int(np.sum(err > 0)))
    assert err.max() <= 1e-6
    assert np.all(geo["wallD"][~fl] == 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("komega", [False, True])
def test_steps_identical_with_either_builder(kofm_lib, komega):
    """The wavy channel stepped from the same state on a geometry from the
    host builder and one from the device builder: identical fields."""
    nx, ny, yb, yt, _, _, _ = _walls("wavy")
    ch = G.channel_from_walls(nx, ny, yb, yt)
    f = perturbed_state(ch, seed=3, u_mean=0.02)
    if komega:
        k, o, nut, s = komega_state(ch)
        f, k, o, nut = fp32_state(f, k, o, nut)
    else:
        (f,) = fp32_state(f)
    out = []
    for device in (False, True):
        with Lattice(_desc(nx, ny, komega=komega)) as L:
            if device:
                L.set_walls(yb, yt)
            else:
                L.set_geometry(ch.ntype, ch.wallD if komega else None, ch.dX if komega else None,
                               ch.ibb_idx, ch.ibb_q)
            L.set_state(f, k, o, nut, s) if komega else L.set_state(f)
            L.step(20)
            rho, ux, uy = L.get_macro()
            st = L.get_state()
            out.append((rho, ux, uy, st[1] if komega else None))
    for a, b in zip(out[0], out[1]):
        if a is None:
            continue
        if komega:   # wall distances may differ in the last FP32 bit
            assert np.allclose(a, b, rtol=1e-6, atol=1e-12)
        else:
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_walls_moving_on_a_live_context(kofm_lib):
    """A deposit grows while the lattice runs: kofm_set_walls on the live
    context gives the same steps as kofm_set_geometry with the host builder's
    arrays for the grown walls."""
    nx, ny = 256, 48
    x = np.arange(nx)
    yb0, yt0 = np.full(nx, 0.5), np.full(nx, ny - 1.5)
    grow = lambda a: 0.5 + a * (1 - np.cos(2 * np.pi * x / 128)) / 2  # noqa: E731
    ch0 = G.channel_from_walls(nx, ny, yb0, yt0)
    (f,) = fp32_state(perturbed_state(ch0, seed=7, u_mean=0.02))
    runs = []
    for device in (False, True):
        with Lattice(_desc(nx, ny)) as L:
            L.set_walls(yb0, yt0)
            L.set_state(f)
            L.step(10)
            for a in (2.0, 3.7, 5.2):
                yb, yt = grow(a), ny - 1 - grow(a)
                if device:
                    L.set_walls(yb, yt, yb0, yt0)
                else:
                    ch = G.channel_from_walls(nx, ny, yb, yt, y_bot0=yb0, y_top0=yt0)
                    L.set_geometry(ch.ntype, None, None, ch.ibb_idx, ch.ibb_q)
                L.step(10)
            runs.append(L.get_macro())
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_workload_with_device_geometry(kofm_lib):
    """A workload whose lattice geometry comes from kofm_set_walls (as the
    batched sweep's) steps exactly as the same workload with the host
    builder's arrays."""
    from komegafoulingmodel_b200 import workloads as W
    nx, ny, yb, yt, _, _, _ = _walls("wavy")
    full = G.channel_from_walls(nx, ny, yb, yt)
    bare = G.channel_from_walls(nx, ny, yb, yt, wall_distance=False)
    nu, u = 5e-4, 0.05
    f = G.equilibrium_state(full, ux=u)
    k, o, nut = G.komega_fields(full, 1.5 * (0.05 * u) ** 2, 0.003)
    out = []
    for ch, dev in ((full, False), (bare, True)):
        w = W.Workload("wavy", ch, 1.0 / (3 * nu + 0.5), 1e-7, nu, True, f, k, o, nut,
                       np.zeros(3 * ch.n), device_geometry=dev)
        with Lattice(W.descriptor(w)) as L:
            W.apply(L, w)
            L.step(10)
            out.append(L.get_state())
    for a, b in zip(*out):
        if a is not None:
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_komega_walls_moving_zero_the_new_solid_nodes(kofm_lib):
    """k-omega channel, deposit grown on the live context: kofm_set_walls sets
    k, omega, nu_t, the strain rates and the moments of the nodes turned solid
    to 0 (updateNType) and leaves them unchanged everywhere else."""
    nx, ny = 256, 48
    x = np.arange(nx)
    yb0, yt0 = np.full(nx, 0.5), np.full(nx, ny - 1.5)
    h = 0.5 + 3.7 * (1 - np.cos(2 * np.pi * x / 128)) / 2
    ch0 = G.channel_from_walls(nx, ny, yb0, yt0)
    ch1 = G.channel_from_walls(nx, ny, h, ny - 1 - h, y_bot0=yb0, y_top0=yt0)
    f = perturbed_state(ch0, seed=8, u_mean=0.02)
    k, o, nut, s = komega_state(ch0)
    f, k, o, nut = fp32_state(f, k, o, nut)
    with Lattice(_desc(nx, ny, komega=True)) as L:
        L.set_walls(yb0, yt0)
        L.set_state(f, k, o, nut, s)
        L.step(5)
        before = L.get_state()[1:]
        mbefore = L.get_macro()
        L.set_walls(h, ny - 1 - h, yb0, yt0)
        after = L.get_state()[1:]
        mafter = L.get_macro()
    gone = ch0.fluid_mask().ravel() & ~ch1.fluid_mask().ravel()
    assert gone.sum() > 0
    for b, a in zip(before + tuple(mbefore), after + tuple(mafter)):
        b, a = np.asarray(b).reshape(-1, ch0.n), np.asarray(a).reshape(-1, ch0.n)
        assert np.all(a[:, gone] == 0.0)
        assert np.array_equal(a[:, ~gone], b[:, ~gone])
