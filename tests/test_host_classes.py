"""The C++ host classes (clVariablesLB / kOmega / clProblem step loop over the
C ABI) driven by host/kofm_host_run, against the Python path through the same
ABI.  Restart files use the reference's raw FP64 layout (lbf.bin = 9 planes of
XsizeFull * nY, lbkappa.bin, lbomega.bin)."""
import json
import os
import subprocess

import numpy as np
import pytest

from komegafoulingmodel_b200 import build
from komegafoulingmodel_b200 import geometry as G
from tests.test_komega_gpu import channel_case, make_lattice

RUN = build.HOST_RUN


def write_case(d, ch, f, k=None, o=None, rate=1.25, g=0.0, nu=0.1, komega=False, thermal=False):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params.txt"), "w") as fh:
        fh.write(f"nX {ch.nx}\nXsizeFull {ch.nx_full}\nnY {ch.ny}\ntau {rate!r}\n"
                 f"Fval {g!r}\nMuVal {nu!r}\nkOmega {int(komega)}\nthermal {int(thermal)}\n")
    ch.ntype.astype(np.int16).tofile(os.path.join(d, "ntype.bin"))
    np.asarray(f, dtype=np.float64).tofile(os.path.join(d, "lbf.bin"))
    if komega or thermal:
        np.asarray(ch.dX, dtype=np.float64).tofile(os.path.join(d, "dX.bin"))
    if komega:
        np.asarray(ch.wallD, dtype=np.float64).tofile(os.path.join(d, "wallD.bin"))
        np.asarray(k, dtype=np.float64).tofile(os.path.join(d, "lbkappa.bin"))
        np.asarray(o, dtype=np.float64).tofile(os.path.join(d, "lbomega.bin"))
    if ch.ibb_idx is not None and len(ch.ibb_idx):
        np.asarray(ch.ibb_idx, dtype=np.int32).tofile(os.path.join(d, "ibbArr.bin"))
        np.asarray(ch.ibb_q, dtype=np.float64).tofile(os.path.join(d, "ibbDistArr.bin"))


def test_driver_builds_and_fails_loudly_without_a_device(tmp_path):
    """On a machine without a GPU the step loop stops with the library's
    NO_DEVICE status instead of falling back to anything."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    build.build()
    ch = G.straight_channel(64, 8)
    write_case(str(tmp_path), ch, G.equilibrium_state(ch))
    r = subprocess.run([RUN, str(tmp_path), "1"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "device" in r.stderr.lower()


def test_restart_file_layout(tmp_path):
    """lbf.bin holds the 9 population planes one after another."""
    ch = G.straight_channel(64, 8)
    f = G.equilibrium_state(ch, ux=0.01)
    write_case(str(tmp_path), ch, f)
    raw = np.fromfile(os.path.join(str(tmp_path), "lbf.bin"), dtype=np.float64)
    assert raw.size == 9 * ch.nx_full * ch.ny
    assert np.array_equal(raw.reshape(9, -1), f.reshape(9, -1))


@pytest.mark.gpu
def test_host_step_loop_matches_python_path(tmp_path, kofm_lib):
    from komegafoulingmodel_b200 import _abi
    ch, f, k, o, nut, rate, g, nu = channel_case(nx=128, ny=34)
    d = str(tmp_path)
    write_case(d, ch, f, k, o, rate, g, nu, komega=True)
    r = subprocess.run([RUN, d, "25"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    with make_lattice(ch, rate, g, nu) as L:
        L.set_state(f, k, o, None, np.zeros(3 * ch.n))
        L.step(25)
        f2, k2, o2, _, _ = L.get_state()
        sum_rho = L.reduce(_abi.FIELD_RHO)
        sum_k = L.reduce(_abi.FIELD_K)
    out = os.path.join(d, "out")
    fo = np.fromfile(os.path.join(out, "lbf.bin"))
    ko = np.fromfile(os.path.join(out, "lbkappa.bin"))
    oo = np.fromfile(os.path.join(out, "lbomega.bin"))
    # same kernels, same inputs, same order: identical results
    assert np.array_equal(fo, f2.ravel())
    assert np.array_equal(ko, k2) and np.array_equal(oo, o2)
    assert res["sum_rho"] == sum_rho and res["sum_k"] == sum_k
    # a restart from the written files continues the run
    write_case(os.path.join(d, "again"), ch, fo, ko, oo, rate, g, nu, komega=True)
    r2 = subprocess.run([RUN, os.path.join(d, "again"), "1"], capture_output=True, text=True,
                        timeout=300)
    assert r2.returncode == 0, r2.stderr


@pytest.mark.gpu
def test_host_thermal_step_loop_matches_python_path(tmp_path, kofm_lib):
    """clProblem::step with a clVariablesFD attached (collide, kOmega::Solve,
    clVariablesFD::Solve) against kofm_step with use_thermal: identical
    temperature, and temp.bin restarts."""
    from komegafoulingmodel_b200 import Lattice, _abi, desc_default
    from tests.test_thermal import _wavy_case
    ch, f, k, o, nut, rate, g, nu = _wavy_case()
    d = str(tmp_path)
    write_case(d, ch, f, k, o, rate, g, nu, komega=True, thermal=True)
    r = subprocess.run([RUN, d, "8"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    desc = desc_default()
    desc.nx, desc.nx_full, desc.ny = ch.nx, ch.nx_full, ch.ny
    desc.tau, desc.fterm, desc.mu = rate, g, nu
    desc.use_komega = desc.use_thermal = 1
    with Lattice(desc) as L:
        L.set_geometry(ch.ntype, ch.wallD, ch.dX, ch.ibb_idx, ch.ibb_q)
        L.set_state(f, k, o, None, np.zeros(3 * ch.n))
        L.set_temperature(G.temperature_field(ch))
        L.step(8)
        T = L.get_temperature()
        tsum = L.reduce(_abi.FIELD_TEMP)
    To = np.fromfile(os.path.join(d, "out", "temp.bin"))
    assert np.array_equal(To, T)
    assert res["sum_temp"] == tsum


@pytest.mark.gpu
def test_host_walls_and_update_match_python_path(tmp_path, kofm_lib):
    """clVariablesLB with wall heights (geometry built on the device at ini)
    and clVariablesLB::update after the walls moved, driven by kofm_host_run,
    against Lattice.set_walls on the same live context path."""
    from komegafoulingmodel_b200 import Lattice, _abi, desc_default
    from tests.cases import fp32_state
    nx, ny = 128, 34
    x = np.arange(nx)
    h1 = 0.5 + 2.0 * (1 - np.cos(2 * np.pi * x / 64)) / 2
    h2 = 0.5 + 3.5 * (1 - np.cos(2 * np.pi * x / 64)) / 2
    ch = G.channel_from_walls(nx, ny, h1, ny - 1 - h1)
    (f,) = fp32_state(G.equilibrium_state(ch, ux=0.01))
    d = str(tmp_path)
    write_case(d, ch, f, rate=1.25, g=1e-6, nu=0.1)
    with open(os.path.join(d, "params.txt"), "a") as fh:
        fh.write("moveAt 10\n")
    np.concatenate([h1, ny - 1 - h1]).tofile(os.path.join(d, "walls.bin"))
    np.concatenate([h2, ny - 1 - h2, h1, ny - 1 - h1]).tofile(os.path.join(d, "walls_moved.bin"))
    r = subprocess.run([RUN, d, "20"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    dd = desc_default()
    dd.nx, dd.nx_full, dd.ny, dd.tau, dd.fterm, dd.mu = nx, nx, ny, 1.25, 1e-6, 0.1
    with Lattice(dd) as L:
        L.set_walls(h1, ny - 1 - h1)
        L.set_state(f)
        L.step(10)
        L.set_walls(h2, ny - 1 - h2, h1, ny - 1 - h1)
        L.step(10)
        f2 = L.get_state()[0]
        sum_rho = L.reduce(_abi.FIELD_RHO)
    fo = np.fromfile(os.path.join(d, "out", "lbf.bin"))
    assert np.array_equal(fo, f2.ravel())
    assert res["sum_rho"] == sum_rho
