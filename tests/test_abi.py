"""The C-ABI library loads and exports every entry point of include/kofm.h.
Host-only calls (version, defaults, error strings, descriptor validation)
run on CPU; nothing here launches device code."""
import ctypes as C
import os
import re

import pytest

from komegafoulingmodel_b200 import _abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "kofm.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\*\s]+?\b(kofm_\w+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    for s in ("kofm_create", "kofm_set_geometry", "kofm_set_state", "kofm_get_state",
              "kofm_lb_step", "kofm_komega_assemble", "kofm_komega_solve", "kofm_step",
              "kofm_reduce", "kofm_sync", "kofm_destroy"):
        assert s in syms


def test_library_exports_every_declared_symbol(kofm_lib):
    missing = [s for s in declared_symbols() if not hasattr(kofm_lib, s)]
    assert not missing, missing
    # and the Python bindings declare exactly the header's set
    assert sorted(_abi.SIGNATURES) == declared_symbols()


def test_host_only_calls(kofm_lib):
    assert kofm_lib.kofm_abi_version() == 3
    d = _abi.KofmDesc()
    assert kofm_lib.kofm_desc_default(C.byref(d)) == 0
    assert (d.krylov_dim, d.komega_max_iters) == (10, 1000)
    # thermal defaults of ConstDef.h (THERMAL_MAX_*, PR_NUMBER, PR_TURB_NUMBER, TFD_X_IN)
    assert (d.use_thermal, d.thermal_every, d.thermal_max_iters) == (0, 1, 1000)
    assert (d.pr_number, d.pr_turb_number, d.t_in, d.thermal_dt) == (0.708, 0.9, 2.0, 1.0)
    assert abs(d.thermal_rel_tol - 1e-4) < 1e-18 and abs(d.thermal_abs_tol - 1e-7) < 1e-20
    # the Python mirror of the structs has the C sizes
    assert C.sizeof(_abi.KofmDesc) == 168 and C.sizeof(_abi.KofmStats) == 176
    assert abs(d.komega_rel_tol - 1e-4) < 1e-18 and abs(d.komega_abs_tol - 1e-7) < 1e-20
    assert d.max_turb_visc == 10.0
    assert kofm_lib.kofm_error_string(-204) == b"bounded device wait expired"
    assert kofm_lib.kofm_desc_default(None) == -200


def test_create_rejects_bad_descriptors_before_touching_a_device(kofm_lib):
    d = _abi.KofmDesc()
    kofm_lib.kofm_desc_default(C.byref(d))
    ctx = C.c_void_p()
    bad = []
    for field, val in (("nx", 2), ("ny", 2), ("tau", 2.5), ("krylov_dim", 40),
                       ("storage", 7), ("komega_max_iters", 0)):
        dd = _abi.KofmDesc.from_buffer_copy(d)
        setattr(dd, field, val)
        bad.append(kofm_lib.kofm_create(C.byref(dd), C.byref(ctx)))
    assert all(s == -110 for s in bad), bad
    assert kofm_lib.kofm_create(None, C.byref(ctx)) == -200


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) != "" and
                    os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_create_without_gpu_reports_no_device(kofm_lib):
    d = _abi.KofmDesc()
    kofm_lib.kofm_desc_default(C.byref(d))
    ctx = C.c_void_p()
    assert kofm_lib.kofm_create(C.byref(d), C.byref(ctx)) == -201
