import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and libkofm.so")


@pytest.fixture(scope="session")
def oracle():
    """The FP64 CPU restatement (built on demand; test infrastructure only)."""
    from oracle.orc import LIB_ORACLE, Oracle
    # make rebuilds it when a source is newer than the library
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=False)
    if r.returncode != 0 and not os.path.exists(LIB_ORACLE):
        raise RuntimeError("oracle/liboracle.so could not be built")
    return Oracle(LIB_ORACLE)


@pytest.fixture(scope="session")
def refk():
    """The reference's own kernels compiled for the CPU (oracle/_ref)."""
    from oracle.orc import LIB_REF, RefKernels
    if not os.path.exists(LIB_REF):
        from __graft_entry__ import REFERENCE_MOUNT
        ref = os.environ.get("KOFM_REFERENCE") or REFERENCE_MOUNT
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref",
                        "REF=" + (ref if os.path.isdir(ref) else "")], check=False)
    if not os.path.exists(LIB_REF):
        pytest.skip("oracle/_ref not built (reference tree absent); golden fixtures cover the pin")
    return RefKernels()


@pytest.fixture(scope="session")
def kofm_lib():
    from komegafoulingmodel_b200 import build
    build.build()
    from komegafoulingmodel_b200 import _abi
    return _abi.load()
