"""Run parameters from a reference-style multi-document YAML file."""
import pytest

from komegafoulingmodel_b200 import params

DOC = """\
--- # System
ParamsName: 1
nX: !!int 1000
nY: !!int 130
Pipe Radius: !!float 6.4e+001
--- # Fluid
ParamsName: 2
Tau: !!float 1.9
Re: !!float 5.0e+003
--- # k-omega
ParamsName: 4
Use Turb Model: True
Kappa Max Rel Tol: 1.0e-5
"""


def test_tau_and_re_derivations():
    p = params.run_params(DOC)
    assert (p.nX, p.nY, p.XsizeFull) == (1000, 130, 1024)
    assert p.tau == 1.9 and p.mu == pytest.approx((1 / 1.9 - 0.5) / 3)
    assert p.fval == pytest.approx(5000 * 3 * p.mu ** 2 / 64.0 ** 3)
    assert p.use_komega and p.rel_tol == 1e-5 and p.abs_tol == 1e-7 and p.max_iters == 1000


def test_mu_and_fval_alternatives():
    doc = DOC.replace("Tau: !!float 1.9", "Mu: !!float 0.01").replace("Re: !!float 5.0e+003",
                                                                   "Fval: !!float 1.0e-6")
    p = params.run_params(doc)
    assert p.tau == pytest.approx(1 / (0.03 + 0.5))
    assert p.re == pytest.approx(1e-6 * 64.0 ** 3 / 3 / 0.01 ** 2)


def test_defaults_when_absent():
    doc = "nX: 256\nnY: 64\nPipe Radius: 31.0\n"
    p = params.run_params(doc)
    assert p.tau == params.LB_TAU_NUMBER and p.re == params.RE_NUMBER
    assert p.XsizeFull == 256
