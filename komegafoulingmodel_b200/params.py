"""Run parameters from the reference's YAML parameter files.

The reference reads its parameters from a multi-document YAML file
(load/RunParam.yaml; clProblem::loadParams, clProblem.cpp:337-405, 460-480;
clVariablesLB::loadParams, clVariablesLB.cpp:550-610; kOmega::loadParams,
kOmega.cpp:350-380).  `run_params` flattens such a file and applies the same
derivations the reference applies, so a run described by a reference
parameter file gets the same lattice parameters here:

  * XsizeFull = nX rounded up to a multiple of 128 (BLOCKSIZE);
  * "Mu" or "Tau" (the relaxation RATE; tau = 1 / (3 Mu + 0.5) when only Mu
    is given, Mu = (1/Tau - 0.5) / 3 when only Tau is given, LB_TAU_NUMBER
    = 1.99 when neither is);
  * "Re" or "Fval" with Fval = Re * 3 Mu^2 / R^3 (R = "Pipe Radius"), and
    RE_NUMBER = 10800 when neither is given;
  * "Use Turb Model" (USE_TURBULENCE_MODEL = true), "Kappa Max Rel Tol",
    "Kappa Max Abs Tol", "Kappa Max Iterations" (KOMEGA_MAX_* defaults).

When both members of a pair are present the reference's getParameter(a, b)
prefers the first (returns 1); so does this loader.
"""
from __future__ import annotations

from dataclasses import dataclass

import yaml

LB_TAU_NUMBER = 1.99
RE_NUMBER = 10800.0
BLOCKSIZE = 128


@dataclass
class RunParams:
    nX: int
    nY: int
    XsizeFull: int
    pipe_radius: float
    tau: float          # relaxation rate
    mu: float
    re: float
    fval: float
    use_komega: bool
    rel_tol: float = 1.0e-4
    abs_tol: float = 1.0e-7
    max_iters: int = 1000
    wall_d_search_radius: int = 50

    def descriptor(self, storage: int = 0):
        """A kofm_desc filled from these parameters (needs libkofm.so)."""
        from .lattice import desc_default
        d = desc_default()
        d.nx, d.nx_full, d.ny = self.nX, self.XsizeFull, self.nY
        d.tau, d.fterm, d.mu = self.tau, self.fval, self.mu
        d.use_komega = 1 if self.use_komega else 0
        d.komega_rel_tol, d.komega_abs_tol = self.rel_tol, self.abs_tol
        d.komega_max_iters = self.max_iters
        d.storage = storage
        return d


def flatten(text: str) -> dict:
    """All key / value pairs of every document of a reference YAML file."""
    out: dict = {}
    for doc in yaml.safe_load_all(text):
        if isinstance(doc, dict):
            out.update(doc)
    return out


def run_params(text: str) -> RunParams:
    p = flatten(text)
    nx, ny = int(p["nX"]), int(p["nY"])
    xsf = -(-nx // BLOCKSIZE) * BLOCKSIZE
    R = float(p["Pipe Radius"])
    if "Mu" in p:
        mu = float(p["Mu"])
        tau = 1.0 / (mu * 3.0 + 0.5)
    elif "Tau" in p:
        tau = float(p["Tau"])
        mu = (1.0 / tau - 0.5) / 3.0
    else:
        tau = LB_TAU_NUMBER
        mu = (1.0 / tau - 0.5) / 3.0
    if "Re" in p:
        re = float(p["Re"])
        fval = re * 3.0 * mu * mu / R ** 3
    elif "Fval" in p:
        fval = float(p["Fval"])
        re = fval * R ** 3 / 3.0 / mu / mu
    else:
        re = RE_NUMBER
        fval = re * 3.0 * mu * mu / R ** 3
    return RunParams(
        nX=nx, nY=ny, XsizeFull=xsf, pipe_radius=R, tau=tau, mu=mu, re=re, fval=fval,
        use_komega=bool(p.get("Use Turb Model", True)),
        rel_tol=float(p.get("Kappa Max Rel Tol", 1.0e-4)),
        abs_tol=float(p.get("Kappa Max Abs Tol", 1.0e-7)),
        max_iters=int(p.get("Kappa Max Iterations", 1000)),
        wall_d_search_radius=int(p.get("Wall D Search Rad", 50)))


def load(path: str) -> RunParams:
    with open(path) as fh:
        return run_params(fh.read())
