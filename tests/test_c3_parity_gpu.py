"""Parity at the full size of the precision-study channel: the straight k-omega
channel of 16384 x 1024 nodes (16.7M) that the throughput benchmark runs,
stepped on the GPU and by the FP64 oracle (the reference's step loop,
Solve_no_TR, LBLS.cpp:185-205: collide + push, then kOmega::Solve with the
restarted simpler GMRES at the reference's tolerances) from the same
FP32-rounded state.  A few steps: the oracle takes seconds per step at this
size on the host cores."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice
from komegafoulingmodel_b200 import workloads as W
from oracle.orc import OracleSim, make_cfg
from tests.cases import fp32_state, rel_l2

pytestmark = pytest.mark.gpu

STEPS = 3


def test_full_size_channel_matches_oracle(kofm_lib, oracle):
    """rho, u, k and omega within rel-L2 1e-5 of the oracle after each of 3
    steps at 16384 x 1024, with the same number of GMRES restarts per step for
    both systems."""
    w = W.komega_channel(16384, 1024)
    ch = w.channel
    f, k, o, nut = fp32_state(w.f, w.k, w.omega, w.nut)
    cfg = make_cfg(ch.nx, ch.ny, w.tau, w.fterm, w.mu)
    sim = OracleSim(oracle, cfg, ch.ntype, ch.dX, ch.wallD, f, k, o, nut, komega=True)
    fl = ch.fluid_mask().ravel()
    with Lattice(W.descriptor(w)) as L:
        L.set_geometry(ch.ntype, ch.wallD, ch.dX)
        L.set_state(f, k, o, nut, np.zeros(3 * ch.n))
        for step in range(STEPS):
            L.step(1)
            sim.step(1)
            st = L.stats()
            assert (st.omega_restarts, st.k_restarts) == (
                sim.kst.last_o.restarts, sim.kst.last_k.restarts), step
            rho, ux, uy = L.get_macro()
            _, k2, o2, _, _ = L.get_state()
            errs = dict(rho=rel_l2(rho, sim.rho, fl), ux=rel_l2(ux, sim.ux, fl),
                        k=rel_l2(k2, sim.K, fl), omega=rel_l2(o2, sim.O, fl))
            print(step + 1, errs, (st.omega_restarts, st.k_restarts), (st.omega_iters, st.k_iters))
            for key, e in errs.items():
                assert e < 1e-5, (step, errs)
