"""Steps a seeded workload through the C ABI and prints each step's solver
statistics: the program the ncu launch lists and kernel captures of the
k-omega step run.

    python -m komegafoulingmodel_b200.steprun --workload komega_straight_16384x1024 \\
        --steps 4 --form 3

--form is kofm_desc.komega_classic: 0 the device-driven update graph
(default), 1 one Krylov vector per sweep, 2 the one-launch solve, 3 the
phase kernels with the host enqueueing each round (the kernels of form 0;
ncu lists kernels that conditional graph nodes launch only in this form).
"""
from __future__ import annotations

import argparse

from . import workloads as W
from .lattice import Lattice


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", default="komega_straight_16384x1024")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--form", type=int, default=0, choices=(0, 1, 2, 3))
    args = ap.parse_args(argv)
    w = W.by_name(args.workload)
    d = W.descriptor(w)
    d.komega_classic = args.form
    with Lattice(d) as L:
        W.apply(L, w)
        print("step omega_powers k_powers solver_launches solver_rounds", flush=True)
        for step in range(args.steps):
            L.step(1)
            st = L.stats()
            print(step, st.omega_powers, st.k_powers, st.solver_launches, st.solver_rounds, flush=True)


if __name__ == "__main__":
    main()
