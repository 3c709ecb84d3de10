"""Batched channels: several lattices advanced by one CUDA graph per two steps
(kofm_batch_*), and the seeded 48-channel sweep of uneven size and Re.

    python -m komegafoulingmodel_b200.batch [--channels 48] [--steps 20]

prints one JSON line with the aggregate throughput of the sweep advanced as a
batch (one graph launch per two steps, the lattices' kernels running
concurrently) and of the same channels stepped one launch sequence each.  The
batch's solver grid sizes come from `autotune`, which times a few batched
steps under each sizing policy and keeps the fastest.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time

import numpy as np

from . import _abi
from . import geometry as G
from . import workloads as W
from ._abi import check
from .lattice import Lattice


class Batch:
    """kofm_batch over existing Lattice objects (each already stepped once).
    tile_rows: block rows (4 lattice rows each) per tile of the persistent
    multi-lattice collide (0: the library's default, -1: one collide launch
    per lattice)."""

    def __init__(self, lattices, tile_rows: int = 0):
        self.lib = _abi.load()
        self.lattices = list(lattices)
        arr = (C.c_void_p * len(self.lattices))(*[L._ctx for L in self.lattices])
        out = C.c_void_p()
        check("kofm_batch_create_tiled",
              self.lib.kofm_batch_create_tiled(arr, len(self.lattices), int(tile_rows), C.byref(out)))
        self._b = out

    def step(self, nsteps: int = 2) -> None:
        check("kofm_batch_step", self.lib.kofm_batch_step(self._b, nsteps))

    def close(self) -> None:
        if self._b:
            self.lib.kofm_batch_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def sweep_channels(n: int = 48, seed: int = 0, u_mean: float = 0.05):
    """The batched-sweep channels: nx from {512, 1024, 2048, 4096}, ny from
    {64, 128, 256}, Re log-uniform in [500, 30000] on the opening, a
    sinusoidal wall of amplitude uniform in [0, 0.15 ny] and wavelength from
    {128, 256, 512}; laminar below Re = 2000, k-omega above (the rule used
    here).  Velocity scale u_mean = 0.05; nu = u_mean H / Re."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = int(rng.choice([512, 1024, 2048, 4096]))
        ny = int(rng.choice([64, 128, 256]))
        re = float(np.exp(rng.uniform(np.log(500.0), np.log(30000.0))))
        amp = float(rng.uniform(0.0, 0.15 * ny))
        lam = int(rng.choice([128, 256, 512]))
        # the host builds the flags and the start state; the device builds the
        # geometry the lattice uses (the same, and the wall distance of a
        # million-node channel in milliseconds instead of seconds)
        ch = G.wavy_channel(nx, ny, amp, lam, wall_distance=False)
        R = ch.pipe_radius
        H = 2.0 * R
        nu = u_mean * H / re
        komega = re >= 2000.0
        u_max = 1.5 * u_mean
        yb, yt = ch.y_bot[None, :], ch.y_top[None, :]
        y = np.arange(ny)[:, None]
        ux = np.clip(u_max * 4.0 * (y - yb) * (yt - y) / np.maximum(yt - yb, 1.0) ** 2, 0.0, None)
        f = G.equilibrium_state(ch, ux=ux)
        g = G.force_from_re(u_mean * R / nu, nu, R)
        w = W.Workload(f"sweep{i}_{nx}x{ny}_re{re:.0f}", ch, 1.0 / (3.0 * nu + 0.5), g, nu, komega, f,
                       device_geometry=True)
        if komega:
            k0 = 1.5 * (0.05 * u_max) ** 2
            o0 = np.sqrt(k0) / (0.09 ** 0.25 * 0.07 * H)
            w.k, w.omega, w.nut = G.komega_fields(ch, k0, o0)
            w.sxy = np.zeros(3 * ch.n)
        out.append(w)
    return out


def open_lattices(workloads, storage=_abi.STORE_FP16_NEQ, caps=None):
    lats = []
    for i, w in enumerate(workloads):
        d = W.descriptor(w, storage=storage)
        if caps is not None:
            d.solver_max_blocks = int(caps[i])
        L = Lattice(d)
        W.apply(L, w)
        L.step(1)
        lats.append(L)
    return lats


def solver_caps(workloads, policy, sms: int):
    """Per-lattice caps on the solver grid for one tuning policy:
    "auto" -- none (each solver may take two blocks per SM);
    "share" -- two blocks per SM split over the k-omega lattices in proportion
    to their node counts (at least 8 each), so concurrent solvers fit side by
    side; an integer -- that cap for every lattice."""
    if policy == "auto":
        return [0] * len(workloads)
    if policy == "share":
        tot = sum(w.nodes for w in workloads if w.komega) or 1
        return [max(8, int(2 * sms * w.nodes / tot)) if w.komega else 0 for w in workloads]
    return [int(policy)] * len(workloads)


def _time_batch(workloads, storage, caps, tile_rows, steps):
    """MLUPS of `steps` batched steps, or None when the batch refuses the
    lattices (a k-omega lattice whose first step halved dt: the library says
    which on stderr)."""
    nodes = sum(w.nodes for w in workloads)
    lats = open_lattices(workloads, storage, caps)
    try:
        with Batch(lats, tile_rows) as B:
            B.step(2)
            t0 = time.perf_counter()
            B.step(steps)
            return nodes * steps / (time.perf_counter() - t0) / 1e6
    except _abi.KofmError as e:
        states = [(i, L.stats().steps_per_lb) for i, L in enumerate(lats) if L.stats().steps_per_lb != 1]
        print(f"batch refused ({e}); lattices with steps_per_lb != 1: {states}", file=sys.stderr, flush=True)
        return None
    finally:
        for L in lats:
            L.close()


def autotune(workloads, tile_rows=(1, 2, 4, 8), policies=("auto", "share", 148, 74), steps: int = 4,
             storage=_abi.STORE_FP16_NEQ):
    """Times `steps` batched steps per tile shape of the multi-lattice collide
    (block rows per tile, with the default solver grids), then per solver grid
    policy with the best tile shape; returns ((tile_rows, policy), {setting: MLUPS})."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    res = {}
    for r in tile_rows:
        res[f"tile_rows={r}"] = _time_batch(workloads, storage, None, r, steps)
    best_r = max(tile_rows, key=lambda r: res[f"tile_rows={r}"] or 0.0)
    for pol in policies:
        key = f"tile_rows={best_r},solver={pol}"
        if pol == "auto":
            res[key] = res[f"tile_rows={best_r}"]
            continue
        res[key] = _time_batch(workloads, storage, solver_caps(workloads, pol, sms), best_r, steps)
    best_p = max(policies, key=lambda p: res[f"tile_rows={best_r},solver={p}"] or 0.0)
    return (best_r, best_p), res


def measure(channels: int = 48, steps: int = 20, seed: int = 0, storage=_abi.STORE_FP16_NEQ,
            tune: bool = True):
    import torch
    ws = sweep_channels(channels, seed)
    nodes = sum(w.nodes for w in ws)
    (rows, pol), table = autotune(ws, storage=storage) if tune else ((0, "auto"), {})
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    lats = open_lattices(ws, storage)
    try:
        # each lattice stepped on its own (its own stream; the k-omega update
        # as the device-driven graph, so the lattices' steps overlap)
        for L in lats:
            L.step(2)
        for L in lats:
            L.sync()
        t0 = time.perf_counter()
        for _ in range(steps):
            for L in lats:
                L.step(1)
        for L in lats:
            L.sync()
        t_seq = time.perf_counter() - t0
    finally:
        for L in lats:
            L.close()
    # the batch graph with one collide launch per lattice (its branch), and
    # with the tuned multi-lattice collide and solver grids
    per_lattice = _time_batch(ws, storage, None, -1, steps)
    tuned = _time_batch(ws, storage, solver_caps(ws, pol, sms), rows, steps)
    return {"channels": channels, "komega_channels": sum(w.komega for w in ws), "nodes": nodes,
            "steps": steps, "unit": "MLUPS",
            "batched_mlups": tuned,
            "batched_per_lattice_collide_mlups": per_lattice,
            "one_by_one_mlups": nodes * steps / t_seq / 1e6,
            "storage": {0: "fp32", 1: "fp16", 2: "bf16", 3: "fp16neq"}[storage],
            "tile_rows": rows, "solver_grid_policy": str(pol), "autotune_mlups": table,
            "timing": "host wall clock around the steps, synchronised at both ends"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--channels", type=int, default=48)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-tune", action="store_true")
    args = ap.parse_args()
    print(json.dumps(measure(args.channels, args.steps, args.seed, tune=not args.no_tune)), flush=True)


if __name__ == "__main__":
    main()
