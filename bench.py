"""Benchmark of the D2Q9 + k-omega time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--storage fp32|fp16|bf16]

One "step" is one full time step of the reference's Solve_no_TR path over the
whole lattice: collide-stream with the k-omega eddy viscosity, the fused k/omega
assembly and the implicit GMRES solves of omega and k.  Default workload:
komega_straight_16384x1024 (16.7M nodes, synthetic seeded channel).  The
populations (1.2 GB) and solver vectors exceed the 126 MB L2, so no flush is
needed between steps.

With N > 1 (launched by torch.distributed.run) every rank advances its own
replica of the channel; the path has no exchange step ("replicas only"), value
is the lattice updates of all ranks over the slowest rank's time.

--impl reference times the reference's own CPU code of the path on the host
cores: its OpenCL kernel sources compiled as C++ (oracle/_ref) for the collide
and k-omega assembly, with the oracle's C restatement of its GMRES solver, all
OpenMP-parallel.  Only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "D2Q9+k-omega MLUPS & % HBM roofline; FP16-storage vs FP32 at <=1e-3 rel-L2"
UNIT = "MLUPS"
FALLBACK_HBM_GBS = 6650.0


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.proc, self.lines = gpu, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [l.split(", ") for l in self.lines if l]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
STORAGE_NAMES = {"fp32": "fp32 f-w deviation", "fp16": "fp16 f-w deviation",
                 "bf16": "bf16 f-w deviation", "fp16neq": "fp16 f-feq (FP32 reference moments)",
                 "fp64": "fp64 f-w deviation, fp64 fields",
                 "fp16neq32": "fp16 f-feq (FP32 reference moments), fp32 collide",
                 "fp16row": "fp16 f-feq (one reference per row), fp32 collide"}


def workload_config(w, args, world: int) -> dict:
    """The `config` object of both arms' JSON lines."""
    # resident bytes per node: populations (two buffers), node fields and, for
    # k-omega, both systems' solver vectors (coefficients, b', r, x twice, basis)
    per_node = 2 * 9 * STORE_BYTES.get(args.storage, 4) + 60 + (2 * 8 * (4 + 5 + 10) if w.komega else 0)
    big = per_node * w.nodes > 126e6
    cfg = {"workload": w.name, "nx": w.channel.nx, "ny": w.channel.ny, "nodes": w.nodes,
           "storage": STORAGE_NAMES[args.storage], "krylov_dim": 10, "rel_tol": 1.0e-4,
           "abs_tol": 1.0e-7, "parallelism": f"replicas x{world}",
           "l2": ("inputs larger than L2 (populations and solver vectors), no flush" if big else
                  "working set within the 126 MB L2, no flush: steps of an L2-resident lattice")}
    if getattr(args, "thermal", False):
        cfg["thermal"] = "implicit FD temperature update every step (BiCGStab to 1e-4)"
    return cfg


def thermal_bytes_per_node(checks: int) -> float:
    """Algorithmic bytes per node of one thermal update (one solve ending
    after `checks` residual checks): the assembly (ntype, link-fraction index,
    u, v, nu_t, T in; 4 coefficients, b and the saved T out: 74), pass R (b,
    x, coefficients, ntype in; r, r0 out: 66), per iteration pass B (r, p, v,
    coefficients, ntype, r0 in; p, v out: 82; 50 in the first, where p = r0),
    pass C (r, v in; s out: 24) and pass D (s, coefficients, ntype, x, p, r0
    in; x, r out: 82); a solve that stops at the check after pass C ends with
    x += alpha p, r = s (40)."""
    n_c = (checks + 1) // 2
    n_d = checks // 2
    b = 74 + 66 + 50 + (n_c - 1) * 82 + n_c * 24 + n_d * 82
    if checks % 2 == 1:
        b += 40
    return float(b)


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The slowest rank's time: all-reduce MAX over the process group (NCCL
    on the GPU box; gloo with a CPU tensor in the tests)."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(nodes: int, steps: int, world: int, ms: float) -> float:
    """Whole-job MLUPS of N independent replicas: every rank's node updates
    over the slowest rank's time."""
    return nodes * steps * world / (ms * 1e-3) / 1e6


# DRAM traffic over algorithmic bytes of one solver launch, from an ncu capture
# of the 8192x512 case (profiles/<kernel>_komega_straight_8192x512.md); the
# bench's traffic figure is this ratio times its average launch's algorithmic
# bytes (traffic grows with the nodes and the sweeps of a launch).
SOLVER_TRAFFIC_RATIO = {
    "gmres_kernel": 4.7967e9 / (1076 * 4194304),   # one vector per sweep
    "sstep_kernel": None,                          # one sweep per cycle's powers
    "sstep_phases": None,                          # the same, one launch per sweep
}

STORE_BYTES = {"fp32": 4, "fp16": 2, "bf16": 2, "fp16neq": 2, "fp16neq32": 2, "fp16row": 2, "fp64": 8}
# laminar collide (no macro fields saved by the plain step): f read + write, flags
LB_BYTES_LAMINAR = {"fp32": 74, "fp16": 38, "bf16": 38, "fp16neq": 62, "fp16neq32": 62, "fp16row": 38,
                    "fp64": 146}
LB_BYTES = {"fp32": 126, "fp16": 90, "bf16": 90,   # k-omega collide, per node
            "fp16neq": 114, "fp16neq32": 114,  # + reference moments read and written
            "fp16row": 90,                      # row references: a few KB, cached
            "fp64": 250}                      # FP64 populations and fields
ASM_BYTES = {"fp64": 162}                           # fused assembly, per node (FP64 fields)
ASM_BYTES_FP32 = 122                                # ... FP32 fields


def run_ours(args, rank, world, local_rank):
    import ctypes as C

    import numpy as np
    import torch

    from komegafoulingmodel_b200 import _abi, build
    from komegafoulingmodel_b200 import workloads as W
    from komegafoulingmodel_b200.lattice import Lattice

    build.build()
    lib = _abi.load()
    torch.cuda.set_device(local_rank)
    storage = {"fp32": _abi.STORE_FP32, "fp16": _abi.STORE_FP16_DEV, "bf16": _abi.STORE_BF16_DEV,
               "fp16neq": _abi.STORE_FP16_NEQ, "fp64": _abi.STORE_FP64,
               "fp16neq32": _abi.STORE_FP16_NEQ32, "fp16row": _abi.STORE_FP16_ROW}[args.storage]
    asm_bytes = ASM_BYTES.get(args.storage, ASM_BYTES_FP32)
    w = W.by_name(args.workload)
    d = W.descriptor(w, storage=storage)
    d.device = local_rank
    d.komega_classic = {"sstep": 0, "classic": 1, "sstep_coop": 2, "sstep_host": 3}[args.solver]
    solver_kernel = {"sstep": "sstep_phases", "classic": "gmres_kernel", "sstep_coop": "sstep_kernel",
                     "sstep_host": "sstep_phases"}[args.solver]
    d.use_thermal = 1 if args.thermal else 0
    L = Lattice(d)
    W.apply(L, w)
    if args.thermal:
        from komegafoulingmodel_b200 import geometry as G
        L.set_temperature(G.temperature_field(w.channel))
    stream = torch.cuda.ExternalStream(L.stream, device=local_rank)
    nodes = w.nodes

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---- warm-up and timed region (inputs resident in HBM) --------------------
    for _ in range(args.warmup):
        L.step(1)
    L.sync()
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = L.stats().solver_launches_total if w.komega else 0
    e0.record(stream)
    for _ in range(args.steps):
        L.step(1)
    e1.record(stream)
    L.sync()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, f"cuda:{local_rank}")
    st = L.stats()
    solver_launches = (st.solver_launches_total - launches0) if w.komega else 0
    value = replica_value(nodes, args.steps, world, ms)
    # kernels of the timed steps: one collide per step plus the k-omega
    # updates' kernels (assembly, solver, the graph's control kernels), which
    # the library counts on the device
    launches_per_step = (1 + solver_launches / args.steps) if w.komega else 1
    if args.thermal:  # assembly, control-block init and BiCGStab per solve
        launches_per_step += 3 * max(1, st.thermal_solves)

    # ---- per-kernel breakdown (same stream, CUDA events) ------------------------
    nb = max(3, min(args.steps, 10))
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(nb)]
    passes, bytes_solver = [], []
    for i in range(nb):
        ev[i][0].record(stream)
        L.lb_step(_abi.OPTION_SAVE_MACRO_FIELDS if w.komega else 0)
        ev[i][1].record(stream)
        if w.komega:
            L.komega_assemble(1.0)
        ev[i][2].record(stream)
        if w.komega:
            L.komega_solve(raise_on_error=False)
        ev[i][3].record(stream)
        if w.komega:
            s = L.stats()
            passes.append(s.solver_passes)
            bytes_solver.append(s.solver_bytes_per_node)
    torch.cuda.synchronize()
    t_lb = sum(ev[i][0].elapsed_time(ev[i][1]) for i in range(nb)) / nb
    t_as = sum(ev[i][1].elapsed_time(ev[i][2]) for i in range(nb)) / nb
    t_sv = sum(ev[i][2].elapsed_time(ev[i][3]) for i in range(nb)) / nb
    b_sv = sum(bytes_solver) / nb if bytes_solver else 0.0
    thermal = None
    if args.thermal:
        tev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(nb)]
        tchecks = []
        for i in range(nb):
            L.lb_step(_abi.OPTION_SAVE_MACRO_FIELDS)
            L.komega_update()
            tev[i][0].record(stream)
            L.thermal_update()
            tev[i][1].record(stream)
            tchecks.append(L.stats().thermal_checks)
        torch.cuda.synchronize()
        t_th = sum(tev[i][0].elapsed_time(tev[i][1]) for i in range(nb)) / nb
        b_th = sum(thermal_bytes_per_node(c) for c in tchecks) / nb
        thermal = {"ms": t_th, "bytes_per_node": b_th, "gbs": b_th * nodes / (t_th * 1e-3) / 1e9,
                   "checks_by_update": tchecks,
                   "kernels": "thermal_assemble_kernel + bicgstab_kernel (+ T copy, control init)"}
    peak, peak_kind = measured_peaks()
    lb_bytes = LB_BYTES[args.storage] if w.komega else LB_BYTES_LAMINAR[args.storage]
    kern = {"lb_step_kernel": {"ms": t_lb, "bytes_per_node": lb_bytes,
                               "gbs": lb_bytes * nodes / (t_lb * 1e-3) / 1e9}}
    if w.komega:
        kern["komega_assemble_kernel"] = {"ms": t_as, "bytes_per_node": asm_bytes,
                                          "gbs": asm_bytes * nodes / (t_as * 1e-3) / 1e9}
        kern[solver_kernel] = {"ms": t_sv, "bytes_per_node": b_sv,
                               "gbs": b_sv * nodes / (t_sv * 1e-3) / 1e9,
                               "passes": sum(passes) / nb,
                               "bytes_per_node_by_launch": bytes_solver}
    dom = max(kern, key=lambda k: kern[k]["ms"])
    ratio = SOLVER_TRAFFIC_RATIO.get(dom)
    roof = {"kernel": dom, "bound": "hbm", "achieved": kern[dom]["gbs"], "peak": peak,
            "unit": "GB/s", "frac": kern[dom]["gbs"] / peak, "peak_kind": peak_kind,
            "traffic": (ratio * kern[dom]["bytes_per_node"] * nodes if ratio else None),
            "traffic_source": "ncu dram bytes / algorithmic bytes of one launch on "
                              "komega_straight_8192x512, times this run's average launch",
            "bytes_per_node": kern[dom]["bytes_per_node"]}
    step_bytes = lb_bytes + (asm_bytes + b_sv if w.komega else 0.0)
    step_ms = t_lb + t_as + t_sv

    # ---- end to end through the public API with host buffers ---------------------
    e2e = None
    if not args.no_e2e:
        n = w.channel.n
        pin = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        hf, hk, ho, hn, hs = pin(w.f), pin(w.k), pin(w.omega), pin(w.nut), pin(w.sxy)
        hr, hu = torch.empty(n, dtype=torch.float64).pin_memory(), torch.empty(n, dtype=torch.float64).pin_memory()
        dp = lambda t: None if t is None else C.cast(t.data_ptr(), C.POINTER(C.c_double))  # noqa: E731
        out = C.c_double()
        ctx = L._ctx
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _abi.check("set_state", lib.kofm_set_state(ctx, dp(hf), dp(hk), dp(ho), dp(hn), dp(hs)))
        for _ in range(args.steps):
            _abi.check("step", lib.kofm_step(ctx, 1, _abi.OPTION_SAVE_MACRO_FIELDS))
            _abi.check("reduce", lib.kofm_reduce(ctx, _abi.FIELD_RHO, _abi.OP_SUM, C.byref(out)))
            _abi.check("reduce", lib.kofm_reduce(ctx, _abi.FIELD_UX, _abi.OP_SUM, C.byref(out)))
        _abi.check("get_macro", lib.kofm_get_macro(ctx, dp(hr), dp(hu), None))
        t1 = time.perf_counter()
        secs = max_over_ranks(t1 - t0, world, f"cuda:{local_rank}")
        h2d = 8 * (9 * n + (6 * n if w.komega else 0))
        d2h = 8 * 2 * args.steps + 8 * 2 * n
        e2e = {"value": nodes * args.steps * world / secs / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "timing": "host wall clock around set_state (pinned host) + K x "
                         "(kofm_step + 2 kofm_reduce D2H) + kofm_get_macro D2H"}
    L.close()

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.thermal:
        cpu = cpu_reference_sample(w, steps=args.cpu_steps, warmup=0)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.storage in ("fp32", "fp64") else "f32", "data": "synthetic",
            "config": workload_config(w, args, world),
            "roofline": roof,
            "step_roofline": {"bytes_per_node": step_bytes,
                              "achieved": step_bytes * nodes / (step_ms * 1e-3) / 1e9,
                              "frac": step_bytes * nodes / (step_ms * 1e-3) / 1e9 / peak},
            # the whole timed step against the compulsory per-step traffic of
            # the FP32 k-omega form (130 B/node: populations, flags, k, omega,
            # strain rates, wall distance, moments; no solver sweep credited)
            "step_roofline_130": {"bytes_per_node": 130,
                                  "achieved": 130 * nodes / (ms / args.steps * 1e-3) / 1e9,
                                  "frac": 130 * nodes / (ms / args.steps * 1e-3) / 1e9 / peak},
            "kernels": kern,
            **({"thermal": thermal} if thermal else {}),
            "solver": {"omega_iters": st.omega_iters, "k_iters": st.k_iters,
                       "omega_restarts": st.omega_restarts, "k_restarts": st.k_restarts,
                       "omega_vectors": st.omega_vectors, "k_vectors": st.k_vectors,
                       "omega_powers": st.omega_powers, "k_powers": st.k_powers,
                       "passes": st.solver_passes, "form": args.solver},
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": int(round(launches_per_step * args.steps)),
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def cpu_reference_sample(w, steps=2, warmup=0, budget_s=None):
    """The reference's CPU code of the path on this host's cores: the OpenCL
    kernel sources compiled as C++ (oracle/_ref) for collide and assembly plus
    the C restatement of GMRESSolver::solve; full-lattice steps."""
    import ctypes as C

    import numpy as np

    from oracle.orc import LIB_REF, Oracle, OracleSim, RefKernels, make_cfg

    orc = Oracle()
    ch = w.channel
    cfg = make_cfg(ch.nx, ch.ny, w.tau, w.fterm, w.mu, nxf=ch.nx_full)
    ibb = (ch.ibb_idx, ch.ibb_q) if len(ch.ibb_idx) else (None, None)
    sim = OracleSim(orc, cfg, ch.ntype, ch.dX, ch.wallD, w.f, w.k, w.omega, w.nut, w.sxy,
                    komega=w.komega, ibb_idx=ibb[0], ibb_q=ibb[1])
    kind = "port"
    ref = RefKernels() if os.path.exists(LIB_REF) else None
    if ref is not None:
        kind = "reference"
    n = ch.n
    dbg = np.zeros(40 * n) if (ref is not None and w.komega) else None

    def one_step():
        if ref is None:
            sim.step(1)
            return
        cp = C.byref(cfg)
        if w.komega:
            ref.L.ref_collide_komega(cp, sim.rho, sim.ux, sim.uy, sim.FA, sim.FB, sim.m,
                                     sim.wallD, sim.nut, sim.K, sim.O, sim.S, 2)
        else:
            ref.L.ref_collide_laminar(cp, sim.rho, sim.ux, sim.uy, sim.FA, sim.FB, sim.m, 2)
        if len(sim.ibb_idx):  # lbIBB on the post-stream populations
            ref.L.ref_ibb(cp, sim.ibb_idx, sim.ibb_q, sim.FB, len(sim.ibb_idx))
        sim.FA, sim.FB = sim.FB, sim.FA
        if w.komega:
            ref.L.ref_komega_diffusivities(cp, sim.m, sim.K, sim.O, sim.nut, sim.wallD, sim.Dk,
                                           sim.Do, sim.F1, sim.dkdo, sim.rho, sim.dX, dbg)
            ref.L.ref_komega_coeffs(cp, sim.ind, sim.K, sim.O, sim.nut, sim.Dk, sim.Do, sim.F1,
                                    sim.dkdo, sim.S, sim.rho, sim.ux, sim.uy, sim.kA, sim.oA,
                                    sim.kb, sim.ob, sim.dX, sim.wallD, sim.m, 1.0, dbg)
            from oracle.orc import GmresStats
            for A, b, x in ((sim.oA, sim.ob, sim.O), (sim.kA, sim.kb, sim.K)):
                st = GmresStats()
                orc.L.orc_gmres_solve(n, sim.IA, sim.JA, A, b, x, 10, 1000, 1e-4, 1e-7, C.byref(st))

    for _ in range(warmup):
        one_step()
    t0 = time.perf_counter()
    done = 0
    for _ in range(steps):
        one_step()
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    secs = time.perf_counter() - t0
    cores = len(os.sched_getaffinity(0))
    return {"value": w.nodes * done / secs / 1e6, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{done} of {steps} full steps of {w.name} ({w.nodes} nodes), "
                      f"after {warmup} untimed: reference kernels (oracle/_ref) for collide"
                      f"{' + lbIBB' if len(sim.ibb_idx) else ''} + k-omega assembly, C restatement "
                      "of its GMRES(10); OpenMP over rows",
            "seconds": secs, "steps_timed": done}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from komegafoulingmodel_b200 import workloads as W
    w = W.by_name(args.workload)
    # W untimed and up to K timed full-lattice steps; the timed loop stops
    # after ~150 s of host time so the run stays within a few minutes
    res = cpu_reference_sample(w, steps=args.steps, warmup=args.warmup, budget_s=150.0)
    line = {
        "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["seconds"] * 1e3 / res["steps_timed"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(w, args, world),
        "impl": "reference",
        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="komega_straight_16384x1024")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16", "bf16", "fp16neq", "fp16neq32", "fp16row", "fp64"])
    ap.add_argument("--solver", default="sstep", choices=["sstep", "sstep_host", "sstep_coop", "classic"],
                    help="k-omega solve: a cycle's Krylov directions in one sweep, each sweep "
                         "its own launch in a device-driven update graph (default) or enqueued "
                         "round by round by the host (sstep_host), or all in one cooperative "
                         "launch (sstep_coop); or one vector per sweep (classic)")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--thermal", action="store_true",
                    help="add the thermal implicit FD update to every step (reported apart)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
