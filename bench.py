#!/usr/bin/env python
"""Benchmark of the MEUMAPPS-SS time step on B200.

Workload (default): Landau deck 1 -- 128^3 grid, one conserved c and three
tetragonal variants eta_1..3, homogeneous cubic elasticity through the Green
operator, dt = 0.005, FP32 bulk arithmetic (FP64 for Omega(k), the k = 0 mode
and every reduction).  A "step" is one time step of that grid.
--config 0 / 2 select the 64^3 single-variant and the 512^3 heterogeneous decks;
--config 3 the batched ensemble of 96 single-variant runs on 32^3..128^3 grids
(a "step" advances every member once; cells = the members' grid points);
--config 5 the slab-decomposed FFT of one grid over the ranks (512^2 x 512N, weak
scaling; a "step" is one forward and one inverse transform); --config 6 the
reference's own KKS model (128^3, 3 variants, FP64, noise off and on).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); every rank advances its own
independent replica (the single-grid step has no data-parallel exchange), so
scaling is weak and the only collectives are the timing barrier/max.

--impl reference times the CPU FP64 restatement of the reference step
(oracle/, "port": the Fortran/MPI/P3DFFT reference cannot be built in this
image) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s: FP32-bulk vs FP64 plain at stated err; adjoint/forward cost"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--n", type=int, default=0, help="override the grid edge (tests only)")
    ap.add_argument("--schedule", default="",
                    help="pv,threads,tile: fixed schedule of the fused step instead of the autotuner's (profiling)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the extra decks (0 and 2) measured beside the headline")
    ap.add_argument("--profile", action="store_true",
                    help="only the warm-up and timed FP32 steps (for ncu launch lists and captures)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.lines = []
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz)}


# ------------------------------------------------------------ CPU side
def oracle_throughput(params, c, e, steps: int, threads: int):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads)
    s = O.OracleSim(params)
    s.set_fields(c, e)
    t0 = time.perf_counter()
    s.run(steps)
    dt = time.perf_counter() - t0
    s.close()
    n3 = params.nx * params.ny * params.nz
    return n3 * steps / dt / 1e6, dt


def cpu_sample(cfg: int, n_override: int, budget_s: float, min_steps: int, threads: int):
    """Oracle time steps on the deck's grid, or on a smaller grid of the same deck
    when min_steps steps at full size do not fit the budget.  The size is chosen
    from one calibration step at 32^3 scaled by N^3 log N."""
    import math
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    def deck(n):
        # inputs from the oracle's own ran_2: the CPU legs load nothing of the product library
        w = CF.landau_config(cfg, n=n, precision=P.PREC_F64)
        p = w.params
        c, e = O.init_uniform(p.nx, p.ny, p.nz, p.nvar, w.seed, w.c0, w.c_amp, w.eta_amp)
        return w, p, c, e

    w0, p0, c0, e0 = deck(32)
    _, t32 = oracle_throughput(p0, c0, e0, 2, threads)
    t32 /= 2.0
    nmax = n_override or CF.landau_config(cfg, precision=P.PREC_F64).params.nx
    sizes = [nmax] + [s for s in (256, 128, 96, 64, 48, 32) if s < nmax]
    for n in sizes:
        t1 = t32 * (n / 32.0) ** 3 * math.log(n) / math.log(32)
        if t1 * min_steps <= budget_s or n == sizes[-1]:
            w, p, c, e = deck(n)
            steps = max(min_steps, int(budget_s / max(t1, 1e-6)))
            return w, p, c, e, max(1, min(steps, 100000)), t1
    raise RuntimeError("unreachable")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    K, W = args.steps, args.warmup
    budget = 150.0
    # choose the sample grid so that W + K oracle steps take about `budget` seconds
    w, p, c, e, _, t1 = cpu_sample(args.config, args.n, budget, K + W, threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads)
    s = O.OracleSim(p)
    s.set_fields(c, e)
    s.run(W)
    t0 = time.perf_counter()
    s.run(K)
    dt = time.perf_counter() - t0
    n3 = p.nx * p.ny * p.nz
    val = n3 * K / dt / 1e6
    sample = (f"{K} time steps of the {w.name} deck on a {p.nx}^3 grid (FP64 oracle port, {threads} threads; "
              f"the Fortran/MPI/P3DFFT reference cannot be built in this image)")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": K,
        "warmup": W, "ms_per_step": dt / K * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": f"synthetic (ran_2 uniform noise, seed {w.seed})",
        "config": {"workload": w.name, "grid": [p.nx, p.ny, p.nz], "variants": p.nvar, "parallelism": "host threads"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- GPU side
def read_traffic(kernel: str):
    """dram read+write bytes per launch of `kernel` from the committed ncu
    summary (profiles/*.md line 'traffic_bytes_per_launch[<kernel>]: <bytes> at <grid>')."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith(".md"):
            continue
        for ln in open(os.path.join(d, f)):
            key = f"traffic_bytes_per_launch[{kernel}]:"
            if ln.strip().startswith(key):
                try:
                    return float(ln.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


def elasticity_label(p) -> str:
    from meumapps_ss_b200 import params as P
    if p.elastic == P.ELAST_NONE:
        return "none"
    if p.elastic == P.ELAST_HOMOG:
        return "homogeneous cubic 250/150/100, Green operator"
    return (f"heterogeneous: precipitate moduli {p.cela[1][0] / p.cela[0][0]:g}x matrix, compliance mix, "
            f"fixed-point iteration to residual <= {p.el_tol:g} (FP64 residual)")


def measure_deck(cfg: int, stream, K: int, W: int, K64: int, local: int, peak: float = 0.0):
    """One more deck beside the headline: FP32-bulk and FP64 throughput (CUDA events
    around meu_run, graph capture and autotuning outside the timed region), the
    FP32 error against FP64 after W + K steps, the clocks during the FP32 window.
    With peak (GB/s): the FP32 step's algorithmic bytes from two per-kernel-timed
    steps after the window (scaled to the window's elastic iterations per step when
    the moduli are heterogeneous) over the window's step time, as a fraction of it."""
    import numpy as np
    import torch
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200.sim import Simulation

    w = CF.landau_config(cfg, precision=P.PREC_F32)
    p32 = w.params
    p32.flags |= P.FLAG_AUTOTUNE
    n3 = p32.nx * p32.ny * p32.nz
    c0, e0 = _lib.init_uniform(p32.nx, p32.ny, p32.nz, p32.nvar, w.seed, w.c0, w.c_amp, w.eta_amp)
    out = {"workload": w.name, "grid": [p32.nx, p32.ny, p32.nz], "variants": p32.nvar,
           "elasticity": elasticity_label(p32), "dt": p32.dt}
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fields = {}
    for prec, k in ((P.PREC_F32, K), (P.PREC_F64, K64)):
        q = p32.copy()
        q.precision = prec
        sim = Simulation(q)
        sim.set_stream(stream.cuda_stream)
        sim.set_fields(c0, e0)
        sim.run(W, diag=True)
        sampler = ClockSampler(local)
        torch.cuda.synchronize()
        if prec == P.PREC_F32:
            sampler.start()
            time.sleep(0.3)
        rows = (P.MeuDiag * k)()
        a.record(stream)
        sim.run_into(k, rows)  # the driver's call; the rows are converted outside the timed region
        b.record(stream)
        stream.synchronize()
        ms = a.elapsed_time(b)
        d = P.diag_to_dict(list(rows))
        key = "fp32_bulk" if prec == P.PREC_F32 else "fp64_plain"
        out[key] = {"value": n3 * k / (ms / 1e3) / 1e6, "unit": UNIT, "steps": k, "ms_per_step": ms / k}
        if p32.elastic == P.ELAST_HETERO:
            out[key]["elastic_iterations_per_step"] = float(np.mean(d["el_iters"]))
        if prec == P.PREC_F32:
            out["clocks"] = sampler.stop()
            out["schedule"] = sim.schedule
            if peak:
                sim.timing(True)
                tr = (P.MeuDiag * 2)()
                sim.run_into(2, tr)
                rep_t = sim.timing_report()
                sim.timing(False)
                sb = sum(v["bytes"] for v in rep_t.values()) / 2
                if p32.elastic == P.ELAST_HETERO:
                    it_t = float(np.mean(P.diag_to_dict(list(tr))["el_iters"]))
                    sb *= out[key]["elastic_iterations_per_step"] / max(it_t, 1e-9)
                out["step_roofline"] = {"step_algorithmic_bytes": sb, "peak": peak, "unit": "GB/s",
                                        "achieved": sb / (ms / k / 1e3) / 1e9,
                                        "step_frac": sb / (ms / k / 1e3) / 1e9 / peak}
        elif peak:
            sim.run(2, diag=False)  # the FP32 leg's two timed steps: same step count for the error
        if k < K:
            sim.run(K - k, diag=False)
        fields[prec] = sim.get_fields()[:2]
        sim.close()
    (c32, e32), (c64, e64) = fields[P.PREC_F32], fields[P.PREC_F64]
    out["fp32_speedup"] = out["fp32_bulk"]["value"] / out["fp64_plain"]["value"]
    out["err_vs_fp64"] = {"c_rel_l2": float(np.linalg.norm(c32 - c64) / np.linalg.norm(c64)),
                          "eta_rel_l2": float(np.linalg.norm(e32 - e64) / max(np.linalg.norm(e64), 1e-300)),
                          "after_steps": W + K + (2 if peak else 0)}
    return out


def measure_kks(stream, n: int = 128, nvar: int = 3, K: int = 5, W: int = 2):
    """The reference's own model (KKS, plain FP64, heterogeneous elasticity) on an n^3
    deck in the reference's Input.txt format: Mcell-steps/s without noise and with the
    Langevin noise of every step (ran_2 draws on a host thread, meu_run_noise)."""
    import ctypes as C
    import torch
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200.sim import Simulation

    deck = P.parse_input_txt(CF.kks_input_txt(n, nvar, 10 ** 6, radius=max(3, n // 10)))
    p = P.kks_params(deck)
    cons, phi = P.init_fields(deck)
    n3 = n ** 3
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"workload": f"kks-{n}^3-{nvar}var-hetero", "grid": [n, n, n], "variants": nvar, "precision": "f64",
           "elasticity": "heterogeneous cubic moduli, fixed point (ModElastic.f:241-481)",
           "noise_draws_per_step": nvar * n3,
           "noise_note": ("ran_2 is one serial chain: each step's vartot*N^3 langevin draws walk it on one host "
                          "thread (the logarithms on the other host threads), overlapped with the previous step "
                          "on the GPU")}
    for noisy in (False, True):
        q = p.copy()
        q.noise_step = q.step + 10 ** 6 if noisy else 0
        q.flags |= P.FLAG_AUTOTUNE  # the transform passes' radix plan and column tile, timed at meu_create
        with Simulation(q) as g:
            g.set_stream(stream.cuda_stream)
            g.set_fields(cons, phi)
            st = _lib.Ran2State()
            _lib.lib().meu_ran2_init(C.byref(st), -abs(deck.iseed) or -1)
            run = (lambda k: g.run_noise(k, st, deck.sd)) if noisy else (lambda k: g.run(k))
            run(W)
            sched = g.schedule
            torch.cuda.synchronize()
            a.record(stream)
            d = run(K)
            b.record(stream)
            stream.synchronize()
            ms = a.elapsed_time(b)
        key = "noise_on" if noisy else "noise_off"
        out[key] = {"value": n3 * K / (ms / 1e3) / 1e6, "unit": UNIT, "steps": K, "ms_per_step": ms / K,
                    "elastic_iterations_per_step": float(sum(d["el_iters"]) / K), "schedule": list(sched)}
    return out


def measure_ensemble(stream, K: int = 20, W: int = 5, local: int = 0, peak: float = 0.0):
    """Deck 3 beside the headline: the 96-member ensemble (32^3..128^3 grids, one
    variant) in FP32 bulk and plain FP64, CUDA events around meu_ensemble_run (graph
    capture and autotuning outside the timed region), with the FP32 error against FP64
    (worst member) and the clocks of the FP32 window."""
    import numpy as np
    import torch
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200.sim import Ensemble

    out = {"workload": f"landau-ensemble-{ENS_MEMBERS}x1var"}
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fields_out = {}
    # legs: per-bucket kernels replayed as graphs (FP32 autotuned, FP64), and the FP32
    # persistent launch (one launch per run of up to 64 steps, MEU_ENS_PERSISTENT)
    legs = (("fp32_bulk", P.PREC_F32, True, False), ("fp64_plain", P.PREC_F64, False, False),
            ("fp32_persistent", P.PREC_F32, False, True))
    for key, prec, tune, pers in legs:
        ws = CF.ensemble_config(ENS_MEMBERS, precision=prec)
        cells = sum(w.params.nx ** 3 for w in ws)
        ens = Ensemble([w.params for w in ws], autotune=tune, persistent=pers)
        ens.set_stream(stream.cuda_stream)
        for i, w in enumerate(ws):
            ens.set_fields(i, *ensemble_fields(w))
        ens.run(W, diag=True)
        sampler = ClockSampler(local)
        torch.cuda.synchronize()
        if key == "fp32_bulk":
            sampler.start()
            time.sleep(0.3)
        l0 = ens.launch_count
        rows = (P.MeuDiag * (len(ws) * K))()
        a.record(stream)
        ens.run_into(K, rows)
        b.record(stream)
        stream.synchronize()
        ms = a.elapsed_time(b)
        out[key] = {"value": cells * K / (ms / 1e3) / 1e6, "unit": UNIT, "steps": K, "ms_per_step": ms / K,
                    "gpu_launches_per_step": (ens.launch_count - l0) / K}
        if pers:
            out[key]["schedule"] = list(ens.schedule(0)[:3])
        if key == "fp32_bulk":
            out["clocks"] = sampler.stop()
            out["cells_per_step"] = cells
        if peak:
            # two more steps in every leg (same step count for the errors); in the FP32 leg
            # with per-kernel timing, for the step's algorithmic bytes
            if key == "fp32_bulk":
                ens.timing(True)
                ens.run(2, diag=False)
                sb = sum(v["bytes"] for v in ens.timing_report().values()) / 2
                ens.timing(False)
                out["step_roofline"] = {"step_algorithmic_bytes": sb, "peak": peak, "unit": "GB/s",
                                        "achieved": sb / (ms / K / 1e3) / 1e9,
                                        "step_frac": sb / (ms / K / 1e3) / 1e9 / peak}
            else:
                ens.run(2, diag=False)
        fields_out[key] = [ens.get_fields(i)[:2] for i in range(len(ws))]
        ens.close()

    def worst(k32):
        wc = max(float(np.linalg.norm(c32 - c64) / np.linalg.norm(c64))
                 for (c32, _), (c64, _) in zip(fields_out[k32], fields_out["fp64_plain"]))
        we = max(float(np.linalg.norm(e32 - e64) / max(np.linalg.norm(e64), 1e-300))
                 for (_, e32), (_, e64) in zip(fields_out[k32], fields_out["fp64_plain"]))
        return wc, we

    worst_c, worst_e = worst("fp32_bulk")
    pc, pe = worst("fp32_persistent")
    out["fp32_persistent"]["err_vs_fp64"] = {"c_rel_l2_max_member": pc, "eta_rel_l2_max_member": pe,
                                             "after_steps": W + K + (2 if peak else 0)}
    out["fp32_speedup"] = out["fp32_bulk"]["value"] / out["fp64_plain"]["value"]
    out["err_vs_fp64"] = {"c_rel_l2_max_member": worst_c, "eta_rel_l2_max_member": worst_e,
                          "after_steps": W + K + (2 if peak else 0)}
    return out


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200.sim import Simulation

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    K, W = args.steps, max(3, args.warmup)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = CF.landau_config(args.config, n=args.n or None, precision=P.PREC_F32)
    p32 = w.params
    if not args.schedule:
        p32.flags |= P.FLAG_AUTOTUNE  # fused decks: fastest schedule; generic path: fastest transform radix plan
    nx, ny, nz, V, E = p32.nx, p32.ny, p32.nz, p32.nvar, p32.numel
    n3 = nx * ny * nz
    seed = w.seed - rank
    c0, e0 = _lib.init_uniform(nx, ny, nz, V, seed, w.c0, w.c_amp, w.eta_amp)
    stream = torch.cuda.Stream(device=dev)

    free0 = torch.cuda.mem_get_info(dev)[0]
    sim = Simulation(p32)
    footprint = free0 - torch.cuda.mem_get_info(dev)[0]
    if args.schedule:
        sim.set_schedule(*(int(x) for x in args.schedule.split(",")))
    schedule = sim.schedule
    sim.set_stream(stream.cuda_stream)
    sim.set_fields(c0, e0)
    sim.run(W, diag=True)

    # ---------------- timed region: K FP32 steps with the fort.98 diagnostics
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    l0 = sim.launch_count
    rows_k = (P.MeuDiag * K)()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        sim.run_into(K, rows_k)  # the driver's call; rows converted outside the timed region
        ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    launches = sim.launch_count - l0
    clocks = sampler.stop()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = world * n3 * K / (ms / 1e3) / 1e6
    if args.profile:
        sim.close()
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"profile_run": w.name, "steps": K, "warmup": W, "ms_per_step": ms / K}), flush=True)
        return 0
    c32, e32, _, _ = sim.get_fields()

    # ---------------- FP64 plain path, same deck and initial fields
    p64 = p32.copy()
    p64.precision = P.PREC_F64
    sim64 = Simulation(p64)
    sim64.set_stream(stream.cuda_stream)
    sim64.set_fields(c0, e0)
    sim64.run(W, diag=True)
    K64 = min(K, 500)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    rows64 = (P.MeuDiag * K64)()
    a.record(stream)
    sim64.run_into(K64, rows64)
    b.record(stream)
    stream.synchronize()
    ms64 = max_over_ranks(a.elapsed_time(b))
    value64 = world * n3 * K64 / (ms64 / 1e3) / 1e6
    if K > K64:
        sim64.run(K - K64, diag=False)
    c64, e64, _, _ = sim64.get_fields()
    sim64.close()
    err_c = float(np.linalg.norm(c32 - c64) / np.linalg.norm(c64))
    err_e = float(np.linalg.norm(e32 - e64) / max(np.linalg.norm(e64), 1e-300))

    # ---------------- per-kernel CUDA-event timing (roofline of the dominant kernel)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        pk = json.load(open(peaks_path))
        peak, peak_src = float(pk["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    sim.timing(True)
    kt = min(K, 100)
    sim.run(kt, diag=True)
    rep = sim.timing_report()
    sim.timing(False)
    tot = sum(v["ms"] for v in rep.values())
    dom = max(rep, key=lambda k: rep[k]["ms"])
    dr = rep[dom]
    dom_ms = dr["ms"] / dr["launches"]
    achieved = dr["bytes"] / dr["launches"] / (dom_ms / 1e3) / 1e9
    traffic = read_traffic(dom)
    step_bytes = sum(v["bytes"] for v in rep.values()) / kt
    kernels = {k: {"launches": v["launches"], "ms_per_launch": v["ms"] / v["launches"],
                   "share": v["ms"] / tot, "GB/s": v["bytes"] / v["ms"] / 1e6} for k, v in
               sorted(rep.items(), key=lambda kv: -kv[1]["ms"])}

    # ---------------- end to end through the C-ABI with pinned host buffers
    L = _lib.lib()
    hc = torch.empty(E * n3, dtype=torch.float64).pin_memory()
    hp = torch.empty(V * n3, dtype=torch.float64).pin_memory()
    hc.copy_(torch.from_numpy(P.to_fortran(c32)))
    hp.copy_(torch.from_numpy(P.to_fortran(e32)))
    dp = C.POINTER(C.c_double)
    pc = C.cast(hc.data_ptr(), dp)
    pp = C.cast(hp.data_ptr(), dp)
    rows = (P.MeuDiag * 1)()
    ke = min(K, 100) if n3 * (E + V) * 8 <= (1 << 28) else min(K, 3)
    for _ in range(2):
        L.meu_set_fields(sim.h, pc, pp, None)
        L.meu_run(sim.h, 1, rows)
        L.meu_get_fields(sim.h, pc, pp, None, None)
    barrier()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(ke):
        st1 = L.meu_set_fields(sim.h, pc, pp, None)
        st2 = L.meu_run(sim.h, 1, rows)
        st3 = L.meu_get_fields(sim.h, pc, pp, None, None)
        if st1 or st2 or st3:
            raise RuntimeError(f"C-ABI status {st1} {st2} {st3}")
    b.record(stream)
    stream.synchronize()
    ms_e2e = max_over_ranks(a.elapsed_time(b))
    e2e = world * n3 * ke / (ms_e2e / 1e3) / 1e6
    # window form: upload once, K steps with diagnostics, download once
    torch.cuda.synchronize()
    a.record(stream)
    L.meu_set_fields(sim.h, pc, pp, None)
    rowsK = (P.MeuDiag * K)()
    L.meu_run(sim.h, K, rowsK)
    L.meu_get_fields(sim.h, pc, pp, None, None)
    b.record(stream)
    stream.synchronize()
    ms_win = max_over_ranks(a.elapsed_time(b))
    e2e_win = world * n3 * K / (ms_win / 1e3) / 1e6
    sim.close()

    # ---------------- adjoint of deck 4 (gradient call against the forward), rank 0
    adj = None
    if rank == 0 and not args.n:
        adj = measure_adjoint(stream, fd=False)
        adj.pop("kernels_ms", None)

    # ---------------- the other single-grid decks, measured in the same run (rank 0, default workload)
    decks = {}
    if rank == 0 and not args.n and args.config == 1 and not args.no_extra:
        decks["deck0"] = measure_deck(0, stream, K=200, W=W, K64=200, local=local, peak=peak)
        decks["deck2"] = measure_deck(2, stream, K=10, W=W, K64=10, local=local, peak=peak)
        decks["kks"] = measure_kks(stream)
        decks["deck3"] = measure_ensemble(stream, local=local, peak=peak)

    # ---------------- CPU baseline (rank 0, N = 1): the oracle port on host cores
    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        wc, pc64, cc, ec, steps, _ = cpu_sample(args.config, args.n, 20.0, 1, threads)
        v, dt = oracle_throughput(pc64, cc, ec, steps, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{steps} FP64 time steps of {wc.name} on a {pc64.nx}^3 grid ({dt:.1f} s, {threads} threads)"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    l2_mb = 126
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic (ran_2 uniform noise c0={w.c0}+-{w.c_amp}, eta+-{w.eta_amp}, seed {w.seed})",
        "config": {"workload": w.name, "grid": [nx, ny, nz], "variants": V, "free_energy": "landau",
                   "elasticity": elasticity_label(p32), "dt": p32.dt,
                   "precision": "FP32 bulk; FP64 Omega(k), k=0 mode, reductions",
                   "l2": f"device working set {footprint / 2**20:.0f} MiB > {l2_mb} MB L2, no flush",
                   "schedule": schedule,
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "fp64_plain": {"value": value64, "unit": UNIT, "steps": K64, "ms_per_step": ms64 / K64,
                       "fp32_speedup": value / value64},
        "err_vs_fp64": {"c_rel_l2": err_c, "eta_rel_l2": err_e, "after_steps": W + K},
        # t(forward + adjoint, recomputation included) / t(forward) - 1
        "adjoint_forward_cost": None if adj is None else adj["reverse_over_forward"],
        "adjoint": adj,
        "decks": decks,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src,
                     "traffic": traffic, "algorithmic_bytes_per_launch": dr["bytes"] / dr["launches"],
                     "kernel_ms_per_launch": dom_ms,
                     "step_algorithmic_bytes": step_bytes,
                     "step_frac": step_bytes / (ms / K / 1e3) / 1e9 / peak},
        "kernels": kernels,
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": (E + V) * n3 * 8,
                "d2h_bytes_per_step": (E + V) * n3 * 8 + C.sizeof(P.MeuDiag), "steps": ke,
                "form": "per step: meu_set_fields + meu_run(1) + meu_get_fields, pinned host buffers"},
        "e2e_window": {"value": e2e_win, "unit": UNIT, "steps": K,
                       "form": "meu_set_fields once, meu_run(K) with diagnostics, meu_get_fields once"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------- adjoint (deck 4)
def measure_adjoint(stream, n: int = 128, steps: int = 200, fd: bool = True):
    """Gradient of the calibration loss of deck 4 through meu_adjoint: its time
    against the plain forward of the same steps, the FP32 gradient against the
    FP64 one, and central differences (h = 1e-4) of the FP64 loss."""
    import numpy as np
    import torch
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200.sim import Simulation

    K = CF.ADJOINT_CHECKPOINT_EVERY
    w = CF.adjoint_config(n, P.PREC_F64, **CF.ADJOINT_TARGET)
    p = w.params
    c0, e0 = _lib.init_uniform(p.nx, p.ny, p.nz, 1, w.seed, w.c0, w.c_amp, w.eta_amp)
    t = Simulation(p)
    t.set_stream(stream.cuda_stream)
    t.set_fields(c0, e0)
    t.run(steps, diag=False)
    ct, et, _, _ = t.get_fields()
    t.close()

    def loss_fwd(prec, **kw):
        s = Simulation(CF.adjoint_config(n, prec, **kw).params)
        s.set_stream(stream.cuda_stream)
        s.set_fields(c0, e0)
        s.run(steps, diag=False)
        c, e, _, _ = s.get_fields()
        s.close()
        return 0.5 / n ** 3 * (np.sum((e - et) ** 2) + np.sum((c - ct) ** 2))

    def grad(prec):
        s = Simulation(CF.adjoint_config(n, prec, **CF.ADJOINT_START).params)
        s.set_stream(stream.cuda_stream)
        s.set_fields(c0, e0)
        J, g, ge = s.adjoint(steps, K, ct, et)
        st = CF.ADJOINT_START
        out = {"kappa": g["beta_eta"] / st["kappa"] + g["kappa_c"], "L": g["L"], "M": g["M"],
               "eps0": g["alpha"] / st["eps0"]}
        return J, out, ge, s

    J32, g32, ge32, s32 = grad(P.PREC_F32)
    J64, g64, ge64, s64 = grad(P.PREC_F64)
    s64.close()
    # timing: the gradient call and the plain forward of the same steps, FP32, same handle
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    s32.set_fields(c0, e0)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        s32.set_fields(c0, e0)
        s32.adjoint(steps, K, ct, et, want_field=True)
    b.record(stream)
    stream.synchronize()
    t_grad = a.elapsed_time(b) / reps
    s32.set_fields(c0, e0)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        s32.set_fields(c0, e0)
        s32.run(steps, diag=True)
    b.record(stream)
    stream.synchronize()
    t_fwd = a.elapsed_time(b) / reps
    s32.timing(True)
    s32.set_fields(c0, e0)
    s32.adjoint(steps, K, ct, et)
    rep = s32.timing_report()
    s32.timing(False)
    s32.close()
    out = {"workload": w.name.replace("-adjoint-", "-adjoint-calibration-"), "steps": steps, "checkpoint_every": K,
           "loss_fp32": J32, "loss_fp64": J64, "gradient_fp32": g32, "gradient_fp64": g64,
           "fp32_vs_fp64_rel": {k: abs(g32[k] - g64[k]) / max(abs(g64[k]), 1e-300) for k in g64},
           "eta0_grad_fp32_vs_fp64_rel_l2": float(np.linalg.norm(ge32 - ge64) / np.linalg.norm(ge64)),
           "ms_gradient": t_grad, "ms_forward": t_fwd,
           "gradient_over_forward": t_grad / t_fwd,
           "reverse_over_forward": (t_grad - t_fwd) / t_fwd,
           "kernels_ms": {k: v["ms"] for k, v in sorted(rep.items(), key=lambda kv: -kv[1]["ms"])}}
    if fd:
        h = 1e-4
        rel = {}
        for k in ("kappa", "L", "M", "eps0"):
            up, dn = dict(CF.ADJOINT_START), dict(CF.ADJOINT_START)
            up[k] += h
            dn[k] -= h
            fdv = (loss_fwd(P.PREC_F64, **up) - loss_fwd(P.PREC_F64, **dn)) / (2 * h)
            rel[k] = {"fd": fdv, "adjoint_fp64": g64[k], "rel": abs(g64[k] - fdv) / max(abs(fdv), 1e-300)}
        out["central_fd_h1e-4"] = rel
    return out


def run_adjoint_bench(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    sampler = ClockSampler(local)
    sampler.start()
    r = measure_adjoint(stream, n=args.n or 128, steps=200)
    clocks = sampler.stop()
    if rank != 0:
        return 0
    n = args.n or 128
    cells = n ** 3 * r["steps"]
    line = {
        "metric": METRIC, "value": cells / (r["ms_gradient"] / 1e3) / 1e6, "unit": UNIT, "n_gpus": 1,
        "steps": r["steps"], "warmup": 1, "ms_per_step": r["ms_gradient"] / r["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (ran_2 uniform noise, seed -1)",
        "config": {"workload": r["workload"], "grid": [n, n, n], "variants": 1,
                   "value_is": "cell-steps of the gradient call (forward with checkpoints + reverse sweep) per second"},
        "adjoint_forward_cost": r["reverse_over_forward"], "adjoint": r, "clocks": clocks,
        "gpu_launches": None, "e2e": None, "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------- ensemble (deck 3)
ENS_MEMBERS = 96


def ensemble_fields(w, rank: int = 0, oracle_rng: bool = False):
    p = w.params
    if oracle_rng:  # CPU legs: the oracle's own ran_2 (same numbers, no product library)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        return O.init_uniform(p.nx, p.ny, p.nz, p.nvar, w.seed - 1000 * rank, w.c0, w.c_amp, w.eta_amp)
    from meumapps_ss_b200 import _lib
    return _lib.init_uniform(p.nx, p.ny, p.nz, p.nvar, w.seed - 1000 * rank, w.c0, w.c_amp, w.eta_amp)


def ensemble_cpu_sample(budget_s: float, threads: int):
    """Oracle steps over members of the ensemble deck taken in order (each member's
    own grid), about budget_s seconds in all; returns (cells*steps, seconds, text)."""
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    ws = CF.ensemble_config(ENS_MEMBERS, precision=P.PREC_F64)
    cells, secs, used = 0, 0.0, []
    for w in ws:
        c, e = ensemble_fields(w, oracle_rng=True)
        _, dt1 = oracle_throughput(w.params, c, e, 1, threads)
        steps = max(1, min(50, int((budget_s - secs) / max(dt1, 1e-6) * 0.5)))
        v, dt = oracle_throughput(w.params, c, e, steps, threads)
        n3 = w.params.nx ** 3
        cells += n3 * (steps + 1)
        secs += dt + dt1
        used.append(f"{w.params.nx}^3x{steps + 1}")
        if secs >= budget_s:
            break
    return cells, secs, f"FP64 oracle steps of the first {len(used)} ensemble members ({', '.join(used)}), {threads} threads"


def run_ensemble(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200.sim import Ensemble

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    K, W = args.steps, max(3, args.warmup)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from meumapps_ss_b200.shard import gather_by_member, shard_members

    # whole members per rank, balanced by grid points (strong scaling of one ensemble)
    ws_all = CF.ensemble_config(ENS_MEMBERS, precision=P.PREC_F32)
    cells_all = [w.params.nx ** 3 for w in ws_all]
    mine = shard_members(cells_all, world)[rank]
    ws = [ws_all[i] for i in mine]
    cells = sum(cells_all)  # value counts the whole ensemble; time is the max over ranks
    local_cells = sum(cells_all[i] for i in mine)
    fields = [ensemble_fields(w) for w in ws]
    stream = torch.cuda.Stream(device=dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    ens = Ensemble([w.params for w in ws], autotune=True)
    footprint = free0 - torch.cuda.mem_get_info(dev)[0]
    ens.set_stream(stream.cuda_stream)
    scheds = {}
    for i, w in enumerate(ws):
        ens.set_fields(i, *fields[i])
        scheds[w.params.nx] = ens.schedule(i)[:3]
    ens.run(W, diag=True)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    l0 = ens.launch_count
    rows_e = (P.MeuDiag * (len(ws) * K))()
    with torch.cuda.stream(stream):
        ev0.record(stream)
        ens.run_into(K, rows_e)
        ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    launches = ens.launch_count - l0
    clocks = sampler.stop()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = cells * K / (ms / 1e3) / 1e6
    if args.profile:
        ens.close()
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"profile_run": "ensemble", "steps": K, "warmup": W, "ms_per_step": ms / K}), flush=True)
        return 0
    out32 = [ens.get_fields(i)[:2] for i in range(len(ws))]

    # FP64 plain ensemble: same members and fields
    ws64 = [CF.ensemble_config(ENS_MEMBERS, precision=P.PREC_F64)[i] for i in mine]
    e64 = Ensemble([w.params for w in ws64])
    e64.set_stream(stream.cuda_stream)
    for i in range(len(ws64)):
        e64.set_fields(i, *fields[i])
    e64.run(W, diag=True)
    K64 = min(K, 500)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    rows_e64 = (P.MeuDiag * (len(ws64) * K64))()
    a.record(stream)
    e64.run_into(K64, rows_e64)
    b.record(stream)
    stream.synchronize()
    ms64 = max_over_ranks(a.elapsed_time(b))
    value64 = cells * K64 / (ms64 / 1e3) / 1e6
    if K > K64:
        e64.run(K - K64, diag=False)
    errs = {}
    for i in range(len(ws)):
        c64, f64, _ = e64.get_fields(i)
        c32, f32 = out32[i]
        errs[mine[i]] = (float(np.linalg.norm(c32 - c64) / np.linalg.norm(c64)),
                         float(np.linalg.norm(f32 - f64) / max(np.linalg.norm(f64), 1e-300)))
    e64.close()
    # per-member errors gathered on the host (rank 0 gets every member's)
    all_errs = gather_by_member(errs, ENS_MEMBERS)
    err_c = max(x[0] for x in all_errs) if all_errs else 0.0
    err_e = max(x[1] for x in all_errs) if all_errs else 0.0

    # per-kernel timing (all buckets together)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    ens.timing(True)
    kt = min(K, 50)
    ens.run(kt, diag=True)
    rep = ens.timing_report()
    ens.timing(False)
    tot = sum(v["ms"] for v in rep.values())
    dom = max(rep, key=lambda k: rep[k]["ms"])
    dr = rep[dom]
    dom_ms = dr["ms"] / dr["launches"]
    achieved = dr["bytes"] / dr["launches"] / (dom_ms / 1e3) / 1e9
    step_bytes = sum(v["bytes"] for v in rep.values()) / kt
    kernels = {k: {"launches": v["launches"], "ms_per_launch": v["ms"] / v["launches"], "share": v["ms"] / tot,
                   "GB/s": v["bytes"] / v["ms"] / 1e6} for k, v in sorted(rep.items(), key=lambda kv: -kv[1]["ms"])}

    # end to end through the C-ABI: every member's fields in and out each step, pinned host buffers
    L = _lib.lib()
    host = []
    for i, w in enumerate(ws):
        n3 = w.params.nx ** 3
        hc = torch.empty(n3, dtype=torch.float64).pin_memory()
        hp = torch.empty(n3, dtype=torch.float64).pin_memory()
        hc.copy_(torch.from_numpy(P.to_fortran(out32[i][0])))
        hp.copy_(torch.from_numpy(P.to_fortran(out32[i][1])))
        host.append((hc, hp))
    dp = C.POINTER(C.c_double)
    ptrs = [(C.cast(hc.data_ptr(), dp), C.cast(hp.data_ptr(), dp)) for hc, hp in host]
    rows = (P.MeuDiag * len(ws))()

    def e2e_step():
        for i, (pc, pp) in enumerate(ptrs):
            if L.meu_ensemble_set_fields(ens.h, i, pc, pp):
                raise RuntimeError(L.meu_ensemble_last_error(ens.h).decode())
        if L.meu_ensemble_run(ens.h, 1, rows):
            raise RuntimeError(L.meu_ensemble_last_error(ens.h).decode())
        for i, (pc, pp) in enumerate(ptrs):
            if L.meu_ensemble_get_fields(ens.h, i, pc, pp, None):
                raise RuntimeError(L.meu_ensemble_last_error(ens.h).decode())

    e2e_step()
    ke = min(K, 5)
    barrier()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(ke):
        e2e_step()
    b.record(stream)
    stream.synchronize()
    ms_e2e = max_over_ranks(a.elapsed_time(b))
    e2e = cells * ke / (ms_e2e / 1e3) / 1e6
    ens.close()

    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        cc, secs, txt = ensemble_cpu_sample(20.0, threads)
        cpu = {"value": cc / secs / 1e6, "unit": UNIT, "cores": threads, "kind": "port", "sample": txt}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    sizes = {}
    for w in ws_all:
        sizes[w.params.nx] = sizes.get(w.params.nx, 0) + 1
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (ran_2 uniform noise per member, seeds -1..-96; member parameters drawn with ran_2 seed -3)",
        "config": {"workload": f"landau-ensemble-{len(ws)}x1var", "members": len(ws),
                   "grids": {f"{n}^3": k for n, k in sorted(sizes.items())}, "cells_per_step": cells,
                   "schedules": {f"{n}^3": list(s) for n, s in sorted(scheds.items())},
                   "launch": "one batched launch per kernel and size bucket, buckets on parallel streams, "
                             "8-step CUDA graph replays",
                   "l2": f"device working set {footprint / 2**20:.0f} MiB > 126 MB L2, no flush",
                   "parallelism": (f"members sharded over {world} ranks by grid points "
                                   f"(rank 0: {len(mine)} members, {local_cells} cells)") if world > 1 else "single GPU"},
        "fp64_plain": {"value": value64, "unit": UNIT, "steps": K64, "ms_per_step": ms64 / K64,
                       "fp32_speedup": value / value64},
        "err_vs_fp64": {"c_rel_l2_max_member": err_c, "eta_rel_l2_max_member": err_e, "after_steps": W + K},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": read_traffic(dom + "@ensemble"),
                     "algorithmic_bytes_per_launch": dr["bytes"] / dr["launches"], "kernel_ms_per_launch": dom_ms,
                     "step_algorithmic_bytes": step_bytes, "step_frac": step_bytes / (ms / K / 1e3) / 1e9 / peak},
        "kernels": kernels,
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 2 * cells * 8,
                "d2h_bytes_per_step": 2 * cells * 8 + C.sizeof(P.MeuDiag) * len(ws), "steps": ke,
                "form": "per step: meu_ensemble_set_fields of every member + meu_ensemble_run(1) + "
                        "meu_ensemble_get_fields of every member, pinned host buffers"},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_ensemble(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    K, W = args.steps, args.warmup
    # each "step" of the sample: oracle steps over ensemble members, about 150 s in all
    cc, secs, txt = ensemble_cpu_sample(150.0, threads)
    val = cc / secs / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": K,
        "warmup": W, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (ran_2 uniform noise per member)",
        "config": {"workload": f"landau-ensemble-{ENS_MEMBERS}x1var", "parallelism": "host threads"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": txt},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------- slab-decomposed FFT (multi-GPU)
def run_slab(args):
    """--config 5: f_trans + inv_trans of one grid split over the N ranks in z slabs
    (meu_slab_fft_*, one NCCL all-to-all per transform).  Weak scaling: the grid is
    512 x 512 x (512 N), so every rank holds a 512^3 slab; FP32.  A step is one forward
    and one inverse transform; value = grid cells / step time (max over ranks)."""
    import datetime

    import torch
    import torch.distributed as dist

    from meumapps_ss_b200 import params as P
    from meumapps_ss_b200.slab_fft import SlabFFT

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference's P3DFFT build needs MPI and a "
                              "Fortran compiler, neither of which this image has"}), flush=True)
        return 0
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    n = args.n or 512
    nx, ny, nz = n, n, n * world
    K, W = args.steps, max(3, args.warmup)
    f = SlabFFT(nx, ny, nz, precision=P.PREC_F32)
    g = torch.Generator(device="cuda").manual_seed(1 + rank)
    real = torch.rand(f.real_shape, dtype=torch.float32, device="cuda", generator=g)
    for _ in range(W):
        real = f.inverse(f.forward(real))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    a.record()
    for _ in range(K):
        real = f.inverse(f.forward(real))
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    f.close()
    if rank == 0:
        cells = nx * ny * nz
        print(json.dumps({"metric": "Mcell/s (slab FFT forward + inverse)", "value": cells * K / (ms / 1e3) / 1e6,
                          "unit": "Mcell/s", "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms / K,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic (uniform random slabs)",
                          "config": {"workload": f"slab-fft-{nx}x{ny}x{nz}", "grid": [nx, ny, nz],
                                     "parallelism": f"z slabs over {world} ranks, NCCL all-to-all"}}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------ the reference's own model (KKS)
def run_kks(args):
    """--config 6: the reference's KKS model (plain FP64, 3 variants, heterogeneous
    cubic moduli, deck in its Input.txt format) on a 128^3 grid (--n to change it),
    Langevin noise off and on; one rank.  A step is one time step."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.impl == "reference":
        return run_kks_reference(args)
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.Stream()
    n = args.n or 128
    r = measure_kks(stream, n=n, K=args.steps, W=max(1, args.warmup))
    off = r["noise_off"]
    print(json.dumps({"metric": "Mcell-steps/s (KKS, plain FP64)", "value": off["value"], "unit": UNIT, "n_gpus": 1,
                      "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": off["ms_per_step"],
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic (the reference's InitFields restated, ran_2 with the deck's seed)",
                      "config": {"workload": r["workload"], "grid": r["grid"], "variants": r["variants"]},
                      "noise_on": r["noise_on"], "elastic_iterations_per_step": off["elastic_iterations_per_step"]}),
          flush=True)
    return 0


def run_kks_reference(args):
    """--config 6 --impl reference: the oracle port of the reference's KKS step (FP64,
    all host threads) on the same deck, inputs from the pure-Python set-up mirror; after
    one untimed step, as many of the K steps as fit about two minutes."""
    from meumapps_ss_b200 import configs as CF
    from meumapps_ss_b200 import params as P
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n = args.n or 128
    deck = P.parse_input_txt(CF.kks_input_txt(n, 3, 10 ** 6, radius=max(3, n // 10)))
    p = P.kks_params(deck)
    p.noise_step = 0
    cons, phi = P.init_fields(deck)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    s = O.OracleSim(p)
    s.set_fields(cons, phi)
    t0 = time.perf_counter()
    s.run(1)
    t1 = time.perf_counter() - t0
    k = max(1, min(args.steps, int(120.0 / max(t1, 1e-3))))
    t0 = time.perf_counter()
    s.run(k)
    dt = time.perf_counter() - t0
    s.close()
    value = n ** 3 * k / dt / 1e6
    sample = (f"{k} FP64 KKS time steps of kks-{n}^3-3var-hetero after one untimed step (oracle port, "
              f"{threads} threads; the Fortran/MPI/P3DFFT reference cannot be built in this image)")
    print(json.dumps({"impl": "reference", "metric": "Mcell-steps/s (KKS, plain FP64)", "value": value, "unit": UNIT,
                      "n_gpus": 1, "steps": k, "warmup": 1, "ms_per_step": dt / k * 1e3, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic (the reference's InitFields restated, ran_2 with the deck's seed)",
                      "config": {"workload": f"kks-{n}^3-3var-hetero", "grid": [n, n, n], "variants": 3},
                      "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)
    return 0


def main():
    args = parse()
    if args.config == 5:
        return run_slab(args)
    if args.config == 6:
        return run_kks(args)
    if args.config == 4:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint"}), flush=True)
            return 0
        return run_adjoint_bench(args)
    if args.config == 3:
        return run_reference_ensemble(args) if args.impl == "reference" else run_ensemble(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
