"""Benchmark of the DNS_GKM_LPT hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the body of the reference's Evolve loop on a 256^3 periodic cube
(FP64, Mt 0.3, Re_lambda 60, cfl 0.5) with 10^6 Lagrangian particles: x/y/z
fused WENO + gas-kinetic sweeps, halo wrap, dt reduction, velocity splines,
Heun advection.  The state stays resident in HBM; "value" is Gcell-updates/s
of the Eulerian step (n^3 x steps / its device time), "particle_steps_per_s"
the particle part.  "e2e" runs the reference's GPU plug point evolve(W, dt)
through the C ABI with pinned host buffers: H2D of W, one step, D2H of W,
every step.

N > 1 (torchrun): each rank advances its own independent replica (the path
does not shard: no inter-GPU exchange); value sums all ranks over the slowest
rank's time.

"forms" (one GPU): the mixed-precision form on the same 256^3 input; the
batched ensemble (32 cubes of uneven sizes) in FP64 and mixed precision,
against its members stepped one after another and against one cube of the
same cell count;
c2_256_curves, both forms over 200 steps of the 256^3 case with the
PrintStats curves every 10 steps; c3_512, the 512^3 case (Mt 0.5,
Re_lambda 100, 4 x 10^6 particles) over 500 steps in both forms, with the
mixed form's field and curve errors against the FP64 run.

--impl reference: the reference's own CPU code (oracle/_ref, compiled from
the reference sources) on all host cores, one 64^3 cube per process (the
per-cell rate stands in for the 256^3 cube: extrapolated), all processes
concurrent, --warmup untimed and --steps timed reference steps each.  Where
that build is absent, the oracle's C restatement of the Eulerian step runs
instead ("kind": "port").  The GPU arm's cpu_baseline is the same
measurement.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 256
N_PART = 1_000_000
MT, RE, CFL, SEED = 0.3, 60.0, 0.5, 1234
PERTURBATION = 1e-7   # relative size of the long runs' FP64 control perturbation
REF_N = 64                   # reference CPU sample: one 64^3 cube per process
REF_PART = N_PART * REF_N ** 3 // N_CELLS ** 3   # same particle density
C3_PART = 4_000_000          # particles of the 512^3 mixed-precision case
HBM_FALLBACK_GBS = 6650.0    # an earlier copy-bandwidth measurement on these B200s, used only without a
                             # measured-peaks file beside this script
# DRAM bytes per cell of one sweep launch: mean over the x, y, z sweeps of the ncu capture of this
# benchmark's 256^3 cube (83.8, 123.3, 141.4 B; compulsory 80, 120, 120)
SWEEP_DRAM_BYTES_PER_CELL = 116.2


def hbm_peak():
    """(GB/s, source) of the HBM copy bandwidth measured on this machine's GPUs (MEASURED_PEAKS.json
    beside this script, written by the machine's set-up), else the fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            v = float(json.load(f)["hbm_gbs"])
        if v > 0:
            return v, "measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError, KeyError, TypeError):
        pass
    return HBM_FALLBACK_GBS, "fallback: earlier copy-bandwidth measurement (no MEASURED_PEAKS.json)"


# batched ensemble: 16 x 32^3 + 8 x 48^3 + 6 x 64^3 + 2 x 96^3 (4.75 M cells), Mt ~ U[0.1, 0.6],
# Re_lambda ~ U[20, 80], 10^4 particles each; member m uses seed 10000 + m
ENSEMBLE = [(32, 16), (48, 8), (64, 6), (96, 2)]
ENS_PART = 10_000


def ensemble_specs():
    import numpy as np
    rng = np.random.default_rng(10000)
    specs = []
    for n, count in ENSEMBLE:
        for _ in range(count):
            specs.append((n, float(rng.uniform(0.1, 0.6)), float(rng.uniform(20.0, 80.0)), 10000 + len(specs)))
    return specs


def max_over_ranks(values, device=None):
    """Element-wise maximum of per-rank timings over all ranks of the default process group
    (identity without one).  Every rank must call it, in the same order, with the same length."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()) or tdist.get_world_size() == 1:
        return [float(v) for v in values]
    if device is None:
        device = "cuda" if tdist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return t.tolist()


def cells_of(n: int) -> int:
    return n ** 3


# (Mt, Re_lambda) per cube size: 64^3 and 256^3 as the 64^3 / 256^3 cases, 512^3 and 1024^3 the large ones
SIZES = {64: (0.3, 30.0), 256: (MT, RE), 512: (0.5, 100.0), 1024: (0.4, 150.0)}


def case_of(n: int):
    return SIZES.get(n, (MT, RE))


def workload(n=N_CELLS, npart=N_PART, precision="fp64", spline_precision="fp64"):
    Mt, Re = case_of(n)
    form = {"fp64": "FP64 drop-in", "mixed": "mixed precision (FP32 WENO + flux, FP64 state)"}.get(
        precision, "FP64 drop-in and mixed precision from the same field")
    nt = n + 6
    spl = "natural_ghost3 splines" + (", FP32 velocity-spline coefficients" if spline_precision == "fp32" else "")
    return {"workload": f"{n}^3 periodic cube, {form}, Mt {Mt}, Re_lambda {Re:g}, {npart} particles, "
                        f"cfl {CFL}, {spl}",
            "n": n, "particles": npart, "cfl": CFL, "precision": precision, "seed": SEED,
            "l2": f"no flush: resident state 2 x {5 * nt ** 3 * 8 / 1e9:.2f} GB exceeds the 126 MB L2",
            "parallelism": "replicas"}


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------- reference arm ----
def _reference_built() -> bool:
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    return os.path.exists(O.REF_SO)


def _ref_worker(args):
    """One process: the reference CPU build on one seeded REF_N^3 cube, or, where that build is
    absent, the oracle's C restatement of the Eulerian step (no particles) on the same cube."""
    n, npart, seed, warm, steps = args
    sys.path.insert(0, ROOT)
    from dns_gkm_lpt_b200 import ic
    from oracle import oracle as O
    P, u, v, w, rho, p = ic.make_field(n, MT, RE, seed)
    if not os.path.exists(O.REF_SO):
        orc = O.Oracle()
        W = ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))
        par = orc.params(P, CFL)

        def one():
            t = time.perf_counter()
            orc.step(par, W, orc.timestep(par, W))
            return time.perf_counter() - t, 0.0

        for _ in range(warm):
            one()
        return [one() for _ in range(steps)]
    d = tempfile.mkdtemp(prefix="gkm_ref_")
    ic.write_reference_inputs(d, P, u, v, w, rho, p, ic.make_particles(npart, seed))
    ref = O.ReferenceRun(d, CFL, True)
    if warm:
        ref.time_steps(warm)
    return [ref.time_steps(1) for _ in range(steps)]


def run_reference(workers: int, warm: int, steps: int, n=REF_N, npart=REF_PART):
    kind = "reference" if _reference_built() else "port"
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(workers) as pool:
        res = pool.map(_ref_worker, [(n, npart, SEED + 17 * w, warm, steps) for w in range(workers)])
    wall = time.time() - t0
    te = [sum(s[0] for s in r) for r in res]   # Eulerian seconds per worker
    tp = [sum(s[1] for s in r) for r in res]   # particle seconds per worker
    gcell = sum(n ** 3 * steps / t for t in te) / 1e9
    psteps = sum(npart * steps / t for t in tp) if all(t > 0 for t in tp) else None
    ms_step = 1e3 * statistics.mean([(a + b) / steps for a, b in zip(te, tp)])
    return {"gcell": gcell, "psteps": psteps, "ms_per_step": ms_step, "workers": workers, "wall_s": wall,
            "kind": kind}


def reference_sample_text(workers, warm, steps, wall_s, kind="reference"):
    what = ("timed reference steps each" if kind == "reference" else
            "timed Eulerian steps each of the oracle's C restatement (the reference build was absent)")
    return (f"{REF_N}^3 cube per process (same spectrum recipe, Mt {MT}, Re_lambda {RE:g}), {REF_PART} particles "
            f"per process (the 256^3 case's particle density), {workers} concurrent single-rank processes on "
            f"{workers} host cores, {warm} warm-up + {steps} {what} ({wall_s:.1f} s wall); "
            f"Gcell-updates/s is the per-cell rate of those cubes, standing in for the 256^3 cube "
            f"(extrapolated: a 256^3 step takes ~2 min on one core, and the reference parallelises only "
            f"through MPI, which this box lacks)")


def reference_config(workers):
    cfg = workload()
    cfg["workload"] = (f"{cfg['workload']}; reference CPU build measured on {REF_N}^3 cubes, one per process, "
                       f"x {workers} processes (per-cell rate; stands in for 256^3, extrapolated)")
    cfg["reference_sample"] = {"n": REF_N, "processes": workers, "particles_per_process": REF_PART}
    return cfg


def reference_arm(args, world: int):
    workers = max(1, min(os.cpu_count() or 1, 96))
    # every timed step is one reference step of every process (a 64^3 step takes ~2 s on one core)
    r = run_reference(workers, args.warmup, args.steps)
    line = {"impl": "reference", "metric": "Gcell-updates/s", "value": r["gcell"], "unit": "Gcell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded solenoidal field (init_DNS recipe), uniform particles",
            "config": reference_config(workers), "particle_steps_per_s": r["psteps"],
            "cpu_baseline": {"value": r["gcell"], "unit": "Gcell-updates/s", "cores": workers, "kind": r["kind"],
                             "sample": reference_sample_text(workers, args.warmup, args.steps, r["wall_s"], r["kind"])},
            "e2e": {"value": r["gcell"], "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------ batched ensemble --
def _rel_l2(a, b):
    import numpy as np
    sl = slice(3, -3)
    return max(float(np.linalg.norm(a[q, sl, sl, sl] - b[q, sl, sl, sl]) / np.linalg.norm(b[q, sl, sl, sl]))
               for q in range(5))


def batched_forms(args, local_rank: int, stream):
    """C4 ensemble in FP64 and mixed precision (one launch per stage, graph-captured
    step) against the same members stepped one after another as single cubes."""
    import torch

    from dns_gkm_lpt_b200 import ic
    from dns_gkm_lpt_b200.solver import Ensemble, Solver

    specs = ensemble_specs()
    inputs = []
    for n, Mt, Re, seed in specs:
        P, u, v, w, rho, p = ic.make_field(n, Mt, Re, seed)
        inputs.append((P, ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p)),
                       ic.particles_to_reference_order(ic.make_particles(ENS_PART, seed))))
    cells = sum(n ** 3 for n, _, _, _ in specs)
    steps = args.steps
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def eul(ph):
        return ph["sweep_x"] + ph["sweep_y"] + ph["sweep_z"] + ph["halo"]

    def run_ensemble(precision):
        E = Ensemble([{"params": P, "cfl": CFL, "max_particles": ENS_PART} for P, _, _ in inputs],
                     device=local_rank, precision=precision)
        for m, (_, W0, pos) in enumerate(inputs):
            E[m].upload_state(W0)
            E[m].particles_upload(pos)
        cfg = E.autotune(2)
        E.step_timed(args.warmup)
        ph = E.step_timed(steps)
        st = torch.cuda.ExternalStream(E.stream())
        E.step(1)                                  # graph instantiation, untimed
        l0 = E.launch_count()
        ev[0].record(st)
        E.step(steps)
        ev[1].record(st)
        torch.cuda.synchronize()
        graph_ms = ev[0].elapsed_time(ev[1])
        launches = E.launch_count() - l0
        states = [E[m].download_state() for m in range(len(E))]
        tke = [E[m].print_stats()["TKE"] for m in range(len(E))]
        E.close()
        return ph, graph_ms, launches, cfg, states, tke

    def run_sequential():
        ph_sum, graph_ms, states = {}, 0.0, []
        for P, W0, pos in inputs:
            s = Solver(P, cfl=CFL, max_particles=ENS_PART, device=local_rank)
            s.set_stream(stream.cuda_stream)
            s.upload_state(W0)
            s.particles_upload(pos)
            s.autotune(1)
            s.step_timed(args.warmup, True)
            ph = s.step_timed(steps, True)
            for k, v in ph.items():
                ph_sum[k] = ph_sum.get(k, 0.0) + v
            s.step(1)
            ev[0].record(stream)
            s.step(steps)
            ev[1].record(stream)
            torch.cuda.synchronize()
            graph_ms += ev[0].elapsed_time(ev[1])
            states.append(s.download_state())
            s.close()
        return ph_sum, graph_ms, states

    def same_cells_cube(precision):
        # one cube holding the ensemble's cell count (the nearest even n), the same form, no particles
        n_eq = int(round(cells ** (1.0 / 3.0) / 2.0)) * 2
        P, u, v, w, rho, p = ic.make_field(n_eq, MT, RE, SEED)
        s = Solver(P, cfl=CFL, device=local_rank, precision=precision)
        s.set_stream(stream.cuda_stream)
        s.upload_state(ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p)))
        if args.autotune_reps > 0:
            s.autotune(args.autotune_reps)
        s.step_timed(args.warmup, False)
        ph = s.step_timed(steps, False)
        s.close()
        return {"n": n_eq, "value": n_eq ** 3 * steps / (eul(ph) * 1e-3) / 1e9,
                "what": "one cube of the ensemble's cell count, same form"}

    out = {}
    ph64, g64, l64, cfg64, W64, tke64 = run_ensemble(0)
    phs, gs, Ws = run_sequential()
    members = " + ".join(f"{c} x {n}^3" for n, c in ENSEMBLE)
    common = {"members": members, "cells": cells, "particles_per_member": ENS_PART}
    out["batched_fp64"] = dict(common, **{
        "value": cells * steps / (eul(ph64) * 1e-3) / 1e9, "unit": "Gcell-updates/s",
        "particle_steps_per_s": len(specs) * ENS_PART * steps / ((ph64["splines"] + ph64["particles"]) * 1e-3),
        "graph_ms_per_step": g64 / steps, "graph_launches_per_step": l64 / steps,
        "sequential_single_cubes": {"value": cells * steps / (eul(phs) * 1e-3) / 1e9,
                                    "graph_ms_per_step": gs / steps,
                                    "what": "same members, one handle each, stepped one after another"},
        "speedup_vs_sequential_graph": gs / g64,
        "max_rel_l2_vs_single_cubes": max(_rel_l2(a, b) for a, b in zip(W64, Ws)),
        "sweep_shapes": cfg64})
    eq64 = same_cells_cube(0)
    out["batched_fp64"]["single_cube_same_cells"] = eq64
    out["batched_fp64"]["over_single_cube_same_cells"] = out["batched_fp64"]["value"] / eq64["value"]
    del Ws
    phm, gm, lm, cfgm, Wm, tkem = run_ensemble(1)
    out["batched_mixed"] = dict(common, **{
        "value": cells * steps / (eul(phm) * 1e-3) / 1e9, "unit": "Gcell-updates/s",
        "particle_steps_per_s": len(specs) * ENS_PART * steps / ((phm["splines"] + phm["particles"]) * 1e-3),
        "graph_ms_per_step": gm / steps, "graph_launches_per_step": lm / steps,
        "speedup_vs_sequential_graph": gs / gm,
        "max_rel_l2_vs_fp64": max(_rel_l2(a, b) for a, b in zip(Wm, W64)),
        "max_tke_rel_err_vs_fp64": max(abs(a - b) / b for a, b in zip(tkem, tke64)),
        "steps_compared": args.warmup + 2 * steps + 1, "sweep_shapes": cfgm})
    eqm = same_cells_cube(1)
    out["batched_mixed"]["single_cube_same_cells"] = eqm
    out["batched_mixed"]["over_single_cube_same_cells"] = out["batched_mixed"]["value"] / eqm["value"]
    return out


# ------------------------------------------------ long runs: FP64 vs mixed --
STAT_KEYS = ("TKE", "Diss", "SijSij", "SKEWu", "SKEWv", "SKEWw", "KURTu", "KURTv", "KURTw", "Prms", "Trms", "Vrms")


def long_run_pair(n, npart, steps, seed, local_rank, stream, autotune_reps=2, stats_every=10):
    """The FP64 drop-in and the mixed-precision form advanced from the same seeded field for
    `steps` full steps, with the PrintStats line every `stats_every` steps (as the reference prints it,
    src/update.cpp:135-144, 835-841): per form Gcell-updates/s and particle-steps/s over all steps
    (CUDA events per phase), and the mixed form's errors against the FP64 run: relative L2 of rho,
    rho u, rho v, rho w, rho E and of the velocities u, v, w after the last step, and the largest
    relative difference of every PrintStats curve over the run.  A control run, the FP64 drop-in
    from the same field with relative noise of single-precision rounding size, gives the
    same errors for a difference that no precision choice makes: how far the flow itself grows one.
    Its noise enters after every step, as the mixed form's rounding does."""
    import numpy as np
    import torch

    from dns_gkm_lpt_b200 import ic
    from dns_gkm_lpt_b200.solver import Solver

    Mt, Re = case_of(n)
    dev = f"cuda:{local_rank}"
    if n > 256:
        P, W0 = ic.make_state_device(n, Mt, Re, seed, device=dev)
    else:
        P, u, v, w, rho, p = ic.make_field(n, Mt, Re, seed)
        W0 = ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))
        del u, v, w, rho, p
    pos0 = ic.particles_to_reference_order(ic.make_particles(npart, seed))
    nt = n + 6

    g = torch.Generator(device=dev)
    g.manual_seed(seed + 7)

    def perturb(Wd):
        # the control's step: the state's interior times (1 + PERTURBATION N(0, 1)), seeded, then the
        # periodic ghosts rewrapped; on the solver's stream, between two steps
        with torch.cuda.stream(stream):
            for q in range(5):
                Wd[q, 3:n + 3, 3:n + 3, 3:n + 3] *= 1.0 + PERTURBATION * torch.randn(
                    (n, n, n), generator=g, device=dev, dtype=torch.float64)
            for ax in (1, 2, 3):
                Wd.narrow(ax, 0, 3).copy_(Wd.narrow(ax, n, 3))
                Wd.narrow(ax, n + 3, 3).copy_(Wd.narrow(ax, 3, 3))

    out, finals, curves, pos = {}, {}, {}, {}
    for name, prec in (("fp64", 0), ("mixed", 1), ("fp64_perturbed", 0)):
        s = Solver(P, cfl=CFL, max_particles=npart, device=local_rank, precision=prec)
        s.set_stream(stream.cuda_stream)
        s.upload_state(W0)
        s.particles_upload(pos0)
        cfg = s.autotune(autotune_reps) if autotune_reps > 0 else s.sweep_config()
        curve, ph_sum, done = [], {}, 0
        while done < steps:
            st = s.print_stats()
            curve.append([st["t_over_t0"]] + [st[k] for k in STAT_KEYS])
            k = min(stats_every, steps - done)
            if name == "fp64_perturbed":
                for _ in range(k):
                    s.step(1)
                    perturb(s.device_state())
            else:
                for key, v in s.step_timed(k, True).items():
                    ph_sum[key] = ph_sum.get(key, 0.0) + v
            done += k
        st = s.print_stats()
        curve.append([st["t_over_t0"]] + [st[k] for k in STAT_KEYS])
        Wf = torch.empty((5, nt, nt, nt), dtype=torch.float64, device=dev)
        s.download_state(Wf)
        pos[name] = s.particles_download()[0]
        s.close()
        finals[name] = Wf
        curves[name] = np.array(curve)
        if name == "fp64_perturbed":
            continue
        eul = ph_sum["sweep_x"] + ph_sum["sweep_y"] + ph_sum["sweep_z"] + ph_sum["halo"]
        part = ph_sum["splines"] + ph_sum["particles"]
        out[name] = {"value": n ** 3 * steps / (eul * 1e-3) / 1e9, "unit": "Gcell-updates/s",
                     "particle_steps_per_s": npart * steps / (part * 1e-3),
                     "ms_per_step": ph_sum["total"] / steps,
                     "phases_ms_per_step": {k: v / steps for k, v in ph_sum.items()}, "sweep_shapes": cfg}
    del W0
    sl = (slice(3, nt - 3),) * 3

    def rl2(x, y):
        return float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))

    def field_err(a, b):
        e = {nm: rl2(a[q][sl], b[q][sl]) for q, nm in enumerate(("rho", "rho_u", "rho_v", "rho_w", "rho_E"))}
        for q, nm in ((1, "u"), (2, "v"), (3, "w")):
            e[nm] = rl2(a[q][sl] / a[0][sl], b[q][sl] / b[0][sl])
        return e

    err = field_err(finals["mixed"], finals["fp64"])
    err_control = field_err(finals["fp64_perturbed"], finals["fp64"])
    del finals
    torch.cuda.empty_cache()
    cm, cf, cp = curves["mixed"], curves["fp64"], curves["fp64_perturbed"]

    def curve_errs(c):
        return {k: float(np.max(np.abs(c[:, i + 1] - cf[:, i + 1]) / np.maximum(np.abs(cf[:, i + 1]), 1e-300)))
                for i, k in enumerate(STAT_KEYS)}

    curve_err = curve_errs(cm)
    # kinetic-energy decay: TKE(t) / TKE(0) of each run
    decay_m, decay_f, decay_p = cm[:, 1] / cm[0, 1], cf[:, 1] / cf[0, 1], cp[:, 1] / cp[0, 1]
    decay_err = float(np.max(np.abs(decay_m - decay_f) / decay_f))
    dx = 2 * np.pi / n
    fields_max = max(err[k] for k in ("rho", "u", "v", "w", "rho_E"))
    out.update({
        "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
        "steps": steps, "stats_every": stats_every, "curve_points": len(cf),
        "rel_l2_mixed_vs_fp64": err,
        "curve_max_rel_err_mixed_vs_fp64": curve_err,
        "tke_decay_max_rel_err": decay_err,
        "t_over_t0_final": {"fp64": float(cf[-1, 0]), "mixed": float(cm[-1, 0])},
        "tke_decay_final": {"fp64": float(decay_f[-1]), "mixed": float(decay_m[-1])},
        "particle_pos_max_abs_err": float(np.abs(pos["mixed"] - pos["fp64"]).max()),
        "particle_cells_equal_fraction": float(np.mean(np.all(
            np.floor(pos["mixed"] / dx) == np.floor(pos["fp64"] / dx), axis=1))),
        "bars": {"fields_rel_l2": 1e-5, "tke_decay": 1e-3},
        "within_bars": bool(fields_max < 1e-5 and decay_err < 1e-3),
        "fp64_perturbed_control": {
            "what": f"the FP64 drop-in from the same field, its state's interior multiplied by (1 + "
                    f"{PERTURBATION:g} N(0,1)) after every step (seeded noise of single-precision rounding "
                    "size, as the mixed form's rounding enters every step), against the unperturbed FP64 run",
            "rel_l2_vs_fp64": err_control,
            "curve_max_rel_err_vs_fp64": curve_errs(cp),
            "tke_decay_max_rel_err": float(np.max(np.abs(decay_p - decay_f) / decay_f))},
        "curves": {"columns": ["t_over_t0"] + list(STAT_KEYS),
                   "fp64": cf.tolist(), "mixed": cm.tolist()}})
    return out


# ------------------------------------------------------------- our arm ----
def ours(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch

    from dns_gkm_lpt_b200 import ic, opcount
    from dns_gkm_lpt_b200.solver import Solver, probe_fma_peak

    torch.cuda.set_device(local_rank)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
    n, npart = args.n, args.particles
    Mt, Re = case_of(n)
    prec = 1 if args.precision == "mixed" else 0
    if n > 256:
        # cuFFT-based restatement of the recipe: the NumPy one needs tens of GB of host memory here
        P, W0 = ic.make_state_device(n, Mt, Re, SEED + rank, device=f"cuda:{local_rank}")
        torch.cuda.empty_cache()
    else:
        P, u, v, w, rho, p = ic.make_field(n, Mt, Re, SEED + rank)
        W0 = ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))
        del u, v, w, rho, p
    pos0 = ic.particles_to_reference_order(ic.make_particles(npart, SEED + rank))

    fp64_peak, fp32_peak = probe_fma_peak(local_rank)
    stream = torch.cuda.Stream()
    sp32 = args.spline_precision == "fp32"
    free0 = torch.cuda.mem_get_info(local_rank)[0]
    s = Solver(P, cfl=CFL, max_particles=npart, device=local_rank, precision=prec, spline_precision=1 if sp32 else 0)
    free1 = torch.cuda.mem_get_info(local_rank)[0]
    Ms = (n + 6) + 2   # natural_ghost3 spline grid: N = n + 6 points, N + 2 coefficients per axis
    memory = {"handle_bytes": free0 - free1,
              "spline_coefficient_bytes": 3 * Ms ** 3 * (4 if sp32 else 8),
              "spline_scratch_bytes": Ms * Ms * (n + 6) * 8,
              "spline_coefficient_bytes_fp64": 3 * Ms ** 3 * 8}
    s.set_stream(stream.cuda_stream)
    s.upload_state(W0)
    s.particles_upload(pos0)
    if args.shapes:
        # fixed sweep shapes, e.g. "x=2:64,y=2:64,z=1:64" (window variant : segment length per direction)
        shapes = dict(item.split("=") for item in args.shapes.split(","))
        s.set_sweep_config([tuple(int(v) for v in shapes[d].split(":")) for d in "xyz"])
        sweep_cfg = s.sweep_config()
    else:
        sweep_cfg = s.autotune(args.autotune_reps) if args.autotune_reps > 0 else s.sweep_config()
    s.step_timed(args.warmup, True)
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    sampler.start()
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    l0 = s.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ph = s.step_timed(args.steps, True)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    launches = s.launch_count() - l0
    total_ms = e0.elapsed_time(e1)
    eul_ms = ph["sweep_x"] + ph["sweep_y"] + ph["sweep_z"] + ph["halo"]
    part_ms = ph["splines"] + ph["particles"]
    eul_ms, part_ms, total_ms = max_over_ranks([eul_ms, part_ms, total_ms])
    nt = s.nt
    state_bytes = 5 * nt ** 3 * 8
    # the side forms run on one GPU only (the scaling runs time the main line alone)
    do_forms = not args.no_forms and prec == 0 and world == 1
    # the particle statistics build five more splines (the 41-column property path): at 1024^3 they
    # do not fit beside the state, the velocity splines and the initial field
    with_pstats = n <= 512
    if do_forms:   # FP64 state after warmup + steps, the reference point of the mixed form
        W64 = s.download_state()
        st64 = s.print_stats()
        tke64 = st64["TKE"]
        pos64, _ = s.particles_download()
        pst64 = s.particle_stats() if with_pstats else None

    # end to end through the plug point evolve(W, dt): pinned host W in, one step, W out
    e2e = None
    if not args.no_e2e:
        Wh = torch.empty((5, nt, nt, nt), dtype=torch.float64, pin_memory=True)
        Wn = Wh.numpy()
        s.download_state(Wn)
        dt = s.timestep()
        s.evolve(Wn, dt)   # warm-up of the copy path
        torch.cuda.synchronize()
        if dist:
            tdist.barrier()
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x0.record(stream)
        for _ in range(args.steps):
            s.evolve(Wn, dt)
        x1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks([x0.elapsed_time(x1)])[0]
        if dist:
            tdist.barrier()
        del Wh, Wn
        e2e = {"value": world * n ** 3 * args.steps / (e2e_ms * 1e-3) / 1e9, "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
               "api": "gkm_evolve(h, W, dt): the reference's evolve(W, dev, dt) plug point"}
    clocks = sampler.stop()

    # the mixed-precision form on the same input and step count; error against the FP64 run
    forms = {}
    s.close()
    if do_forms:
        m = Solver(P, cfl=CFL, max_particles=npart, device=local_rank, precision=1)
        m.set_stream(stream.cuda_stream)
        m.upload_state(W0)
        m.particles_upload(pos0)
        m_cfg = m.autotune(args.autotune_reps) if args.autotune_reps > 0 else m.sweep_config()
        m.step_timed(args.warmup, True)
        mph = m.step_timed(args.steps, True)
        Wm = m.download_state()
        stm = m.print_stats()
        tkem = stm["TKE"]
        posm, _ = m.particles_download()
        pstm = m.particle_stats() if with_pstats else None
        m.close()
        sl = slice(3, -3)
        err = [float(np.linalg.norm(Wm[q, sl, sl, sl] - W64[q, sl, sl, sl]) / np.linalg.norm(W64[q, sl, sl, sl]))
               for q in range(5)]
        m_eul, m_part = max_over_ranks([mph["sweep_x"] + mph["sweep_y"] + mph["sweep_z"] + mph["halo"],
                                        mph["splines"] + mph["particles"]])
        forms["mixed"] = {"value": world * n ** 3 * args.steps / (m_eul * 1e-3) / 1e9, "unit": "Gcell-updates/s",
                          "particle_steps_per_s": world * npart * args.steps / (m_part * 1e-3),
                          "ms_per_step": mph["total"] / args.steps,
                          "phases_ms_per_step": {k: v / args.steps for k, v in mph.items()},
                          "rel_l2_vs_fp64": dict(zip(("rho", "rho_u", "rho_v", "rho_w", "rho_E"), err)),
                          "tke_rel_err_vs_fp64": abs(tkem - tke64) / tke64,
                          # every PrintStats statistic and the particles, against the FP64 run
                          "stats_rel_err_vs_fp64": {k: abs(stm[k] - st64[k]) / max(abs(st64[k]), 1e-300)
                                                    for k in st64 if k != "t_over_t0"},
                          "t_over_t0_rel_err_vs_fp64": abs(stm["t_over_t0"] - st64["t_over_t0"]) / st64["t_over_t0"],
                          "particle_stats_rel_err_vs_fp64": {k: abs(pstm[k] - pst64[k]) / max(abs(pst64[k]), 1e-300)
                                                             for k in ("TKE", "SijSij", "SKEWu", "SKEWw")}
                                                            if with_pstats else None,
                          "particle_pos_max_abs_err_vs_fp64": float(np.abs(posm - pos64).max()),
                          "particle_cells_equal_fraction": float(np.mean(np.all(
                              np.floor(posm / P.dx) == np.floor(pos64 / P.dx), axis=1))),
                          "steps_compared": args.warmup + args.steps, "sweep_shapes": m_cfg}
        del W64, Wm
        if not args.no_batched:
            forms.update(batched_forms(args, local_rank, stream))
        if args.c2_steps > 0:
            # the 256^3 case over its full run: PrintStats curves of both forms every 10 steps
            forms["c2_256_curves"] = dict(long_run_pair(256, N_PART, args.c2_steps, SEED, local_rank, stream,
                                                        args.autotune_reps),
                                          config=workload(256, N_PART))
        if args.c3_steps > 0:
            # the mixed-precision target case: 512^3, Mt 0.5, Re_lambda 100, 4 x 10^6 particles
            forms["c3_512"] = dict(long_run_pair(512, C3_PART, args.c3_steps, SEED + 512, local_rank, stream,
                                                 args.autotune_reps),
                                   config=workload(512, C3_PART, "both"))
        fp64_256 = world * n ** 3 * args.steps / (eul_ms * 1e-3) / 1e9
        for key in ("batched_fp64", "batched_mixed"):
            if key in forms:
                forms[key]["over_fp64_single_cube_256"] = forms[key]["value"] / fp64_256
                if "c3_512" in forms:
                    forms[key]["over_fp64_single_cube_512"] = forms[key]["value"] / forms["c3_512"]["fp64"]["value"]
    if rank != 0:
        return

    cells = n ** 3
    value = world * cells * args.steps / (eul_ms * 1e-3) / 1e9
    oc = opcount.load()
    flops_cell = oc["flops_per_cell_update"]
    sweep_ms = ph["sweep_x"] + ph["sweep_y"] + ph["sweep_z"]
    launch_s = sweep_ms * 1e-3 / (3 * args.steps)          # average sweep launch
    flops_launch = flops_cell * cells / 3                   # one of the three sweeps
    achieved = flops_launch / launch_s / 1e12
    bytes_launch = (80 + 120 + 120) / 3 * cells             # compulsory W read + accumulator traffic
    traffic = None if SWEEP_DRAM_BYTES_PER_CELL is None else SWEEP_DRAM_BYTES_PER_CELL * cells
    peak = fp32_peak if prec else fp64_peak
    hbm_gbs, hbm_src = hbm_peak()

    line = {"metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if prec else "f64",
            "data": "synthetic: seeded solenoidal field (init_DNS recipe), uniform particles",
            "config": workload(n, npart, args.precision, args.spline_precision),
            "particle_steps_per_s": world * npart * args.steps / (part_ms * 1e-3),
            "memory": memory,
            "phases_ms_per_step": {k: v / args.steps for k, v in ph.items()},
            "roofline": {"kernel": "sweep_kernel (x/y/z, one launch each per step)", "bound": "fp32" if prec else "fp64",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic if not prec else None, "flops_per_cell_update": flops_cell,
                         "peak_source": "FMA probe run by this bench (gkm_probe_fma_peak)",
                         "hbm": {"achieved_gbs": bytes_launch / launch_s / 1e9, "peak_gbs": hbm_gbs,
                                 "frac": bytes_launch / launch_s / 1e9 / hbm_gbs, "peak_source": hbm_src}},
            "fma_peaks_tflops": {"fp64": fp64_peak, "fp32": fp32_peak},
            "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, "sweep_shapes": sweep_cfg, "forms": forms}
    if world == 1 and not args.no_cpu_baseline:
        # the same measurement as --impl reference: all host cores, the same steps and warm-up
        workers = max(1, min(os.cpu_count() or 1, 96))
        r = run_reference(workers, args.warmup, args.steps)
        line["cpu_baseline"] = {"value": r["gcell"], "unit": "Gcell-updates/s", "cores": workers,
                                "kind": r["kind"],
                                "sample": reference_sample_text(workers, args.warmup, args.steps, r["wall_s"], r["kind"]),
                                "particle_steps_per_s": r["psteps"]}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_CELLS)
    ap.add_argument("--particles", type=int, default=N_PART)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed-precision and batched forms")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched ensemble forms")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer plug-point measurement")
    ap.add_argument("--c2-steps", type=int, default=200,
                    help="steps of the 256^3 FP64-vs-mixed curve comparison (0 skips it)")
    ap.add_argument("--c3-steps", type=int, default=500,
                    help="steps of the 512^3 FP64-vs-mixed run with its error budget (0 skips it)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="form of the main line")
    ap.add_argument("--spline-precision", default="fp64", choices=["fp64", "fp32"],
                    help="velocity-spline coefficients of the main line (fp32: same FP64 solves, stored rounded)")
    ap.add_argument("--shapes", default="",
                    help="fixed sweep shapes of the main line instead of the autotuner's, e.g. x=2:64,y=2:64,z=1:64 "
                         "(window variant:segment length)")
    ap.add_argument("--autotune-reps", type=int, default=2,
                    help="timed launches per sweep shape; 0 keeps the default shapes (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
