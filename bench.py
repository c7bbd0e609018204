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

--impl reference: the reference's own CPU code (oracle/_ref, compiled from
the reference sources) on the host cores, one 64^3 cube per process, all
processes concurrent, each timed step one reference step.
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
REF_N = 64                   # reference CPU sample: one 64^3 cube per process
REF_PART = N_PART * REF_N ** 3 // N_CELLS ** 3   # same particle density
HBM_PEAK_GBS = 6550.7        # measured copy bandwidth of this pool's B200s
# DRAM bytes per cell of one sweep launch, from the ncu capture of a 128^3 case (traffic scales with
# the cells a launch processes; mean over the x, y, z sweeps)
SWEEP_DRAM_BYTES_PER_CELL = 97.9   # mean DRAM bytes per cell of the x, y, z sweep launches (ncu, 128^3)


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


def workload(n=N_CELLS, npart=N_PART, precision="fp64"):
    Mt, Re = case_of(n)
    form = "FP64 drop-in" if precision == "fp64" else "mixed precision (FP32 WENO + flux, FP64 state)"
    nt = n + 6
    return {"workload": f"{n}^3 periodic cube, {form}, Mt {Mt}, Re_lambda {Re:g}, {npart} particles, "
                        f"cfl {CFL}, natural_ghost3 splines",
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
def _ref_worker(args):
    """One process: the reference CPU build on one seeded REF_N^3 cube."""
    n, npart, seed, warm, steps = args
    sys.path.insert(0, ROOT)
    from dns_gkm_lpt_b200 import ic
    from oracle import oracle as O
    d = tempfile.mkdtemp(prefix="gkm_ref_")
    P, u, v, w, rho, p = ic.make_field(n, MT, RE, seed)
    ic.write_reference_inputs(d, P, u, v, w, rho, p, ic.make_particles(npart, seed))
    ref = O.ReferenceRun(d, CFL, True)
    if warm:
        ref.time_steps(warm)
    return [ref.time_steps(1) for _ in range(steps)]


def run_reference(workers: int, warm: int, steps: int, n=REF_N, npart=REF_PART):
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
    return {"gcell": gcell, "psteps": psteps, "ms_per_step": ms_step, "workers": workers, "wall_s": wall}


def reference_arm(args, world: int):
    ncpu = os.cpu_count() or 1
    workers = max(1, min(ncpu, 96))
    # a bounded sample: a reference step of a 64^3 cube takes ~2 s on one core, so at most 10 timed
    # and 1 warm-up step per process keep the arm within a minute whatever --steps says
    ref_steps, ref_warm = max(1, min(args.steps, 10)), min(args.warmup, 1)
    r = run_reference(workers, ref_warm, ref_steps)
    sample = (f"{REF_N}^3 cube per process (same spectrum recipe, Mt {MT}, Re_lambda {RE:g}), {REF_PART} particles "
              f"per process, {workers} concurrent processes, {ref_steps} timed reference steps each "
              f"after {ref_warm} warm-up ({r['wall_s']:.1f} s wall)")
    line = {"impl": "reference", "metric": "Gcell-updates/s", "value": r["gcell"], "unit": "Gcell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded solenoidal field (init_DNS recipe), uniform particles",
            "config": workload(), "particle_steps_per_s": r["psteps"],
            "cpu_baseline": {"value": r["gcell"], "unit": "Gcell-updates/s", "cores": workers, "kind": "reference",
                             "sample": sample},
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
    s = Solver(P, cfl=CFL, max_particles=npart, device=local_rank, precision=prec)
    s.set_stream(stream.cuda_stream)
    s.upload_state(W0)
    s.particles_upload(pos0)
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
    do_forms = not args.no_forms and prec == 0
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

    line = {"metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if prec else "f64",
            "data": "synthetic: seeded solenoidal field (init_DNS recipe), uniform particles",
            "config": workload(n, npart, args.precision),
            "particle_steps_per_s": world * npart * args.steps / (part_ms * 1e-3),
            "phases_ms_per_step": {k: v / args.steps for k, v in ph.items()},
            "roofline": {"kernel": "sweep_kernel (x/y/z, one launch each per step)", "bound": "fp32" if prec else "fp64",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic if not prec else None, "flops_per_cell_update": flops_cell,
                         "peak_source": "FMA probe run by this bench (gkm_probe_fma_peak)",
                         "hbm": {"achieved_gbs": bytes_launch / launch_s / 1e9, "peak_gbs": HBM_PEAK_GBS,
                                 "frac": bytes_launch / launch_s / 1e9 / HBM_PEAK_GBS,
                                 "peak_source": "measured copy bandwidth"}},
            "fma_peaks_tflops": {"fp64": fp64_peak, "fp32": fp32_peak},
            "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, "sweep_shapes": sweep_cfg, "forms": forms}
    if world == 1 and not args.no_cpu_baseline:
        workers = max(1, min(os.cpu_count() or 1, 8))
        r = run_reference(workers, 0, 2)
        line["cpu_baseline"] = {"value": r["gcell"], "unit": "Gcell-updates/s", "cores": workers,
                                "kind": "reference",
                                "sample": f"{REF_N}^3 cube per process, same recipe, {REF_PART} particles, 2 steps, "
                                          f"{workers} concurrent processes ({r['wall_s']:.1f} s wall)",
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
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="form of the main line")
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
