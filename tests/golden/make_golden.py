"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs the reference CPU sources compiled by oracle/Makefile (oracle/_ref/
libgkm_ref.so, built from the reference tree in place) on seeded inputs and
stores inputs and outputs as .npz.  The reference ships no tests, fixtures or
golden data of its own, so these are the pins for the oracle restatement.

    python tests/golden/make_golden.py        (needs the reference tree to build oracle/_ref)

Cases
  field_16 : 16^3, Mt 0.3, Re_lambda 30, cfl 0.5, 64 particles, 10 steps of Evolve's loop body
  field_12 : 12^3, Mt 0.6, Re_lambda 20, cfl 0.3, 24 particles, 5 steps
  faces    : single-face flux() and ApplyWENO() inputs/outputs (stencils cut from field_16 plus edge cases)
  outputs_12 : the field_12 case at iteration 0 and after 3 steps: getParticleProp table,
             GetParticleStats, and the files of writeField / writeParticleData (+ T file) /
             WriteReInit as bytes
  curve_32 : 32^3, Mt 0.3, Re_lambda 30, cfl 0.5, 200 steps: the PrintStats line every 10 steps
  curve_64 : 64^3, Mt 0.3, Re_lambda 30, cfl 0.5, 100 steps (the 64^3 benchmark case), same

    python tests/golden/make_golden.py --curves    (only the two curve cases; several minutes)
    python tests/golden/make_golden.py --outputs   (only outputs_12)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from dns_gkm_lpt_b200 import ic  # noqa: E402

CASES = {
    "field_16": dict(n=16, Mt=0.3, Re=30.0, seed=1234, np=64, cfl=0.5, steps=10),
    "field_12": dict(n=12, Mt=0.6, Re=20.0, seed=99, np=24, cfl=0.3, steps=5),
}


def field_case(name: str, c: dict) -> dict:
    d = O.tmpdir()
    P, u, v, w, rho, p = ic.make_field(c["n"], c["Mt"], c["Re"], c["seed"])
    xyz = ic.make_particles(c["np"], c["seed"])
    ic.write_reference_inputs(d, P, u, v, w, rho, p, xyz)
    ref = O.ReferenceRun(d, c["cfl"], True)
    sl = slice(3, -3)
    out = dict(n=c["n"], cfl=c["cfl"], gam=P.gam, den0=P.den0, Mt=P.Mt, Re=P.Re, mu0=P.mu0, p0=P.p0, t0=P.t0,
               u=u, v=v, w=w, particles_xyz=xyz)
    stats0 = ref.stats()
    dts1, _ = ref.run(1)
    out["W_step1"] = ref.W()[:, sl, sl, sl]
    dts_rest, _ = ref.run(c["steps"] - 1)
    out["W_final"] = ref.W()[:, sl, sl, sl]
    out["dt"] = np.concatenate([dts1, dts_rest])
    out["dt_next"] = ref.dt
    ref.particle_props()
    pos, U, tags = ref.particles(c["np"] * 2)
    out.update(pos_final=pos, U_final=U, tags=tags, stats_step0=stats0, stats_final=ref.stats())
    return out


CURVES = {
    "curve_32": dict(n=32, Mt=0.3, Re=30.0, seed=4321, cfl=0.5, steps=200),
    "curve_64": dict(n=64, Mt=0.3, Re=30.0, seed=1235, cfl=0.5, steps=100),
}


def curve_case(c: dict) -> dict:
    """Long run of Evolve's loop body (no particles): dt of every step and the
    PrintStats line at iterations 0, 10, 20, ... (gkmref_run)."""
    d = O.tmpdir()
    P, u, v, w, rho, p = ic.make_field(c["n"], c["Mt"], c["Re"], c["seed"])
    ic.write_reference_inputs(d, P, u, v, w, rho, p, None)
    ref = O.ReferenceRun(d, c["cfl"], False)
    dts, stats = ref.run(c["steps"])
    return dict(n=c["n"], cfl=c["cfl"], gam=P.gam, den0=P.den0, Mt=P.Mt, Re=P.Re, mu0=P.mu0, p0=P.p0, t0=P.t0,
                seed=c["seed"], steps=c["steps"], dt=dts, stats=stats)


def _read(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        return np.frombuffer(f.read(), dtype=np.uint8)


def outputs_case() -> dict:
    c = CASES["field_12"]
    d = O.tmpdir()
    P, u, v, w, rho, p = ic.make_field(c["n"], c["Mt"], c["Re"], c["seed"])
    ic.write_reference_inputs(d, P, u, v, w, rho, p, ic.make_particles(c["np"], c["seed"]))
    ref = O.ReferenceRun(d, c["cfl"], True)
    out = {}
    for it in (0, 3):
        if it:
            ref.run(it)
        props, tags = ref.particle_table(c["np"] * 2)
        out[f"props_{it}"] = props
        out[f"tags_{it}"] = tags
        out[f"pstats_{it}"] = ref.particle_stats()
        od = O.tmpdir()
        ref.write_outputs(od)
        out[f"field_{it}"] = _read(os.path.join(od, "Results", "Field", f"Field_0_{it}"))
        out[f"particles_{it}"] = _read(os.path.join(od, "Results", "Particles", f"P_0_{it}"))
        out[f"time_{it}"] = _read(os.path.join(od, "Results", "Time", f"T_{it}"))
        out[f"reinit_{it}"] = _read(os.path.join(od, "InitialCondition", "Init000"))
    return out


def face_inputs(rng, W, nt):
    """Cut real WENO stencils and flux inputs out of a ghost-extended field."""
    stencils = []
    for _ in range(48):
        j, i, k = rng.integers(3, nt - 6, size=3)
        d = rng.integers(0, 3)
        s = []
        for o in range(-2, 4):
            idx = [j, i, k]
            idx[d] += o
            s.append(W[:, idx[0], idx[1], idx[2]])
        stencils.append(np.array(s))
    return np.array(stencils)


def faces_case(field_W: np.ndarray, P, cfl: float) -> dict:
    rng = np.random.default_rng(2024)
    nt = field_W.shape[1]
    stencils = face_inputs(rng, field_W, nt)
    # edge cases: a uniform stencil (all smoothness indicators 0) and a density/energy jump
    uni = np.tile(stencils[0][2], (6, 1))
    jump = stencils[1].copy()
    jump[3:, 0] *= 1.5
    jump[3:, 4] *= 1.3
    stencils = np.concatenate([stencils, uni[None], jump[None]])
    d = O.tmpdir()
    Pf, u, v, w, rho, p = ic.make_field(8, 0.3, 30.0, 5)
    ic.write_reference_inputs(d, Pf, u, v, w, rho, p, None)
    ref = O.ReferenceRun(d, cfl, False)
    wl, wr = [], []
    for s in stencils:
        a, b = ref.weno(s, P.gam)
        wl.append(a)
        wr.append(b)
    wl, wr = np.array(wl), np.array(wr)
    # flux inputs: face states from the reconstructions, slopes of realistic size
    nf = len(stencils)
    dx = 2 * np.pi / 16
    dt = 3e-4
    WL = stencils[:, 2]
    WR = stencils[:, 3]
    DW = rng.normal(size=(nf, 6, 5)) * np.abs(WL)[:, None, :] * 0.3 / dx
    DW[-2] = 0.0  # uniform flow: zero slopes
    tau = rng.uniform(1e-6, 5e-5, size=nf)
    F = []
    for f in range(nf):
        F.append(ref.flux(WL[f], WR[f], wl[f], wr[f], DW[f, 0], DW[f, 1], DW[f, 2], DW[f, 3], DW[f, 4], DW[f, 5],
                          tau[f], dt, dx, P.gam))
    return dict(stencils=stencils, Wl=wl, Wr=wr, WL=WL, WR=WR, DW=DW, tau=tau, dt=dt, dx=dx, gam=P.gam,
                F=np.array(F))


def main() -> None:
    O.build(ref=True)
    if "--outputs" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "outputs_12.npz"), **outputs_case())
        print("outputs_12 written")
        return
    if "--curves" in sys.argv:
        for name, c in CURVES.items():
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **curve_case(c))
            print(name, "written")
        return
    results = {}
    for name, c in CASES.items():
        results[name] = field_case(name, c)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **results[name])
        print(name, "written")
    r = results["field_16"]
    P = ic.Params(n=16, gam=r["gam"], den0=r["den0"], Mt=r["Mt"], Re=r["Re"], mu0=r["mu0"], p0=r["p0"], t0=r["t0"])
    W0 = ic.embed_ghost(ic.primitive_to_conserved(P, r["u"], r["v"], r["w"], np.ones_like(r["u"]),
                                                  np.full_like(r["u"], P.p0)))
    np.savez_compressed(os.path.join(HERE, "faces.npz"), **faces_case(W0, P, 0.5))
    print("faces written")


if __name__ == "__main__":
    main()
