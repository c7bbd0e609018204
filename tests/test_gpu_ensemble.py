"""The batched ensemble (gkm_ensemble_*): cubes of different sizes, Mach and
Reynolds numbers and particle counts stepped together, one launch per stage.

Checks
  * the two reference-generated goldens (12^3 after 5 steps, 16^3 after 10)
    run as members of one ensemble: fields rel-L2 <= 1e-12, particles <= 1e-10
    (the bars of the single-cube parity tests);
  * every member of a ragged ensemble (n = 12..40, one member without
    particles) against the same cube stepped alone through gkm_step:
    fields rel-L2 <= 1e-13, particles <= 1e-12, clocks equal (the per-member
    arithmetic is the single-cube code; the report says whether it was bit
    for bit);
  * the same for the mixed-precision form (FP32 flux): fields <= 3e-6 and
    particles <= 1e-6 against the single mixed cube (FP32 rounding differs
    between the two kernel builds, and each build is about 1e-6 from FP64
    after these steps, so two builds may differ by twice that), fields <= 1e-5
    against FP64;
  * graph replay == the event-timed path; autotuning keeps the state;
  * member handles refuse gkm_destroy / gkm_set_stream and a member stepped
    outside the ensemble stops the ensemble with GKM_ERR_STATE.
"""
import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic
from dns_gkm_lpt_b200.solver import Ensemble, GkmError, Solver
from tests.gpu_helpers import analytic_case, case, rel_l2, w0_of

pytestmark = pytest.mark.gpu

# (n, Mt, Re, seed, particles)
RAGGED = [(16, 0.3, 40.0, 11, 200), (24, 0.5, 20.0, 12, 0), (20, 0.1, 80.0, 13, 150), (40, 0.4, 60.0, 14, 300),
          (12, 0.6, 30.0, 15, 64)]


def _member_inputs(spec):
    n, Mt, Re, seed, npart = spec
    P, W0 = case(n, Mt, Re, seed)
    pos = ic.particles_to_reference_order(ic.make_particles(npart, seed)) if npart else None
    return P, W0, pos


def _outputs(s, npart):
    W = s.download_state()
    pos, U = s.particles_download() if npart else (None, None)
    return W, pos, U, s.clock()


def test_ensemble_matches_reference_goldens(golden):
    gs = [golden["field_12"], golden["field_16"]]
    members, inputs = [], []
    for g in gs:
        P, W0 = w0_of(g)
        pos0 = ic.particles_to_reference_order(g["particles_xyz"])
        members.append({"params": P, "cfl": float(g["cfl"]), "max_particles": len(pos0)})
        inputs.append((W0, pos0))
    with Ensemble(members) as E:
        for m, (W0, pos0) in enumerate(inputs):
            E[m].upload_state(W0)
            E[m].particles_upload(pos0)
        done = 0
        for m, g in enumerate(gs):
            E.step(len(g["dt"]) - done)
            done = len(g["dt"])
            W = E[m].download_state()
            pos, U = E[m].particles_download()
            err = rel_l2(W, g["W_final"])
            order = np.argsort(g["tags"])
            print(f"member n={int(g['n'])} after {done} steps: rel-L2 {err.max():.3e}")
            assert err.max() <= 1e-12
            assert np.abs(pos - g["pos_final"][order]).max() <= 1e-10
            assert np.abs(U - g["U_final"][order]).max() <= 1e-10 * max(1.0, np.abs(g["U_final"]).max())


def _single_runs(precision, nsteps):
    out = []
    for spec in RAGGED:
        P, W0, pos = _member_inputs(spec)
        with Solver(P, cfl=0.5, max_particles=spec[4], precision=precision) as s:
            s.upload_state(W0)
            if pos is not None:
                s.particles_upload(pos)
            s.step(nsteps)
            out.append(_outputs(s, spec[4]))
    return out


def _ensemble_runs(precision, nsteps, timed=False, autotune=False):
    members = [{"params": _member_inputs(s)[0], "cfl": 0.5, "max_particles": s[4]} for s in RAGGED]
    with Ensemble(members, precision=precision) as E:
        for m, spec in enumerate(RAGGED):
            _, W0, pos = _member_inputs(spec)
            E[m].upload_state(W0)
            if pos is not None:
                E[m].particles_upload(pos)
        if autotune:
            cfg = E.autotune(1)
            print("ensemble sweep config:", cfg)
        if timed:
            E.step_timed(nsteps)
        else:
            E.step(nsteps)
            assert E.launch_count() == nsteps * 8
        return [_outputs(E[m], spec[4]) for m, spec in enumerate(RAGGED)]


def _compare(a, b, field_tol, part_tol, label, clock_tol=1e-13):
    report = []
    for m, (x, y) in enumerate(zip(a, b)):
        err = rel_l2(x[0], y[0]).max()
        same = bool(np.array_equal(x[0], y[0]))
        assert err <= field_tol, (label, m, err)
        if x[1] is not None:
            assert np.abs(x[1] - y[1]).max() <= part_tol, (label, m)
            assert np.abs(x[2] - y[2]).max() <= part_tol * max(1.0, np.abs(y[2]).max()), (label, m)
            same &= bool(np.array_equal(x[1], y[1]))
        t0, dt0, it0 = x[3]
        t1, dt1, it1 = y[3]
        assert it0 == it1
        assert abs(t0 - t1) <= clock_tol * abs(t1) and abs(dt0 - dt1) <= clock_tol * abs(dt1)
        report.append(f"n={x[0].shape[1] - 6}: {'bitwise' if same else f'{err:.1e}'}")
    print(f"{label}: " + ", ".join(report))


def test_ensemble_members_match_single_cubes_fp64():
    single = _single_runs(0, 6)
    ens = _ensemble_runs(0, 6)
    _compare(ens, single, 1e-13, 1e-12, "FP64 ensemble vs single cubes")
    timed = _ensemble_runs(0, 6, timed=True)
    _compare(timed, ens, 1e-13, 1e-12, "FP64 ensemble timed path vs graph")


def test_ensemble_members_match_single_cubes_mixed():
    single = _single_runs(1, 6)
    ens = _ensemble_runs(1, 6)
    _compare(ens, single, 3e-6, 1e-6, "mixed ensemble vs single mixed cubes", clock_tol=1e-6)
    fp64 = _single_runs(0, 6)
    for m, (x, y) in enumerate(zip(ens, fp64)):
        assert rel_l2(x[0], y[0]).max() <= 1e-5, m


def test_ensemble_autotune_keeps_state():
    base = _ensemble_runs(0, 3)
    tuned = _ensemble_runs(0, 3, autotune=True)
    _compare(tuned, base, 1e-13, 1e-12, "FP64 ensemble autotuned vs default")


def test_ensemble_member_rules():
    members = [{"params": _member_inputs(s)[0], "cfl": 0.5, "max_particles": s[4]} for s in RAGGED[:2]]
    with Ensemble(members) as E:
        for m, spec in enumerate(RAGGED[:2]):
            E[m].upload_state(_member_inputs(spec)[1])
        L = E.L
        assert L.gkm_destroy(E[0].h) == 5          # GKM_ERR_STATE
        assert L.gkm_set_stream(E[0].h, None) == 5
        E.step(1, with_particles=False)
        E[1].evolve_eulerian(1)                    # member stepped alone
        with pytest.raises(GkmError) as ei:
            E.step(1)
        assert ei.value.status == 5
        assert "outside the ensemble" in str(ei.value)


def test_ensemble_eulerian_only_equals_evolve_eulerian():
    specs = RAGGED[:3]
    single = []
    for spec in specs:
        P, W0, _ = _member_inputs(spec)
        with Solver(P, cfl=0.5) as s:
            s.upload_state(W0)
            s.evolve_eulerian(4)
            single.append(s.download_state())
    members = [{"params": _member_inputs(s)[0], "cfl": 0.5} for s in specs]
    with Ensemble(members) as E:
        for m, spec in enumerate(specs):
            E[m].upload_state(_member_inputs(spec)[1])
        E.step(4, with_particles=False)
        for m in range(len(specs)):
            assert rel_l2(E[m].download_state(), single[m]).max() <= 1e-13


def test_ensemble_warp_specialized_sweeps_match_single_cubes():
    """Window variant 2 in the ensemble: the persistent warp-specialized kernel for x and y (each
    warpgroup looping over the work items with its own register budget), 16 x 16 windows for z; the
    members must match single cubes stepped with the warp-specialized sweeps (bitwise where the
    arithmetic is the same; the single cubes' z sweep is the warp-specialized kernel there, so
    within rounding) and the plain ensemble."""
    members = [{"params": _member_inputs(s)[0], "cfl": 0.5, "max_particles": s[4]} for s in RAGGED]
    out = {}
    for var in (1, 2):
        with Ensemble(members) as E:
            E.set_sweep_config([(var, 16)] * 3)
            assert [c["variant"] for c in E.sweep_config()] == [var] * 3
            for m, spec in enumerate(RAGGED):
                _, W0, pos = _member_inputs(spec)
                E[m].upload_state(W0)
                if pos is not None:
                    E[m].particles_upload(pos)
            E.step(5)
            out[var] = [_outputs(E[m], spec[4]) for m, spec in enumerate(RAGGED)]
    _compare(out[2], out[1], 1e-14, 1e-12, "FP64 ensemble variant 2 vs variant 1")
    single = []
    for spec in RAGGED:
        P, W0, pos = _member_inputs(spec)
        with Solver(P, cfl=0.5, max_particles=spec[4]) as s:
            s.set_sweep_config([(2, 16)] * 3)
            s.upload_state(W0)
            if pos is not None:
                s.particles_upload(pos)
            s.step(5)
            single.append(_outputs(s, spec[4]))
    _compare(out[2], single, 1e-14, 1e-12, "FP64 ensemble variant 2 vs single cubes variant 2")
    with Ensemble(members[:1]) as E, pytest.raises(GkmError):
        E.set_sweep_config([(3, 16)] * 3)


@pytest.mark.parametrize("precision,variant,tol", [(0, 1, 1e-13), (0, 2, 1e-13), (1, 0, 1e-6)])
def test_ensemble_with_odd_grid_members_matches_single_cubes(precision, variant, tol):
    """Odd n gives an odd extent nt, so those members have no tensor maps: their work items take
    the per-element copies inside the same persistent launches whose other items use tensor copies
    (FP64: the plain kernel for variant 1; for variant 2 the warp-specialized x and y kernel, whose
    producer and consumer warpgroups decide per item; mixed: its one window variant)."""
    cases = [analytic_case(13, 61), case(16, 0.3, 40.0, 62), analytic_case(21, 63), case(24, 0.4, 30.0, 64)]
    single = []
    for P, W0 in cases:
        with Solver(P, cfl=0.5, precision=precision) as s:
            s.set_sweep_config([(variant, 16)] * 3)
            s.upload_state(W0)
            s.evolve_eulerian(4)
            single.append(s.download_state())
    with Ensemble([{"params": P, "cfl": 0.5} for P, _ in cases], precision=precision) as E:
        E.set_sweep_config([(variant, 16)] * 3)
        for m, (_, W0) in enumerate(cases):
            E[m].upload_state(W0)
        E.step(4, with_particles=False)
        for m in range(len(cases)):
            assert rel_l2(E[m].download_state(), single[m]).max() <= tol, m

