"""Parity of the CUDA path (libgkm_b200.so through the C ABI) with the
reference's CPU build (golden vectors) and with the CPU oracle.

Tolerances (FP64 drop-in):
  * fields after 1 and 10 steps: relative L2 per conserved component <= 1e-12
    (the parity bar of the FP64 form); the CUDA path rounds differently (reciprocals, FMA,
    reorganised moment sums) but computes the same algorithm;
  * single-face flux: |dF| <= 1e-11 * max|F| of the face; WENO faces 1e-13 relative;
  * spline coefficients: bit-exact with the oracle (same rounding order);
  * particle cell indices: exact; positions 1e-10 absolute (they live in [0, 2 pi));
  * PrintStats moments: 1e-10 relative.
"""
import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic
from dns_gkm_lpt_b200.solver import GkmError, Solver, flux_faces, weno_faces
from tests.gpu_helpers import analytic_case, case, params_of, rel_l2, w0_of

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12


def test_weno_faces_match_reference(golden):
    f = golden["faces"]
    Wl, Wr = weno_faces(f["stencils"], float(f["gam"]))
    for got, ref in ((Wl, f["Wl"]), (Wr, f["Wr"])):
        scale = np.abs(ref).max(axis=1, keepdims=True)
        assert np.all(np.abs(got - ref) <= 1e-13 * np.maximum(np.abs(ref), 1e-3 * scale))


def test_flux_faces_match_reference(golden):
    f = golden["faces"]
    nf = len(f["F"])
    inp = np.concatenate([f["WL"], f["WR"], f["Wl"], f["Wr"], f["DW"].reshape(nf, 30), f["tau"][:, None]], axis=1)
    F = flux_faces(inp, float(f["gam"]), float(f["dt"]), float(f["dx"]))
    err = np.abs(F - f["F"]).max(axis=1) / np.abs(f["F"]).max(axis=1)
    assert err.max() <= 1e-11, err.max()


@pytest.mark.parametrize("name", ["field_16", "field_12"])
def test_field_and_particles_match_reference(golden, name):
    g = golden[name]
    P, W0 = w0_of(g)
    pos0 = ic.particles_to_reference_order(g["particles_xyz"])
    with Solver(P, cfl=float(g["cfl"]), max_particles=len(pos0)) as s:
        s.upload_state(W0)
        s.particles_upload(pos0)
        s.step(1)
        assert rel_l2(s.download_state(), g["W_step1"]).max() <= FIELD_TOL
        s.step(len(g["dt"]) - 1)
        W = s.download_state()
        assert rel_l2(W, g["W_final"]).max() <= FIELD_TOL
        t, dt_last, it = s.clock()
        assert it == len(g["dt"])
        assert dt_last == pytest.approx(g["dt"][-1], rel=1e-13)
        # the reference's time accounting: each step adds the dt of the next one
        # (src/update.cpp:167-168, timestep(W); t += dt)
        assert t == pytest.approx(g["dt"][1:].sum() + float(g["dt_next"]), rel=1e-13)
        assert s.timestep() == pytest.approx(float(g["dt_next"]), rel=1e-13)
        pos, U = s.particles_download()
    order = np.argsort(g["tags"])
    ref_pos, ref_U = g["pos_final"][order], g["U_final"][order]
    dx = P.dx
    assert np.array_equal(np.floor(pos / dx).astype(int), np.floor(ref_pos / dx).astype(int))
    assert np.abs(pos - ref_pos).max() <= 1e-10
    assert np.abs(U - ref_U).max() <= 1e-10 * np.abs(ref_U).max()


def test_stats_match_reference(golden):
    g = golden["field_16"]
    P, W0 = w0_of(g)
    ref = g["stats_step0"]
    with Solver(P, cfl=float(g["cfl"])) as s:
        s.upload_state(W0)
        st = s.print_stats()
    for k, i in (("TKE", 1), ("Diss", 2), ("SijSij", 3), ("SKEWu", 4), ("SKEWv", 5), ("SKEWw", 6),
                 ("KURTu", 7), ("KURTv", 8), ("KURTw", 9)):
        assert st[k] == pytest.approx(ref[i], rel=1e-10), k
    assert st["Prms"] == pytest.approx(ref[10], rel=1e-8, abs=1e-12)
    assert st["Trms"] == pytest.approx(ref[11], rel=1e-8, abs=1e-12)


@pytest.mark.parametrize("build", [1, 2])
@pytest.mark.parametrize("mode", [0, 1])
def test_spline_coefficients_bitexact_with_oracle(oracle, golden, mode, build):
    """All three velocity splines, both launch forms of the build (one component per launch,
    or each pass for all three components in one launch)."""
    g = golden["field_12"]
    P, W0 = w0_of(g)
    p = oracle.params(P, 0.5)
    start, dinv = oracle.grid(p, mode)
    with Solver(P, cfl=0.5, spline_mode=mode, spline_build=build) as s:
        s.upload_state(W0)
        s.generate_splines()
        got = [s.spline_coefs(c) for c in range(3)]
    for c in range(3):
        data = W0[1 + c] / W0[0]
        if mode == 1:
            data = np.ascontiguousarray(data[3:-3, 3:-3, 3:-3])
        _, ref = oracle.spline3d(data, mode, start, dinv)
        assert np.array_equal(got[c], ref), c


@pytest.mark.parametrize("build", [1, 2])
@pytest.mark.parametrize("mode", [0, 1])
def test_spline_coefficients_bitexact_on_an_odd_grid(oracle, mode, build):
    """n = 13: lines of 19 (natural) or 13 (periodic) points, an odd count of both lines and
    points per line, in both launch forms."""
    P, W0 = analytic_case(13, 5)
    p = oracle.params(P, 0.5)
    start, dinv = oracle.grid(p, mode)
    with Solver(P, cfl=0.5, spline_mode=mode, spline_build=build) as s:
        s.upload_state(W0)
        s.generate_splines()
        got = [s.spline_coefs(c) for c in range(3)]
    for c in range(3):
        data = W0[1 + c] / W0[0]
        if mode == 1:
            data = np.ascontiguousarray(data[3:-3, 3:-3, 3:-3])
        _, ref = oracle.spline3d(data, mode, start, dinv)
        assert np.array_equal(got[c], ref), c


@pytest.mark.parametrize("mode", [0, 1])
def test_particles_match_oracle_both_spline_modes(oracle, mode):
    P, W0 = case(16, 0.4, 40.0, 31)
    pos0 = ic.particles_to_reference_order(ic.make_particles(200, 31))
    p = oracle.params(P, 0.4)
    Wo = W0.copy()
    r = oracle.run(p, Wo, 6, mode, pos0, stats=False)
    with Solver(P, cfl=0.4, spline_mode=mode, max_particles=200) as s:
        s.upload_state(W0)
        s.particles_upload(pos0)
        s.step(6)
        pos, U = s.particles_download()
        assert rel_l2(s.download_state(), Wo).max() <= FIELD_TOL
    assert np.array_equal(np.floor(pos / P.dx), np.floor(r["pos"] / P.dx))
    assert np.abs(pos - r["pos"]).max() <= 1e-10


def test_64cube_step_matches_oracle(oracle):
    P, W0 = case(64, 0.3, 30.0, 5)
    p = oracle.params(P, 0.5)
    Wo = W0.copy()
    dt = oracle.timestep(p, Wo)
    oracle.step(p, Wo, dt)
    with Solver(P, cfl=0.5) as s:
        s.upload_state(W0)
        assert s.timestep() == dt
        s.evolve_eulerian(1)
        assert rel_l2(s.download_state(), Wo).max() <= FIELD_TOL


@pytest.mark.parametrize("n", [13, 21, 8, 10, 18])
def test_odd_and_small_grids_match_oracle(oracle, n):
    """Odd n: slabs, z boxes and accumulators by per-element copies.  Even n below or just past one
    16 x 16 window (8, 10, 18): the tensor-copy paths with boxes and bricks that reach past the
    grid (elements beyond the tensor not read or written, ghost cells stored back unchanged)."""
    P, W0 = analytic_case(n, 40 + n)
    p = oracle.params(P, 0.5)
    W = W0.copy()
    r = oracle.run(p, W, 3, 0, None, stats=False)
    with Solver(P, cfl=0.5) as s:
        s.upload_state(W0)
        s.evolve_eulerian(3)
        Wg = s.download_state()
        _, dt_last, it = s.clock()
    assert it == 3 and dt_last == pytest.approx(r["dt"][-1], rel=1e-13)
    assert rel_l2(Wg, W).max() <= FIELD_TOL


def test_plug_point_evolve_matches_eulerian_step():
    P, W0 = case(24, 0.3, 30.0, 8)
    with Solver(P, cfl=0.5) as s:
        s.upload_state(W0)
        dt = s.timestep()
        s.evolve_eulerian(1)
        Wa = s.download_state()
        Wb = W0.copy()
        s.evolve(Wb, dt)
    assert np.array_equal(Wa, Wb)


def test_graph_replay_is_bitwise_equal_to_direct_launches():
    P, W0 = case(32, 0.3, 30.0, 9)
    pos0 = ic.particles_to_reference_order(ic.make_particles(500, 9))
    out = []
    for graphs in (True, False):
        with Solver(P, cfl=0.5, max_particles=500, use_graphs=graphs) as s:
            s.upload_state(W0)
            s.particles_upload(pos0)
            s.step(3)
            out.append((s.download_state(), s.particles_download()[0]))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_uniform_flow_stays_uniform():
    n = 32
    P = ic.Params(n=n, gam=1.4, den0=1.0, Mt=0.3, Re=30.0, mu0=1.0, p0=86100.0, t0=0.01)
    sh = (n, n, n)
    W0 = ic.embed_ghost(ic.primitive_to_conserved(P, np.full(sh, 100.0), np.full(sh, -50.0), np.full(sh, 30.0),
                                                  np.ones(sh), np.full(sh, 86100.0)))
    with Solver(P, cfl=0.5) as s:
        s.upload_state(W0)
        s.evolve_eulerian(3)
        W = s.download_state()
    assert rel_l2(W, W0).max() <= 1e-14


def test_nonfinite_state_is_reported_not_faulted():
    P, W0 = case(16, 0.3, 30.0, 3)
    W0[0, 10, 10, 10] = -1.0   # negative density: sqrt of a negative pressure, a NaN wave speed
    with Solver(P, cfl=0.5) as s:
        s.upload_state(W0)
        with pytest.raises(GkmError) as e:
            s.timestep()
        assert e.value.status == 4


def test_full_size_conservation_and_decay():
    """256^3: total mass and momentum are conserved to round-off, kinetic energy decays."""
    P, W0 = case(256, 0.3, 60.0, 1234)
    sl = slice(3, -3)
    with Solver(P, cfl=0.5) as s:
        s.upload_state(W0)
        e0 = s.print_stats()["TKE"]
        s.evolve_eulerian(3)
        W = s.download_state()
        e1 = s.print_stats()["TKE"]
    m0 = W0[0, sl, sl, sl].sum(dtype=np.float64)
    m1 = W[0, sl, sl, sl].sum(dtype=np.float64)
    assert abs(m1 - m0) <= 1e-12 * m0
    for q in (1, 2, 3):   # net momentum of the periodic cube stays ~0 (relative to |rho u| scale)
        scale = np.abs(W0[q, sl, sl, sl]).sum()
        assert abs(W[q, sl, sl, sl].sum() - W0[q, sl, sl, sl].sum()) <= 1e-12 * scale
    assert e1 < e0


def _jump_field(n, seed):
    """A periodic field of piecewise-constant blocks: density 0.2 .. 5, pressure 2e4 .. 1e6,
    velocities up to about Mach 1 in each block, so every sweep meets contact, shear and
    pressure jumps (WENO on discontinuities, strongly different face states)."""
    P, _ = case(n, 0.3, 30.0, seed)
    rng = np.random.default_rng(seed)
    b = n // 4
    def blocks(lo, hi, log=False):
        v = rng.uniform(np.log(lo), np.log(hi), (4, 4, 4)) if log else rng.uniform(lo, hi, (4, 4, 4))
        v = np.exp(v) if log else v
        return np.repeat(np.repeat(np.repeat(v, b, 0), b, 1), b, 2)
    rho = blocks(0.2, 5.0, log=True)
    p = blocks(2e4, 1e6, log=True)
    c = np.sqrt(P.gam * p / rho)
    u, v, w = (blocks(-0.6, 0.6) * c for _ in range(3))
    return P, ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))


def test_strong_jumps_match_oracle(oracle):
    """Two steps from a field of density, pressure and velocity jumps against the oracle: the
    grouped divisions of the reconstruction and the flux (shared among denominators that span
    many orders of magnitude here) keep the FP64 parity bar."""
    P, W0 = _jump_field(32, 3)
    p = oracle.params(P, 0.3)
    Wo = W0.copy()
    for _ in range(2):
        dt = oracle.timestep(p, Wo)
        oracle.step(p, Wo, dt)
    with Solver(P, cfl=0.3) as s:
        s.upload_state(W0)
        s.evolve_eulerian(2)
        Wg = s.download_state()
    assert np.all(np.isfinite(Wg))
    err = rel_l2(Wg, Wo).max()
    print(f"jump field, 2 steps: rel-L2 {err:.1e}")
    assert err <= FIELD_TOL


@pytest.mark.parametrize("prec", [0, 1])
def test_autotune_keeps_state_and_results(prec):
    P, W0 = case(48, 0.3, 30.0, 12)
    with Solver(P, cfl=0.5, precision=prec) as s:
        s.upload_state(W0)
        dt0 = s.timestep()
        cfg = s.autotune(1)
        assert len(cfg) == 3 and all(c["segment"] >= 8 for c in cfg)
        assert np.array_equal(s.download_state(), W0)   # the tuner only writes the accumulator
        assert s.clock() == (0.0, s.clock()[1], 0) and s.timestep() == dt0
        s.evolve_eulerian(3)
        tuned = s.download_state()
    with Solver(P, cfl=0.5, precision=prec) as s:
        s.upload_state(W0)
        s.evolve_eulerian(3)
        plain = s.download_state()
    # every face sees the same inputs whatever the window or segment, so the results agree
    assert rel_l2(tuned, plain).max() <= 1e-13


def test_warp_specialized_sweep_matches_reference_and_plain_sweep(golden):
    """Window variant 2 (a producer warpgroup reconstructs the next face plane while two consumer
    warpgroups compute fluxes) against the reference CPU build's 16^3 fields (1e-12) and against
    the plain 16 x 16 sweep (variant 1) at 48^3 (1e-14: the same arithmetic, rounded differently
    only where the plain sweep splits a window's last cells into single WENO scalars)."""
    g = golden["field_16"]
    P, W0 = w0_of(g)
    pos0 = ic.particles_to_reference_order(g["particles_xyz"])
    with Solver(P, cfl=float(g["cfl"]), max_particles=len(pos0)) as s:
        s.set_sweep_config([(2, 8), (2, 16), (2, 5)])
        assert [c["variant"] for c in s.sweep_config()] == [2, 2, 2]
        s.upload_state(W0)
        s.particles_upload(pos0)
        s.step(len(g["dt"]))
        assert rel_l2(s.download_state(), g["W_final"]).max() <= FIELD_TOL
    P, W0 = case(48, 0.4, 50.0, 5)
    out = {}
    for var in (1, 2):
        with Solver(P, cfl=0.5) as s:
            s.set_sweep_config([(var, 24)] * 3)
            s.upload_state(W0)
            s.evolve_eulerian(4)
            out[var] = s.download_state()
            s.clock()
    assert rel_l2(out[2], out[1]).max() <= 1e-14


def test_z_sweep_pairs_do_not_depend_on_segmentation():
    """The z sweep moves cells k, k+1 (k + 3 even) as accumulator bricks when both lie in its
    segment and reads and writes the other cells directly; its slabs land two planes per bulk copy.
    z segments of 1, 2, 3, 5 and 7 faces (every mix of edge and paired cells) on a 24^3 grid, whose
    last windows end inside their boxes, must reproduce the one-segment state: bit for bit in
    FP64, within single-precision rounding in the mixed form."""
    P, W0 = case(24, 0.4, 50.0, 11)
    for prec, var in ((0, 1), (0, 0), (1, 0)):
        ref = None
        for L in (24, 1, 2, 3, 5, 7):
            with Solver(P, cfl=0.5, precision=prec) as s:
                s.set_sweep_config([(var, 24), (var, 24), (var, L)])
                s.upload_state(W0)
                s.evolve_eulerian(3)
                W = s.download_state()
            if ref is None:
                ref = W
            elif prec == 0:
                assert np.array_equal(W, ref), (var, L)
            else:
                assert rel_l2(W, ref).max() <= 1e-6, L
