"""The mixed-precision form (GKM_PREC_MIXED): WENO and the gas-kinetic flux in
non-dimensional FP32, time coefficients, flux differences, update and
reductions in FP64.  Checked against the FP64 path and the reference goldens.

Tolerances: field relative L2 per conserved component <= 1e-5 after 10 steps
(the error bar of the mixed form); exact properties (uniform flow,
conservation) as for FP64.
"""
import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic
from dns_gkm_lpt_b200.solver import Solver
from tests.gpu_helpers import analytic_case, case, rel_l2, w0_of

pytestmark = pytest.mark.gpu
MIXED = 1


def test_mixed_matches_reference_goldens(golden):
    g = golden["field_16"]
    P, W0 = w0_of(g)
    pos0 = ic.particles_to_reference_order(g["particles_xyz"])
    with Solver(P, cfl=float(g["cfl"]), max_particles=len(pos0), precision=MIXED) as s:
        s.upload_state(W0)
        s.particles_upload(pos0)
        s.step(len(g["dt"]))
        W = s.download_state()
        pos, _ = s.particles_download()
    err = rel_l2(W, g["W_final"])
    print("mixed vs reference after 10 steps, rel-L2 per component:", err)
    assert err.max() <= 1e-5
    order = np.argsort(g["tags"])
    assert np.abs(pos - g["pos_final"][order]).max() <= 1e-6


def test_mixed_vs_fp64_64cube():
    P, W0 = case(64, 0.3, 30.0, 5)
    out = []
    for prec in (0, MIXED):
        with Solver(P, cfl=0.5, precision=prec) as s:
            s.upload_state(W0)
            s.evolve_eulerian(5)
            out.append(s.download_state())
    err = rel_l2(out[1], out[0])
    print("mixed vs FP64 after 5 steps at 64^3:", err)
    assert err.max() <= 1e-5


def test_mixed_uniform_flow_and_conservation():
    n = 32
    P = ic.Params(n=n, gam=1.4, den0=1.0, Mt=0.3, Re=30.0, mu0=1.0, p0=86100.0, t0=0.01)
    sh = (n, n, n)
    W0 = ic.embed_ghost(ic.primitive_to_conserved(P, np.full(sh, 100.0), np.full(sh, -50.0), np.full(sh, 30.0),
                                                  np.ones(sh), np.full(sh, 86100.0)))
    with Solver(P, cfl=0.5, precision=MIXED) as s:
        s.upload_state(W0)
        s.evolve_eulerian(3)
        W = s.download_state()
    assert rel_l2(W, W0).max() <= 1e-14
    P, W0 = case(48, 0.4, 40.0, 6)
    with Solver(P, cfl=0.5, precision=MIXED) as s:
        s.upload_state(W0)
        s.evolve_eulerian(3)
        W = s.download_state()
    sl = slice(3, -3)
    m0, m1 = W0[0, sl, sl, sl].sum(), W[0, sl, sl, sl].sum()
    assert abs(m1 - m0) <= 1e-12 * m0


@pytest.mark.parametrize("n", [13, 21, 10])
def test_mixed_odd_and_small_grids_track_fp64(n):
    """Odd n: no tensor maps, so the mixed sweeps load and convert every slab cell by cell and the
    z sweep moves single cells; n = 10: boxes and bricks that reach past the grid.  Both stay within
    the mixed form's error bar of the FP64 path."""
    P, W0 = analytic_case(n, 70 + n)
    out = []
    for prec in (0, MIXED):
        with Solver(P, cfl=0.5, precision=prec) as s:
            s.upload_state(W0)
            s.evolve_eulerian(3)
            out.append(s.download_state())
    err = rel_l2(out[1], out[0])
    print(f"mixed vs FP64 after 3 steps at {n}^3:", err)
    assert err.max() <= 1e-5

