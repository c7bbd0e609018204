"""FP32 velocity-spline coefficients (gkm_config.spline_precision =
GKM_SPLINE_COEF_FP32), the large-grid option: the same FP64 line solves as the
FP64 splines (generateSplines / get_bsplinep, src/update.cpp:1235-1247,
src/Interpolation.cpp:3-31), with the coefficients stored rounded to single
precision, built one component at a time in one FP64 buffer of (N+P)^2 N
values, and read as floats by the tricubic evaluation (FP64 arithmetic).

Checks: the stored coefficients are the FP64 coefficients rounded to float,
bit for bit, in both spline modes; the Eulerian fields do not depend on the
splines (bitwise equal); after 20 full steps particle positions stay within
1e-6 (absolute, in [0, 2 pi)) of the FP64-spline run with >= 99.9 % of the
particles in the same cell, and the spline-gradient statistics of PrintStats
(Diss, SijSij, skewness) within 1e-5 relative; particle properties, which need
FP64 coefficients, are refused with GKM_ERR_CONFIG.
"""
import numpy as np
import pytest

from dns_gkm_lpt_b200 import _capi, ic
from dns_gkm_lpt_b200.solver import GkmError, Solver
from tests.gpu_helpers import case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
def test_fp32_coefficients_are_the_fp64_ones_rounded(mode):
    P, W0 = case(24, 0.3, 30.0, 41)
    coefs = {}
    for sp in (0, 1):
        with Solver(P, cfl=0.5, spline_mode=mode, spline_precision=sp) as s:
            s.upload_state(W0)
            s.generate_splines()
            coefs[sp] = [s.spline_coefs(c) for c in range(3)]
    for c in range(3):
        assert np.array_equal(coefs[1][c], coefs[0][c].astype(np.float32).astype(np.float64)), c


def test_fp32_splines_track_particles_like_fp64():
    n, npart, steps = 48, 20000, 20
    P, W0 = case(n, 0.4, 50.0, 42)
    pos0 = ic.particles_to_reference_order(ic.make_particles(npart, 42))
    out = {}
    for sp in (0, 1):
        with Solver(P, cfl=0.5, max_particles=npart, spline_precision=sp) as s:
            s.upload_state(W0)
            s.particles_upload(pos0)
            s.step(steps)
            out[sp] = (s.download_state(), s.particles_download()[0], s.print_stats())
            if sp == 1:
                with pytest.raises(GkmError) as ei:
                    s.particle_props()
                assert ei.value.status == _capi.GKM_ERR_CONFIG
    assert np.array_equal(out[0][0], out[1][0])   # the Eulerian step never reads the splines
    p64, p32 = out[0][1], out[1][1]
    assert np.abs(p32 - p64).max() <= 1e-6
    dx = P.dx
    same = np.all(np.floor(p32 / dx) == np.floor(p64 / dx), axis=1)
    assert same.mean() >= 0.999
    s64, s32 = out[0][2], out[1][2]
    assert s32["TKE"] == s64["TKE"]               # from the cell averages
    for k in ("Diss", "SijSij", "SKEWu", "SKEWv", "SKEWw"):
        assert abs(s32[k] - s64[k]) <= 1e-5 * abs(s64[k]), k
