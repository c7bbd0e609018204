"""The device numerics header compiled for the host (tests/native/hostnum.cpp)
against golden faces from the reference build: the FP64 formulation the
kernels run, and the mixed-precision formulation (non-dimensional FP32 flux,
FP64 time coefficients).

Tolerances: FP64 flux 1e-11 of the face's largest component (as on the GPU);
mixed flux 5e-6 of the face's largest component (single-precision moments; measured 9e-7).
"""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def hostnum():
    out = os.path.join(tempfile.mkdtemp(), "libhostnum.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off",
                    "-I", os.path.join(ROOT, "dns_gkm_lpt_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "hostnum.cpp"), "-o", out], check=True)
    L = C.CDLL(out)
    L.hn_flux_double.argtypes = [_dp, C.c_double, C.c_double, C.c_double, _dp]
    L.hn_flux_double_mcal.argtypes = [_dp, C.c_double, C.c_double, C.c_double, _dp]
    L.hn_flux_mixed.argtypes = [_dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _dp]
    L.hn_weno_double.argtypes = [_dp, C.c_double, _dp, _dp]
    L.hn_weno_float.argtypes = [_dp, C.c_double, _dp, _dp]
    return L


def _faces(golden):
    f = golden["faces"]
    nf = len(f["F"])
    inp = np.concatenate([f["WL"], f["WR"], f["Wl"], f["Wr"], f["DW"].reshape(nf, 30), f["tau"][:, None]], axis=1)
    return f, np.ascontiguousarray(inp)


def _p(a):
    return a.ctypes.data_as(_dp)


def test_fp64_flux_formulation(hostnum, golden):
    f, inp = _faces(golden)
    for i in range(len(inp)):
        F = np.zeros(5)
        hostnum.hn_flux_double(_p(inp[i]), float(f["gam"]), float(f["dt"]), float(f["dx"]), _p(F))
        assert np.abs(F - f["F"][i]).max() <= 1e-11 * np.abs(f["F"][i]).max(), i


def test_mixed_flux_formulation(hostnum, golden):
    f, inp = _faces(golden)
    g = golden["field_16"]
    errs = []
    for i in range(len(inp)):
        F = np.zeros(5)
        hostnum.hn_flux_mixed(_p(inp[i]), float(f["gam"]), float(f["dt"]), float(f["dx"]), float(g["den0"]),
                              float(g["p0"]), _p(F))
        errs.append(np.abs(F - f["F"][i]).max() / np.abs(f["F"][i]).max())
    assert max(errs) <= 5e-6, max(errs)


def test_weno_float_branch_handles_flat_stencils(hostnum):
    l, r = C.c_double(), C.c_double()
    s = np.full(6, 0.7)
    hostnum.hn_weno_float(_p(s), 1e-16, C.byref(l), C.byref(r))
    assert abs(l.value - 0.7) < 1e-7 and abs(r.value - 0.7) < 1e-7
    s = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])   # a step: both sides stay on their own plateau
    hostnum.hn_weno_float(_p(s), 1e-10, C.byref(l), C.byref(r))
    a, b = C.c_double(), C.c_double()
    hostnum.hn_weno_double(_p(s), 1e-10, C.byref(a), C.byref(b))
    assert abs(l.value - a.value) < 1e-6 and abs(r.value - b.value) < 1e-6


def _face_state(rng, gam, c, mach):
    rho = rng.uniform(0.2, 5.0)
    u = rng.normal(0.0, c * mach, 3)
    p = 1e5 * rng.uniform(0.1, 10.0)
    return np.array([rho, rho * u[0], rho * u[1], rho * u[2], p / (gam - 1) + 0.5 * rho * (u @ u)])


def test_fp64_flux_functional_form_equals_mcal_form(hostnum, golden):
    """The kernels' flux (moments as tangential functionals contracted with the normal
    tables, grouped reciprocals) against the reference's MCal algebra on the same faces: the
    golden faces, and 3000 random faces with density ratios up to 25, pressure ratios up to
    100, velocities up to Mach 3 and slopes up to three times the state per cell.  Same
    moments summed in another order: within 1e-10 of each face's largest component."""
    f, inp = _faces(golden)
    gam, dx = float(f["gam"]), float(f["dx"])
    worst = 0.0
    for i in range(len(inp)):
        a, b = np.zeros(5), np.zeros(5)
        hostnum.hn_flux_double(_p(inp[i]), gam, float(f["dt"]), dx, _p(a))
        hostnum.hn_flux_double_mcal(_p(inp[i]), gam, float(f["dt"]), dx, _p(b))
        worst = max(worst, np.abs(a - b).max() / np.abs(b).max())
    assert worst <= 1e-14, worst
    rng = np.random.default_rng(11)
    c = 347.0
    for _ in range(3000):
        x = np.zeros(51)
        for k in range(4):
            x[5 * k:5 * k + 5] = _face_state(rng, gam, c, rng.uniform(0.05, 1.0))
        scale = np.abs(x[0:5]) + 1.0
        x[20:50] = rng.normal(0.0, 1.0, 30) * np.tile(scale, 6) * rng.uniform(0.01, 3.0) / dx
        x[50] = 10 ** rng.uniform(-9, -5)
        dt = 10 ** rng.uniform(-7, -5)
        a, b = np.zeros(5), np.zeros(5)
        hostnum.hn_flux_double(_p(x), gam, dt, dx, _p(a))
        hostnum.hn_flux_double_mcal(_p(x), gam, dt, dx, _p(b))
        assert np.all(np.isfinite(b))
        assert np.all(np.isfinite(a))
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), (x, a, b)
