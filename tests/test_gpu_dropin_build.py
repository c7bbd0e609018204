"""The reference's own -D UseGPU build with this library as its GPU plug point.

oracle/Makefile (target refgpu) compiles the reference's update.cpp with
-D UseGPU (as makefileGPU does), FlowField.cpp, param.cpp, ParticleTrack.cpp
and Interpolation.cpp where they lie, and links them with
dns_gkm_lpt_b200/plug/GPUupdate_b200.cpp in place of the reference's
GPUupdate.cu and GPUAlloc.cu, so DevAlloc::DevAlloc() and
evolve(W, dev, dt) (src/GPUAlloc.h:8-26, src/GPUupdate.h:33) are the shim's,
compiled against the reference's headers and calling libgkm_b200.so.  The
reference's loop body (src/update.cpp:124-170) then runs unmodified:
evolveEulerian(W, dev) -> evolve -> gkm_evolve on the GPU, everything else on
the host as the reference does it.

After 1 and 10 steps of the 16^3 golden case the fields must equal the
reference CPU build's (tests/golden/field_16) within relative L2 1e-12 per
component (the FP64 parity bar), every dt within 1e-13, particle cell indices
exactly and positions within 1e-10.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic
from tests.gpu_helpers import params_of, rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU_SO = os.path.join(ROOT, "oracle", "_ref", "libgkm_ref_gpu.so")
_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


@pytest.mark.skipif(not os.path.exists(REF_GPU_SO),
                    reason="oracle/_ref/libgkm_ref_gpu.so is built by `make -C oracle` where the reference tree exists")
def test_reference_gpu_build_with_the_plug_point_matches_the_cpu_build(golden):
    g = golden["field_16"]
    P = params_of(g)
    u, v, w = g["u"], g["v"], g["w"]
    d = tempfile.mkdtemp(prefix="gkm_refgpu_")
    ic.write_reference_inputs(d, P, u, v, w, np.ones_like(u), np.full_like(u, P.p0), g["particles_xyz"])

    L = C.CDLL(REF_GPU_SO)
    L.gkmrefgpu_setup.argtypes = [C.c_char_p, C.c_double]
    L.gkmrefgpu_setup.restype = C.c_int
    L.gkmrefgpu_run.argtypes = [C.c_int, _dp]
    L.gkmrefgpu_nt.restype = C.c_int
    L.gkmrefgpu_dt.restype = C.c_double
    L.gkmrefgpu_get_W.argtypes = [_dp]
    L.gkmrefgpu_get_particles.argtypes = [_dp, _dp, C.POINTER(C.c_int)]
    L.gkmrefgpu_get_particles.restype = C.c_int

    assert L.gkmrefgpu_setup(d.encode(), float(g["cfl"])) == 0
    nt = L.gkmrefgpu_nt()
    assert nt == P.n + 6
    W = np.zeros((5, nt, nt, nt))
    nsteps = len(g["dt"])
    dts = np.zeros(nsteps)
    L.gkmrefgpu_run(1, _ptr(dts[:1]))
    L.gkmrefgpu_get_W(_ptr(W))
    assert rel_l2(W, g["W_step1"]).max() <= 1e-12
    rest = np.zeros(nsteps - 1)
    L.gkmrefgpu_run(nsteps - 1, _ptr(rest))
    dts[1:] = rest
    L.gkmrefgpu_get_W(_ptr(W))
    assert rel_l2(W, g["W_final"]).max() <= 1e-12
    assert np.allclose(dts, g["dt"], rtol=1e-13, atol=0)
    assert L.gkmrefgpu_dt() == pytest.approx(float(g["dt_next"]), rel=1e-13)

    npart = len(g["particles_xyz"])
    pos = np.zeros((2 * npart, 3))
    U = np.zeros((2 * npart, 3))
    tags = np.zeros(2 * npart, dtype=np.int32)
    cnt = L.gkmrefgpu_get_particles(_ptr(pos), _ptr(U), tags.ctypes.data_as(C.POINTER(C.c_int)))
    assert cnt == npart
    pos, U, tags = pos[:cnt], U[:cnt], tags[:cnt]
    # both runs list the particles in the reference's own order (its tags)
    assert np.array_equal(tags, g["tags"])
    dx = P.dx
    assert np.array_equal(np.floor(pos / dx).astype(int), np.floor(g["pos_final"] / dx).astype(int))
    assert np.abs(pos - g["pos_final"]).max() <= 1e-10
    assert np.abs(U - g["U_final"]).max() <= 1e-10 * np.abs(g["U_final"]).max()
    L.gkmrefgpu_finish()
