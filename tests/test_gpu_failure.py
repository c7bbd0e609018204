"""Failure detection on the GPU without a fault: the sweeps' bounded waits.

The FP64 x and y sweeps land each stencil slab with a bulk tensor copy that
completes on an mbarrier.  Every wait on it polls a bounded number of times;
a wait that runs out raises bit 1 of the device status word, the kernel
carries on, and the next synchronising call returns GKM_ERR_CUDA.  The test
hook gkm_config.test_wait_probe makes one such wait run out per launch
without any failing copy: the first CTA expects 16 bytes more than its first
copy delivers and polls only 256 times, then takes the extra bytes back and
waits for the copy, which lands normally.  Nothing faults, nothing waits
without a bound and nothing is left in flight, so the step's result is the
normal one and the GPU stays usable: a fresh handle then steps the 16^3
golden case to parity with the reference CPU build.
"""
import numpy as np
import pytest

from dns_gkm_lpt_b200 import _capi, ic
from dns_gkm_lpt_b200.solver import GkmError, Solver
from tests.gpu_helpers import rel_l2, w0_of

pytestmark = pytest.mark.gpu


def test_bounded_copy_wait_that_runs_out_is_reported_and_the_gpu_stays_usable(golden):
    g = golden["field_16"]
    P, W0 = w0_of(g)
    cfl = float(g["cfl"])
    with Solver(P, cfl=cfl) as ref:
        ref.upload_state(W0)
        ref.evolve_eulerian(1)
        W_ref = ref.download_state()
        ref.clock()   # no error without the hook

    with Solver(P, cfl=cfl, test_wait_probe=1) as s:
        s.upload_state(W0)
        s.evolve_eulerian(1)
        with pytest.raises(GkmError) as ei:
            s.clock()
        assert ei.value.status == _capi.GKM_ERR_CUDA
        assert "did not complete in time" in str(ei.value)
        W = np.empty_like(W_ref)
        with pytest.raises(GkmError):
            s.download_state(W)   # the data is copied, then the status is reported
    # every copy landed: the step's result is the normal one, bit for bit
    assert np.array_equal(W, W_ref)

    pos0 = ic.particles_to_reference_order(g["particles_xyz"])
    with Solver(P, cfl=cfl, max_particles=len(pos0)) as s2:
        s2.upload_state(W0)
        s2.particles_upload(pos0)
        s2.step(len(g["dt"]))
        assert rel_l2(s2.download_state(), g["W_final"]).max() <= 1e-12
        assert s2.clock()[2] == len(g["dt"])

