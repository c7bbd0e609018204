"""gkm_spline_build_noalloc, the spline build for callers that cannot allocate
device memory (their GPU memory already belongs to their own pool allocator,
or an allocation's implicit device synchronisation is not acceptable).

The entry point gets the state and the coefficient array from the caller
(here: torch tensors) and keeps its intermediate results in a static device
array.  Its coefficients must equal those of the handle-based path
(gkm_generate_splines + gkm_spline_coefs) bit for bit, the tolerance of the
other spline tests, on two calls in a row: the second call finds the first
call's leftovers in the static array.
"""
import numpy as np
import pytest
import torch

from dns_gkm_lpt_b200 import _capi
from dns_gkm_lpt_b200.solver import Solver
from tests.gpu_helpers import case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_spline_build_matches_handle_path_twice(mode):
    P, W0 = case(24, 0.3, 30.0, 77)
    with Solver(P, cfl=0.5, spline_mode=mode) as s:
        s.upload_state(W0)
        s.generate_splines()
        ref = [s.spline_coefs(c) for c in range(3)]
    L = _capi.lib()
    Wd = torch.from_numpy(W0).to("cuda")
    M = ref[0].shape[0]
    out = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for c in (1, 2, 3):
            out.fill_(float("nan"))
            rc = L.gkm_spline_build_noalloc(Wd.data_ptr(), P.n, mode, c, out.data_ptr(), stream)
            assert rc == _capi.GKM_OK, (call, c, rc)
            torch.cuda.synchronize()
            got = out.cpu().numpy().reshape(M, M, M)
            assert np.array_equal(got, ref[c - 1]), (call, c)


def test_noalloc_rejects_grids_beyond_the_static_buffer():
    L = _capi.lib()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")   # never read: the size check comes first
    assert L.gkm_spline_build_noalloc(buf.data_ptr(), 200, 0, 1, buf.data_ptr(), None) == _capi.GKM_ERR_CONFIG
    assert L.gkm_spline_build_noalloc(buf.data_ptr(), 24, 0, 4, buf.data_ptr(), None) == _capi.GKM_ERR_ARG
