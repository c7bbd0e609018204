"""gkm_spline_build_noalloc, the spline build for callers that cannot allocate
device memory (their GPU memory already belongs to their own pool allocator,
or an allocation's implicit device synchronisation is not acceptable).

The entry point gets the state and the coefficient array from the caller
(here: torch tensors) and keeps its intermediate results in a static device
array.  Its coefficients must equal those of the handle-based path
(gkm_generate_splines + gkm_spline_coefs) bit for bit, the tolerance of the
other spline tests, on two calls in a row: the second call finds the first
call's leftovers in the static array.  The device's free memory must not
change across calls made after a first (set-up) call, and the largest grids
the static array accepts must still match.
"""
import numpy as np
import pytest
import torch

from dns_gkm_lpt_b200 import _capi
from dns_gkm_lpt_b200.solver import Solver
from tests.gpu_helpers import case

pytestmark = pytest.mark.gpu

# largest grids whose line-solve intermediates fit the 32 MiB array: natural_ghost3 N = n + 6,
# (N + 2)^2 N doubles; periodic N = n, (N + 3)^2 N doubles; at most 4 Mi doubles
LARGEST = {0: 153, 1: 159}


def _fits(n, mode):
    N = n + 6 if mode == 0 else n
    M = N + (2 if mode == 0 else 3)
    return M * M * N <= 4 * 1024 * 1024


def test_largest_accepted_sizes_are_the_documented_ones():
    for mode, n in LARGEST.items():
        assert _fits(n, mode) and not _fits(n + 1, mode)


def _handle_coefs(P, W0, mode):
    with Solver(P, cfl=0.5, spline_mode=mode) as s:
        s.upload_state(W0)
        s.generate_splines()
        return [s.spline_coefs(c) for c in range(3)]


def _check_twice(P, W0, mode, ref):
    L = _capi.lib()
    Wd = torch.from_numpy(W0).to("cuda")
    M = ref[0].shape[0]
    out = torch.empty(M ** 3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # the set-up call: the first call on a device looks up the static array's address
    assert L.gkm_spline_build_noalloc(Wd.data_ptr(), P.n, mode, 1, out.data_ptr(), stream) == _capi.GKM_OK
    # the torch kernels the loop uses run once here too: their modules load on first use, which
    # takes device memory that is not the entry point's
    out.fill_(float("nan"))
    out.cpu()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for call in range(2):
        for c in (1, 2, 3):
            out.fill_(float("nan"))
            rc = L.gkm_spline_build_noalloc(Wd.data_ptr(), P.n, mode, c, out.data_ptr(), stream)
            assert rc == _capi.GKM_OK, (call, c, rc)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0, "the entry point changed the device's free memory"
            got = out.cpu().numpy().reshape(M, M, M)
            assert np.array_equal(got, ref[c - 1]), (call, c)


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_spline_build_matches_handle_path_twice(mode):
    P, W0 = case(24, 0.3, 30.0, 77)
    _check_twice(P, W0, mode, _handle_coefs(P, W0, mode))


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_spline_build_near_the_largest_accepted_grid(mode):
    n = LARGEST[mode] - 1   # the seeded field generator takes even n only
    P, W0 = case(n, 0.3, 30.0, 78)
    _check_twice(P, W0, mode, _handle_coefs(P, W0, mode))


def test_noalloc_rejects_grids_beyond_the_static_buffer():
    L = _capi.lib()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")   # never read: the size check comes first
    assert L.gkm_spline_build_noalloc(buf.data_ptr(), LARGEST[0] + 1, 0, 1, buf.data_ptr(), None) == \
        _capi.GKM_ERR_CONFIG
    assert L.gkm_spline_build_noalloc(buf.data_ptr(), LARGEST[1] + 1, 1, 1, buf.data_ptr(), None) == \
        _capi.GKM_ERR_CONFIG
    assert L.gkm_spline_build_noalloc(buf.data_ptr(), 200, 0, 1, buf.data_ptr(), None) == _capi.GKM_ERR_CONFIG
    assert L.gkm_spline_build_noalloc(buf.data_ptr(), 24, 0, 4, buf.data_ptr(), None) == _capi.GKM_ERR_ARG
