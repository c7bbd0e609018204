"""The plug point evolve(W, dt) (gkm_evolve) with pinned host or device
buffers, which runs as a pipeline over chunks of y-planes (copy-in, sweeps
and copy-out of consecutive chunks overlap), against the resident step and
the one-shot path of pageable buffers.

Bars: the new state (ghosts included) within relative L2 1e-13 per component
of the resident step (the y sweep's segments follow the chunks, so rounding
may differ; the report says whether it was bit for bit), ghosts equal to the
periodic images of the interior, clock advanced by dt and one step, several
grid sizes whose last chunk is ragged, odd sizes (no tensor maps: per-element copies in every
chunk's launches), both precisions.
"""
import numpy as np
import pytest
import torch

from dns_gkm_lpt_b200.solver import Solver
from tests.gpu_helpers import analytic_case, case, rel_l2

pytestmark = pytest.mark.gpu


def _ghosts_are_periodic(W):
    n = W.shape[1] - 6
    inner = W[:, 3:n + 3, 3:n + 3, 3:n + 3]
    return np.array_equal(np.pad(inner, ((0, 0), (3, 3), (3, 3), (3, 3)), mode="wrap"), W)


@pytest.mark.parametrize("n,prec", [(12, 0), (20, 0), (36, 0), (64, 0), (70, 1), (128, 0), (21, 0), (13, 1)])
def test_pipelined_plug_point_matches_resident_step(n, prec):
    P, W0 = case(n, 0.3, 40.0, 30 + n) if n % 2 == 0 else analytic_case(n, 30 + n)
    with Solver(P, cfl=0.5, precision=prec) as s:
        s.upload_state(W0)
        dt = s.timestep()
        s.evolve_eulerian(1)
        Wa = s.download_state()
        t_a, _, it_a = s.clock()
    # pinned host buffers
    Wp = torch.from_numpy(W0.copy()).pin_memory()
    with Solver(P, cfl=0.5, precision=prec) as s:
        Wn = Wp.numpy()
        s.evolve(Wn, dt)
        t_b, dt_b, it_b = s.clock()
        Wb = Wn.copy()
        # device buffers, a second step from the first one's result
        Wd = torch.from_numpy(Wb).cuda()
        torch.cuda.synchronize()
        s.evolve(Wd, dt)
        torch.cuda.synchronize()
        Wc = Wd.cpu().numpy()
    err = rel_l2(Wb, Wa).max()
    print(f"n={n} prec={prec}: pipelined vs resident {'bitwise' if np.array_equal(Wb, Wa) else f'{err:.1e}'}")
    assert err <= 1e-13
    assert _ghosts_are_periodic(Wb)
    assert it_b == 1 and dt_b == dt and t_b == pytest.approx(dt, rel=1e-15)
    # second step: the pageable one-shot path from the same state
    with Solver(P, cfl=0.5, precision=prec) as s:
        Wr = Wb.copy()
        s.evolve(Wr, dt)
    assert rel_l2(Wc, Wr).max() <= 1e-13
    assert _ghosts_are_periodic(Wc)


@pytest.mark.parametrize("prec", [0, 1])
def test_pipeline_stream_counts_are_bitwise_identical(prec):
    """One, two and three compute streams launch the same sweeps on the same planes, so
    their results agree bit for bit; 16-plane chunks at 64^3 give four chunks, so chunks on
    different streams really overlap."""
    n = 64
    P, W0 = case(n, 0.3, 40.0, 77)
    out = {}
    with Solver(P, cfl=0.5, precision=prec) as s:
        s.upload_state(W0)
        dt = s.timestep()
        for streams in (1, 2, 3):
            s.set_pipeline(16, streams)
            Wp = torch.from_numpy(W0.copy()).pin_memory()
            s.evolve(Wp.numpy(), dt)
            out[streams] = Wp.numpy().copy()
    for streams in (2, 3):
        assert np.array_equal(out[streams], out[1]), streams
    assert _ghosts_are_periodic(out[1])
