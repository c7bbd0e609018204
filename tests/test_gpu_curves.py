"""Long-run kinetic-energy decay and dissipation curves against the reference.

The goldens curve_32 (32^3, 200 steps) and curve_64 (64^3, 100 steps) hold
the reference CPU build's PrintStats line every 10 iterations
(tests/golden/make_golden.py --curves).  The initial field is regenerated
here from the same seed and recipe (checked through mu0 and t0, which depend
on every value of the field).

Bar: TKE and Diss within 0.5% at every sampled iteration (FP64 and the
mixed-precision form); the FP64 form is also held to 1e-9.  t/t0 is compared
with the reference's printed value (6 significant digits, %e): 1e-6.
"""
import os

import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic
from dns_gkm_lpt_b200.solver import Solver

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# inputs of the curve cases (tests/golden/make_golden.py CURVES)
CASES = {"curve_32": dict(n=32, Mt=0.3, Re=30.0, seed=4321, cfl=0.5),
         "curve_64": dict(n=64, Mt=0.3, Re=30.0, seed=1235, cfl=0.5)}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tke_and_dissipation_curves(name, precision):
    g = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    c = CASES[name]
    P, u, v, w, rho, p = ic.make_field(c["n"], c["Mt"], c["Re"], c["seed"])
    assert P.mu0 == pytest.approx(float(g["mu0"]), rel=1e-12)
    assert P.t0 == pytest.approx(float(g["t0"]), rel=1e-12)
    W0 = ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))
    ref = g["stats"]
    rows = []
    with Solver(P, cfl=c["cfl"], precision=precision) as s:
        s.upload_state(W0)
        for r in range(len(ref)):
            if r:
                s.evolve_eulerian(10)
            st = s.print_stats()
            rows.append((st["t_over_t0"], st["TKE"], st["Diss"]))
    rows = np.array(rows)
    err_tke = np.abs(rows[:, 1] / ref[:, 1] - 1)
    err_diss = np.abs(rows[:, 2] / ref[:, 2] - 1)
    err_t = np.abs(rows[1:, 0] / ref[1:, 0] - 1)
    print(f"{name} precision={precision}: max rel err TKE {err_tke.max():.2e}, Diss {err_diss.max():.2e}, "
          f"t/t0 {err_t.max():.2e} over {10 * (len(ref) - 1)} steps")
    assert err_tke.max() <= 5e-3 and err_diss.max() <= 5e-3
    if precision == 0:
        assert err_tke.max() <= 1e-9 and err_diss.max() <= 1e-9
    assert err_t.max() <= 1e-6
