"""The C restatement (oracle/gkm_oracle.c) against golden vectors produced by
the reference's own CPU build (tests/golden/make_golden.py): bit-exact."""
import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic


def _params(g):
    return ic.Params(n=int(g["n"]), gam=float(g["gam"]), den0=float(g["den0"]), Mt=float(g["Mt"]),
                     Re=float(g["Re"]), mu0=float(g["mu0"]), p0=float(g["p0"]), t0=float(g["t0"]))


def _w0(g):
    P = _params(g)
    u = g["u"]
    return P, ic.embed_ghost(ic.primitive_to_conserved(P, u, g["v"], g["w"], np.ones_like(u), np.full_like(u, P.p0)))


def test_weno_faces_bitexact(oracle, golden):
    f = golden["faces"]
    for s, wl, wr in zip(f["stencils"], f["Wl"], f["Wr"]):
        a, b = oracle.weno(s, float(f["gam"]))
        assert np.array_equal(a, wl) and np.array_equal(b, wr)


def test_flux_faces_bitexact(oracle, golden):
    f = golden["faces"]
    for i in range(len(f["F"])):
        D = f["DW"][i]
        F = oracle.flux(f["WL"][i], f["WR"][i], f["Wl"][i], f["Wr"][i], D[0], D[1], D[2], D[3], D[4], D[5],
                        float(f["tau"][i]), float(f["dt"]), float(f["dx"]), float(f["gam"]))
        assert np.array_equal(F, f["F"][i]), (i, F, f["F"][i])


def test_uniform_face_has_no_mass_flux_without_velocity(oracle):
    # a uniform gas at rest: mass and energy fluxes vanish, momentum flux is the pressure impulse p*dt
    W = np.array([1.0, 0.0, 0.0, 0.0, 86100.0 / 0.4])
    Z = np.zeros(5)
    F = oracle.flux(W, W, W, W, Z, Z, Z, Z, Z, Z, 1e-5, 3e-4, 0.4, 1.4)
    assert abs(F[0]) < 1e-12 and abs(F[4]) < 1e-6
    assert F[1] == pytest.approx(86100.0 * 3e-4, rel=1e-12)


@pytest.mark.parametrize("case", ["field_16", "field_12"])
def test_field_run_bitexact(oracle, golden, case):
    g = golden[case]
    P, W = _w0(g)
    p = oracle.params(P, float(g["cfl"]))
    W1 = W.copy()
    pos = ic.particles_to_reference_order(g["particles_xyz"])
    r1 = oracle.run(p, W1, 1, 0, pos)
    assert np.array_equal(W1[:, 3:-3, 3:-3, 3:-3], g["W_step1"])
    steps = len(g["dt"])
    r = oracle.run(p, W, steps, 0, pos)
    assert np.array_equal(r["dt"], g["dt"])
    assert np.array_equal(W[:, 3:-3, 3:-3, 3:-3], g["W_final"])
    assert oracle.timestep(p, W) == float(g["dt_next"])
    order = np.argsort(g["tags"])
    assert np.array_equal(r["pos"], g["pos_final"][order])
    assert np.array_equal(r["U"], g["U_final"][order])
    # PrintStats globals (TKE, Diss, SijSij, skewness, kurtosis) at step 0
    s0 = r1["stats"][0]
    for k, idx in (("TKE", 1), ("Diss", 2), ("SijSij", 3), ("SKEWu", 4), ("SKEWv", 5), ("SKEWw", 6),
                   ("KURTu", 7), ("KURTv", 8), ("KURTw", 9)):
        assert s0[k] == g["stats_step0"][idx], k
    # Prms/Trms are printed by the reference with 9 significant digits
    assert s0["Prms"] == pytest.approx(g["stats_step0"][10], rel=1e-8, abs=1e-12)
    assert s0["Trms"] == pytest.approx(g["stats_step0"][11], rel=1e-8, abs=1e-12)
    if steps % 10 == 0:
        assert r["stats"][-1]["TKE"] == g["stats_final"][1]
        assert r["stats"][-1]["Diss"] == g["stats_final"][2]


def test_halo_is_periodic_wrap(oracle, golden):
    g = golden["field_12"]
    P, W = _w0(g)
    p = oracle.params(P, 0.5)
    V = W.copy()
    V[:, :3] = 0
    V[:, :, -3:] = -1
    oracle.halo(p, V)
    assert np.array_equal(V, W)


def _outputs_golden():
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "outputs_12.npz")
    return dict(np.load(path))


def test_particle_props_and_stats_bitexact(oracle, golden):
    """getParticleProp (all eight splines) and GetParticleStats at iteration 0."""
    g = golden["field_12"]
    o = _outputs_golden()
    P, W = _w0(g)
    p = oracle.params(P, float(g["cfl"]))
    oracle.halo(p, W)
    pos = ic.particles_to_reference_order(g["particles_xyz"])
    props = oracle.particle_props(p, W, pos)
    order = np.argsort(o["tags_0"])
    assert np.array_equal(props, o["props_0"][order])
    assert np.array_equal(oracle.particle_stats(props), o["pstats_0"])
