"""Shared helpers of the GPU tests (no test functions here)."""
import numpy as np

from dns_gkm_lpt_b200 import ic


def params_of(g):
    return ic.Params(n=int(g["n"]), gam=float(g["gam"]), den0=float(g["den0"]), Mt=float(g["Mt"]),
                     Re=float(g["Re"]), mu0=float(g["mu0"]), p0=float(g["p0"]), t0=float(g["t0"]))


def w0_of(g):
    P = params_of(g)
    u = g["u"]
    return P, ic.embed_ghost(ic.primitive_to_conserved(P, u, g["v"], g["w"], np.ones_like(u), np.full_like(u, P.p0)))


def rel_l2(a, b):
    """Per-component relative L2 error over the interior, as ||a-b|| / ||b||."""
    a = a[:, 3:-3, 3:-3, 3:-3] if a.shape[1] > b.shape[1] else a
    b = b[:, 3:-3, 3:-3, 3:-3] if b.shape[1] > a.shape[1] else b
    return np.array([np.linalg.norm(a[q] - b[q]) / max(np.linalg.norm(b[q]), 1e-300) for q in range(5)])


def case(n, Mt, Re, seed):
    P, u, v, w, rho, p = ic.make_field(n, Mt, Re, seed)
    return P, ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))
