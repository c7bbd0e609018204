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


def analytic_case(n, seed):
    """A smooth random-phase velocity field for any n (odd included; the spectral generator
    needs even n)."""
    rng = np.random.default_rng(seed)
    P = ic.Params(n=n, gam=1.4, den0=1.0, Mt=0.3, Re=30.0, mu0=0.9, p0=86100.0, t0=0.01)
    x = (np.arange(n) + 0.5) * (2 * np.pi / n)
    Y, X, Z = np.meshgrid(x, x, x, indexing="ij")
    u, v, w = [sum(rng.uniform(20, 60) * np.sin(kx * X + ky * Y + kz * Z + rng.uniform(0, 2 * np.pi))
                   for kx, ky, kz in ((1, 0, 1), (0, 2, 1), (1, 1, 0))) for _ in range(3)]
    rho = 1.0 + 0.05 * np.cos(X + 2 * Z)
    return P, ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, np.full_like(u, P.p0)))
