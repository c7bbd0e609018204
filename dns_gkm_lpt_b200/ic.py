"""Seeded synthetic initial conditions in the reference's formats.

A NumPy restatement of the reference's MATLAB pre-processing
(InitialConditions/init_DNS.m, InitialConditions/Part_Gen.m), which MATLAB or
Octave would otherwise have to run.  The recipe:

* uniform random u, v, w on an N^3 grid -> 3-D FFT            (init_DNS.m:28-32)
* solenoidal projection u_hat -= (k . u_hat) k / |k|^2        (init_DNS.m:35-43)
* shell rescale to E(k) = A k^4 exp(-2 (k/k0)^2) on 1<=|k|<=8 (init_DNS.m:16-18,47-63)
  using |u_hat|^2 (the MATLAB script squares the complex value instead, which
  rotates phases; the magnitude form is the spectrum the script intends)
* inverse FFT, real part; scale to the turbulent Mach number  (init_DNS.m:65-92)
* mu0 from Re_lambda with central differences, t0 = lam/urms  (init_DNS.m:96-126)
* rho = rho0 = 1, p = p0 = rho0 R T0 uniform, T0 = 300 K      (init_DNS.m:78-82,147-148)

Array convention: fields are returned as (y, x, z) arrays, the reference's
(j, i, k) order (src/param.h:39-45).  Files are written exactly as the MATLAB
script writes them (column-major), so the reference's own readers
(src/FlowField.cpp:9-114, src/update.cpp:1286-1302) load them unchanged.
"""
from __future__ import annotations

import dataclasses
import os
import struct

import numpy as np

R_GAS = 287.0


@dataclasses.dataclass
class Params:
    """Contents of InitialConditions/params (init_DNS.m:165-175, read at FlowField.cpp:16-50)."""

    n: int
    gam: float
    den0: float
    Mt: float
    Re: float
    mu0: float
    p0: float
    t0: float

    @property
    def T0(self) -> float:
        return self.p0 / (R_GAS * self.den0)

    @property
    def dx(self) -> float:
        return 2.0 * (np.arctan(1.0) * 4.0) / self.n


def _kfft(n: int) -> np.ndarray:
    # MATLAB kfft = [0:kmax kmin:-1] with kmax = floor(N/2), kmin = -floor(N/2)+1
    return np.concatenate([np.arange(0, n // 2 + 1), np.arange(-(n // 2) + 1, 0)]).astype(np.float64)


def make_field(n: int, Mt: float, Re: float, seed: int, k0: float = 4.0, kcmin: float = 1.0,
               kcmax: float = 8.0, gam: float = 1.4, rho0: float = 1.0, T0: float = 300.0):
    """Return (params, u, v, w, rho, p) with u, v, w, rho, p shaped (y, x, z)."""
    rng = np.random.default_rng(seed)
    Np = float(n) ** 3
    A = np.sqrt(2.0 / np.pi) * (16.0 / 3.0) * Mt ** 2 / k0 ** 5
    # MATLAB dims (1, 2, 3) = (y, x, z); u pairs with k1 along dim 2 (x),
    # v with k2 along dim 1 (y), w with k3 along dim 3 (z) (meshgrid semantics)
    uk = np.fft.fftn(rng.random((n, n, n)))
    vk = np.fft.fftn(rng.random((n, n, n)))
    wk = np.fft.fftn(rng.random((n, n, n)))
    kf = _kfft(n)
    k2 = kf[:, None, None]  # along dim 1 (y)
    k1 = kf[None, :, None]  # along dim 2 (x)
    k3 = kf[None, None, :]  # along dim 3 (z)
    ksq = np.maximum(k1 ** 2 + k2 ** 2 + k3 ** 2, 1e-14)
    kdot = k1 * uk + k2 * vk + k3 * wk
    uk -= kdot * k1 / ksq
    vk -= kdot * k2 / ksq
    wk -= kdot * k3 / ksq
    kk = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2)
    shell = (kk >= kcmin) & (kk <= kcmax)
    ee = A * kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2) * Np ** 2
    ee = np.where(shell, ee / (4.0 * np.pi * np.where(shell, kk, 1.0) ** 2), 0.0)
    umag2 = np.abs(uk) ** 2 + np.abs(vk) ** 2 + np.abs(wk) ** 2
    fac = np.where(shell & (umag2 > 0), np.sqrt(ee / np.where(umag2 > 0, umag2, 1.0)), 0.0)
    uk *= fac / Np
    vk *= fac / Np
    wk *= fac / Np
    u = np.real(np.fft.ifftn(uk))
    v = np.real(np.fft.ifftn(vk))
    w = np.real(np.fft.ifftn(wk))
    del uk, vk, wk

    p0 = rho0 * R_GAS * T0
    ek0 = 0.5 * np.mean(u * u + v * v + w * w)
    M = np.sqrt(2 * ek0) / np.sqrt(gam * p0 / rho0)
    eta = Mt / M
    u *= eta
    v *= eta
    w *= eta
    ek0 = 0.5 * np.mean(u * u + v * v + w * w)
    Mt_out = np.sqrt(2 * ek0) / np.sqrt(gam * p0 / rho0)

    dx = 2 * np.pi / n

    def d(f, axis):
        return 0.5 * (np.roll(f, -1, axis) - np.roll(f, 1, axis)) / dx

    # dim 2 (axis 1) = x, dim 1 (axis 0) = y, dim 3 (axis 2) = z
    grads = [d(f, ax) for f in (u, v, w) for ax in (1, 0, 2)]
    sqdu = float(np.mean(sum(g * g for g in grads)))
    del grads
    mu = 2 * ek0 * np.sqrt(5 / (3 * sqdu)) / Re
    lam = np.sqrt(10 * ek0 / sqdu)
    urms = np.sqrt(2 * ek0 / 3)
    t0 = lam / urms
    params = Params(n=n, gam=gam, den0=rho0, Mt=float(Mt_out), Re=float(Re), mu0=float(mu), p0=p0, t0=float(t0))
    rho = np.full((n, n, n), rho0)
    p = np.full((n, n, n), p0)
    return params, u, v, w, rho, p


def make_particles(num: int, seed: int) -> np.ndarray:
    """Uniform particles in [0, 2pi)^3 (Part_Gen.m:1-9).  Returns (num, 3) as (x, y, z)."""
    rng = np.random.default_rng(seed + 7919)
    return rng.random((num, 3)) * (2 * np.pi)


def primitive_to_conserved(params: Params, u, v, w, rho, p) -> np.ndarray:
    """Interior conserved state (5, n, n, n) as Initialize_DHIT builds it (FlowField.cpp:99-104)."""
    g = params.gam
    vsq = u * u + v * v + w * w
    W = np.empty((5,) + u.shape)
    W[0] = rho
    W[1] = u * rho
    W[2] = v * rho
    W[3] = w * rho
    W[4] = rho * (p / (rho * (g - 1.0)) + 0.5 * vsq)
    return W


def embed_ghost(Wint: np.ndarray) -> np.ndarray:
    """Place an interior (5, n, n, n) state into the reference layout (5, n+6, n+6, n+6)
    with periodic ghosts filled (HaloTransfer on one rank)."""
    return np.pad(Wint, ((0, 0), (3, 3), (3, 3), (3, 3)), mode="wrap")


def write_reference_inputs(directory: str, params: Params, u, v, w, rho, p, particles_xyz=None) -> None:
    """Write InitialConditions/{params,Init000,unirand,particleCount} under directory."""
    d = os.path.join(directory, "InitialConditions")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params"), "wb") as f:
        f.write(struct.pack("<i", params.n))
        f.write(struct.pack("<7d", params.gam, params.den0, params.Mt, params.Re, params.mu0, params.p0, params.t0))
    with open(os.path.join(d, "Init000"), "wb") as f:
        for a in (u, v, w, rho, p):
            f.write(np.asarray(a, dtype=np.float64).tobytes(order="F"))
    np_ = 0 if particles_xyz is None else len(particles_xyz)
    with open(os.path.join(d, "particleCount"), "wb") as f:
        f.write(struct.pack("<i", np_))
    with open(os.path.join(d, "unirand"), "wb") as f:
        if np_:
            for c in range(3):
                f.write(np.ascontiguousarray(particles_xyz[:, c], dtype=np.float64).tobytes())


def read_reference_params(directory: str) -> Params:
    with open(os.path.join(directory, "InitialConditions", "params"), "rb") as f:
        n = struct.unpack("<i", f.read(4))[0]
        gam, den0, Mt, Re, mu0, p0, t0 = struct.unpack("<7d", f.read(56))
    return Params(n=n, gam=gam, den0=den0, Mt=Mt, Re=Re, mu0=mu0, p0=p0, t0=t0)


def particles_to_reference_order(xyz: np.ndarray) -> np.ndarray:
    """(x, y, z) -> the reference's particle position order (y, x, z) (ParticleTrack.cpp:15-17)."""
    return np.ascontiguousarray(xyz[:, [1, 0, 2]])
