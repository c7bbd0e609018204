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
    if n % 2:
        raise ValueError("n must be even (the wavenumber layout of init_DNS.m)")
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


def make_state_device(n: int, Mt: float, Re: float, seed: int, device="cuda", k0: float = 4.0, kcmin: float = 1.0,
                      kcmax: float = 8.0, gam: float = 1.4, rho0: float = 1.0, T0: float = 300.0, rand=None):
    """The make_field recipe computed with torch (cuFFT on a GPU), returning
    (params, W) with W the conserved state already in the reference layout,
    a (5, n+6, n+6, n+6) float64 tensor on ``device`` whose ghosts are left
    for gkm_upload_state to wrap.  For the large grids (512^3, 1024^3) the
    NumPy path would need tens to hundreds of GB of host memory.

    The random u, v, w come from torch's generator seeded with ``seed`` (a
    different stream from NumPy's), unless ``rand`` supplies the three
    (n, n, n) arrays; with NumPy's draws it reproduces make_field to rounding.
    Real-to-complex transforms halve the spectral memory: the projection and
    the shell rescale keep the spectrum Hermitian and the shell (|k| <= 8)
    never reaches the Nyquist planes for n >= 32, so irfftn equals the real
    part of the full inverse transform.
    """
    import torch

    if n % 2:
        raise ValueError("n must be even (the wavenumber layout of init_DNS.m)")
    dev = torch.device(device)
    f64 = torch.float64
    Np = float(n) ** 3
    A = np.sqrt(2.0 / np.pi) * (16.0 / 3.0) * Mt ** 2 / k0 ** 5
    kf = torch.tensor(_kfft(n), dtype=f64, device=dev)
    k2 = kf.view(n, 1, 1)                       # dim 0 (y) pairs with v
    k1 = kf.view(1, n, 1)                       # dim 1 (x) pairs with u
    k3 = kf[: n // 2 + 1].view(1, 1, n // 2 + 1)  # dim 2 (z, half spectrum) pairs with w
    if rand is None:
        g = torch.Generator(device=dev)
        g.manual_seed(int(seed))
    spec = []
    for c in range(3):
        r = (torch.as_tensor(rand[c], dtype=f64, device=dev) if rand is not None
             else torch.rand((n, n, n), generator=g, dtype=f64, device=dev))
        spec.append(torch.fft.rfftn(r))
        del r
    uk, vk, wk = spec
    del spec
    ksq = (k1 * k1 + k2 * k2 + k3 * k3).clamp_min(1e-14)
    kdot = uk * k1
    kdot += vk * k2
    kdot += wk * k3
    kdot /= ksq
    uk -= kdot * k1
    vk -= kdot * k2
    wk -= kdot * k3
    del kdot
    kk = ksq.sqrt_()                            # ksq is not needed any more
    del ksq
    shell = (kk >= kcmin) & (kk <= kcmax)
    ee = A * kk ** 4 * torch.exp(-2.0 * (kk / k0) ** 2) * Np ** 2
    ee = torch.where(shell, ee / (4.0 * np.pi * torch.where(shell, kk, torch.ones_like(kk)) ** 2),
                     torch.zeros_like(ee))
    umag2 = uk.real ** 2 + uk.imag ** 2
    umag2 += vk.real ** 2 + vk.imag ** 2
    umag2 += wk.real ** 2 + wk.imag ** 2
    ok = shell & (umag2 > 0)
    fac = torch.where(ok, torch.sqrt(ee / torch.where(umag2 > 0, umag2, torch.ones_like(umag2))),
                      torch.zeros_like(ee))
    del ee, umag2, ok, shell, kk
    fac /= Np
    vel = []
    for sk in (uk, vk, wk):
        sk *= fac
        vel.append(torch.fft.irfftn(sk, s=(n, n, n)))
    del uk, vk, wk, fac
    u, v, w = vel
    del vel

    p0 = rho0 * R_GAS * T0
    ek0 = 0.5 * float(((u * u).mean() + (v * v).mean() + (w * w).mean()).item())
    M = np.sqrt(2 * ek0) / np.sqrt(gam * p0 / rho0)
    eta = Mt / M
    for a in (u, v, w):
        a *= eta
    ek0 = 0.5 * float(((u * u).mean() + (v * v).mean() + (w * w).mean()).item())
    Mt_out = np.sqrt(2 * ek0) / np.sqrt(gam * p0 / rho0)
    dx = 2 * np.pi / n
    sqdu = 0.0
    for a in (u, v, w):
        for ax in (1, 0, 2):
            d = (torch.roll(a, -1, ax) - torch.roll(a, 1, ax)) * (0.5 / dx)
            sqdu += float((d * d).mean().item())
            del d
    mu = 2 * ek0 * np.sqrt(5 / (3 * sqdu)) / Re
    lam = np.sqrt(10 * ek0 / sqdu)
    urms = np.sqrt(2 * ek0 / 3)
    params = Params(n=n, gam=gam, den0=rho0, Mt=float(Mt_out), Re=float(Re), mu0=float(mu), p0=p0,
                    t0=float(lam / urms))
    nt = n + 6
    W = torch.zeros((5, nt, nt, nt), dtype=f64, device=dev)
    inner = (slice(3, nt - 3),) * 3
    W[0][inner] = rho0
    W[1][inner] = u * rho0
    W[2][inner] = v * rho0
    W[3][inner] = w * rho0
    e = u * u
    e += v * v
    e += w * w
    del u, v, w
    W[4][inner] = rho0 * (p0 / (rho0 * (gam - 1.0))) + 0.5 * rho0 * e
    return params, W
