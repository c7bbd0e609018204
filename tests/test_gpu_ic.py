"""The GPU initial-condition generator (ic.make_state_device, cuFFT through
torch.fft) on cuda against the NumPy restatement of init_DNS.m
(InitialConditions/init_DNS.m:34-126).  It produces every 512^3 and 1024^3
benchmark input, so it is checked on the device that runs it: with NumPy's
random draws it must reproduce make_field + primitive_to_conserved to rounding
(1e-14 of each component's largest value); with the device generator's own
draws the field must keep the recipe's properties (solenoidal, scaled to the
requested turbulent Mach number, uniform density and pressure)."""
import numpy as np
import pytest
import torch

from dns_gkm_lpt_b200 import ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,Mt,Re,seed", [(32, 0.4, 50.0, 7), (64, 0.3, 30.0, 1234)])
def test_device_generator_matches_numpy_recipe_on_gpu(n, Mt, Re, seed):
    rng = np.random.default_rng(seed)
    rand = [rng.random((n, n, n)) for _ in range(3)]
    P, u, v, w, rho, p = ic.make_field(n, Mt, Re, seed)
    Wref = ic.primitive_to_conserved(P, u, v, w, rho, p)
    P2, W2 = ic.make_state_device(n, Mt, Re, seed, device="cuda", rand=rand)
    assert W2.is_cuda and W2.dtype == torch.float64 and tuple(W2.shape) == (5, n + 6, n + 6, n + 6)
    W2 = W2.cpu().numpy()[:, 3:-3, 3:-3, 3:-3]
    for q in range(5):
        assert np.abs(W2[q] - Wref[q]).max() <= 1e-14 * np.abs(Wref[q]).max(), q
    assert P2.mu0 == pytest.approx(P.mu0, rel=1e-13)
    assert P2.t0 == pytest.approx(P.t0, rel=1e-13)
    assert P2.Mt == pytest.approx(P.Mt, rel=1e-13)
    assert P2.p0 == P.p0 and P2.n == P.n


def test_device_generator_own_draws_keep_the_recipe_properties():
    n, Mt = 64, 0.5
    P, W = ic.make_state_device(n, Mt, 100.0, 99, device="cuda")
    W = W.cpu().numpy()[:, 3:-3, 3:-3, 3:-3]
    rho = W[0]
    u, v, w = W[1] / rho, W[2] / rho, W[3] / rho
    assert np.all(rho == 1.0)
    # pressure from E: p = (gamma - 1)(E - rho |u|^2 / 2) is the uniform p0
    p = (P.gam - 1.0) * (W[4] - 0.5 * rho * (u * u + v * v + w * w))
    assert np.abs(p - P.p0).max() <= 1e-9 * P.p0
    # Mt = sqrt(<|u|^2>) / c0 with c0 = sqrt(gamma p0 / rho0) (init_DNS.m:84-92)
    c0 = np.sqrt(P.gam * P.p0 / 1.0)
    assert np.sqrt(np.mean(u * u + v * v + w * w)) / c0 == pytest.approx(Mt, rel=1e-10)
    # spectral divergence (u pairs with axis 1, v with axis 0, w with axis 2) away from Nyquist
    k = ic._kfft(n)
    div = (np.fft.fftn(u) * k[None, :, None] + np.fft.fftn(v) * k[:, None, None] + np.fft.fftn(w) * k[None, None, :])
    mask = (np.abs(k)[:, None, None] < n // 2) & (np.abs(k)[None, :, None] < n // 2) & (np.abs(k)[None, None, :] < n // 2)
    assert np.abs(div[mask]).max() < 1e-9 * np.abs(np.fft.fftn(u)).max()
