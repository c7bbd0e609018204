"""The seeded initial-condition generator (restatement of init_DNS.m / Part_Gen.m)."""
import os
import struct
import tempfile

import numpy as np
import pytest

from dns_gkm_lpt_b200 import ic


def test_field_is_solenoidal_and_scaled_to_mach():
    P, u, v, w, rho, p = ic.make_field(32, 0.3, 30.0, seed=7)
    assert P.Mt == pytest.approx(0.3, rel=1e-12)
    k = ic._kfft(32)
    div = (np.fft.fftn(u) * k[None, :, None] + np.fft.fftn(v) * k[:, None, None] + np.fft.fftn(w) * k[None, None, :])
    # the Nyquist plane breaks exact symmetry of the real part; away from it divergence is round-off
    mask = (np.abs(k)[:, None, None] < 16) & (np.abs(k)[None, :, None] < 16) & (np.abs(k)[None, None, :] < 16)
    assert np.abs(div[mask]).max() < 1e-9 * np.abs(np.fft.fftn(u)).max()
    assert np.all(rho == 1.0) and np.all(p == 86100.0)
    assert P.T0 == pytest.approx(300.0)


def test_reference_file_formats_roundtrip():
    P, u, v, w, rho, p = ic.make_field(8, 0.3, 30.0, seed=1)
    xyz = ic.make_particles(10, 1)
    d = tempfile.mkdtemp()
    ic.write_reference_inputs(d, P, u, v, w, rho, p, xyz)
    Q = ic.read_reference_params(d)
    assert Q == P
    raw = np.fromfile(os.path.join(d, "InitialConditions", "Init000"))
    # MATLAB column-major: file index k*ny*nx + i*ny + j holds (j, i, k) (FlowField.cpp:96-97)
    j, i, k = 1, 2, 3
    assert raw[k * 64 + i * 8 + j] == u[j, i, k]
    with open(os.path.join(d, "InitialConditions", "particleCount"), "rb") as f:
        assert struct.unpack("<i", f.read(4))[0] == 10
    un = np.fromfile(os.path.join(d, "InitialConditions", "unirand"))
    assert np.array_equal(un[:10], xyz[:, 0]) and np.array_equal(un[10:20], xyz[:, 1])
    yxz = ic.particles_to_reference_order(xyz)
    assert np.array_equal(yxz[:, 0], xyz[:, 1])


def test_seed_determinism():
    a = ic.make_field(8, 0.3, 30.0, seed=3)
    b = ic.make_field(8, 0.3, 30.0, seed=3)
    assert np.array_equal(a[1], b[1]) and a[0] == b[0]


def test_device_state_generator_matches_numpy_recipe():
    """make_state_device (torch, run here on the CPU) with NumPy's random draws
    reproduces make_field + primitive_to_conserved to rounding."""
    import torch  # noqa: F401

    n = 32
    rng = np.random.default_rng(7)
    rand = [rng.random((n, n, n)) for _ in range(3)]
    P, u, v, w, rho, p = ic.make_field(n, 0.4, 50.0, 7)
    Wref = ic.primitive_to_conserved(P, u, v, w, rho, p)
    P2, W2 = ic.make_state_device(n, 0.4, 50.0, 7, device="cpu", rand=rand)
    W2 = W2.numpy()[:, 3:-3, 3:-3, 3:-3]
    for q in range(5):
        assert np.abs(W2[q] - Wref[q]).max() <= 1e-14 * np.abs(Wref[q]).max()
    assert P2.mu0 == pytest.approx(P.mu0, rel=1e-13)
    assert P2.t0 == pytest.approx(P.t0, rel=1e-13)
    assert P2.Mt == pytest.approx(P.Mt, rel=1e-13)
