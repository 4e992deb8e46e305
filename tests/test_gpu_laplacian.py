"""Spectral Laplacian (radon_inversion/backprojection/laplace3dfft.m) on the
GPU and the backprojection inversion it completes: against the numpy
restatement (FP64 FFTs both sides), exact on eigenfunctions, the device entry
point equal to the host one, and the whole chain forward transform ->
backprojection -> -1/(8 pi^2) Laplacian recovering a smooth phantom."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32, 27, 64])
def test_laplacian_matches_restatement(ctx, n):
    u = np.random.default_rng(n).standard_normal((n, n, n))
    got = ctx.spectral_laplacian(u, 2.0)
    assert rel_l2(got, O.spectral_laplacian(u, 2.0)) < 1e-12
    got3 = ctx.spectral_laplacian(u, 3.0)
    assert rel_l2(got3, O.spectral_laplacian(u, 3.0)) < 1e-12


def test_laplacian_eigenfunction_and_device_entry(ctx):
    n = 48
    c = -1.0 + (2.0 * np.arange(n) + 1.0) / n
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    u = np.sin(np.pi * 5 * X) * np.cos(np.pi * 2 * Y) * np.sin(np.pi * 7 * Z)
    got = ctx.spectral_laplacian(u, 2.0)
    assert np.abs(got + np.pi ** 2 * (25 + 4 + 49) * u).max() < 1e-9
    din, dout = wrt.DeviceBuffer(ctx, u.nbytes), wrt.DeviceBuffer(ctx, u.nbytes)
    din.upload(u)
    ctx.check(wrt.lib().wrt_spectral_laplacian_device(ctx.handle, din.ptr, n, 2.0, dout.ptr),
              "laplacian device")
    assert np.array_equal(dout.download(np.empty_like(u)), got)
    din.close(); dout.close()


def test_backprojection_inversion_recovers_a_smooth_phantom(ctx):
    n, sig = 32, 0.15
    x = -1.0 + 2.0 * np.arange(n) / (n - 1)  # nodes of the input grid
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / (2 * sig ** 2))
    R = ctx.radon_grid(f, 48, 24, 96, sampler=wrt.TRILINEAR, half_extent=n)
    rec = ctx.backprojection_inversion(R, n)  # [iz][ix][iy] at cell centres
    c = -1.0 + (2.0 * np.arange(n) + 1.0) / n
    Zc, Xc, Yc = np.meshgrid(c, c, c, indexing="ij")
    fc = np.exp(-(Xc ** 2 + Yc ** 2 + Zc ** 2) / (2 * sig ** 2))
    inner = Xc ** 2 + Yc ** 2 + Zc ** 2 < 0.25
    err = rel_l2(rec[inner], fc[inner])
    print(f"backprojection inversion: rel. L2 {err:.3e} inside radius 0.5")
    assert err < 0.05
    # the same chain in the oracle
    ref = O.spectral_laplacian(O.adjoint_forward(R, n), 2.0) * (-1.0 / (8.0 * np.pi ** 2))
    assert rel_l2(rec, ref) < 1e-5
