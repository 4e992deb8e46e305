"""Fourier-slice inversion (radon_inversion/rtft3d.m + nfft_reconstruct_3d.m)
on the GPU: against the FP64 numpy restatement on the same data, against the
closed form of a Gaussian, and recovering a smooth phantom from the library's
own forward transform."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt

pytestmark = pytest.mark.gpu


def test_matches_restatement(ctx):
    nphi, ntheta, nshift, n = 16, 8, 33, 12
    R = np.random.default_rng(1).standard_normal((nshift, nphi, ntheta))
    got = ctx.fourier_slice_inversion(R, n)
    ref = O.fourier_slice_inversion(R, n)
    assert rel_l2(got, ref) < 1e-5
    got2 = ctx.fourier_slice_inversion(R, n, rsupp=0.9, padding=3)
    assert rel_l2(got2, O.fourier_slice_inversion(R, n, rsupp=0.9, padding=3)) < 1e-5


def test_gaussian_closed_form(ctx):
    sig, nphi, ntheta, nshift, n = 0.12, 48, 24, 65, 32
    _, _, _, s = O.radon_grid(nphi, ntheta, nshift)
    R = np.broadcast_to((2 * np.pi * sig ** 2 * np.exp(-s ** 2 / (2 * sig ** 2)))[:, None, None],
                        (nshift, nphi, ntheta)).copy()
    got = ctx.fourier_slice_inversion(R, n)
    g = -1.0 + 2.0 * np.arange(n) / n
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    r2 = X ** 2 + Y ** 2 + Z ** 2
    exact = np.exp(-r2 / (2 * sig ** 2))
    # The 48 x 24 direction grid resolves the phase e^{2 pi i nu w.y} for
    # |y| < 0.8 (FP64 error 8e-10 there); further out the quadrature itself is
    # off by up to ~5e-4 in FP64 as well, so there the GPU is held to the FP64
    # restatement of the same discretisation instead.
    inner = r2 < 0.8 ** 2
    err_in = np.abs(got - exact)[inner].max()
    idx = np.random.default_rng(3).integers(0, n, (300, 3))
    ref = O.fourier_slice_inversion(R, n, points=g[idx])
    err_all = np.abs(got[idx[:, 0], idx[:, 1], idx[:, 2]] - ref).max()
    print(f"Fourier-slice inversion of a Gaussian: max abs error {err_in:.2e} against the closed "
          f"form (|y| < 0.8), {err_all:.2e} against the FP64 restatement (300 points)")
    assert err_in < 1e-5 and err_all < 1e-5


def test_recovers_a_smooth_phantom_from_the_forward_transform(ctx):
    n, sig = 40, 0.15
    x = -1.0 + 2.0 * np.arange(n) / (n - 1)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.exp(-((X - 0.1) ** 2 + Y ** 2 + (Z + 0.05) ** 2) / (2 * sig ** 2))
    R = ctx.radon_grid(f, 48, 24, 97, sampler=wrt.TRILINEAR, half_extent=n)
    rec = ctx.fourier_slice_inversion(R, 32)
    g = -1.0 + 2.0 * np.arange(32) / 32
    Xg, Yg, Zg = np.meshgrid(g, g, g, indexing="ij")
    fg = np.exp(-((Xg - 0.1) ** 2 + Yg ** 2 + (Zg + 0.05) ** 2) / (2 * sig ** 2))
    err = rel_l2(rec, fg)
    print(f"forward transform -> Fourier-slice inversion: rel. L2 {err:.2e}")
    assert err < 5e-2  # trilinear sampling of the phantom (3.3e-2 in the FP64 restatement)
