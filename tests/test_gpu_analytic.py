"""Analytic-function transforms (radon_analytic, ray_analytic) on the GPU
against the reference's own integrators compiled here with its two example
functions (oracle/_ref: radon_analytic/src/integral.c and
ray_analytic/integral.c with exponential_bump.c / sinusoidal_bump.c), and
against closed forms: a plane through a radially symmetric term integrates to
2 pi times a 1D integral, which the lattice sum approaches."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5
FUNCS = {"exp": wrt.exp_bump(), "sine": wrt.sine_bumps()}


@pytest.mark.parametrize("family", ["exp", "sine"])
def test_plane_integrals_match_the_reference(ctx, family):
    n, nphi, ntheta, nshift = 48, 32, 16, 40
    got = ctx.radon_analytic(FUNCS[family], n, nphi, ntheta, nshift)
    phi, theta, _, shift = O.radon_grid(nphi, ntheta, nshift)
    rng = np.random.default_rng(3)
    sel = rng.integers(0, [nshift, nphi, ntheta], size=(512, 3))
    ref = O.Reference().analytic_planes(family, n, phi[sel[:, 1]], theta[sel[:, 2]],
                                        shift[sel[:, 0]])
    err = rel_l2(got[sel[:, 0], sel[:, 1], sel[:, 2]], ref)
    print(f"radon_analytic {family}: rel. L2 {err:.2e} on 512 planes")
    assert err < TOL_L2


@pytest.mark.parametrize("family", ["exp", "sine"])
def test_ray_integrals_match_the_reference(ctx, family):
    n, nshift, nphi = 40, 36, 24
    got = ctx.ray_analytic(FUNCS[family], n, nshift, nphi)
    shifts, phis = O.ray_grid(nshift, nphi)
    z = -1.0 + np.arange(n) * 2.0 / (n - 1)
    iz, i_s, ip = np.meshgrid(np.arange(n), np.arange(nshift), np.arange(nphi), indexing="ij")
    ref = O.Reference().analytic_rays(family, n, z[iz.ravel()], shifts[i_s.ravel()],
                                      phis[ip.ravel()]).reshape(n, nshift, nphi)
    err = rel_l2(got, ref)
    print(f"ray_analytic {family}: rel. L2 {err:.2e} on all rays")
    assert err < TOL_L2


def test_plane_integral_of_a_radial_term_approaches_its_closed_form(ctx):
    # one ball of the sine family: f(r) = a (r < rin), transition, 0 beyond rout;
    # a plane at distance d from the centre integrates 2 pi int_d^rout f(r) r dr
    a, rin, rout = 1.0, 0.3, 0.5
    f = wrt.sine_bumps([(0.0, 0.0, 0.0, a, rin, rout)])
    n = 160
    got = ctx.radon_analytic(f, n, 4, 2, 21)[:, 0, 0]
    shifts = O.radon_grid(4, 2, 21)[3]

    def radial(r):
        t = np.pi * (r - rout) / (rout - rin)
        v = (a / (20 * np.pi)) * (-np.sin(6 * t) / 3 + 3 * np.sin(4 * t) - 15 * np.sin(2 * t) + 20 * t)
        return np.where(r < rin, a, np.where(r < rout, v, 0.0))
    r = np.linspace(0.0, rout, 400001)
    closed = np.array([2 * np.pi * np.trapezoid(np.where(r >= abs(d), radial(r) * r, 0.0), r)
                       for d in shifts])
    err = np.abs(got - closed).max() / np.abs(closed).max()
    print(f"radial closed form: max rel. difference {err:.2e} at n = {n}")
    assert err < 2e-2  # the lattice's discretisation of the jump at rin
