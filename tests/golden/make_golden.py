"""Generate the golden fixtures from the reference's own code.

Runs the reference's hot-path functions, compiled unmodified from the
reference sources into oracle/_ref (``make -C oracle``), on small seeded
inputs and stores inputs and FP64 outputs in golden_*.npz next to this file.
The fixtures pin the oracle restatement (tests/test_oracle_pins.py) on
machines where the reference tree is absent.

    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "wrt-project_b200"))

import oracle as O  # noqa: E402
from phantom import ellipsoid_phantom  # noqa: E402


def main():
    ref = O.Reference()
    rng = np.random.default_rng(20240601)
    n = 16
    phantom = ellipsoid_phantom(n, 6, 77)
    noise = rng.standard_normal((n, n, n))

    # radon_grid: plane_integral (nearest sampler, lattice [-2n,2n)^2)
    nphi, ntheta, nshift = 8, 5, 7
    phi, theta, shift = ref.radon_grid(nphi, ntheta, nshift)
    P, T, S = np.meshgrid(phi, theta, shift, indexing="ij")
    planes = {}
    for name, v in (("phantom", phantom), ("noise", noise)):
        out = ref.plane_integrals(v, P.ravel(), T.ravel(), S.ravel(), nthreads=1)
        # reorder (phi, theta, shift) -> the program's (shift, phi, theta)
        planes[name] = out.reshape(nphi, ntheta, nshift).transpose(2, 0, 1).copy()
    np.savez_compressed(HERE / "golden_radon_grid.npz", phantom=phantom, noise=noise,
                        grid=np.array([nphi, ntheta, nshift]), phi=phi, theta=theta, shift=shift,
                        out_phantom=planes["phantom"], out_noise=planes["noise"])

    # samplers at random points (both reference samplers)
    x, y, z = rng.uniform(-1.05, 1.05, (3, 4000))
    near, tri = ref.samplers(noise, x, y, z)
    np.savez_compressed(HERE / "golden_samplers.npz", x=x, y=y, z=z, nearest=near, trilinear=tri)

    # ray_grid: the program's loop nest
    nsl, nsr, nph = n, 9, 8
    rays_ph = ref.ray_forward(phantom, nsl, nsr, nph, nthreads=1)
    rays_no = ref.ray_forward(noise, nsl, nsr, nph, nthreads=1)
    np.savez_compressed(HERE / "golden_ray_grid.npz", grid=np.array([nsl, nsr, nph]),
                        out_phantom=rays_ph, out_noise=rays_no)

    # radon_reduction on the phantom's rays (coupled grids, as the program).
    # An even ntheta keeps theta = pi/2 off the grid: with it on the grid the
    # slice coordinate z falls one rounding below the first node of the
    # quadratic in z (radon_reduction/slicing.c:67-72) and GSL's default error
    # handler aborts the program; golden_reduction_odd.npz records that case
    # (NaN where the reference's interpolation call fails).
    for name, nth in (("golden_reduction.npz", 6), ("golden_reduction_odd.npz", 5)):
        idx = np.array([(a, b, c) for a in range(nsr) for b in range(nph) for c in range(nth)])
        red = ref.reduction_planes(rays_ph, nth, idx[:, 0], idx[:, 1], idx[:, 2], nthreads=1)
        np.savez_compressed(HERE / name, rays=rays_ph, ntheta=nth, out=red.reshape(nsr, nph, nth))

    # backprojection adjoint at cell centres of an m^3 grid
    m = 6
    radon = rng.standard_normal((9, 8, 5))
    c = -1.0 + 1.0 / m + np.arange(m) * (2.0 / m)
    Z, X, Y = np.meshgrid(c, c, c, indexing="ij")
    adj = ref.adjoint_points(radon, X.ravel(), Y.ravel(), Z.ravel(), nthreads=1)
    np.savez_compressed(HERE / "golden_adjoint.npz", radon=radon, m=m, out=adj.reshape(m, m, m))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
