"""The benchmark configurations beyond the headline one, at their full sizes,
checked against the FP64 oracle on seeded random subsets (the oracle at these
sizes would take hours in full):

* the CPU configuration on the GPU at its own grid: 64^3, 32 x 64 sphere grid
  x 128 shifts, 128^2 trilinear lattice, and the reference's default nearest
  sampler on its 4n x 4n lattice, 4,096 seeded planes each;

* ray transform + reduction at 128^3: 64 layer orientations x 128 layers x
  128 ray angles x 128 ray offsets (24 seeded rays of every orientation against
  the oracle); ray data reduced to a 64 x 128 sphere grid with 256 shifts
  (decoupled from the 128 ray offsets);
* 64 volumes of uneven edge lengths, each with its own sphere grid and shift
  count, in ONE batched launch; relative error per volume;
* 256^3 in FP32 and BF16 storage on a 96 x 192 sphere grid with 384 shifts
  (4,096 seeded planes each); the backprojection back to 256^3 of seeded
  Gaussian Radon data (a 32^3 voxel block and 256 scattered voxels); and the
  inner-product test <R f, g> = <f, R^T g> with the exact transpose.

Each volume is a sum of seeded ellipsoids (centres in the ball of radius 0.6,
semi-axes U[0.05, 0.3], random rotations, densities U[-0.5, 1.0])."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt
from wrt_b200.phantom import ellipsoid_phantom, layer_frames

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5


def _planes_subset(rng, nphi, ntheta, nshift, count):
    phi, theta, _, shift = O.radon_grid(nphi, ntheta, nshift)
    idx = rng.integers(0, nphi * ntheta * nshift, size=count)
    it, ip, i_s = idx % ntheta, (idx // ntheta) % nphi, idx // (ntheta * nphi)
    return (i_s, ip, it), (phi[ip], theta[it], shift[i_s])


@pytest.mark.parametrize("sampler", [O.TRILINEAR, O.NEAREST])
def test_cpu_configuration_64_cubed_at_its_grid(ctx, sampler):
    n, nphi, ntheta, nshift = 64, 64, 32, 128
    vol = ellipsoid_phantom(n, 8, 1000)
    L = n if sampler == O.TRILINEAR else 2 * n  # 128^2 trilinear; reference 4n x 4n nearest
    got = ctx.radon_grid(vol, nphi, ntheta, nshift, sampler=sampler, half_extent=L)
    rng = np.random.default_rng(64 + sampler)
    (i_s, ip, it), (p, t, s) = _planes_subset(rng, nphi, ntheta, nshift, 4096)
    ref = O.radon_planes(vol, p, t, s, sampler=sampler, half_extent=L)
    err = rel_l2(got[i_s, ip, it], ref)
    print(f"64^3 {'trilinear' if sampler else 'nearest'}: rel. L2 {err:.2e} on 4096 planes")
    assert err < TOL_L2


def test_rays_64_orientations_and_decoupled_reduction_128(ctx):
    n = 128
    vol = ellipsoid_phantom(n, 16, 1001)
    frames = layer_frames(64, 1101)
    rng = np.random.default_rng(12)
    shifts, phis = O.ray_grid(128, 128)
    errs = []
    for k, F in enumerate(frames):
        rays = ctx.ray_grid(vol, n, 128, 128, frame=None if k == 0 else F)
        # oracle on 24 seeded rays of every orientation
        iz, i_s, ip = (rng.integers(0, 128, 24) for _ in range(3))
        got = rays[iz, i_s, ip]
        ref = np.array([O.ray_transform(vol, -1.0 + 2.0 * a / (n - 1), shifts[b], phis[c],
                                        frame=None if k == 0 else F)
                        for a, b, c in zip(iz, i_s, ip)])
        errs.append(rel_l2(got, ref))
        if k == 0:
            rays0 = rays
    assert max(errs) < TOL_L2, errs
    # reduction of orientation 0's rays (128 offsets) to 256 Radon shifts
    radon = ctx.radon_reduction(rays0, 256, 64)
    assert radon.shape == (256, 128, 64)
    sel = rng.integers(0, [256, 128, 64], size=(1024, 3))
    ref = O.reduction_planes(rays0, 256, 64, sel[:, 0], sel[:, 1], sel[:, 2])
    assert rel_l2(radon[sel[:, 0], sel[:, 1], sel[:, 2]], ref) < TOL_L2


def test_64_uneven_volumes_in_one_batched_launch(ctx):
    rng = np.random.default_rng(2002)
    reqs, keep = [], []
    for k in range(64):
        n = int(rng.choice([48, 64, 96, 128, 160, 192]))
        nth = int(rng.integers(16, 97))
        ns = int(rng.integers(64, 257))
        vol = ellipsoid_phantom(n, int(rng.integers(4, 25)), 3000 + k)
        v = wrt.Volume(ctx, n)
        v.upload(vol)
        g = wrt.Grid(ctx, 2 * nth, nth, ns)
        out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
        reqs.append((v, g, out.ptr, n))
        keep.append((vol, v, g, out, (ns, 2 * nth, nth)))
    ctx.timer_start()
    wrt.radon_forward_batch(ctx, reqs)
    ms = ctx.timer_stop()
    planes = sum(np.prod(s) for *_, s in keep)
    errs = []
    for k, (vol, v, g, out, shape) in enumerate(keep):
        res = out.download(np.empty(shape))
        (i_s, ip, it), (p, t, s) = _planes_subset(rng, shape[1], shape[2], shape[0], 8)
        ref = O.radon_planes(vol, p, t, s, sampler=O.TRILINEAR, half_extent=vol.shape[0])
        errs.append(rel_l2(res[i_s, ip, it], ref))
        out.close(); g.close(); v.close()
    print(f"64 volumes, {planes} planes in one launch: {ms:.1f} ms; per-volume rel. L2 "
          f"max {max(errs):.2e}, median {np.median(errs):.2e}")
    assert max(errs) < TOL_L2


@pytest.fixture(scope="module")
def vol256():
    return ellipsoid_phantom(256, 16, 1003)


@pytest.mark.parametrize("storage", [wrt.STORAGE_F32, wrt.STORAGE_BF16])
def test_256_cubed_fp32_and_bf16(ctx, vol256, storage):
    n, nphi, ntheta, nshift = 256, 192, 96, 384
    v = wrt.Volume(ctx, n, storage=storage)
    v.upload(vol256)
    g = wrt.Grid(ctx, nphi, ntheta, nshift)
    out = wrt.DeviceBuffer(ctx, g.nplanes * 8)
    wrt.radon_forward_batch(ctx, [(v, g, out.ptr, n)])
    res = out.download(np.empty((nshift, nphi, ntheta)))
    rng = np.random.default_rng(31 + storage)
    (i_s, ip, it), (p, t, s) = _planes_subset(rng, nphi, ntheta, nshift, 4096)
    got = res[i_s, ip, it]
    if storage == wrt.STORAGE_BF16:
        held = O.radon_planes(wrt.round_bf16(vol256), p, t, s, sampler=O.TRILINEAR, half_extent=n)
        assert rel_l2(got, held) < TOL_L2  # the FP32 path on the values stored
        exact = O.radon_planes(vol256, p, t, s, sampler=O.TRILINEAR, half_extent=n)
        err = rel_l2(got, exact)
        print(f"256^3 BF16 storage: rel. L2 {err:.2e} against the unrounded volume")
        assert err < 4e-3  # bf16 keeps 8 significant bits
    else:
        exact = O.radon_planes(vol256, p, t, s, sampler=O.TRILINEAR, half_extent=n)
        assert rel_l2(got, exact) < TOL_L2
    out.close(); g.close(); v.close()


def test_256_cubed_backprojection_and_inner_product(ctx, vol256):
    n, nphi, ntheta, nshift = 256, 192, 96, 384
    rng = np.random.default_rng(4004)
    # the reference's backprojection of seeded Gaussian Radon data, back to 256^3
    g = rng.standard_normal((nshift, nphi, ntheta))
    adj = ctx.radon3d_adjoint(g, n)  # [iz][ix][iy], cell centres
    c = lambda i: -1.0 + 1.0 / n + i * (2.0 / n)
    # a 32^3 block of voxels at a seeded corner, and 256 voxels anywhere
    z0, x0, y0 = rng.integers(0, n - 32, 3)
    bz, bx, by = np.meshgrid(np.arange(z0, z0 + 32), np.arange(x0, x0 + 32),
                             np.arange(y0, y0 + 32), indexing="ij")
    iz = np.concatenate([bz.ravel(), rng.integers(0, n, 256)])
    ix = np.concatenate([bx.ravel(), rng.integers(0, n, 256)])
    iy = np.concatenate([by.ravel(), rng.integers(0, n, 256)])
    ref = O.adjoint_points(g, c(ix), c(iy), c(iz))
    err = rel_l2(adj[iz, ix, iy], ref)
    print(f"256^3 backprojection: rel. L2 {err:.2e} on a 32^3 block + 256 voxels")
    assert err < TOL_L2
    # inner-product test of the forward transform against its exact transpose:
    # g seeded Gaussian on 2048 random planes (zero elsewhere)
    gs = np.zeros((nshift, nphi, ntheta))
    idx = rng.choice(gs.size, size=2048, replace=False)
    gs.flat[idx] = rng.standard_normal(2048)
    v = wrt.Volume(ctx, n)
    v.upload(vol256)
    grid = wrt.Grid(ctx, nphi, ntheta, nshift)
    out = wrt.DeviceBuffer(ctx, grid.nplanes * 8)
    wrt.radon_forward_batch(ctx, [(v, grid, out.ptr, n)])
    Rf = out.download(np.empty((nshift, nphi, ntheta)))
    RTg = ctx.radon_transpose(gs, n, sampler=wrt.TRILINEAR, half_extent=n)
    lhs, rhs = float((Rf * gs).sum()), float((vol256 * RTg).sum())
    print(f"<Rf, g> = {lhs:.12e}, <f, R^T g> = {rhs:.12e}, rel. diff "
          f"{abs(lhs - rhs) / abs(lhs):.2e}")
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    out.close(); grid.close(); v.close()
