"""Device-resident forms of the ray transform, the ray-to-Radon reduction and
the backprojection (wrt_ray_forward_device, wrt_radon_reduction_device,
wrt_radon3d_adjoint_device): the same numbers as the host-array drop-in calls
(bit for bit: same kernels, same tables), within the FP32 tolerance of the
FP64 oracle, chained on the device without a host round trip (ray_grid ->
radon_reduction), and warm drop-in calls of one size allocate no further
device memory."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2, wrt
from wrt_b200.phantom import ellipsoid_phantom, layer_frames

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-5


def test_ray_then_reduction_on_the_device_match_the_drop_in_calls(ctx):
    n, nslices, nsr, nphi, nshift, ntheta = 40, 40, 48, 36, 64, 18
    vol = ellipsoid_phantom(n, 8, 77)
    v = wrt.Volume(ctx, n)
    v.upload(vol)
    grid = wrt.Grid(ctx, nphi, ntheta, nshift)
    rays_d = wrt.DeviceBuffer(ctx, nslices * nsr * nphi * 8)
    radon_d = wrt.DeviceBuffer(ctx, grid.nplanes * 8)
    for frame in (None, layer_frames(3, 5)[2]):
        wrt.ray_forward_device(ctx, v, nslices, nsr, nphi, rays_d.ptr, frame=frame)
        rays = rays_d.download(np.empty((nslices, nsr, nphi)))
        assert np.array_equal(rays, ctx.ray_grid(vol, nslices, nsr, nphi, frame=frame))
        assert rel_l2(rays, O.ray_forward(vol, nslices, nsr, nphi, frame=frame)) < TOL_L2
    # reduction of the reference-frame rays straight from device memory
    wrt.ray_forward_device(ctx, v, n, nsr, nphi, rays_d.ptr)
    wrt.radon_reduction_device(ctx, rays_d.ptr, n, nsr, grid, radon_d.ptr)
    radon = radon_d.download(np.empty((nshift, nphi, ntheta)))
    rays = ctx.ray_grid(vol, n, nsr, nphi)
    assert np.array_equal(radon, ctx.radon_reduction(rays, nshift, ntheta))
    assert rel_l2(radon, O.reduction_forward(rays, nshift, ntheta)) < TOL_L2
    for b in (rays_d, radon_d):
        b.close()
    grid.close()
    v.close()


def test_adjoint_on_the_device_matches_the_drop_in_call(ctx):
    n, nphi, ntheta, nshift = 24, 30, 14, 41
    rng = np.random.default_rng(9)
    radon = rng.standard_normal((nshift, nphi, ntheta))
    grid = wrt.Grid(ctx, nphi, ntheta, nshift)
    din = wrt.DeviceBuffer(ctx, radon.nbytes)
    dout = wrt.DeviceBuffer(ctx, n ** 3 * 8)
    din.upload(radon)
    wrt.radon3d_adjoint_device(ctx, din.ptr, grid, n, dout.ptr)
    got = dout.download(np.empty((n, n, n)))
    assert np.array_equal(got, ctx.radon3d_adjoint(radon, n))
    assert rel_l2(got, O.adjoint_forward(radon, n)) < TOL_L2
    din.close(); dout.close(); grid.close()


def test_warm_drop_in_calls_allocate_nothing():
    n = 32
    vol = ellipsoid_phantom(n, 6, 3)
    rng = np.random.default_rng(4)
    radon = rng.standard_normal((48, 24, 12))
    with wrt.Context(0) as c:
        calls = [lambda: c.radon_grid(vol, 24, 12, 48, sampler=wrt.TRILINEAR, half_extent=n),
                 lambda: c.ray_grid(vol, n, 40, 24),
                 lambda: c.radon_reduction(c.ray_grid(vol, n, 40, 24), 48, 12),
                 lambda: c.radon3d_adjoint(radon, n)]
        for call in calls:
            first = call()
            held = c.bytes_in_use
            again = call()
            assert c.bytes_in_use == held
            assert np.array_equal(first, again)
